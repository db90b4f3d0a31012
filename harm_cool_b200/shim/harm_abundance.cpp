/*
 * harm_abundance.cpp -- the reference's Fortran entry point abundance_() over
 * libharm_b200's restatement of it.
 *
 * The reference's COOL_EOS code fills its table cache node by node through
 *
 *   extern "C" void abundance_(double *rho, double *T, double *HdFac, double *e,
 *                              double *p, double *Qnu, double *tau,
 *                              double *xnee, double *xnep);        cooleos.c:58-59
 *
 * called from calc_cache_val (cooleos.c:171-194) on its cache worker threads,
 * and links the gfortran objects of abundance.f90 and its modules for it
 * (Makefile:60-67).  Linking this file and libharm_b200 in their place gives
 * the same symbol, with the same arguments and units, on a build host without
 * a Fortran compiler.  Each call computes its node on the calling thread.  A
 * failed library call prints harm_last_error() and exits(1).
 */
#include "harm_b200.h"

#include <stdio.h>
#include <stdlib.h>

extern "C" void abundance_(double *rho, double *T, double *HdFac, double *e, double *p, double *Qnu, double *tau,
                           double *xnee, double *xnep)
{
  double out[7];
  if (harm_nu_abundance(rho, T, HdFac, 1, 1, out)) {
    fprintf(stderr, "harm_b200: harm_nu_abundance: %s\n", harm_last_error());
    exit(1);
  }
  *e = out[0];
  *p = out[1];
  *Qnu = out[2];
  *tau = out[3];
  *xnee = out[4];
  *xnep = out[5];
}
