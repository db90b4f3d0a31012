/*
 * Stand-in for the reference's Fortran EOS/neutrino table generator, for the
 * COOL_EOS checker build only (TEST INFRASTRUCTURE ONLY).
 *
 * The reference fills its EOS tables by calling abundance_() (abundance.f90:6-243)
 * through calc_cache_val (cooleos.c:171-194).  No Fortran compiler exists here, so
 * this file supplies a function with the same signature and a smooth, analytic
 * equation of state in its place: nucleons and electrons as ideal gases (Ye = 1/2)
 * plus black-body radiation, and power-law placeholders for the neutrino
 * emissivity and optical depth.  The checker then exercises the reference's own
 * run-time EOS code -- its lazily filled (rho, T) cache, the Akima interpolation
 * and the Newton solve for T -- on these tables; the values themselves carry no
 * physics of the reference's generator.
 */
void abundance_(double *rho, double *T, double *HdFac, double *e, double *p, double *Qnu, double *tau,
                double *xnee, double *xnep)
{
  const double kB = 1.380649e-16, mu = 1.66053907e-24, arad = 7.5657e-15;
  const double nb = *rho / mu;
  const double pgas = 1.5 * nb * kB * (*T);          /* ions + electrons, Ye = 1/2 */
  const double T2 = (*T) * (*T);
  const double prad = arad * T2 * T2 / 3.0;
  *p = pgas + prad;
  *e = 1.5 * pgas + 3.0 * prad;
  *Qnu = 1.0e-30 * (*rho) * T2 * (*T) * 1.0e-9;
  *tau = 1.0e-10 * (*Qnu) * (*HdFac);
  *xnee = 0.5 * (*rho) / 1.66e15;                    /* fm^-3: Yee = 1/2 in calc_cache_val */
  *xnep = 0.0;
}
