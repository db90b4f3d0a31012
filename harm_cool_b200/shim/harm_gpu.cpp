/*
 * harm_gpu.cpp -- HARM-COOL's per-zone update on a B200, behind the
 * reference's own calling surface.
 *
 * This file is the reference-side binding of libharm_b200.  It is compiled
 * with the reference's sources, against its decs.h, and takes the place of
 * step_ch.c, bounds.c, fixup.c and utoprim_2d.c in the link.  The reference
 * compiles its .c files as C++ (Makefile:17-29), so the routines below keep
 * C++ linkage and the reference's exact prototypes (decs.h:548-610):
 *
 *   void step_ch(void)                                   step_ch.c:90-140
 *   void bound_prim(double *_pr)                         bounds.c:54-331
 *   void fixup(double *_pv)                              fixup.c:51-60
 *   void fixup1zone(int h, int i, int j, double pv[NPR]) fixup.c:142-383
 *   void fixup_utoprim(double *_pv)                      fixup.c:432-538
 *   void set_Katm(void)                                  fixup.c:555-585
 *   int  Utoprim_2d(U, gcov, gcon, gdet, prim)           utoprim_2d.c:126-176
 *
 * The rest of the reference (main.c, init.c, diag.c, dump.c, restart.c,
 * the other inversions) is unchanged.  The device keeps the state between
 * steps; the host arrays _p and _pflag are brought up to date after every
 * step_ch(), since the reference's main loop reads them (diag, dump,
 * restart) without announcing it.  A host that reads them only at its own
 * output times can turn that off with harm_gpu_set_sync(0) and call
 * harm_gpu_sync_to_host() before each read; a host that writes _p between
 * steps calls harm_gpu_invalidate() so the next step uploads it.
 *
 * Errors: a failed library call prints harm_last_error() and exits(1); a
 * physics failure recorded on the device goes to the reference's fail(),
 * after the state is brought back; dt < 1e-9 exits(11) as step_ch.c:126-129
 * does.
 */
#include "decs.h"
#include "harm_b200.h"

#include <stdio.h>
#include <stdlib.h>

static harm_ctx *g_ctx;        /* the device state */
static int g_stepping;         /* g_ctx was made by step_ch(), with the run's final parameters */
static int g_host_newer = 1;   /* the host arrays hold the state: upload before the next step */
static int g_sync_every = 1;   /* bring _p and _pflag back after every step */

static void gpu_check(int rc, const char *what)
{
  if (rc) {
    fprintf(stderr, "harm_b200: %s: %s\n", what, harm_last_error());
    exit(1);
  }
}

static harm_grid_spec grid_spec(void)
{
  harm_grid_spec g;
  g.n1 = N1;
  g.n2 = N2;
  g.n3 = N3;
  g.a = a;
  g.Rin = Rin;
  g.Rout = Rout;
  g.R0 = R0;
  g.hslope = hslope;
  return g;
}

/* the device context for the reference's current globals (geometry from
   set_grid(), Katm from set_Katm(), the run parameters) */
static harm_ctx *gpu(void)
{
  if (!g_ctx) {
    harm_params prm;
    prm.n1 = N1;
    prm.n2 = N2;
    prm.n3 = N3;
    prm.lim = lim;
    prm.a = a;
    prm.gam = gam;
    prm.cour = cour;
    prm.defcon = defcon;
    prm.tf = tf;
    for (int k = 0; k < NDIM; k++) {
      prm.dx[k] = dx[k];
      prm.startx[k] = startx[k];
    }
    gpu_check(harm_create(&prm, _gcov, _gcon, _gdet, _conn, _coords, Katm, 0, &g_ctx), "harm_create");
  }
  return g_ctx;
}

static void drop_context(void)
{
  if (g_ctx) harm_destroy(g_ctx);
  g_ctx = NULL;
  g_stepping = 0;
  g_host_newer = 1;
}

extern "C" void harm_gpu_invalidate(void) { g_host_newer = 1; }

extern "C" void harm_gpu_set_sync(int every_step) { g_sync_every = every_step; }

extern "C" void harm_gpu_sync_to_host(void)
{
  if (g_ctx && g_stepping && !g_host_newer)
    gpu_check(harm_get_prims(g_ctx, _p, (signed char *)_pflag), "harm_get_prims");
}

extern "C" void harm_gpu_release(void) { drop_context(); }

void step_ch(void)
{
  if (!g_stepping) {
    /* a context made during init() carried its parameters (defcon, tf) of that
       moment and the Katm before set_Katm(): the stepping one is made now */
    drop_context();
    gpu();
    g_stepping = 1;
  }
  if (g_host_newer) {
    gpu_check(harm_put_prims(g_ctx, _p, (const signed char *)_pflag), "harm_put_prims");
    gpu_check(harm_set_time(g_ctx, t, dt), "harm_set_time");
    gpu_check(harm_set_mass(g_ctx, mass_in, mass_out), "harm_set_mass");
    g_host_newer = 0;
  }
  if (rank == 0) fprintf(stdout, "hf");
  const int rc = harm_step_ch(g_ctx);
  if (rc == HARM_E_DT) {
    harm_gpu_sync_to_host();
    fprintf(stderr, "^timestep too small\n");
    exit(11);
  }
  gpu_check(rc, "harm_step_ch");
  harm_diag d;
  gpu_check(harm_get_time(g_ctx, &t, &dt), "harm_get_time");
  gpu_check(harm_get_diag(g_ctx, &d), "harm_get_diag");
  mdot = d.mdot;
  edot = d.edot;
  ldot = d.ldot;
  mdot_in = d.mdot_in;
  mdot_out = d.mdot_out;
  mass_curr = d.mass_curr;
  mass_in = d.mass_in;
  mass_out = d.mass_out;
  if (d.fail_code) {
    harm_gpu_sync_to_host();
    fail(d.fail_code);
  }
  if (g_sync_every) harm_gpu_sync_to_host();
}

/* the per-array routines run on the host array passed, as the reference's do
   (init() calls them on _p before the first step, init.c:311-313, 419-423) */
void bound_prim(double *_pr)
{
  if (_pr == _p) harm_gpu_sync_to_host();
  gpu_check(harm_bound_prim(gpu(), _pr), "harm_bound_prim");
  if (_pr == _p) g_host_newer = 1;
}

void fixup(double *_pv)
{
  if (_pv == _p) harm_gpu_sync_to_host();
  gpu_check(harm_fixup(gpu(), _pv), "harm_fixup");
  if (_pv == _p) g_host_newer = 1;
}

void fixup_utoprim(double *_pv)
{
  if (_pv == _p) harm_gpu_sync_to_host();
  gpu_check(harm_fixup_utoprim(gpu(), _pv), "harm_fixup_utoprim");
  if (_pv == _p) g_host_newer = 1;
}

void fixup1zone(int h, int i, int j, double pv[NPR])
{
  char(*pflag)[SN1][SN2] = (char(*)[SN1][SN2])(_pflag);
  const int hij[3] = {h, i, j};
  signed char flag = 0;
  gpu_check(harm_fixup1zone(gpu(), 1, hij, pv, &flag), "harm_fixup1zone");
  if (flag == -33) pflag[h][i][j] = -33;
}

void set_Katm(void)
{
  double G_tmp;
  get_G_ATM(&G_tmp);
  fflush(stdout);
  fprintf(stdout, "G_tmp = %26.20e \n", G_tmp);
  fflush(stdout);
  harm_grid_spec g = grid_spec();
  gpu_check(harm_set_katm(&g, gam, _coords, Katm), "harm_set_katm");
  /* a context holds the Katm it was made with */
  if (g_ctx && !g_stepping) drop_context();
}

int Utoprim_2d(double U[NPR], double gcov[NDIM][NDIM], double gcon[NDIM][NDIM], double gdet, double prim[NPR])
{
  int ret = 0;
  gpu_check(harm_utoprim_2d_batch_noalloc(U, &gcov[0][0], &gcon[0][0], &gdet, prim, &ret, 1, gam),
            "harm_utoprim_2d_batch_noalloc");
  return ret;
}
