/*
 * Driver for the HARM-COOL reference compiled as a CPU checker library
 * (oracle/_ref/<config>/libharmref.so).  TEST INFRASTRUCTURE ONLY.
 *
 * The reference's own main() (main.c:97-274) redirects stdout/stderr to
 * files and writes dumps; this driver reproduces only the part of its
 * start-up that the step path needs, in the same order:
 *   MPI_Init + set_MPI("1x1x1")        main.c:110-141
 *   init()                             main.c:164 (init.c:70)
 *   mass_start, diag_mass(0)           main.c:171-182
 *   defcon = 1                         main.c:204
 * and then exposes step_ch() (step_ch.c:90) and the reference's global
 * arrays to a ctypes caller.  It is compiled together with the reference
 * sources, with decs.h resolved to a per-configuration patched copy.
 */
#include "decs.h"
#include <vector>
#include <string.h>
#include <time.h>
#include <unistd.h>
#include <fcntl.h>
#include <signal.h>

#ifdef MPI_USED
void set_MPI(int argc, char *argv[]);
#endif
double advance(double *_pi, double *_pb, double Dt, double *_pf, int fullstep);
double fluxcalc(double *_pr, double *_F, const int dir, const int fullstep);
#if TRACERSDUMP
void init_tracers(void);
#endif

static int g_stdout_saved = -1;

static void quiet(int on)
{
  /* step_ch() prints progress letters on stdout (step_ch.c:99-100) */
  fflush(stdout);
  if (on) {
    if (g_stdout_saved < 0) g_stdout_saved = dup(1);
    int fd = open("/dev/null", O_WRONLY);
    dup2(fd, 1); close(fd);
  } else if (g_stdout_saved >= 0) {
    dup2(g_stdout_saved, 1);
  }
}

extern "C" {

int ref_init(void)
{
  quiet(1);
  static char a0[] = "harm", a1[] = "1x1x1";
  char *argv[] = {a0, a1, NULL};
  int argc = 2;
  nstep = 0;
#ifdef MPI_USED
  MPI_Init(&argc, (char ***)&argv);
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  MPI_Comm_size(MPI_COMM_WORLD, &nprocs);
  set_MPI(argc, argv);
#endif
#if COOL_EOS
  /* SetupCache_CoolEOS (cooleos.c:977-986) installs process-wide signal handlers:
     keep the caller's */
  static const int sigs[] = {SIGINT, SIGQUIT, SIGHUP, SIGTERM, SIGCHLD};
  struct sigaction saved[5];
  for (int k = 0; k < 5; k++) sigaction(sigs[k], NULL, &saved[k]);
#endif
  init();
#if COOL_EOS
  for (int k = 0; k < 5; k++) sigaction(sigs[k], &saved[k], NULL);
#endif
  {
    double (*p)[SN1][SN2][NPR] = (double (*)[SN1][SN2][NPR])(_p);
    double (*gdet)[SN2][NPG] = (double (*)[SN2][NPG])(_gdet);
    int h, i, j;
    mass_start = 0.;
    ZLOOP { mass_start += p[h][i][j][RHO] * gdet[i][j][CENT] * dx[RR] * dx[TH] * dx[PH]; }
  }
  diag_mass(0.);
#if TRACERSDUMP
  init_tracers();  /* main.c:184-186 */
#endif
  defcon = 1.;
  quiet(0);
  return 0;
}

void ref_step(void) { quiet(1); step_ch(); nstep++; quiet(0); }

void ref_dims(int *out)
{
  out[0] = N1; out[1] = N2; out[2] = N3; out[3] = SN1; out[4] = SN2; out[5] = SN3;
  out[6] = NPR; out[7] = NPG; out[8] = istart; out[9] = istop; out[10] = jstart;
  out[11] = jstop; out[12] = hstart; out[13] = hstop;
}

void *ref_ptr(const char *name)
{
  if (!strcmp(name, "p")) return _p;
  if (!strcmp(name, "ph")) return _ph;
  if (!strcmp(name, "dq")) return _dq;
  if (!strcmp(name, "F1")) return _F1;
  if (!strcmp(name, "F2")) return _F2;
  if (!strcmp(name, "F3")) return _F3;
  if (!strcmp(name, "pflag")) return _pflag;
  if (!strcmp(name, "gcov")) return _gcov;
  if (!strcmp(name, "gcon")) return _gcon;
  if (!strcmp(name, "gdet")) return _gdet;
  if (!strcmp(name, "conn")) return _conn;
  if (!strcmp(name, "coords")) return _coords;
  if (!strcmp(name, "A")) return _A;
#if DO_FONT_FIX
  if (!strcmp(name, "Katm")) return Katm;
#endif
  return NULL;
}

static double *scalar(const char *name)
{
  static double dx1, dx2, dx3, sx1, sx2, sx3, lim_d;
  if (!strcmp(name, "dt")) return &dt;
  if (!strcmp(name, "t")) return &t;
  if (!strcmp(name, "tf")) return &tf;
  if (!strcmp(name, "a")) return &a;
  if (!strcmp(name, "gam")) return &gam;
  if (!strcmp(name, "cour")) return &cour;
  if (!strcmp(name, "defcon")) return &defcon;
  if (!strcmp(name, "Rin")) return &Rin;
  if (!strcmp(name, "Rout")) return &Rout;
  if (!strcmp(name, "hslope")) return &hslope;
  if (!strcmp(name, "R0")) return &R0;
  if (!strcmp(name, "mdot")) return &mdot;
  if (!strcmp(name, "edot")) return &edot;
  if (!strcmp(name, "ldot")) return &ldot;
  if (!strcmp(name, "mdot_in")) return &mdot_in;
  if (!strcmp(name, "mdot_out")) return &mdot_out;
  if (!strcmp(name, "mass_start")) return &mass_start;
  if (!strcmp(name, "mass_curr")) return &mass_curr;
  if (!strcmp(name, "mass_in")) return &mass_in;
  if (!strcmp(name, "mass_out")) return &mass_out;
  if (!strcmp(name, "dx1")) { dx1 = dx[1]; return &dx1; }
  if (!strcmp(name, "dx2")) { dx2 = dx[2]; return &dx2; }
  if (!strcmp(name, "dx3")) { dx3 = dx[3]; return &dx3; }
  if (!strcmp(name, "startx1")) { sx1 = startx[1]; return &sx1; }
  if (!strcmp(name, "startx2")) { sx2 = startx[2]; return &sx2; }
  if (!strcmp(name, "startx3")) { sx3 = startx[3]; return &sx3; }
  if (!strcmp(name, "lim")) { lim_d = lim; return &lim_d; }
  return NULL;
}

double ref_get(const char *name) { double *s = scalar(name); return s ? *s : NAN; }

int ref_set(const char *name, double v)
{
  if (!strcmp(name, "lim")) { lim = (int)v; return 0; }
  double *s = scalar(name);
  if (!s || !strncmp(name, "dx", 2) || !strncmp(name, "startx", 6)) return -1;
  *s = v;
  return 0;
}

/* single-function known-answer hooks (quiet: no output on the success path) */
int ref_utoprim_2d(double *U, int i, int j, double *prim)
{
  struct of_geom geom;
  get_geometry(0, i, j, CENT, &geom);
  return Utoprim_2d(U, geom.gcov, geom.gcon, geom.g, prim);
}

int ref_utoprim_fix(double *U, int i, int j, double *prim, double K, int which)
{
  struct of_geom geom;
  get_geometry(0, i, j, CENT, &geom);
  if (which == 1) return Utoprim_1dvsq2fix1(U, geom.gcov, geom.gcon, geom.g, prim, K);
  return Utoprim_1dfix1(U, geom.gcov, geom.gcon, geom.g, prim, K);
}

/* conserved variables of a primitive state at zone (i, j), CENT (phys.c:99-105) */
void ref_prim_to_U(double *pr, int i, int j, double *U)
{
  struct of_geom geom;
  struct of_state q;
  get_geometry(0, i, j, CENT, &geom);
  get_state(pr, &geom, &q);
  primtoU(pr, &q, &geom, U);
}

void ref_fixup(double *pv) { fixup(pv); }
void ref_bound_prim(double *pv) { bound_prim(pv); }
void ref_fixup_utoprim(double *pv) { fixup_utoprim(pv); }
#ifndef HARM_SHIM_BUILD
/* (the drop-in build has no advance(): step_ch.c is not linked) */
double ref_advance(double *pi, double *pb, double Dt, double *pf, int fullstep)
{
  quiet(1);
  double r = advance(pi, pb, Dt, pf, fullstep);
  quiet(0);
  return r;
}
#endif

/* diag(INIT_OUT) (diag.c:59-375) run in directory dir (which must hold a dumps/
   subdirectory): it appends the energy line to dir/ener.out and writes its LOG
   line, with divbmax and its zone, to dir/diag_stderr.txt */
int ref_diag_init(const char *dir)
{
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(dir)) return -1;
  fflush(stderr);
  int saved = dup(2);
  int fd = open("diag_stderr.txt", O_WRONLY | O_CREAT | O_TRUNC, 0644);
  dup2(fd, 2);
  close(fd);
  quiet(1);
  diag(INIT_OUT);
  quiet(0);
  fflush(stderr);
  dup2(saved, 2);
  close(saved);
  return chdir(cwd);
}

/* restart_write() (restart.c:73-186) in directory dir (with a dumps/
   subdirectory): the file ends up as dir/dumps/rdump1.0_1x1x1 */
int ref_restart_write(const char *dir)
{
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(dir)) return -1;
  quiet(1);
  fflush(stderr);
  int saved = dup(2);
  int fd = open("/dev/null", O_WRONLY);
  dup2(fd, 2);
  close(fd);
  restart_write();
  fflush(stderr);
  dup2(saved, 2);
  close(saved);
  quiet(0);
  return chdir(cwd);
}

/* restart_init() (restart.c:197-303) from dir/dumps/: the reference's own
   reader; it allocates new global arrays, so callers fetch pointers again */
int ref_restart_init(const char *dir)
{
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(dir)) return -1;
  quiet(1);
  fflush(stderr);
  int saved = dup(2);
  int fd = open("/dev/null", O_WRONLY);
  dup2(fd, 2);
  close(fd);
  int ok = restart_init();
  fflush(stderr);
  dup2(saved, 2);
  close(saved);
  quiet(0);
  if (chdir(cwd)) return -1;
  return ok ? 0 : -2;
}

/* the reference's ASCII dump() (dump.c:1710-2047) of the current state, into
   the file at path; the header's counters are the globals as they stand */
int ref_dump(const char *path)
{
  FILE *fp = fopen(path, "w");
  if (!fp) return -1;
  quiet(1);
  dump(fp);
  quiet(0);
  fclose(fp);
  return 0;
}

/* CPU throughput of the reference's step_ch(): warm-up steps, then timed steps */
double ref_time_steps(int warm, int steps)
{
  quiet(1);
  for (int s = 0; s < warm; s++) { step_ch(); nstep++; }
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int s = 0; s < steps; s++) { step_ch(); nstep++; }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  quiet(0);
  return (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
}

#if TRACERSDUMP
} /* extern "C" */
/* the tracer list of tracers.c (tracers.c:19-24) */
struct of_tracer {
  int h, i, j;
  double X[NDIM];
};
extern std::vector<of_tracer> vtr;
extern "C" {
long ref_tracers_count(void) { return (long)vtr.size(); }
/* ids[n][3] = (i, j, h) of the zone each tracer started in, X[n][3] = X1, X2, X3 */
void ref_tracers_get(int *ids, double *X)
{
  for (size_t k = 0; k < vtr.size(); k++) {
    ids[3 * k] = vtr[k].i; ids[3 * k + 1] = vtr[k].j; ids[3 * k + 2] = vtr[k].h;
    X[3 * k] = vtr[k].X[1]; X[3 * k + 1] = vtr[k].X[2]; X[3 * k + 2] = vtr[k].X[3];
  }
}
/* replace the tracer list: ids[n][3] = (i, j, h) labels, X[n][3] = X1, X2, X3 */
void ref_tracers_set(const int *ids, const double *X, long n)
{
  vtr.clear();
  for (long k = 0; k < n; k++) {
    of_tracer t;
    t.i = ids[3 * k]; t.j = ids[3 * k + 1]; t.h = ids[3 * k + 2];
    t.X[0] = 0.;
    t.X[1] = X[3 * k]; t.X[2] = X[3 * k + 1]; t.X[3] = X[3 * k + 2];
    vtr.push_back(t);
  }
}
#endif
} /* extern "C" */
