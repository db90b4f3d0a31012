/*
 * CPU oracle for the HARM-COOL step_ch() path.  TEST INFRASTRUCTURE ONLY:
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it as
 * the checker; nothing in the product links or calls it.
 *
 * A plain-C restatement of the reference's gamma-law predictor/corrector
 * zone update (step_ch.c:90-318 and the routines it calls).  Each function
 * in harm_oracle.c cites the reference file:line it follows.  Floating point
 * follows the reference's expression order so that, built with
 * -ffp-contract=off on SSE2, it reproduces the reference bit for bit; this is
 * pinned by tests against the reference compiled from its own sources
 * (oracle/_ref) and against fixtures generated from it (tests/golden).
 *
 * State layout is the reference's: prims p[SN3][SN1][SN2][NPR] with
 * SN1=N1+4, SN2=N2+4, SN3=N3+2 (or 1 when N3==1); geometry is 2D:
 * gcov/gcon[SN1][SN2][NPG][4][4], gdet[SN1][SN2][NPG],
 * conn[SN1][SN2][4][4][4], coords[SN1][SN2][4] (decs.h:288-303, main.c:384-388).
 */
#ifndef HARM_ORACLE_H
#define HARM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* run parameters; same field order as harm_params in include/harm_b200.h */
typedef struct {
  int n1, n2, n3;      /* active zones in r, theta, phi */
  int lim;             /* slope limiter: 0 MC, 1 van Leer, 2 minmod (decs.h:214-216) */
  double a;            /* black-hole spin */
  double gam;          /* adiabatic index */
  double cour;         /* Courant number */
  double defcon;       /* Courant safety factor in advance() (main.c:204) */
  double tf;           /* end time */
  double dx[4];        /* coordinate spacing, dx[1..3] used */
  double startx[4];    /* coordinate origin, startx[1..3] used */
} ora_params;

typedef struct {
  double mdot, edot, ldot;               /* diag_flux (diag.c:437-465) */
  double mdot_in, mdot_out, mass_curr;   /* diag_mass (diag.c:477-580) */
  double mass_in, mass_out;
  double ndt;                            /* Courant dt proposed by the corrector */
  int fail_code, fail_h, fail_i, fail_j; /* first fail() the reference would take */
} ora_diag;

typedef struct ora_state ora_state;

ora_state *ora_create(const ora_params *prm, const double *gcov, const double *gcon,
                      const double *gdet, const double *conn, const double *coords,
                      const double *katm);
void ora_destroy(ora_state *s);

/* the state's own arrays (reference layout); the caller may read and write them */
double *ora_p(ora_state *s);
double *ora_ph(ora_state *s);
signed char *ora_pflag(ora_state *s);
double *ora_flux(ora_state *s, int dir);

void ora_set_time(ora_state *s, double t, double dt);
void ora_get_time(const ora_state *s, double *t, double *dt);
void ora_set_mass(ora_state *s, double mass_in, double mass_out);
void ora_get_diag(const ora_state *s, ora_diag *d);

/* one full step (step_ch.c:90-140); returns 0, or 11 where the reference exits(11) */
int ora_step_ch(ora_state *s);

/* the reference's per-array entry points, applied to an array of the state's shape */
void ora_fixup(ora_state *s, double *pv);          /* fixup.c:51-60 */
void ora_bound_prim(ora_state *s, double *pv);     /* bounds.c:54-331 */
void ora_fixup_utoprim(ora_state *s, double *pv);  /* fixup.c:432-538 */
double ora_advance(ora_state *s, double *pi, double *pb, double Dt, double *pf, int fullstep);

/* single-zone inversions on explicit geometry (utoprim_2d.c:126, utoprim_1dvsq2fix1.c:143,
   utoprim_1dfix1.c:137); gam is the adiabatic index */
int ora_utoprim_2d(double gam, const double U[8], const double *gcov, const double *gcon,
                   double gdet, double *prim);
int ora_utoprim_1dvsq2fix1(double gam, const double U[8], const double *gcov,
                           const double *gcon, double gdet, double *prim, double K);
int ora_utoprim_1dfix1(double gam, const double U[8], const double *gcov,
                       const double *gcon, double gdet, double *prim, double K);

/* face flux of one direction for given left/right states on explicit geometry:
   F, U and wave speeds as fluxcalc computes them (step_ch.c:429-473) */
void ora_face_flux(double gam, int dir, const double pl[8], const double pr[8],
                   const double *gcov, const double *gcon, double gdet,
                   double F[8], double *ctop);

/* tracer particles (tracers.c): ids[n][3] labels (i, j, h), X[n][3] code
   coordinates X1..X3, status[n] 0 active, 1 fell in, 2 left inside the theta
   window, 3 left in the jet, -1 dropped by the search.  Once tracers exist,
   ora_step_ch() moves them after diag_mass (step_ch.c:121-123).  bl_coord()
   needs the grid's R0 and hslope. */
void ora_tracers_geometry(ora_state *s, double R0, double hslope);
long ora_tracers_init(ora_state *s);
void ora_tracers_put(ora_state *s, const int *ids, const double *X, long n);
long ora_tracers_count(const ora_state *s);
void ora_tracers_get(const ora_state *s, int *ids, double *X, signed char *status);
/* diag()'s integrals (diag.c:113-230) over the active zones of the state's p:
   out[0] = sum U[RHO] dV, out[1] = sum U[U3] dV, out[2] = sum U[UU] dV,
   out[3] = max |div B| (flux-CT definition), imax = its zone (r, theta, phi from 0) */
void ora_diag_integrals(ora_state *s, double *out, int *imax);

/* run-time COOL_EOS (cooleos_oracle.c): tables of the values e, p, Qnu, tau, Yee
   (cooleos.c:32-37) at the nodes of a rho axis xa[nx] and a T axis ya[ny], one table
   per radial index, val[ntab][nx][ny][nd] (the reference's MValues order), with the
   unit and range constants of cooleos.c:83-135, 840-940 */
enum { ORA_EOS_E = 0, ORA_EOS_P = 1 };
typedef struct {
  int nx, ny, nd, ntab;
  const double *xa, *ya, *val;
  double rho_unit, u_unit, p_unit, kbol, mav, cl, rho_min, rho_max, t_min, t_max, hh, gam;
} OraEos;
double ora_eos_pressure(const OraEos *E, int tab, double rho0, double u, double *lastT);
double ora_eos_dpdu(const OraEos *E, int tab, double rho0, double u, double *lastT);
double ora_eos_dpdrho(const OraEos *E, int tab, double rho0, double u, double *lastT);
void ora_eos_batch(const OraEos *E, int what, long n, const int *tab, const double *rho0, const double *u,
                   double *lastT, double *out);
int ora_eos_value(const OraEos *E, int tab, int d, double rho, double T, double *val, double *der);
#ifdef __cplusplus
}
#endif
#endif
