/*
 * harm_b200.h -- C ABI of the B200 implementation of HARM-COOL's per-zone
 * GRMHD update (the step_ch() path).
 *
 * Plain C types only.  Arrays use the reference's own layouts:
 *   primitives   p[SN3][SN1][SN2][8]       (decs.h:190-197, main.c:318-342)
 *   pflag        signed char [SN3][SN1][SN2]
 *   gcov, gcon   [SN1][SN2][5][4][4]        (main.c:384-386; locations FACE1,
 *   gdet         [SN1][SN2][5]               FACE2, CORN, CENT, FACE3)
 *   conn         [SN1][SN2][4][4][4]         (main.c:384)
 *   coords       [SN1][SN2][4]               (main.c:388)
 *   katm         [SN1]                       (decs.h:306)
 * with SN1 = N1+4, SN2 = N2+4, SN3 = N3+2 (N3 > 1) or 1 (N3 == 1).
 *
 * Every function returns 0 on success or a negative HARM_E* code; the text
 * of the last error on the calling thread is available from
 * harm_last_error().  Physical failures that the reference handles by
 * calling fail() and exiting (diag.c:381-397) are reported instead through
 * harm_diag.fail_code after the step that met them, and the state is left as
 * the reference leaves it just before the exit.
 */
#ifndef HARM_B200_H
#define HARM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define HARM_NPR 8
#define HARM_NPG 5

enum {
  HARM_OK = 0,
  HARM_E_ARG = -1,      /* bad argument or grid size */
  HARM_E_CUDA = -2,     /* a CUDA runtime call failed */
  HARM_E_NODEV = -3,    /* no usable sm_100 device */
  HARM_E_DT = -11,      /* dt < 1e-9: where the reference calls exit(11) (step_ch.c:126-129) */
  HARM_E_ADJOINT = -13  /* the adjoint cannot follow the steps (a step failed; see harm_last_error) */
};

/* Arithmetic of the step (harm_set_precision). */
enum {
  HARM_FP64 = 0,   /* everything in FP64, bit-compatible with the reference (default) */
  HARM_MIXED = 1   /* FP32 reconstruction, wave speeds and face fluxes; FP64 geometry
                      source, accumulation, inversion and floors */
};

/* Run parameters (decs.h:263-283, init.c:104-125). */
typedef struct harm_params {
  int n1, n2, n3;   /* active zones in r, theta, phi; n3 == 1 or even n3 >= 4 */
  int lim;          /* slope limiter: 0 MC, 1 van Leer, 2 minmod */
  double a;         /* black-hole spin */
  double gam;       /* adiabatic index */
  double cour;      /* Courant number */
  double defcon;    /* Courant safety factor (main.c:204) */
  double tf;        /* end time: dt is clipped so that t never passes tf */
  double dx[4];     /* coordinate spacing; dx[1..3] used */
  double startx[4]; /* coordinate origin; startx[1..3] used */
} harm_params;

/* Modified Kerr-Schild grid (coord.c:61-81, 202-262). */
typedef struct harm_grid_spec {
  int n1, n2, n3;
  double a;       /* spin */
  double Rin;     /* inner radius of the grid */
  double Rout;    /* outer radius of the grid */
  double R0;      /* radial offset of the exponential map */
  double hslope;  /* theta concentration */
} harm_grid_spec;

/* Fishbone-Moncrief torus (init.c:70-472). */
typedef struct harm_torus_spec {
  double rin;    /* torus inner edge */
  double rmax;   /* radius of pressure maximum */
  double kappa;  /* polytropic constant */
  double beta;   /* target gas-to-magnetic pressure ratio */
} harm_torus_spec;

/* Per-step diagnostics (diag.c:437-580) and the first recorded failure. */
typedef struct harm_diag {
  double mdot, edot, ldot;
  double mdot_in, mdot_out, mass_curr;
  double mass_in, mass_out;
  double ndt;       /* Courant time step proposed by the corrector */
  int fail_code;    /* 0, or the fail() code the reference would exit with */
  int fail_h, fail_i, fail_j;
} harm_diag;

const char *harm_last_error(void);

/* ---- host-side grid set-up (CPU only; no device needed) ---- */

/* set_points() (coord.c:202-262): dx[] and startx[] of the grid. */
int harm_set_points(const harm_grid_spec *g, double dx[4], double startx[4]);

/* set_grid() (main.c:413-520): metric, inverse metric, sqrt(-g), connection
   and Boyer-Lindquist coordinates on the whole 2D (r, theta) grid. */
int harm_set_grid(const harm_grid_spec *g, const double dx[4], const double startx[4],
                  double *gcov, double *gcon, double *gdet, double *conn, double *coords);

/* set_Katm() (fixup.c:555-585): entropy constant of the floor state per radius. */
int harm_set_katm(const harm_grid_spec *g, double gam, const double *coords, double *katm);

/* ---- device context: state resident on one GPU ---- */

typedef struct harm_ctx harm_ctx;

/* Allocate the device state for one grid and upload its geometry.
   Replaces the reference's set_arrays()/set_grid() storage (main.c:288-520). */
int harm_create(const harm_params *prm, const double *gcov, const double *gcon,
                const double *gdet, const double *conn, const double *coords,
                const double *katm, int device, harm_ctx **out);
void harm_destroy(harm_ctx *ctx);

/* Fishbone-Moncrief torus with a normalised poloidal loop, as init() builds it
   (init.c:70-472), left resident on the device; sets t = 0, dt = 1e-5 and the
   mass counters as main() does after init (main.c:166-182). */
int harm_init_torus(harm_ctx *ctx, const harm_grid_spec *g, const harm_torus_spec *torus);

/* Copy primitives (and optionally pflag) between host and device, reference layout. */
int harm_put_prims(harm_ctx *ctx, const double *p, const signed char *pflag);
int harm_get_prims(harm_ctx *ctx, double *p, signed char *pflag);

int harm_set_time(harm_ctx *ctx, double t, double dt);
int harm_get_time(harm_ctx *ctx, double *t, double *dt);
int harm_set_mass(harm_ctx *ctx, double mass_in, double mass_out);
int harm_get_diag(harm_ctx *ctx, harm_diag *d);

/* Select HARM_FP64 or HARM_MIXED for the following steps (no reference
   counterpart: the reference is FP64 throughout). */
int harm_set_precision(harm_ctx *ctx, int mode);

/* step_ch() (step_ch.c:90-140): predictor to dt/2, floors, boundaries,
   failure repair, corrector to dt, the same again, mass diagnostics and the
   next dt.  Asynchronous on the context's stream; returns after launch. */
int harm_step_ch(harm_ctx *ctx);

/* n steps captured once into a CUDA graph and replayed; synchronises at the end
   and returns HARM_E_DT if any step met dt < 1e-9. */
int harm_run(harm_ctx *ctx, int nsteps);

/* step_ch() on host primitives: upload p, one step, download p.  The call a
   host that owns its primitive array (the reference's _p) makes per step. */
int harm_step_ch_host(harm_ctx *ctx, double *p);

/* ---- device-timed variants (CUDA events on the context's stream) ---- */

/* harm_run() with the elapsed device time of the n graph launches in *ms. */
int harm_run_timed(harm_ctx *ctx, int nsteps, double *ms);

/* nsteps steps with the state in the host array p: each step uploads p,
   steps and downloads into p, as nsteps calls of harm_step_ch_host() do.  The
   upload of each step's input is cut into chunks that follow the previous
   step's download chunk by chunk, so that with p in pinned memory the link
   carries both directions at once.  Returns when p holds the final state. */
int harm_run_host(harm_ctx *ctx, double *p, int nsteps);

/* harm_run_host() with the elapsed device time in *ms. */
int harm_step_ch_host_timed(harm_ctx *ctx, double *p, int nsteps, double *ms);

/* Runs reps ordinary steps launched kernel by kernel with a CUDA event after
   each, and returns the average device time per launch of each kind, into
   ms[HARM_NKERNELS] in this order: flux (all three directions), update
   (flux-CT + source + inversion + floors), bound_prim, fixup_utoprim (flag
   flip + repair), diagnostics (flux and mass sums, next dt, per step).  The
   state advances by reps steps. */
#define HARM_NKERNELS 5
int harm_time_kernels(harm_ctx *ctx, int reps, double *ms);

/* Block until the context's stream is idle; returns any pending device error. */
int harm_sync(harm_ctx *ctx);

/* ---- restart files (restart.c, the reference's ASCII format) ---- */

/* The restart header in file order (restart.c:103-136).  On write, t, dt,
   mass_in and mass_out come from the context and the other fields from the
   caller (they are the host driver's: output cadence, counters, the grid's
   parameters); on read, every field is returned. */
typedef struct harm_restart_header {
  int n1, n2, n3;
  double t, tf;
  int nstep;
  double a, gam, cour, DTd, DTl, DTi;
  int DTr, dump_cnt, image_cnt, rdump_cnt;
  double dt;
  int lim, failed;
  double Rin, Rout, hslope, R0, mass_start, mass_in, mass_out, tdump, timage, tlog, defcon;
  int nfailed;
  double Rbr, cyl_R0, cyl_Th0;
  int ener_size;  /* the ener.out size stored after the body (restart.c:150-158) */
} harm_restart_header;

/* restart_write() (restart.c:73-186): the context's primitives (phi ghost planes as
   periodic copies), and its active tracers when it has any (tracers.c:565-603;
   per-tracer file sizes written as 0).  g is needed only when there are tracers. */
int harm_restart_write(harm_ctx *ctx, const harm_restart_header *hdr, const harm_grid_spec *g,
                       const char *path);
/* restart_init()/restart_read() (restart.c:197-383): primitives, t, dt, mass
   counters and tracers into the context, pflag cleared, then bound_prim as the
   reference does after reading.  The file's grid, spin and adiabatic index must
   match the context's. */
int harm_restart_read(harm_ctx *ctx, const char *path, const harm_grid_spec *g, harm_restart_header *hdr);

/* dump() (dump.c:1710-2047, the ASCII dump of HDFDUMP 0) of the device state
   into the file at path: the header line (from hdr's fields and the context's
   t, dt and grid), then one line per active zone in the reference's order with
   its coordinates, primitives, cooling values (zeros without COOL_EOS), div B,
   u^mu, u_mu, b^mu, b_mu, wave speeds, sqrt(-g), |v|, sound speed, radial
   velocity and Mach number; hdr->failed != 0 stops each line after div B, as
   the reference does.  g gives R0 and hslope.  With COOL_EOS the zones'
   temperature guesses move as the reference's dump() moves them. */
int harm_dump_write(harm_ctx *ctx, const harm_restart_header *hdr, const harm_grid_spec *g, const char *path);

/* Discrete adjoint of nsteps steps of step_ch() (2D gamma-law FP64 step; no
   reference counterpart).  Runs the steps from the context's state (the
   context ends where they end, as after harm_run), sets *J to the mass that
   crossed the inner radial boundary meanwhile -- the change of mass_in
   (diag.c:578, mass_in += mdot_in*Dt) -- and grad to dJ/dp of the state at the
   call, in harm_get_prims' layout (every cell and primitive, ghosts included).
   Reverse sweep: states kept every checkpoint_every steps, each segment
   recomputed by the step's own kernels, then transposed step by step (limiter
   branches, floors and wave-speed choices frozen at the forward's; the
   inversion differentiated through its converged Newton system).  ms, if not
   NULL, gets the device time of the forward pass (ms[0]) and of the reverse
   sweep with its recomputation (ms[1]).  The call allocates device memory for
   the checkpoints and for two segments' records (about 20 MB per step of a
   segment at 192x192), works on the context's stream and on two streams of
   its own, and returns when the results are in J and grad.  Refused for 3D,
   COOL_EOS, the mixed step and attached tracers; HARM_E_ADJOINT if a step
   fails. */
int harm_adjoint_mass_in(harm_ctx *ctx, int nsteps, int checkpoint_every, double *J, double *grad, double *ms);

/* ---- diagnostics ---- */

/* diag()'s integrals (diag.c:113-230) over the active zones of the current state. */
typedef struct harm_integrals {
  double mass;      /* sum of U[RHO] dV (rmed) */
  double ang_mom;   /* sum of U[U3] dV (pp) */
  double energy;    /* sum of U[UU] dV (e) */
  double divbmax;   /* largest |div B| in the flux-CT form */
  int imax[3];      /* its zone: r, theta, phi indices from 0 (the first in loop order) */
  /* with COOL_EOS (diag.c:137-251, ener.out columns 10-13): the neutrino
     luminosities from CoolVal_rho0_u_CoolEOS; 0 otherwise */
  double lnu;       /* sum of Lambda_sim sqrt(-g) */
  double lnu_rho;   /* sum of Lambda_sim sqrt(-g) rho / sum of sqrt(-g) rho */
  double lnu_rho_2; /* sum of sqrt(-g) rho */
  double lnu2;      /* per (phi, r) row, Qnu sqrt(-g) at the first theta from the equator
                       where |r tan theta| reaches the row's mean scale height */
} harm_integrals;
/* With COOL_EOS tables attached, this also moves each zone's temperature guess
   as diag() does (InitCache_CoolEOS, primtoU, CoolVal_rho0_u_CoolEOS per zone,
   diag.c:137-149); those guesses carry into the following steps. */
int harm_diag_integrals(harm_ctx *ctx, harm_integrals *out);

/* ---- tracer particles (tracers.c) ----
   Tracers live on the device with the state.  Once a context has tracers,
   every step moves them after the mass diagnostics, as step_ch() calls
   update_tracers(dt) (step_ch.c:121-123).  ids[n][3] are labels (the zone i, j, h
   a tracer started in, as tracers.c names its files); X[n][3] are code
   coordinates X1, X2, X3; status[n] is 0 while active, 1 after falling in
   (r < inner tracer radius or theta outside [0, pi]), 2 after leaving through the
   outer tracer radius inside the theta window [0.02 pi, 0.98 pi], 3 after leaving
   in the jet, -1 when the zone search failed -- where the reference erases the
   tracer and moves its file to tracers/in, out or jet.  g gives R0 and hslope. */

/* init_tracers() (tracers.c:109-188): one tracer at the centre of every active zone
   whose zone holds rho > RHOMIN, in the reference's loop order; *count tracers. */
int harm_tracers_init(harm_ctx *ctx, const harm_grid_spec *g, long *count);
/* Replace the tracers with n given ones, all active. */
int harm_tracers_put(harm_ctx *ctx, const harm_grid_spec *g, const int *ids, const double *X, long n);
int harm_tracers_count(harm_ctx *ctx, long *n);
/* Read back all tracers, retired ones included (any pointer may be NULL). */
int harm_tracers_get(harm_ctx *ctx, int *ids, double *X, signed char *status);

/* ---- tile shapes (no reference counterpart: the reference runs on CPUs) ---- */

/* Threads per block of the face and zone kernels: bx along theta by by along r,
   bx * by = 128, bx a multiple of 8 (default 32 x 4). */
int harm_set_tile(harm_ctx *ctx, int bx, int by);
int harm_get_tile(harm_ctx *ctx, int *bx, int *by);

/* Autotuner: times `steps` steps with each candidate tile (32x4, 64x2, 16x8,
   128x1), every trial from the same saved state, restores that state, keeps
   the fastest tile and returns it in *bx, *by (either may be NULL). */
int harm_autotune_tile(harm_ctx *ctx, int steps, int *bx, int *by);

/* ---- ensembles: many independent grids on one GPU (no reference counterpart:
   the reference advances one compile-time grid per run) ---- */

typedef struct harm_ensemble harm_ensemble;

/* Bind n contexts created on the same device.  Each ensemble step advances every
   member by one step_ch() with its own dt, as harm_step_ch would; the members'
   step sequences are captured as parallel branches of one CUDA graph, launched
   once per ensemble step.  The members stay usable on their own; a member whose
   precision or tile changes is re-captured at the next run. */
int harm_ensemble_create(harm_ctx *const *members, int n, harm_ensemble **out);
void harm_ensemble_destroy(harm_ensemble *ens);

/* nsteps ensemble steps; synchronises and returns the first member error. */
int harm_ensemble_run(harm_ensemble *ens, int nsteps);

/* harm_ensemble_run() with the device time of the nsteps graph launches in *ms. */
int harm_ensemble_run_timed(harm_ensemble *ens, int nsteps, double *ms);

/* ---- the reference's per-array entry points, on host arrays of the context's shape ---- */

int harm_fixup(harm_ctx *ctx, double *pv);                        /* fixup.c:51-60, decs.h:567 */
int harm_bound_prim(harm_ctx *ctx, double *pv);                   /* bounds.c:54, decs.h:548 */
int harm_fixup_utoprim(harm_ctx *ctx, double *pv);                /* fixup.c:432, decs.h:569 */
/* fixup1zone() (fixup.c:142-383, decs.h:568) at n zones of the context's grid:
   hij[n][3] = (h, i, j) in the reference's indices, pv[n][8] the primitives
   (floored in place), flag[n] = -33 where the reference sets pflag to -33 (a
   gamma failure, left to fixup_utoprim), else 0.  Host arrays. */
int harm_fixup1zone(harm_ctx *ctx, long n, const int *hij, double *pv, signed char *flag);

/* Utoprim_2d() (utoprim_2d.c:126, decs.h:608) over n independent zones on the
   device: U[n][8], gcov[n][16], gcon[n][16], gdet[n], prim[n][8] (guess in,
   result out), ret[n] (the reference's return code).  Host arrays. */
int harm_utoprim_2d_batch(const double *U, const double *gcov, const double *gcon,
                          const double *gdet, double *prim, int *ret, long n, double gam);

/* The isentropic fall-back inversions over n independent zones: which = 1
   Utoprim_1dvsq2fix1() (utoprim_1dvsq2fix1.c:143, decs.h:609), which = 2
   Utoprim_1dfix1() (utoprim_1dfix1.c:137, decs.h:611), with K[n] the entropy
   constant of each zone (the reference passes Katm[i], step_ch.c:277-300);
   arrays as harm_utoprim_2d_batch.  Host arrays. */
int harm_utoprim_fix_batch(int which, const double *U, const double *gcov, const double *gcon,
                           const double *gdet, const double *K, double *prim, int *ret, long n, double gam);

/* x[k]^y[k] rounded to nearest as the fall-back inversions compute it on the
   device (double-double exp(y ln x)), in place of the host libm's pow()
   (utoprim_1dvsq2fix1.c:583-616, utoprim_1dfix1.c:864-880).  Host arrays.  A
   check of the device arithmetic with no counterpart of its own in the
   reference. */
int harm_pow_batch(int device, const double *x, const double *y, double *out, long n);

/* The same inversion as harm_utoprim_2d_batch, for callers that cannot
   allocate device memory: hosts whose GPU memory is already committed to a
   resident simulation state or handed to another allocator, and hosts that
   must not hit the device-wide synchronisation of cudaFree while other streams
   run.  The device copies live in one fixed array inside the library (about
   6.2 MiB per GPU, held until exit), so the call allocates nothing.  At most
   HARM_U2P_NOALLOC_MAX zones per call (HARM_E_ARG beyond).  The first call on
   a device looks up the array's device address and creates the non-blocking
   stream the calls run on; make it before any stream capture, and do not call
   again after resetting the device.  Calls share the array, so calls that
   overlap on the GPU race.
   Blocks until the results are in prim and ret.  No counterpart in the
   reference. */
#define HARM_U2P_NOALLOC_MAX 16384
int harm_utoprim_2d_batch_noalloc(const double *U, const double *gcov, const double *gcon,
                                  const double *gdet, double *prim, int *ret, long n, double gam);

/* Measured FP64 pipe rates of a device, the denominators of the step
   kernels' FP64 roofline: out[0] DFMA, out[1] DADD, out[2] DMUL instructions
   per second (thread instructions, all SMs), out[3] IEEE divisions and out[4]
   IEEE reciprocals per second.
   Runs about 50 ms of device work.  A measurement helper with no counterpart
   in the reference. */
int harm_fp64_peak(int device, double *out);

/* Self-check of the library's division by shared divisors on a device: n
   seeded samples (random, special and near-midpoint numerators) of div_rn
   against the IEEE division a / b.  counts[0]: samples that differ in any bit
   (0 expected); counts[1]: near-midpoint samples drawn.  A self-check with no
   counterpart in the reference. */
int harm_div_check(int device, long n, unsigned long long seed, unsigned long long *counts);
/* The fall-back inversions' power for the gamma = 4/3 exponents (a cube root
   refined in double-double) against the general double-double power, on n
   seeded random densities: counts[0] = results that differ in any bit,
   counts[1] = samples the cube-root path left to the general one. */
int harm_pow_check(int device, long n, unsigned long long seed, unsigned long long *counts);

/* ---- run-time COOL_EOS (cooleos.c, cache4d.c, akima.c, mnewt.h) ---- */

/* Tables of one EOS: per radial index t (the reference's cacheT[t],
   cooleos.c:70, 825-992) the values e, p, Qnu, tau, Yee (cooleos.c:32-37) at
   the nodes of a rho axis and a T axis, values[ntab][nx][ny][5] in the
   reference's node order (Cache4d MValues, cache4d.c:1043).  The tables are
   built on the host, as the reference builds them (calc_cache_val,
   cooleos.c:171-194); the units and ranges are cooleos.c's constants
   (cooleos.c:83-135, 840-940); gam is the gamma-law fall-back's index.
   hdfac[ntab] (each table's HdFac, cooleos.c:945-960) and l_unit serve the
   cooling values of harm_diag_integrals; hdfac may be NULL without them.
   Creating an EOS raises the device's per-thread stack limit to 4 KiB for the
   rest of the process (the EOS calls nest deeper than the default allows). */
typedef struct harm_eos harm_eos;
typedef struct harm_eos_desc {
  int nx, ny, ntab;
  double rho_unit, u_unit, p_unit;  /* RHO_UNIT, U_UNIT, P_UNIT */
  double kbol, mav, cl;             /* KBOL, MAV, CL of the initial T guess */
  double rho_min, rho_max;          /* rhoMin, rhoMax (g/cm^3) */
  double t_min, t_max;              /* TMin, TMax (K) */
  double hh;                        /* relative margin and difference step, 1e-6 */
  double gam;
  double l_unit;                    /* L_UNIT (cm) */
} harm_eos_desc;
int harm_eos_create(const harm_eos_desc *desc, const double *xaxis, const double *yaxis,
                    const double *values, const double *hdfac, harm_eos **out);
int harm_eos_destroy(harm_eos *eos);

/* Tables filled on demand, as the reference's cache fills its nodes as the
   run reads them: nodes not yet computed hold NaN.  After
   harm_eos_track_missing (call it before harm_set_eos: a context keeps the
   tables' description as it was then), every table read, FP64 or the mixed
   path's FP32, that meets a NaN node marks that node; harm_eos_missing copies the marks, [ntab][nx][ny] of
   0 or 1, to the host.  A run that marked nothing read only computed nodes. */
int harm_eos_track_missing(harm_eos *eos);
int harm_eos_missing(const harm_eos *eos, unsigned char *marks);

/* pressure_rho0_u_CoolEOS (cooleos.c:314-444), dpdu_calc_CoolEOS and
   dpdrho_calc_CoolEOS (cooleos.c:667-741) for n independent entries, each with
   its table index tab[k] and its temperature guess lastT[k] (the zone's *LastT
   after InitCache_CoolEOS, cooleos.c:770-807; 0 = none yet), updated in place.
   Host arrays; out[k] receives the value.  precision HARM_FP64: the reference's
   arithmetic, bit for bit; HARM_MIXED: the tables, the interpolation and the T
   solve in FP32 (same branches and fall-backs; HARM_E_ARG when the tables'
   values span more than FP32 holds). */
enum { HARM_EOS_PRESSURE = 0, HARM_EOS_DPDU = 1, HARM_EOS_DPDRHO = 2 };
int harm_eos_batch(harm_eos *eos, int what, int precision, long n, const int *tab,
                   const double *rho0, const double *u, double *lastT, double *out);

/* Utoprim_5d() (utoprim_5d.c:179-245, the COOL_EOS inversion) over n
   independent zones: U, gcov, gcon, gdet, prim as harm_utoprim_2d_batch, tab[n]
   the table (radial index) of each zone and lastT[n] its temperature guess,
   updated in place. */
int harm_utoprim_5d_batch(const harm_eos *eos, const double *U, const double *gcov,
                          const double *gcon, const double *gdet, const int *tab, double *lastT,
                          double *prim, int *ret, long n);

/* Step the context with COOL_EOS (decs.h:110): the run-time EOS pressure in
   the fluxes, wave speeds, source and primtoU, and Utoprim_5d as the
   inversion (step_ch.c:241-300, 437-441).  The tables must have ntab = N1+4,
   table t serving radial index t, and must outlive the attachment; NULL
   detaches them (back to the gamma-law step).  With HARM_MIXED the face
   fluxes' and wave speeds' EOS calls run in FP32 (see harm_eos_batch), the
   update stays FP64.  The context keeps
   the per-zone temperature guesses _aLastT (cooleos.c:69, 836), all unset at
   first, as the reference's calloc leaves them. */
int harm_set_eos(harm_ctx *ctx, const harm_eos *eos);
/* The guesses in the reference's layout double[SN3][SN1][SN2].  After
   harm_put_eos_guess the next step is a seeding step (see harm_run). */
int harm_get_eos_guess(harm_ctx *ctx, double *lastT);
int harm_put_eos_guess(harm_ctx *ctx, const double *lastT);

/* ---- The COOL_EOS table generator ----
   The equation of state and neutrino rates the tables hold: nucleons,
   electron-positron pairs, helium, radiation and trapped neutrinos in beta
   equilibrium (the reference's Fortran abundance(), abundance.f90:6-243, and
   its modules).  Units as abundance() returns them: e and p in erg cm^-3, Qnu
   in erg cm^-2 s^-1, tau dimensionless, n_e- and n_e+ in fm^-3. */

/* abundance() at n nodes on the host's cores (threads <= 0: all of them):
   out[7n] = e, p, Qnu, tau, n_e-, n_e+ and the proton fraction of the free
   nucleons per node.  The library's counterpart of the reference's
   abundance_(rho, T, HdFac, e, p, Qnu, tau, xnee, xnep) (cooleos.c:58-59),
   node by node. */
int harm_nu_abundance(const double *rho, const double *T, const double *hdfac, long n, int threads,
                      double *out);
/* The same on a GPU (host arrays in and out). */
int harm_nu_abundance_dev(int device, const double *rho, const double *T, const double *hdfac, long n,
                          double *out);
/* Every node of ntab tables on a GPU: values[ntab][nx][ny][5] = e, p, Qnu, tau,
   Yee at rho = xaxis[i] (g cm^-3), T = yaxis[j] (K) and the table's HdFac, as
   calc_cache_val packs them (cooleos.c:171-194), ready for harm_eos_create.
   slice: nodes per kernel launch (<= 0: one table).  *ms (may be NULL): the
   device time of the build. */
int harm_nu_tables(int device, const double *xaxis, int nx, const double *yaxis, int ny, const double *hdfac,
                   int ntab, long slice, double *values, float *ms);
/* The generator's quadrature rules, 100 doubles: 20-point Gauss-Legendre
   (10 positive abscissae, 10 weights), 40-point Gauss-Legendre (20, 20),
   20-point Gauss-Laguerre (20 abscissae, 20 weights times e^x). */
int harm_nu_rules(double *out);
/* Generalised Fermi-Dirac integrals F_k(eta, theta) = int_0^inf x^k
   sqrt(1 + theta x / 2) / (e^(x - eta) + 1) dx, k = 1/2, 3/2, 5/2, 7/2, as the
   generator computes them (dfermi, gauss_integral.f90:241-349), on the host:
   F[4n]. */
int harm_nu_fermi(const double *eta, const double *theta, long n, double *F);

#ifdef __cplusplus
}
#endif
#endif
