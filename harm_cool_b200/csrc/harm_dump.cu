// The reference's ASCII dump (dump() with HDFDUMP 0, dump.c:1710-2047) written
// from the device state: a header line, then one line per active zone in the
// reference's loop order (r outermost, then theta, then phi) with the zone's
// coordinates, primitives, cooling values (zeros without COOL_EOS), div B,
// u^mu, u_mu, b^mu, b_mu, the wave speeds in r and theta, sqrt(-g), |v|, and the
// sound speed, radial velocity and Mach number of a gamma = 4/3 gas.  The device
// computes every field but the coordinates, slab by slab of r; the host adds the
// coordinates (as coord() and bl_coord() compute them) and prints with the
// reference's formats.  Built with -fmad=false: the fields are the reference's
// values bit for bit, so the text is too.
//
// With COOL_EOS, each zone's CoolVal_rho0_u_CoolEOS call and its two wave-speed
// calls move the zone's temperature guess, as in the reference.
#include <cstdio>
#include <vector>

#include "harm_common.cuh"
#include "harm_cool.cuh"

namespace harm {
namespace {

constexpr int DUMP_NF = 42;  // device fields per zone

__device__ __forceinline__ double Pz(const Grid &G, const double *P, int k, int h, int i, int j)
{
  return __ldg(P + k * G.nc + cidx(G, h, i, j));
}

// div B as dump() forms it (dump.c:1886-1942): in 2D only where
// 0 < i < N1 and 0 < j < N2 (array indices), in 3D everywhere, with the
// reference's term order (and its gdet[i][j] on the fifth B3 term)
__device__ double dump_divb(const Grid &G, const double *P, const double *gd, int h, int i, int j)
{
  const long s = G.sn2, c = (long)i * s + j;
  const double g00 = __ldg(gd + c), g01 = __ldg(gd + c - 1), g10 = __ldg(gd + c - s), g11 = __ldg(gd + c - s - 1);
  if (G.n3 == 1) {
    if (!(i > 0 && j > 0 && i < G.n1 && j < G.n2)) return 0.;
    return fabs(0.5 * (Pz(G, P, B1, h, i, j) * g00 + Pz(G, P, B1, h, i, j - 1) * g01
                       - Pz(G, P, B1, h, i - 1, j) * g10 - Pz(G, P, B1, h, i - 1, j - 1) * g11) / G.dx1
                + 0.5 * (Pz(G, P, B2, h, i, j) * g00 + Pz(G, P, B2, h, i - 1, j) * g10
                         - Pz(G, P, B2, h, i, j - 1) * g01 - Pz(G, P, B2, h, i - 1, j - 1) * g11) / G.dx2);
  }
  const int m = hwrap(G, h - 1);
  return fabs(0.25 * (+Pz(G, P, B1, m, i, j) * g00 + Pz(G, P, B1, m, i, j - 1) * g01
                      - Pz(G, P, B1, m, i - 1, j) * g10 - Pz(G, P, B1, m, i - 1, j - 1) * g11
                      + Pz(G, P, B1, h, i, j) * g00 + Pz(G, P, B1, h, i, j - 1) * g01
                      - Pz(G, P, B1, h, i - 1, j) * g10 - Pz(G, P, B1, h, i - 1, j - 1) * g11) / G.dx1
              + 0.25 * (+Pz(G, P, B2, m, i, j) * g00 + Pz(G, P, B2, m, i - 1, j) * g10
                        - Pz(G, P, B2, m, i, j - 1) * g01 - Pz(G, P, B2, m, i - 1, j - 1) * g11
                        + Pz(G, P, B2, h, i, j) * g00 + Pz(G, P, B2, h, i - 1, j) * g10
                        - Pz(G, P, B2, h, i, j - 1) * g01 - Pz(G, P, B2, h, i - 1, j - 1) * g11) / G.dx2
              + 0.25 * (+Pz(G, P, B3, h, i, j) * g00 + Pz(G, P, B3, h, i - 1, j) * g10
                        - Pz(G, P, B3, m, i, j) * g00 - Pz(G, P, B3, m, i - 1, j) * g10
                        + Pz(G, P, B3, h, i, j - 1) * g00 + Pz(G, P, B3, h, i - 1, j - 1) * g11
                        - Pz(G, P, B3, m, i, j - 1) * g01 - Pz(G, P, B3, m, i - 1, j - 1) * g11) / G.dx3);
}

// the device fields of one zone: prims, cooling values, div B, the state, wave
// speeds, sqrt(-g), |v| and the gamma = 4/3 sound speed, radial velocity, Mach
template <bool COOL>
__device__ void dump_zone(const Grid &G, const double *__restrict__ P, const double *__restrict__ geo, const EosDev &E,
                          double *lastT, const double *__restrict__ rcent, int h, int i, int j, double *o)
{
  const long c = cidx(G, h, i, j);
  const long gi = (long)i * G.sn2 + j;
  const double *gC = geo_at(geo, G, L_CENT);
  double pr[8];
#pragma unroll
  for (int k = 0; k < 8; k++) o[k] = pr[k] = __ldg(P + k * G.nc + c);
  EosCursor cur = eos_cursor(i, 0.0);
  if (COOL) {
    double T = lastT[c];
    if (T == 0.0 && j > G.jstart) T = lastT[c - 1];
    cur.T = T;
    double cv[NCOOLVAL];
    eos_coolval(E, cur, pr[RHO], pr[UU], __ldg(rcent + gi), cv);
    o[8] = cv[COOL_LAMBDA_SIM];
    o[9] = cv[COOL_P];
    o[10] = cv[COOL_T];
    o[11] = cv[COOL_Hd];
    o[12] = cv[COOL_Qnu];
    o[13] = cv[COOL_Tau];
    o[14] = cv[COOL_Yee];
  } else {
#pragma unroll
    for (int k = 8; k < 15; k++) o[k] = 0.0;
  }
  o[15] = dump_divb(G, P, gC + 17 * G.ng, h, i, j);
  Geo q;
  load_geo(gC, G.ng, gi, q);
  State s;
  int fail = 0;
  get_state(pr, q, s, &fail);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    o[16 + k] = s.ucon[k];
    o[20 + k] = s.ucov[k];
    o[24 + k] = s.bcon[k];
    o[28 + k] = s.bcov[k];
  }
  double vmax, vmin;
  if (COOL) vchar_cool(E, cur, pr, s, q, 1, vmax, vmin, &fail);
  else vchar(G.gam, pr, s, q, 1, vmax, vmin, &fail);
  o[32] = vmin;
  o[33] = vmax;
  if (COOL) vchar_cool(E, cur, pr, s, q, 2, vmax, vmin, &fail);
  else vchar(G.gam, pr, s, q, 2, vmax, vmin, &fail);
  o[34] = vmin;
  o[35] = vmax;
  if (COOL) lastT[c] = cur.T;
  o[36] = q.g;
  {
    const double u1 = s.ucon[1], u2 = s.ucon[2], u3 = s.ucon[3];
    double vsq = 0.;
    vsq += q.v11 * u1 * u1;
    vsq += q.v13 * u1 * u3;
    vsq += q.v22 * u2 * u2;
    vsq += q.v13 * u3 * u1;
    vsq += q.v33 * u3 * u3;
    const double gsqtmp = 1. + vsq;
    vsq /= gsqtmp;
    o[37] = sqrt(vsq);
  }
  const double PS_pressure = pr[UU] * (G.gam - 1.0);
  const double PS_cs = sqrt(4.0 / 3.0 * PS_pressure / (pr[RHO] + 4.0 * PS_pressure));
  const double uur = sqrt(q.v11) * s.ucon[1] / s.ucon[0];
  o[38] = PS_pressure;
  o[39] = PS_cs;
  o[40] = uur;
  o[41] = -uur / PS_cs;
}

// the zones of r rows [i0, i0 + ni); record ((i - i0) * N2 + (j - jstart)) * N3 + h.
// ROWS: one thread per (r, phi) walking theta in order (zones without a guess
// take their theta neighbour's, as the reference's loop gives them)
template <bool COOL, bool ROWS>
__global__ void __launch_bounds__(128) k_dump(Grid G, const double *__restrict__ P, const double *__restrict__ geo,
                                              EosDev E, double *lastT, const double *__restrict__ rcent, int i0,
                                              int ni, double *out)
{
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (ROWS) {
    if (t >= (long)ni * G.n3) return;
    const int i = i0 + (int)(t / G.n3), h = (int)(t % G.n3);
    for (int j = G.jstart; j <= G.jstop; j++)
      dump_zone<COOL>(G, P, geo, E, lastT, rcent, h, i, j,
                      out + ((((long)(i - i0) * G.n2 + (j - G.jstart)) * G.n3 + h) * DUMP_NF));
  } else {
    if (t >= (long)ni * G.n2 * G.n3) return;
    const int h = (int)(t % G.n3), j = G.jstart + (int)((t / G.n3) % G.n2), i = i0 + (int)(t / ((long)G.n3 * G.n2));
    dump_zone<COOL>(G, P, geo, E, lastT, rcent, h, i, j, out + t * DUMP_NF);
  }
}

const char *const FD = "%32.22e";
const char *const FI = "%10d";

}  // namespace
}  // namespace harm

using namespace harm;

extern "C" int harm_dump_write(harm_ctx *h, const harm_restart_header *hdr, const harm_grid_spec *g, const char *path)
{
  if (!h || !hdr || !g || !path) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  const Grid &G = x->G;
  const harm_params &pr = x->prm;
  if (x->cool && !x->eos.hdfac) return fail_with(HARM_E_ARG, "COOL_EOS dumps need each table's HdFac");
  double t = 0., dt = 0.;
  int rc = harm_get_time(h, &t, &dt);
  if (rc) return rc;
  FILE *f = fopen(path, "w");
  if (!f) return fail_with(HARM_E_ARG, std::string("cannot open ") + path);
  struct Closer {
    FILE *f;
    ~Closer() { fclose(f); }
  } closer{f};
  const bool three = G.n3 > 1;
  // header (dump.c:1743-1789)
  fprintf(f, FD, t);
  fprintf(f, FI, G.n1);
  fprintf(f, FI, three ? G.n3 : G.n2);
  fprintf(f, FD, pr.startx[1]);
  fprintf(f, FD, three ? pr.startx[3] : pr.startx[2]);
  fprintf(f, FD, pr.dx[1]);
  fprintf(f, FD, three ? pr.dx[3] : pr.dx[2]);
  fprintf(f, FD, hdr->tf);
  fprintf(f, FI, hdr->nstep);
  fprintf(f, FD, hdr->a);
  fprintf(f, FD, hdr->gam);
  fprintf(f, FD, hdr->cour);
  fprintf(f, FD, hdr->DTd);
  fprintf(f, FD, hdr->DTl);
  fprintf(f, FD, hdr->DTi);
  fprintf(f, FI, hdr->DTr);
  fprintf(f, FI, hdr->dump_cnt);
  fprintf(f, FI, hdr->image_cnt);
  fprintf(f, FI, hdr->rdump_cnt);
  fprintf(f, FD, dt);
  fprintf(f, FI, hdr->lim);
  fprintf(f, FI, hdr->failed);
  fprintf(f, FD, hdr->Rin);
  fprintf(f, FD, hdr->Rout);
  fprintf(f, FD, hdr->hslope);
  fprintf(f, FD, hdr->R0);
  fprintf(f, "\n");
  // the zones, slab by slab of r rows (at most about 256 MB of fields at a time)
  const long per_row = (long)G.n2 * G.n3;
  int rows = (int)((256l << 20) / (per_row * DUMP_NF * (long)sizeof(double)));
  rows = rows < 1 ? 1 : (rows > G.n1 ? G.n1 : rows);
  struct Buf {
    double *d = nullptr;
    ~Buf() { cudaFree(d); }
  } B;
  CK(cudaMalloc(&B.d, (size_t)rows * per_row * DUMP_NF * sizeof(double)));
  std::vector<double> hb((size_t)rows * per_row * DUMP_NF);
  const bool seed = x->cool && x->cool_seed;
  for (int i0 = G.istart; i0 <= G.istop; i0 += rows) {
    const int ni = std::min(rows, G.istop + 1 - i0);
    const long nthr = seed ? (long)ni * G.n3 : (long)ni * per_row;
    const unsigned nb = (unsigned)((nthr + 127) / 128);
    if (x->cool) {
      if (seed) k_dump<true, true><<<nb, 128, 0, x->stream>>>(G, x->p, x->geo, x->eos, x->lastT, x->coolgeo, i0, ni, B.d);
      else k_dump<true, false><<<nb, 128, 0, x->stream>>>(G, x->p, x->geo, x->eos, x->lastT, x->coolgeo, i0, ni, B.d);
    } else {
      k_dump<false, false><<<nb, 128, 0, x->stream>>>(G, x->p, x->geo, x->eos, x->lastT, x->coolgeo, i0, ni, B.d);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hb.data(), B.d, (size_t)ni * per_row * DUMP_NF * sizeof(double), cudaMemcpyDeviceToHost,
                       x->stream));
    CK(cudaStreamSynchronize(x->stream));
    for (int i = i0; i < i0 + ni; i++)
      for (int j = G.jstart; j <= G.jstop; j++)
        for (int hh = 0; hh < G.n3; hh++) {
          const double *o = hb.data() + (((size_t)(i - i0) * G.n2 + (j - G.jstart)) * G.n3 + hh) * DUMP_NF;
          // coord() at CENT and bl_coord() (coord.c:61-125): r and theta from X1, X2
          const double X1 = pr.startx[1] + ((i - 2) + 0.5) * pr.dx[1];
          const double X2 = pr.startx[2] + ((j - 2) + 0.5) * pr.dx[2];
          const double X3 = three ? pr.startx[3] + (hh + 0.5) * pr.dx[3] : pr.startx[3] + hh * pr.dx[3];
          const double r = exp(X1) + g->R0;
          fprintf(f, FD, X1);
          if (three) {
            fprintf(f, FD, X3);
            fprintf(f, FD, r);
            fprintf(f, FD, X3);
          } else {
            double th = M_PI_2 * (1. + X2) + ((1. - g->hslope) / 2.) * sin(M_PI * (1. + X2));
            if (fabs(th) < 1.E-20) th = th >= 0 ? 1.E-20 : -1.E-20;
            if (fabs(M_PI - th) < 1.E-20) th = th >= M_PI ? M_PI + 1.E-20 : M_PI - 1.E-20;
            fprintf(f, FD, X2);
            fprintf(f, FD, r);
            fprintf(f, FD, th);
          }
          const int nf = hdr->failed ? 16 : DUMP_NF;
          for (int k = 0; k < nf; k++) fprintf(f, FD, o[k]);
          fprintf(f, "\n");
        }
  }
  fflush(f);
  if (ferror(f)) return fail_with(HARM_E_ARG, std::string("write error on ") + path);
  return HARM_OK;
}
