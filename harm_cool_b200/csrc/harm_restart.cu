// Restart files in the reference's own ASCII format (restart.c:73-383,
// tracers.c:565-652), written from and read into the device state, so that a
// run can stop on the GPU and resume on the CPU reference or the other way
// round.  Layout: the header (restart.c:103-136: ints as "%10d", doubles as
// "%32.22e", which prints 23 significant digits and so round-trips every
// double), a newline, every cell of p[SN3][SN1][SN2][8] one line per cell,
// the size of ener.out, when tracers exist the tracer section, and with COOL_EOS
// every zone's temperature guess.
//
// The reference's phi ghost planes hold whatever its last MPI exchange left
// there; they are never read before the next exchange refills them.  This
// writer puts the periodic copies of the active planes there.  The per-tracer
// file sizes (the reference stats its tracer files) are written as 0: this
// library keeps no tracer files.
#include <cstdio>
#include <string>
#include <vector>

#include "harm_common.cuh"

namespace harm {
namespace {

const char *const FD = "%32.22e";
const char *const FI = "%10d";

struct File {
  FILE *f;
  explicit File(FILE *x) : f(x) {}
  ~File()
  {
    if (f) fclose(f);
  }
};

// coord() (metric.c:62-115) at CENT, single rank, reference indices
void cent(const harm_params &p, int h, int i, int j, double *X)
{
  i -= 2;
  j -= 2;
  h -= p.n3 > 1 ? 1 : 0;
  X[1] = p.startx[1] + (i + 0.5) * p.dx[1];
  X[2] = p.startx[2] + (j + 0.5) * p.dx[2];
  X[3] = p.n3 > 2 ? p.startx[3] + (h + 0.5) * p.dx[3] : p.startx[3] + h * p.dx[3];
}

}  // namespace
}  // namespace harm

using namespace harm;

extern "C" int harm_restart_write(harm_ctx *h, const harm_restart_header *hdr, const harm_grid_spec *g,
                                  const char *path)
{
  if (!h || !hdr || !path) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  const Dims &d = x->D;
  if (x->ntr && !g) return fail_with(HARM_E_ARG, "a context with tracers needs the grid spec");
  std::vector<double> p((size_t)8 * d.cells());
  int rc = harm_get_prims(h, p.data(), nullptr);
  if (rc) return rc;
  double t, dt;
  rc = harm_get_time(h, &t, &dt);
  if (rc) return rc;
  harm_diag dg;
  rc = harm_get_diag(h, &dg);
  if (rc) return rc;
  File F(fopen(path, "wt"));
  if (!F.f) return fail_with(HARM_E_ARG, std::string("cannot open ") + path);
  FILE *f = F.f;
  // header (restart.c:103-136); t, dt, mass_in and mass_out are the context's
  fprintf(f, FI, d.n1);
  fprintf(f, FI, d.n2);
  fprintf(f, FI, d.n3);
  fprintf(f, FD, t);
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
  fprintf(f, FD, hdr->mass_start);
  fprintf(f, FD, dg.mass_in);
  fprintf(f, FD, dg.mass_out);
  fprintf(f, FD, hdr->tdump);
  fprintf(f, FD, hdr->timage);
  fprintf(f, FD, hdr->tlog);
  fprintf(f, FD, hdr->defcon);
  fprintf(f, FI, hdr->nfailed);
  fprintf(f, FD, hdr->Rbr);
  fprintf(f, FD, hdr->cyl_R0);
  fprintf(f, FD, hdr->cyl_Th0);
  fprintf(f, "\n");
  // body (restart.c:141-145)
  for (long c = 0; c < d.cells(); c++) {
    for (int k = 0; k < 8; k++) fprintf(f, FD, p[(size_t)c * 8 + k]);
    fprintf(f, "\n");
  }
  fprintf(f, FI, hdr->ener_size);
  // tracers (tracers.c:565-603): the active ones, in their order here
  if (x->ntr) {
    const long n = x->ntr;
    std::vector<int> ids(3 * (size_t)n);
    std::vector<double> X(3 * (size_t)n);
    std::vector<signed char> st(n);
    rc = harm_tracers_get(h, ids.data(), X.data(), st.data());
    if (rc) return rc;
    const harm_params &pr = x->prm;
    double Xa[4], Xb[4];
    const double trin = exp(pr.startx[1] - 0.5 * pr.dx[1]) + g->R0;
    const double trout = 0.8 * (exp(pr.startx[1] + pr.n1 * pr.dx[1]) + g->R0);
    cent(pr, d.hstart, d.istart, d.jstart, Xa);
    cent(pr, d.hstart, d.istop + 1, d.jstart, Xb);
    double phin = 0., phout = 0.;
    if (d.n3 > 2) {
      double Xc[4];
      phin = Xa[3];
      cent(pr, d.hstop + 1, d.istart, d.jstart, Xc);
      phout = Xc[3];
    }
    fprintf(f, FD, trin);
    fprintf(f, FD, trout);
    fprintf(f, FD, 0.02 * M_PI);
    fprintf(f, FD, 0.98 * M_PI);
    fprintf(f, FD, Xa[1]);
    fprintf(f, FD, Xb[1]);
    fprintf(f, FD, phin);
    fprintf(f, FD, phout);
    int active = 0;
    for (long k = 0; k < n; k++) active += st[k] == 0;
    fprintf(f, FI, active);
    for (long k = 0; k < n; k++) {
      if (st[k] != 0) continue;
      fprintf(f, FI, ids[3 * k]);
      fprintf(f, FI, ids[3 * k + 1]);
      fprintf(f, FI, ids[3 * k + 2]);
      fprintf(f, FD, 0.);
      for (int m = 0; m < 3; m++) fprintf(f, FD, X[3 * k + m]);
      fprintf(f, FI, 0);
    }
  }
  // COOL_EOS: every zone's temperature guess, _aLastT[SN3][SN1][SN2]
  // (restart_write_CoolEOS, cooleos.c:996-1013)
  if (x->cool) {
    std::vector<double> T(d.cells());
    rc = harm_get_eos_guess(h, T.data());
    if (rc) return rc;
    for (double v : T) fprintf(f, FD, v);
  }
  if (ferror(f)) return fail_with(HARM_E_ARG, std::string("write error on ") + path);
  return HARM_OK;
}

extern "C" int harm_restart_read(harm_ctx *h, const char *path, const harm_grid_spec *g, harm_restart_header *hdr)
{
  if (!h || !path || !hdr) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  const Dims &d = x->D;
  File F(fopen(path, "r"));
  if (!F.f) return fail_with(HARM_E_ARG, std::string("cannot open ") + path);
  FILE *f = F.f;
  harm_restart_header r;
  int ok = 1;
  // restart_read() (restart.c:311-383), same order
  ok &= fscanf(f, "%d", &r.n1) == 1;
  ok &= fscanf(f, "%d", &r.n2) == 1;
  ok &= fscanf(f, "%d", &r.n3) == 1;
  if (!ok || r.n1 != d.n1 || r.n2 != d.n2 || r.n3 != d.n3)
    return fail_with(HARM_E_ARG, "restart file grid differs from the context's");
  ok &= fscanf(f, "%lf", &r.t) == 1;
  ok &= fscanf(f, "%lf", &r.tf) == 1;
  ok &= fscanf(f, "%d", &r.nstep) == 1;
  ok &= fscanf(f, "%lf", &r.a) == 1;
  ok &= fscanf(f, "%lf", &r.gam) == 1;
  ok &= fscanf(f, "%lf", &r.cour) == 1;
  ok &= fscanf(f, "%lf", &r.DTd) == 1;
  ok &= fscanf(f, "%lf", &r.DTl) == 1;
  ok &= fscanf(f, "%lf", &r.DTi) == 1;
  ok &= fscanf(f, "%d", &r.DTr) == 1;
  ok &= fscanf(f, "%d", &r.dump_cnt) == 1;
  ok &= fscanf(f, "%d", &r.image_cnt) == 1;
  ok &= fscanf(f, "%d", &r.rdump_cnt) == 1;
  ok &= fscanf(f, "%lf", &r.dt) == 1;
  ok &= fscanf(f, "%d", &r.lim) == 1;
  ok &= fscanf(f, "%d", &r.failed) == 1;
  ok &= fscanf(f, "%lf", &r.Rin) == 1;
  ok &= fscanf(f, "%lf", &r.Rout) == 1;
  ok &= fscanf(f, "%lf", &r.hslope) == 1;
  ok &= fscanf(f, "%lf", &r.R0) == 1;
  ok &= fscanf(f, "%lf", &r.mass_start) == 1;
  ok &= fscanf(f, "%lf", &r.mass_in) == 1;
  ok &= fscanf(f, "%lf", &r.mass_out) == 1;
  ok &= fscanf(f, "%lf", &r.tdump) == 1;
  ok &= fscanf(f, "%lf", &r.timage) == 1;
  ok &= fscanf(f, "%lf", &r.tlog) == 1;
  ok &= fscanf(f, "%lf", &r.defcon) == 1;
  ok &= fscanf(f, "%d", &r.nfailed) == 1;
  ok &= fscanf(f, "%lf", &r.Rbr) == 1;
  ok &= fscanf(f, "%lf", &r.cyl_R0) == 1;
  ok &= fscanf(f, "%lf", &r.cyl_Th0) == 1;
  if (!ok) return fail_with(HARM_E_ARG, "truncated restart header");
  if (r.a != x->prm.a || r.gam != x->prm.gam)
    return fail_with(HARM_E_ARG, "restart file spin or adiabatic index differs from the context's");
  std::vector<double> p((size_t)8 * d.cells());
  for (size_t k = 0; k < p.size(); k++)
    if (fscanf(f, "%lf", &p[k]) != 1) return fail_with(HARM_E_ARG, "truncated restart body");
  if (fscanf(f, "%d", &r.ener_size) != 1) return fail_with(HARM_E_ARG, "truncated restart file");
  // pflag is not saved: the reference restarts with the zeros of set_arrays()
  std::vector<signed char> fl(d.cells(), 0);
  int rc = harm_put_prims(h, p.data(), fl.data());
  if (rc) return rc;
  // restart_init() bounds the primitives after reading (restart.c:285)
  rc = launch_bound(x, x->p);
  if (rc) return rc;
  CK(cudaGetLastError());
  rc = harm_set_time(h, r.t, r.dt);
  if (rc) return rc;
  rc = harm_set_mass(h, r.mass_in, r.mass_out);
  if (rc) return rc;
  // the tail: the tracer section when the file has one (restart_read_tracers,
  // tracers.c:608-652), then for a COOL_EOS context the zones' temperature
  // guesses (restart_read_CoolEOS, cooleos.c:1018-1030)
  std::vector<std::string> tok;
  {
    char buf[128];
    while (fscanf(f, "%127s", buf) == 1) tok.push_back(buf);
  }
  const size_t nguess = x->cool ? (size_t)d.cells() : 0;
  if (tok.size() < nguess) return fail_with(HARM_E_ARG, "truncated COOL_EOS section");
  const size_t ntr_tok = tok.size() - nguess;
  if (ntr_tok > 0) {
    size_t k = 0;
    auto next_d = [&](double &v) { return k < ntr_tok && sscanf(tok[k++].c_str(), "%lf", &v) == 1; };
    auto next_i = [&](int &v) { return k < ntr_tok && sscanf(tok[k++].c_str(), "%d", &v) == 1; };
    double tr;
    int cnt = 0;
    ok = true;
    for (int m = 0; m < 8; m++) ok &= next_d(tr);
    ok &= next_i(cnt) && cnt >= 0;
    if (!ok) return fail_with(HARM_E_ARG, "truncated tracer section");
    if (!g) return fail_with(HARM_E_ARG, "restart file has tracers: pass the grid spec");
    std::vector<int> ids(3 * (size_t)cnt);
    std::vector<double> X(3 * (size_t)cnt);
    for (int m = 0; m < cnt; m++) {
      double x0;
      int size;
      ok = next_i(ids[3 * m]) && next_i(ids[3 * m + 1]) && next_i(ids[3 * m + 2]);
      ok = ok && next_d(x0) && next_d(X[3 * m]) && next_d(X[3 * m + 1]) && next_d(X[3 * m + 2]);
      ok = ok && next_i(size);
      if (!ok) return fail_with(HARM_E_ARG, "truncated tracer section");
    }
    if (k != ntr_tok) return fail_with(HARM_E_ARG, "unexpected data after the tracer section");
    rc = harm_tracers_put(h, g, ids.data(), X.data(), cnt);
    if (rc) return rc;
  }
  if (nguess) {
    std::vector<double> T(nguess);
    for (size_t m = 0; m < nguess; m++)
      if (sscanf(tok[ntr_tok + m].c_str(), "%lf", &T[m]) != 1) return fail_with(HARM_E_ARG, "bad COOL_EOS section");
    rc = harm_put_eos_guess(h, T.data());
    if (rc) return rc;
  }
  *hdr = r;
  return harm_sync(h);
}
