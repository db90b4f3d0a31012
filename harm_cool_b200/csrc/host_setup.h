// Host-side set-up shared inside libharm_b200: grid geometry and the initial
// torus fields.  The public entry points are declared in include/harm_b200.h.
#pragma once
#include "harm_b200.h"

namespace harm {

// Dimensions of the reference's arrays for one grid (decs.h:266-268, defs.h:49-51).
struct Dims {
  int n1, n2, n3, sn1, sn2, sn3;
  int istart, istop, jstart, jstop, hstart, hstop;
  long zones() const { return (long)n1 * n2 * n3; }
  long cells() const { return (long)sn1 * sn2 * sn3; }
  long plane() const { return (long)sn1 * sn2; }
};

Dims make_dims(int n1, int n2, int n3);
bool valid_grid(int n1, int n2, int n3);

// Fishbone-Moncrief fields in the active zones of p (reference layout),
// before normalisation: rho, u (with the seeded perturbation), u-tilde; B = 0.
// Returns rhomax and umax over the torus as init() computes them (init.c:161-268).
void torus_hydro(const harm_grid_spec &g, const harm_params &prm, const harm_torus_spec &t,
                 const double *gcov, const double *gcon, double *p, double *rhomax, double *umax);

// Corner vector potential from rho (init.c:327-352) and the cell-centred field
// it defines (init.c:360-368), written into B1, B2, B3 of the active zones.
void torus_field(const Dims &d, const harm_params &prm, const double *gdet, double *p);

// get_rho_u_floor() (fixup.c:117-140, BL branch) at every (r, theta) point:
// out[0..n) = rho floor, out[n..2n) = u floor; r from coords[n][4]
void radial_floors(const double *coords, double gam, long n, double *out);

}  // namespace harm
