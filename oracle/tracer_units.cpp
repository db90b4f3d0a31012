// Unit constants for the reference's tracers.c in the checker build (TEST
// INFRASTRUCTURE ONLY).  tracers.c uses RHO_UNIT and T_UNIT only to scale the
// per-tracer dump files (tracers.c:436, 480); the reference defines them in
// cooleos.c, which needs the Fortran EOS library.  The checker never reads
// those files, so unit values serve.
extern const double RHO_UNIT = 1.0;
extern const double T_UNIT = 1.0;
