// The mixed-precision step: FP32 reconstruction, face states, wave speeds and
// fluxes; FP64 geometry source, flux divergence, accumulation, inversion and
// floors, with reciprocal multiplies for the divisions by shared divisors
// (div_rn).  Built with FMA contraction.
#define HARM_VARIANT mixed
#define HARM_STEP_MIXED 1
#ifndef HARM_FLUX_MINB
#define HARM_FLUX_MINB 8   // 64 registers
#endif
#ifndef HARM_CONS_MINB
#define HARM_CONS_MINB 5   // 102 registers
#endif
#ifndef HARM_INV_MINB
#define HARM_INV_MINB 4    // 128 registers
#endif
#include "harm_step.cuh"
