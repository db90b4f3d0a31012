// The mixed-precision step: FP32 reconstruction, face states, wave speeds and
// fluxes; FP64 geometry source, flux divergence, accumulation, inversion and
// floors.  Built with FMA contraction.
#define HARM_VARIANT mixed
#define HARM_STEP_MIXED 1
#include "harm_step.cuh"
