// The FP64 step: built with -fmad=false so every multiply and add stays a
// separate IEEE operation, as in the reference's SSE2 build.
#define HARM_VARIANT exact
#define HARM_STEP_MIXED 0
#ifndef HARM_FLUX_MINB
#define HARM_FLUX_MINB 7   // 72 registers
#endif
#ifndef HARM_CONS_MINB
#define HARM_CONS_MINB 5   // 102 registers
#endif
#ifndef HARM_INV_MINB
#define HARM_INV_MINB 5    // 102 registers
#endif
#include "harm_step.cuh"
