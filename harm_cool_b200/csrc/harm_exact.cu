// The FP64 step: built with -fmad=false so every multiply and add stays a
// separate IEEE operation, as in the reference's SSE2 build.
#define HARM_VARIANT exact
#define HARM_STEP_MIXED 0
#include "harm_step.cuh"
