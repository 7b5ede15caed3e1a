// k_f32.cu -- kernel instances for the PrecF32 arithmetic form.
#include "inst.cuh"
GF_DEFINE_PREC(PrecF32, f32)
