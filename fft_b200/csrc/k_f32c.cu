// k_f32c.cu -- kernel instances for the PrecF32C arithmetic form.
#include "inst.cuh"
GF_DEFINE_PREC(PrecF32C, f32c)
