// k_f32c_ct1.cu -- compile-time-schedule kernel instances (PrecF32C, op group 1).
#include "inst.cuh"
GF_DEFINE_CT(PrecF32C, f32c, 1)
