// k_f32c_ct0.cu -- compile-time-schedule kernel instances (PrecF32C, op group 0).
#include "inst.cuh"
GF_DEFINE_CT(PrecF32C, f32c, 0)
