// k_f32_ct1.cu -- compile-time-schedule kernel instances (PrecF32, op group 1).
#include "inst.cuh"
GF_DEFINE_CT(PrecF32, f32, 1)
