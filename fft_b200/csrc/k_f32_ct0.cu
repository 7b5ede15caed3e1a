// k_f32_ct0.cu -- compile-time-schedule kernel instances (PrecF32, op group 0).
#include "inst.cuh"
GF_DEFINE_CT(PrecF32, f32, 0)
