// k_f32_ew.cu -- elementwise and table kernels (PrecF32).
#include "inst.cuh"
GF_DEFINE_PREC(PrecF32, f32)
