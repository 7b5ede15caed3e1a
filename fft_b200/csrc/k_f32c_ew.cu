// k_f32c_ew.cu -- elementwise and table kernels (PrecF32C).
#include "inst.cuh"
GF_DEFINE_PREC(PrecF32C, f32c)
