// k_f32c_gen0.cu -- run-time-schedule line kernels (PrecF32C, op group 0).
#include "inst.cuh"
GF_DEFINE_GEN(PrecF32C, f32c, 0)
