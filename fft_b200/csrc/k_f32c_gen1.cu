// k_f32c_gen1.cu -- run-time-schedule line kernels (PrecF32C, op group 1).
#include "inst.cuh"
GF_DEFINE_GEN(PrecF32C, f32c, 1)
