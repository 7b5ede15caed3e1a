// k_f32_gen1.cu -- run-time-schedule line kernels (PrecF32, op group 1).
#include "inst.cuh"
GF_DEFINE_GEN(PrecF32, f32, 1)
