// k_f32_gen0.cu -- run-time-schedule line kernels (PrecF32, op group 0).
#include "inst.cuh"
GF_DEFINE_GEN(PrecF32, f32, 0)
