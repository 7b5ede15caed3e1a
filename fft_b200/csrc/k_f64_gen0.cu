// k_f64_gen0.cu -- run-time-schedule line kernels (PrecF64, op group 0).
#include "inst.cuh"
GF_DEFINE_GEN(PrecF64, f64, 0)
