// k_f64_gen1.cu -- run-time-schedule line kernels (PrecF64, op group 1).
#include "inst.cuh"
GF_DEFINE_GEN(PrecF64, f64, 1)
