// k_f64_ew.cu -- elementwise and table kernels (PrecF64).
#include "inst.cuh"
GF_DEFINE_PREC(PrecF64, f64)
