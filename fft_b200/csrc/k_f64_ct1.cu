// k_f64_ct1.cu -- compile-time-schedule kernel instances (PrecF64, op group 1).
#include "inst.cuh"
GF_DEFINE_CT(PrecF64, f64, 1)
