// k_f64_ct0.cu -- compile-time-schedule kernel instances (PrecF64, op group 0).
#include "inst.cuh"
GF_DEFINE_CT(PrecF64, f64, 0)
