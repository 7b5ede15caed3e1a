// k_f64.cu -- kernel instances for the PrecF64 arithmetic form.
#include "inst.cuh"
GF_DEFINE_PREC(PrecF64, f64)
