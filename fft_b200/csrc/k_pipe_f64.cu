// k_pipe_f64.cu -- TMA-fed persistent line kernel instances (PrecF64).
#include "pipe_inst.cuh"
GF_DEFINE_PIPE(PrecF64, f64, true)
