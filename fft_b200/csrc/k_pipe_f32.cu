// k_pipe_f32.cu -- TMA-fed persistent line kernel instances (PrecF32).
#include "pipe_inst.cuh"
GF_DEFINE_PIPE(PrecF32, f32, false)
