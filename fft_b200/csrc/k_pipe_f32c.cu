// k_pipe_f32c.cu -- TMA-fed persistent line kernel instances (PrecF32C).
#include "pipe_inst.cuh"
GF_DEFINE_PIPE(PrecF32C, f32c, false)
