// pipe.h -- host-visible handles of the TMA-fed persistent line kernel.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace gf {

// One compiled instance: the kernel (k_pipe, parameters KArgs, PipeArgs,
// CUtensorMap) and its launch shape.
struct PipeInst {
  const void *fn;
  int lpc, groups, slots, threads;
  size_t smem;
};

// Instance for (op, length, threads per line, radix schedule, column mode)
// in a precision; fn == nullptr if none was built.
PipeInst pipe_kernel_f64(int op, int n, int T, const int *rad, int nst, bool col);
PipeInst pipe_kernel_f32(int op, int n, int T, const int *rad, int nst, bool col);
PipeInst pipe_kernel_f32c(int op, int n, int T, const int *rad, int nst, bool col);

}  // namespace gf
