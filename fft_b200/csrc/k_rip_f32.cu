// k_rip_f32.cu -- in-shared-memory Rader kernel (PrecF32).
#include "rader_ip.cuh"
namespace gf {
const void *rader_ip_kernel_f32(int *threads) {
  *threads = rip_threads<PrecF32>();
  return (const void *)k_rader_ip<PrecF32>;
}
const void *rader_ip2_kernel_f32(int *threads) {
  *threads = rip_threads<PrecF32>();
  return (const void *)k_rader_ip2<PrecF32>;
}
}  // namespace gf
