// k_rip_f32c.cu -- in-shared-memory Rader kernel (PrecF32C).
#include "rader_ip.cuh"
namespace gf {
const void *rader_ip_kernel_f32c(int *threads) {
  *threads = rip_threads<PrecF32C>();
  return (const void *)k_rader_ip<PrecF32C>;
}
const void *rader_ip2_kernel_f32c(int *threads) {
  *threads = rip_threads<PrecF32C>();
  return (const void *)k_rader_ip2<PrecF32C>;
}
}  // namespace gf
