// k_rip_f64.cu -- in-shared-memory Rader kernel (PrecF64).
#include "rader_ip.cuh"
namespace gf {
const void *rader_ip_kernel_f64(int *threads) {
  *threads = rip_threads<PrecF64>();
  return (const void *)k_rader_ip<PrecF64>;
}
const void *rader_ip2_kernel_f64(int *threads) {
  *threads = rip_threads<PrecF64>();
  return (const void *)k_rader_ip2<PrecF64>;
}
}  // namespace gf
