// Stream-collide instantiations for the D3Q19 lattice, f16 storage.
#include "stream_collide_tma.cuh"

namespace aslb {
cudaError_t step_q19_f16(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st) {
  return step_q_s<19, __half>(d, p, closure, parity_in, st);
}
}  // namespace aslb
