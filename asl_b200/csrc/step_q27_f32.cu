// Stream-collide instantiations for the D3Q27 lattice, f32 storage.
#include "stream_collide_tma.cuh"

namespace aslb {
cudaError_t step_q27_f32(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st) {
  return step_q_s<27, float>(d, p, closure, parity_in, st);
}
}  // namespace aslb
