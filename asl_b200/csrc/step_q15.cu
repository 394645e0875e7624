// Stream-collide instantiations for the D3Q15 lattice.
#include "stream_collide_tma.cuh"

namespace aslb {
cudaError_t step_q15(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st) {
  return step_q<15>(d, p, closure, parity_in, st);
}
}  // namespace aslb
