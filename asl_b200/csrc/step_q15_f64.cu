// Stream-collide instantiations for the D3Q15 lattice, f64 storage.
#include "stream_collide_tma.cuh"

namespace aslb {
cudaError_t step_q15_f64(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st) {
  return step_q_s<15, double>(d, p, closure, parity_in, st);
}
}  // namespace aslb
