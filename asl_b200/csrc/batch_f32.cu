// Batched step and links for f32 storage (batch.cuh).
#include "batch.cuh"

namespace aslb {

cudaError_t batch_step_f32(int q, const BatchDom* doms, int ndom, const BatchWork& w, int fused, const StepParams& p,
                           int parity_in, int shape, cudaStream_t st) {
  switch (q) {
    case 15: return batch_step_impl<15, float>(doms, ndom, w, fused, p, parity_in, shape, st);
    case 19: return batch_step_impl<19, float>(doms, ndom, w, fused, p, parity_in, shape, st);
    case 27: return batch_step_impl<27, float>(doms, ndom, w, fused, p, parity_in, shape, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t batch_links_f32(int q, const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st) {
  switch (q) {
    case 15: return batch_links_impl<15, float>(bcs, nbc, nlinks, parity, st);
    case 19: return batch_links_impl<19, float>(bcs, nbc, nlinks, parity, st);
    case 27: return batch_links_impl<27, float>(bcs, nbc, nlinks, parity, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace aslb
