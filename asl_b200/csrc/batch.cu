// Dispatch of the batched step and links to their per-storage instantiations
// (batch_f32.cu, batch_f16.cu, batch_f64.cu; kernels in batch.cuh).
#include "kernels.h"

namespace aslb {

cudaError_t batch_step_f32(int q, const BatchDom* doms, int ndom, long long ntiles, int fused, const StepParams& p,
                           int parity_in, int shape, cudaStream_t st);
cudaError_t batch_step_f16(int q, const BatchDom* doms, int ndom, long long ntiles, int fused, const StepParams& p,
                           int parity_in, int shape, cudaStream_t st);
cudaError_t batch_step_f64(int q, const BatchDom* doms, int ndom, long long ntiles, int fused, const StepParams& p,
                           int parity_in, int shape, cudaStream_t st);
cudaError_t batch_links_f32(int q, const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st);
cudaError_t batch_links_f16(int q, const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st);
cudaError_t batch_links_f64(int q, const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st);

int batch_shape_count() { return 5; }

cudaError_t launch_batch_step(int q, int storage, const BatchDom* doms, int ndom, long long ntiles, int fused,
                              const StepParams& p, int parity_in, int shape, cudaStream_t st) {
  switch (storage) {
    case ST_F32: return batch_step_f32(q, doms, ndom, ntiles, fused, p, parity_in, shape, st);
    case ST_F16: return batch_step_f16(q, doms, ndom, ntiles, fused, p, parity_in, shape, st);
    case ST_F64: return batch_step_f64(q, doms, ndom, ntiles, fused, p, parity_in, shape, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_batch_links(int q, int storage, const BatchBc* bcs, int nbc, long long nlinks, int parity,
                               cudaStream_t st) {
  switch (storage) {
    case ST_F32: return batch_links_f32(q, bcs, nbc, nlinks, parity, st);
    case ST_F16: return batch_links_f16(q, bcs, nbc, nlinks, parity, st);
    case ST_F64: return batch_links_f64(q, bcs, nbc, nlinks, parity, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace aslb
