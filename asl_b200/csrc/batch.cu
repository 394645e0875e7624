// Dispatch of the batched step and links to their per-storage instantiations
// (batch_f32.cu, batch_f16.cu, batch_f64.cu; kernels in batch.cuh).
#include <algorithm>
#include "kernels.h"

namespace aslb {

cudaError_t batch_step_f32(int q, const BatchDom* doms, int ndom, const BatchWork& w, int fused, const StepParams& p,
                           int parity_in, int shape, cudaStream_t st);
cudaError_t batch_step_f16(int q, const BatchDom* doms, int ndom, const BatchWork& w, int fused, const StepParams& p,
                           int parity_in, int shape, cudaStream_t st);
cudaError_t batch_step_f64(int q, const BatchDom* doms, int ndom, const BatchWork& w, int fused, const StepParams& p,
                           int parity_in, int shape, cudaStream_t st);
cudaError_t batch_links_f32(int q, const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st);
cudaError_t batch_links_f16(int q, const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st);
cudaError_t batch_links_f64(int q, const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st);

int batch_shape_count() { return 5; }

void batch_work_tables(const std::vector<long long>& tile_cells, int sms, std::vector<long long>& starts,
                       int (&grid)[3], int (&group)[3], long long (&off)[3]) {
  const long long T = (long long)tile_cells.size();
  long long C = 0;
  for (long long c : tile_cells) C += c;
  starts.clear();
  for (int k = 0; k < 3; ++k) {
    const long long G = std::max(1LL, std::min(T, (long long)sms * (k + 2)));
    const int K = (G % 4 == 0) ? 4 : 1;
    const long long NG = G / K;
    grid[k] = (int)G;
    group[k] = K;
    off[k] = (long long)starts.size();
    // group b starts at the first tile whose preceding cells reach b C / NG
    long long t = 0, before = 0;
    for (long long b = 0; b < NG; ++b) {
      const long long target = (long long)(((__int128)b * C + NG - 1) / NG);
      while (t < T && before < target) before += tile_cells[t++];
      starts.push_back(t);
    }
    starts.push_back(T);
  }
}

cudaError_t launch_batch_step(int q, int storage, const BatchDom* doms, int ndom, const BatchWork& w, int fused,
                              const StepParams& p, int parity_in, int shape, cudaStream_t st) {
  switch (storage) {
    case ST_F32: return batch_step_f32(q, doms, ndom, w, fused, p, parity_in, shape, st);
    case ST_F16: return batch_step_f16(q, doms, ndom, w, fused, p, parity_in, shape, st);
    case ST_F64: return batch_step_f64(q, doms, ndom, w, fused, p, parity_in, shape, st);
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
