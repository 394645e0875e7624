// Batched stream-collide and boundary links (kernels and their launchers):
// many independent domains of different sizes and viscosities advanced by
// one launch per step (plus one per condition position), instead of one
// launch per domain and condition. Each domain keeps its own allocation and
// layout; a device table maps the launch's tiles (one x plane of one domain,
// its cells taken 256 at a time, z fastest across y rows) and links to
// domains. Instantiated per storage in batch_<type>.cu.
#pragma once
#include "kernels.h"
#include "stream_collide.cuh"
#include "bc_links.cuh"

namespace aslb {

// Launch shapes of the persistent batched step: resident blocks of 256
// threads per SM (4: 64 registers, 3: 80, 2: 128). aslb_batch_run times them
// on the batch and keeps the fastest.
constexpr int kBatchShapes = 3;
__host__ __device__ constexpr int batch_shape_blocks(int shape) { return shape == 0 ? 4 : (shape == 1 ? 3 : 2); }

template <int Q, class S, bool ODD, bool FUSED, int BLOCKS>
__global__ void __launch_bounds__(256, BLOCKS)
    k_batch_step(const BatchDom* __restrict__ doms, int ndom, long long ntiles, const StepParams p) {
  using C = typename Store<S>::C;
  using M = typename MacroT<S>::T;
  int d = -1;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // a block's tiles only move forward: advance the domain index
    if (d < 0) {
      int lo = 0, hi = ndom - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (doms[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
      }
      d = lo;
    }
    while (d + 1 < ndom && doms[d + 1].tile0 <= tile) ++d;
    const BatchDom& D = doms[d];
    const GridDesc g = D.g;
    const int x = (int)(tile - D.tile0) + 1;  // one tile = one x plane
    const unsigned plane_cells = (unsigned)(g.ny * g.nz);
    const unsigned nz = (unsigned)g.nz, nz_inv = D.nz_inv;
    S* F = (S*)D.F;
    const uint2* mask = D.mask;
    const C om0 = std::is_same<C, double>::value ? C(D.om0d) : C(D.om0f);
    // storage index of plane cell l (y rows of nz cells, z fastest)
    auto cell_index = [&](unsigned l, int& y, int& z) {
      unsigned yq = __umulhi(l, nz_inv);
      if (yq * nz > l) --yq;  // exact quotient for l < 2^32 / nz
      y = (int)yq + 1;
      z = (int)(l - yq * nz) + 1;
      return (unsigned)sidx(g, x, y, z);
    };
    // the fused-link words of a thread's next cell are loaded one iteration
    // ahead: the population addresses depend on them, so they must not cost
    // a second memory round trip
    uint2 mnext = make_uint2(0u, 0u);
    if (FUSED && mask && threadIdx.x < plane_cells) {
      int y1, z1;
      mnext = mask[cell_index(threadIdx.x, y1, z1)];
    }
    for (unsigned l = threadIdx.x; l < plane_cells; l += 256u) {
      int y, z;
      const unsigned s = cell_index(l, y, z);
      uint32_t bounce = 0, elide = 0;
      if (FUSED && mask) {
        bounce = mnext.x;
        elide = mnext.y;
        if (l + 256u < plane_cells) {
          int y1, z1;
          mnext = mask[cell_index(l + 256u, y1, z1)];
        }
      }
      int ox[3], oy[3], oz[3];
      nb_offsets(g, x, y, z, ox, oy, oz);
      C f[Q];
      cell_load<Q, S, ODD, FUSED>(F, (unsigned)g.dstride, s, ox, oy, oz, bounce, f);
      cell_finish<Q, S, CL_NONE, ODD, FUSED>(F, g, p, (M*)D.rho, (M*)D.u, x, y, z, s, ox, oy, oz, elide, f, om0);
    }
  }
}

template <int Q, class S>
__global__ void __launch_bounds__(256)
    k_batch_links(const BatchBc* __restrict__ bcs, int nbc, long long nlinks, int parity) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nlinks) return;
  int lo = 0, hi = nbc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bcs[mid].link0 <= t) lo = mid; else hi = mid - 1;
  }
  const BatchBc& B = bcs[lo];
  link_apply<Q, S>((S*)B.F, B.dstride, B.links, (int)(t - B.link0), B.ls, B.bp, parity);
}

inline int batch_sm_count() {
  static int g_sms = 0;
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return g_sms;
}

template <int Q, class S, int BLOCKS>
cudaError_t batch_step_shape(const BatchDom* doms, int ndom, long long ntiles, bool fused, const StepParams& p,
                             int parity_in, cudaStream_t st) {
  const long long cap = (long long)batch_sm_count() * BLOCKS;
  const int grid = (int)(ntiles < cap ? ntiles : cap);
  if (parity_in == 0) {
    if (fused) k_batch_step<Q, S, true, true, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, ntiles, p);
    else k_batch_step<Q, S, true, false, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, ntiles, p);
  } else {
    if (fused) k_batch_step<Q, S, false, true, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, ntiles, p);
    else k_batch_step<Q, S, false, false, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, ntiles, p);
  }
  return cudaGetLastError();
}

template <int Q, class S>
cudaError_t batch_step_impl(const BatchDom* doms, int ndom, long long ntiles, bool fused, const StepParams& p,
                            int parity_in, int shape, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  switch (shape) {
    case 0: return batch_step_shape<Q, S, batch_shape_blocks(0)>(doms, ndom, ntiles, fused, p, parity_in, st);
    case 1: return batch_step_shape<Q, S, batch_shape_blocks(1)>(doms, ndom, ntiles, fused, p, parity_in, st);
    case 2: return batch_step_shape<Q, S, batch_shape_blocks(2)>(doms, ndom, ntiles, fused, p, parity_in, st);
  }
  return cudaErrorInvalidValue;
}

template <int Q, class S>
cudaError_t batch_links_impl(const BatchBc* bcs, int nbc, long long nlinks, int parity, cudaStream_t st) {
  if (nlinks <= 0) return cudaSuccess;
  k_batch_links<Q, S><<<(unsigned)((nlinks + 255) / 256), 256, 0, st>>>(bcs, nbc, nlinks, parity);
  return cudaGetLastError();
}

}  // namespace aslb
