// Batched stream-collide and boundary links (kernels and their launchers):
// many independent domains of different sizes and viscosities advanced by
// one launch per step (plus one per condition position), instead of one
// launch per domain and condition. Each domain keeps its own allocation and
// layout; a device table maps the launch's tiles (one x plane of one domain,
// its cells taken 256 at a time, z fastest across y rows) and links to
// domains. Each block of the persistent grid takes a contiguous run of tiles
// holding an equal share of the batch's cells (BatchWork), the blocks of a
// group of four interleaving its planes, so a block's domain changes rarely
// and neighbouring planes of a domain are streamed together.
// Instantiated per storage in batch_<type>.cu.
#pragma once
#include "kernels.h"
#include "stream_collide.cuh"
#include "bc_links.cuh"

namespace aslb {

// Launch shapes of the persistent batched step: one cell per thread at 4, 3
// or 2 resident blocks of 256 threads per SM (64 / 80 / 128 registers), or
// two cells per thread (cells l and l + 256 of a plane, both cells' loads in
// flight before the first collision) at 3 or 2 blocks. aslb_batch_run times
// them on the batch and keeps the fastest.
constexpr int kBatchShapes = 5;
__host__ __device__ constexpr int batch_shape_blocks(int shape) {
  return shape == 0 ? 4 : (shape == 1 || shape == 3 ? 3 : 2);
}
__host__ __device__ constexpr bool batch_shape_pair(int shape) { return shape >= 3; }

// The fused-link words of a cell: the two-word form, or the one-word form
// (bit 31 set: the low bits are elide bits, else bounce bits).
template <bool M32>
__device__ __forceinline__ uint2 batch_links(const BatchDom& D, unsigned s) {
  if (M32) {
    const uint32_t w = D.mask32[s];
    return (w >> 31) ? make_uint2(0u, w & 0x7fffffffu) : make_uint2(w, 0u);
  }
  return D.mask[s];
}

// Collision and stores of one cell whose store offsets are recomputed after
// the collision (y and s are made to depend on its result), so the offsets
// used by the loads die with them instead of living across the collision.
template <int Q, class S, bool ODD, bool MASKED>
__device__ __forceinline__ void batch_finish(S* __restrict__ F, const GridDesc& g, const StepParams& p,
                                             typename MacroT<S>::T* __restrict__ rho_out,
                                             typename MacroT<S>::T* __restrict__ u_out, int x, int y, int z,
                                             unsigned s, uint32_t elide, typename Store<S>::C (&f)[Q],
                                             typename Store<S>::C om0) {
  cell_collide<Q, S, CL_NONE>(g, p, rho_out, u_out, x, y, z, s, f, om0);
  const int y2 = (int)after((unsigned)y, f[0]);
  int ox[3], oy[3], oz[3];
  nb_offsets(g, x, y2, z, ox, oy, oz);
  cell_store<Q, S, ODD, MASKED>(F, p, (unsigned)g.dstride, after(s, f[0]), ox, oy, oz, elide, f);
}

// The domain holding `tile`, searched from d (tiles ascend in the table).
__device__ __forceinline__ int batch_domain(const BatchDom* __restrict__ doms, int ndom, long long tile, int d) {
  if (d < 0) {
    int lo = 0, hi = ndom - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (doms[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
  }
  while (d + 1 < ndom && doms[d + 1].tile0 <= tile) ++d;
  return d;
}

// One cell per thread. The blocks of a group share a run of tiles and take
// every group-th tile of it (block j: tiles j, j + K, ...), so neighbouring
// planes, whose populations each pulls from the other, are streamed at the
// same time by neighbouring blocks; a block's planes of one domain are walked
// as one sequence of cells 256 at a time, so the next cell's link word is
// fetched one step ahead across plane boundaries too and the domain's table
// entry is read once per domain, not once per plane.
template <int Q, class S, bool ODD, bool FUSED, bool M32, int BLOCKS>
__global__ void __launch_bounds__(256, BLOCKS)
    k_batch_step(const BatchDom* __restrict__ doms, int ndom, const long long* __restrict__ starts, int K,
                 const StepParams p) {
  using C = typename Store<S>::C;
  using M = typename MacroT<S>::T;
  const int grp = (int)blockIdx.x / K;
  long long tile = starts[grp] + (int)blockIdx.x % K;
  const long long tend = starts[grp + 1];
  int d = -1;
  while (tile < tend) {
    d = batch_domain(doms, ndom, tile, d);
    const BatchDom& D = doms[d];
    const GridDesc g = D.g;
    // this block's planes of the domain in the run: xa, xa + K, ... <= xb
    const int xa = (int)(tile - D.tile0) + 1;
    const int xb = (int)(min(tend, D.tile0 + g.nx) - D.tile0);
    tile += (long long)K * ((xb - xa) / K + 1);
    const unsigned plane_cells = (unsigned)(g.ny * g.nz);
    const unsigned nz = (unsigned)g.nz, nz_inv = D.nz_inv;
    S* F = (S*)D.F;
    const C om0 = std::is_same<C, double>::value ? C(D.om0d) : C(D.om0f);
    const bool masked = FUSED && (M32 ? D.mask32 != nullptr : D.mask != nullptr);
    // storage index of cell l of plane x (y rows of nz cells, z fastest)
    auto cell_index = [&](int x, unsigned l, int& y, int& z) {
      unsigned yq = __umulhi(l, nz_inv);
      if (yq * nz > l) --yq;  // exact quotient for l < 2^32 / nz
      y = (int)yq + 1;
      z = (int)(l - yq * nz) + 1;
      return (unsigned)sidx(g, x, y, z);
    };
    // (x, l): this thread's cell; advancing by 256 cells may cross planes
    int x = xa;
    unsigned l = threadIdx.x;
    while (l >= plane_cells && x <= xb) {
      l -= plane_cells;
      x += K;
    }
    uint2 mnext = make_uint2(0u, 0u);
    if (masked && x <= xb) {
      int y1, z1;
      mnext = batch_links<M32>(D, cell_index(x, l, y1, z1));
    }
    while (x <= xb) {
      int y, z;
      const unsigned s = cell_index(x, l, y, z);
      const uint32_t bounce = mnext.x, elide = mnext.y;
      int xn = x;
      unsigned ln = l + 256u;
      while (ln >= plane_cells && xn <= xb) {
        ln -= plane_cells;
        xn += K;
      }
      if (masked && xn <= xb) {
        int y1, z1;
        mnext = batch_links<M32>(D, cell_index(xn, ln, y1, z1));
      }
      int ox[3], oy[3], oz[3];
      nb_offsets(g, x, y, z, ox, oy, oz);
      C f[Q];
      cell_load<Q, S, ODD, FUSED>(F, (unsigned)g.dstride, s, ox, oy, oz, bounce, f);
      batch_finish<Q, S, ODD, FUSED>(F, g, p, (M*)D.rho, (M*)D.u, x, y, z, s, elide, f, om0);
      x = xn;
      l = ln;
    }
  }
}

// Two cells per thread: cells l and l + 256 of the plane.
template <int Q, class S, bool ODD, bool FUSED, bool M32, int BLOCKS>
__global__ void __launch_bounds__(256, BLOCKS)
    k_batch_step_pair(const BatchDom* __restrict__ doms, int ndom, const long long* __restrict__ starts, int K,
                      const StepParams p) {
  using C = typename Store<S>::C;
  using M = typename MacroT<S>::T;
  int d = -1;
  const int grp = (int)blockIdx.x / K;
  const long long tend = starts[grp + 1];
  for (long long tile = starts[grp] + (int)blockIdx.x % K; tile < tend; tile += K) {
    d = batch_domain(doms, ndom, tile, d);
    const BatchDom& D = doms[d];
    const GridDesc g = D.g;
    const int x = (int)(tile - D.tile0) + 1;
    const unsigned plane_cells = (unsigned)(g.ny * g.nz);
    const unsigned nz = (unsigned)g.nz, nz_inv = D.nz_inv;
    S* F = (S*)D.F;
    const bool masked = FUSED && D.mask;
    const C om0 = std::is_same<C, double>::value ? C(D.om0d) : C(D.om0f);
    auto cell_index = [&](unsigned l, int& y, int& z) {
      unsigned yq = __umulhi(l, nz_inv);
      if (yq * nz > l) --yq;
      y = (int)yq + 1;
      z = (int)(l - yq * nz) + 1;
      return (unsigned)sidx(g, x, y, z);
    };
    uint2 na = make_uint2(0u, 0u), nb = make_uint2(0u, 0u);
    if (masked) {
      int y1, z1;
      if (threadIdx.x < plane_cells) na = batch_links<M32>(D, cell_index(threadIdx.x, y1, z1));
      if (threadIdx.x + 256u < plane_cells) nb = batch_links<M32>(D, cell_index(threadIdx.x + 256u, y1, z1));
    }
    for (unsigned l = threadIdx.x; l < plane_cells; l += 512u) {
      const bool has_b = l + 256u < plane_cells;
      int ya, za, yb = 0, zb = 0;
      const unsigned sa = cell_index(l, ya, za);
      const unsigned sb = has_b ? cell_index(l + 256u, yb, zb) : 0u;
      const uint2 ma = na, mb = nb;
      if (masked) {
        int y1, z1;
        if (l + 512u < plane_cells) na = batch_links<M32>(D, cell_index(l + 512u, y1, z1));
        if (l + 768u < plane_cells) nb = batch_links<M32>(D, cell_index(l + 768u, y1, z1));
      }
      int ox[3], oya[3], oza[3], oyb[3], ozb[3];
      nb_offsets(g, x, ya, za, ox, oya, oza);
      C fa[Q], fb[Q];
      cell_load<Q, S, ODD, FUSED>(F, (unsigned)g.dstride, sa, ox, oya, oza, ma.x, fa);
      if (has_b) {
        nb_offsets(g, x, yb, zb, ox, oyb, ozb);
        cell_load<Q, S, ODD, FUSED>(F, (unsigned)g.dstride, sb, ox, oyb, ozb, mb.x, fb);
      }
      batch_finish<Q, S, ODD, FUSED>(F, g, p, (M*)D.rho, (M*)D.u, x, ya, za, sa, ma.y, fa, om0);
      if (has_b) batch_finish<Q, S, ODD, FUSED>(F, g, p, (M*)D.rho, (M*)D.u, x, yb, zb, sb, mb.y, fb, om0);
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

template <int Q, class S, int SHAPE, bool M32>
cudaError_t batch_step_shape(const BatchDom* doms, int ndom, const BatchWork& w, bool fused, const StepParams& p,
                             int parity_in, cudaStream_t st) {
  constexpr int BLOCKS = batch_shape_blocks(SHAPE);
  const int grid = w.grid[BLOCKS - 2], K = w.group[BLOCKS - 2];
  const long long* starts = w.starts + w.off[BLOCKS - 2];
  if constexpr (batch_shape_pair(SHAPE)) {
    if (parity_in == 0) {
      if (fused) k_batch_step_pair<Q, S, true, true, M32, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
      else k_batch_step_pair<Q, S, true, false, false, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
    } else {
      if (fused) k_batch_step_pair<Q, S, false, true, M32, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
      else k_batch_step_pair<Q, S, false, false, false, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
    }
  } else {
    if (parity_in == 0) {
      if (fused) k_batch_step<Q, S, true, true, M32, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
      else k_batch_step<Q, S, true, false, false, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
    } else {
      if (fused) k_batch_step<Q, S, false, true, M32, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
      else k_batch_step<Q, S, false, false, false, BLOCKS><<<grid, 256, 0, st>>>(doms, ndom, starts, K, p);
    }
  }
  return cudaGetLastError();
}

// fused: 0 none, 1 two-word link masks, 2 one-word masks in every masked domain
// Two cells per thread are built for D3Q15 / D3Q19 in 4- and 2-byte storage
// with one-word link masks (or none); other cases take the one-cell shape
// with the same residency.
template <int Q, class S, int SHAPE>
cudaError_t batch_step_m(const BatchDom* doms, int ndom, const BatchWork& w, int fused, const StepParams& p,
                         int parity_in, cudaStream_t st) {
  if constexpr (batch_shape_pair(SHAPE)) {
    constexpr int ONE = SHAPE == 3 ? 1 : 2;
    if constexpr (Q == 27 || sizeof(S) == 8) {
      return batch_step_m<Q, S, ONE>(doms, ndom, w, fused, p, parity_in, st);
    } else {
      if (fused == 1) return batch_step_m<Q, S, ONE>(doms, ndom, w, fused, p, parity_in, st);
      return batch_step_shape<Q, S, SHAPE, true>(doms, ndom, w, fused != 0, p, parity_in, st);
    }
  } else {
    if (fused == 2) return batch_step_shape<Q, S, SHAPE, true>(doms, ndom, w, true, p, parity_in, st);
    return batch_step_shape<Q, S, SHAPE, false>(doms, ndom, w, fused != 0, p, parity_in, st);
  }
}

template <int Q, class S>
cudaError_t batch_step_impl(const BatchDom* doms, int ndom, const BatchWork& w, int fused, const StepParams& p,
                            int parity_in, int shape, cudaStream_t st) {
  if (w.ntiles <= 0) return cudaSuccess;
  switch (shape) {
    case 0: return batch_step_m<Q, S, 0>(doms, ndom, w, fused, p, parity_in, st);
    case 1: return batch_step_m<Q, S, 1>(doms, ndom, w, fused, p, parity_in, st);
    case 2: return batch_step_m<Q, S, 2>(doms, ndom, w, fused, p, parity_in, st);
    case 3: return batch_step_m<Q, S, 3>(doms, ndom, w, fused, p, parity_in, st);
    case 4: return batch_step_m<Q, S, 4>(doms, ndom, w, fused, p, parity_in, st);
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
