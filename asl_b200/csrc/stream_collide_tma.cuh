// Stream-collide with TMA staging (sm_100a). A persistent, warp-specialised
// CTA (eight compute warps and one producer warp) walks tiles of R z-rows x
// TZ cells. For every tile the producer warp's lanes issue 1-D bulk copies
// (cp.async.bulk) of the Q population rows the tile reads, plus its row of
// fused-link masks, into one of `stages` shared-memory buffers, tracked by
// full/empty mbarriers with transaction counts; the copies for the next tiles
// are in flight while the compute warps work on the current one, so HBM stays
// busy without registers holding loads. Results go straight to global memory
// (the AA pattern writes the same slots it read).
//
// Alignment: a row's first interior cell is 128-byte aligned and x/y
// neighbour offsets are whole rows, so every copy is exactly the 128-byte
// aligned row segment (widening it to reach the +-1 z neighbours makes the
// copy engine fetch whole extra lines for every row). A direction's +-1 z
// shift is absorbed by indexing inside the buffer; the one lane per row whose
// upstream cell falls outside the segment reads it from global memory.
#pragma once
#include "stream_collide.cuh"
#include "tma.cuh"
#include <algorithm>

namespace aslb {

struct TmaShape {
  int tz;       // cells per row segment (multiple of 32)
  int rows;     // rows per tile (tz * rows = 256)
  int nseg;     // segments per row
  int ntiles;   // row groups * nseg
  int stages;   // pipeline depth
  int span;     // staged elements per row (= tz)
  int stage_bytes;
  int fused;    // masks staged too
};

template <class S>
__device__ __forceinline__ S* stage_pop(unsigned char* smem, const TmaShape& sh, int st, int r, int i, int q) {
  return reinterpret_cast<S*>(smem + (size_t)st * sh.stage_bytes) + ((size_t)r * q + i) * sh.span;
}

template <class S>
__device__ __forceinline__ uint2* stage_mask(unsigned char* smem, const TmaShape& sh, int st, int q) {
  return reinterpret_cast<uint2*>(smem + (size_t)st * sh.stage_bytes + (size_t)sh.rows * q * sh.span * sizeof(S));
}

// Issue the copies of tile `tile` into stage `st`: the 32 lanes of the
// producer warp split the (row, direction) copies; lane 0 first arms the
// stage's barrier with the transaction byte count.
template <int Q, class S, bool ODD>
__device__ __forceinline__ void tma_issue_tile(const S* F, const GridDesc& g, const StepParams& p,
                                               const TmaShape& sh, unsigned char* smem, uint64_t* bar, int st,
                                               int tile, int lane) {
  using Lt = Lattice<Q>;
  const int rg = tile / sh.nseg, seg = tile % sh.nseg;
  const int r0 = rg * sh.rows;
  const int nr = min(sh.rows, g.nx * g.ny - r0);
  const uint32_t row_bytes = (uint32_t)(sh.span * sizeof(S));
  const uint32_t mask_bytes = sh.fused ? (uint32_t)(sh.tz * sizeof(uint2)) : 0u;
  if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)nr * (Q * row_bytes + mask_bytes));
  __syncwarp();
  const int per_row = Q + sh.fused;
  for (int c = lane; c < nr * per_row; c += 32) {
    const int r = c / per_row, i = c % per_row;
    const int row = r0 + r;
    const int x = row / g.ny + 1, y = row % g.ny + 1;
    const long long s0 = sidx(g, x, y, 1 + seg * sh.tz);
    if (i == Q) {
      bulk_g2s(stage_mask<S>(smem, sh, st, Q) + (size_t)r * sh.tz, p.mask + s0, mask_bytes, bar);
      continue;
    }
    long long src;
    if (ODD) {
      int ox[3], oy[3], oz[3];
      nb_offsets(g, x, y, 2, ox, oy, oz);  // z = 2: no z wrap in the row offsets
      src = (long long)i * g.dstride + s0 + ox[1 - Lt::c_rt(i, 0)] + oy[1 - Lt::c_rt(i, 1)];
    } else {
      src = (long long)Lt::inv_rt(i) * g.dstride + s0;
    }
    bulk_g2s(stage_pop<S>(smem, sh, st, r, i, Q), F + src, row_bytes, bar);
  }
}

template <class S, int CL>
struct TmaOccupancy {
  static constexpr int blocks = (CL == CL_NONE && !std::is_same<S, double>::value) ? 3 : 2;
};

constexpr int kConsumerWarps = 8;
constexpr int kTmaThreads = (kConsumerWarps + 1) * 32;

// Warp-specialised persistent kernel: warps 0-7 compute one cell per thread,
// warp 8 produces. full[st] completes when a stage's copies have landed;
// empty[st] when all consumer warps have read it.
template <int Q, class S, int CL, bool ODD>
__global__ void __launch_bounds__(kTmaThreads, TmaOccupancy<S, CL>::blocks)
    k_stream_collide_tma(S* __restrict__ F, const GridDesc g, const StepParams p,
                         typename MacroT<S>::T* __restrict__ rho_out, typename MacroT<S>::T* __restrict__ u_out,
                         const TmaShape sh, int* __restrict__ err) {
  using Lt = Lattice<Q>;
  using C = typename Store<S>::C;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[4], empty[4];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const unsigned ds = (unsigned)g.dstride;

  if (tid == 0) {
    for (int st = 0; st < sh.stages; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kConsumerWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == kConsumerWarps) {
    // ---- producer ----
    int k = 0;
    for (int tile = blockIdx.x; tile < sh.ntiles; tile += gridDim.x, ++k) {
      const int st = k % sh.stages;
      if (k >= sh.stages) {
        int ok = 1;
        if (lane == 0) ok = mbar_wait(&empty[st], (uint32_t)(((k / sh.stages) - 1) & 1));
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
          if (lane == 0) atomicExch(err, 1);
          break;
        }
        fence_proxy_async_smem();
      }
      tma_issue_tile<Q, S, ODD>(F, g, p, sh, smem, &full[st], st, tile, lane);
    }
    return;
  }

  // ---- consumers ----
  const int lr = tid / sh.tz, lz = tid % sh.tz;  // row within tile, cell within segment
  int k = 0;
  for (int tile = blockIdx.x; tile < sh.ntiles; tile += gridDim.x, ++k) {
    const int st = k % sh.stages;
    if (!mbar_wait(&full[st], (uint32_t)((k / sh.stages) & 1))) {
      if (lane == 0) atomicExch(err, 1);
      return;
    }
    const int rg = tile / sh.nseg, seg = tile % sh.nseg;
    const int row = rg * sh.rows + lr;
    const int z = 1 + seg * sh.tz + lz;
    const bool valid = lr < sh.rows && row < g.nx * g.ny && z <= g.nz;
    const int x = valid ? row / g.ny + 1 : 1, y = valid ? row % g.ny + 1 : 1;

    C f[Q];
    uint32_t bounce = 0, elide = 0;
    int ox[3], oy[3], oz[3];
    unsigned s = 0;
    if (valid) {
      s = (unsigned)sidx(g, x, y, z);
      if (sh.fused) {
        const uint2 m = stage_mask<S>(smem, sh, st, Q)[(size_t)lr * sh.tz + lz];
        bounce = m.x;
        elide = m.y;
      }
      nb_offsets(g, x, y, z, ox, oy, oz);
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const bool b = (bounce >> i) & 1u;
        if (b) {
          // bounce-back: the other slot of the pair, read from global memory
          const unsigned up = s + (unsigned)(ox[1 - Lt::c(i, 0)] + oy[1 - Lt::c(i, 1)] + oz[1 - Lt::c(i, 2)]);
          const unsigned idx = ODD ? (unsigned)Lt::inv(i) * ds + s : (unsigned)i * ds + up;
          f[i] = Store<S>::load_c(F + idx);
        } else if (ODD) {
          // upstream cell z - c_z (wrapped on a periodic z axis) inside the staged row
          const int pos = z + oz[1 - Lt::c(i, 2)] - (1 + seg * sh.tz);
          if (pos >= 0 && pos < sh.span) {
            f[i] = Store<S>::load_c(stage_pop<S>(smem, sh, st, lr, i, Q) + pos);
          } else {  // ghost z, or a periodic wrap into another segment of a long row
            const unsigned up = s + (unsigned)(ox[1 - Lt::c(i, 0)] + oy[1 - Lt::c(i, 1)] + oz[1 - Lt::c(i, 2)]);
            f[i] = Store<S>::load_c(F + (unsigned)i * ds + up);
          }
        } else {
          f[i] = Store<S>::load_c(stage_pop<S>(smem, sh, st, lr, i, Q) + lz);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[st]);  // this warp is done with the stage
    if (!valid) continue;

    C rho, u[3];
    const C cs2 = CL == CL_MLP ? C(p.cs2[s]) : C(0);
    collide_cell<Q, C, CL, Store<S>::kDev>(f, p, step_omega<C>(p), cs2, rho, u);
    if (p.write_macro) {
      const long long a = aidx(g, x, y, z);
      if (p.write_rho) rho_out[a] = rho;
      if (p.write_vel) {
        u_out[a] = u[0];
        u_out[g.L + a] = u[1];
        u_out[2 * g.L + a] = u[2];
      }
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      unsigned idx;
      if (ODD)
        idx = (unsigned)Lt::inv(i) * ds + s + (unsigned)(ox[1 + Lt::c(i, 0)] + oy[1 + Lt::c(i, 1)] + oz[1 + Lt::c(i, 2)]);
      else
        idx = (unsigned)i * ds + s;
      store_slot<S>(F + idx, f[i], (elide >> i) & 1u, p);
    }
  }
}

// Tile shape and pipeline depth for a domain; the smem per CTA is
// stages * stage_bytes.
template <int Q, class S>
inline TmaShape tma_shape(const GridDesc& g, bool fused, int blocks_per_sm) {
  TmaShape sh{};
  // tz divides the 256 consumer threads (32, 64, 128 or 256), so that rows * tz
  // is exactly 256 and no consumer thread maps past the tile's staged rows
  int tz = 32;
  while (tz < g.nz && tz < 256) tz *= 2;
  sh.tz = tz;
  sh.rows = 256 / tz;
  sh.nseg = (g.nz + tz - 1) / tz;
  const int rgroups = (g.nx * g.ny + sh.rows - 1) / sh.rows;
  sh.ntiles = rgroups * sh.nseg;
  sh.span = tz;
  sh.fused = fused ? 1 : 0;
  int bytes = sh.rows * Q * sh.span * (int)sizeof(S) + (fused ? sh.rows * tz * (int)sizeof(uint2) : 0);
  sh.stage_bytes = ((bytes + 127) / 128) * 128;
  const int budget = 200 * 1024 / blocks_per_sm;  // shared memory per CTA at the target residency
  sh.stages = std::max(2, std::min(4, budget / sh.stage_bytes));
  return sh;
}

template <int Q, class S, int CL>
cudaError_t step_tma(const DomainDev& d, const StepParams& p, int parity_in, cudaStream_t st) {
  using M = typename MacroT<S>::T;
  constexpr int target = TmaOccupancy<S, CL>::blocks;
  const TmaShape sh = tma_shape<Q, S>(d.g, p.mask != nullptr, target);
  const size_t smem = (size_t)sh.stages * sh.stage_bytes;
  static int sm_count = 0;
  static bool configured[2] = {false, false};
  if (!sm_count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
  }
  auto kern = parity_in == 0 ? k_stream_collide_tma<Q, S, CL, true> : k_stream_collide_tma<Q, S, CL, false>;
  if (!configured[parity_in]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    configured[parity_in] = true;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTmaThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = std::min(sh.ntiles, sm_count * per_sm);
  kern<<<grid, kTmaThreads, smem, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u, sh, d.err);
  return cudaGetLastError();
}

}  // namespace aslb
