// Fused AA-pattern stream-collide kernel (one interior cell per thread) and its
// launch helpers. Instantiated per lattice and storage in step_q<Q>_<type>.cu
// so the instantiations compile in parallel.
#pragma once
#include <type_traits>
#include "kernels.h"
#include "collide.cuh"

namespace aslb {

template <class S>
struct MacroT {
  using T = float;
};
template <>
struct MacroT<double> {
  using T = double;
};

// Storage offsets of the neighbours at displacement d in {-1,0,1} per axis
// (index d + 1), with periodic axes wrapping across the interior.
__device__ __forceinline__ void nb_offsets(const GridDesc& g, int x, int y, int z, int (&ox)[3], int (&oy)[3],
                                           int (&oz)[3]) {
  const int pl = (int)g.plane;
  ox[0] = -pl; ox[1] = 0; ox[2] = pl;
  oy[0] = -g.pitch; oy[1] = 0; oy[2] = g.pitch;
  oz[0] = -1; oz[1] = 0; oz[2] = 1;
  if (g.periodic & 1) {
    if (x == 1) ox[0] = (g.nx - 1) * pl;
    if (x == g.nx) ox[2] = -(g.nx - 1) * pl;
  }
  if (g.periodic & 2) {
    if (y == 1) oy[0] = (g.ny - 1) * g.pitch;
    if (y == g.ny) oy[2] = -(g.ny - 1) * g.pitch;
  }
  if (g.periodic & 4) {
    if (z == 1) oz[0] = g.nz - 1;
    if (z == g.nz) oz[2] = -(g.nz - 1);
  }
}

// Resident blocks of 256 threads per SM the register budget aims for. The
// plain FP32/FP16 kernels must keep enough loads in flight to saturate HBM:
// four blocks (64 registers) with fused links, whose per-direction slot
// selects keep the schedule compact; three (80 registers) without, where the
// compiler hoists all addresses and 64 registers would spill (two, 128
// registers, for D3Q27). Three (80 registers) for the closures, two for FP64.
template <int Q, class S, int CL, bool FUSED>
struct StepOccupancy {
  static constexpr int blocks = std::is_same<S, double>::value
                                    ? 2
                                    : (CL == CL_NONE ? (FUSED ? 4 : (Q == 27 ? 2 : 3)) : 3);
};

// Store one outgoing population. An elided slot keeps its bits: FP32/FP64
// skip the store; 2-byte storage writes back what the slot holds (bits no
// other cell writes this step), so a warp's store covers whole sectors
// instead of leaving partial ones that HBM must read to merge.
template <class S>
__device__ __forceinline__ void store_slot(S* __restrict__ slot, typename Store<S>::C v, bool elided,
                                           const StepParams& p) {
  if (sizeof(S) > 2) {
    if (!elided) *slot = Store<S>::encode(v, p);
  } else {
    S out = Store<S>::encode(v, p);
    if (elided) out = *slot;
    *slot = out;
  }
}

// Gather the Q incoming populations of cell s. MASKED: bounce bits select
// the bounce-back slot (this cell's own outgoing population: the upstream and
// own slots swap roles between representations).
template <int Q, class S, bool ODD, bool MASKED>
__device__ __forceinline__ void cell_load(const S* __restrict__ F, unsigned ds, unsigned s, const int (&ox)[3],
                                          const int (&oy)[3], const int (&oz)[3], uint32_t bounce,
                                          typename Store<S>::C (&f)[Q]) {
  using Lt = Lattice<Q>;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const bool b = MASKED && ((bounce >> i) & 1u);
    unsigned idx;
    if (ODD) {
      idx = b ? (unsigned)Lt::inv(i) * ds + s
              : (unsigned)i * ds + s + (unsigned)(ox[1 - Lt::c(i, 0)] + oy[1 - Lt::c(i, 1)] + oz[1 - Lt::c(i, 2)]);
    } else if (b) {
      idx = (unsigned)i * ds + s + (unsigned)(ox[1 - Lt::c(i, 0)] + oy[1 - Lt::c(i, 1)] + oz[1 - Lt::c(i, 2)]);
    } else {
      idx = (unsigned)Lt::inv(i) * ds + s;
    }
    f[i] = Store<S>::load_c(F + idx);
  }
}

// Collide cell (x, y, z) at storage index s, write rho / u when asked, and
// store the outgoing populations (elide bits keep the slot, store_slot).
template <int Q, class S, int CL, bool ODD, bool MASKED>
__device__ __forceinline__ void cell_finish(S* __restrict__ F, const GridDesc& g, const StepParams& p,
                                            typename MacroT<S>::T* __restrict__ rho_out,
                                            typename MacroT<S>::T* __restrict__ u_out, int x, int y, int z,
                                            unsigned s, const int (&ox)[3], const int (&oy)[3], const int (&oz)[3],
                                            uint32_t elide, typename Store<S>::C (&f)[Q],
                                            typename Store<S>::C om0) {
  using Lt = Lattice<Q>;
  using C = typename Store<S>::C;
  const unsigned ds = (unsigned)g.dstride;
  C rho, u[3];
  const C cs2 = CL == CL_MLP ? C(p.cs2[s]) : C(0);
  collide_cell<Q, C, CL, Store<S>::kDev>(f, p, om0, cs2, rho, u);
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
    store_slot<S>(F + idx, f[i], MASKED && ((elide >> i) & 1u), p);
  }
}

// ---------------------------------------------------------------------------
// Stream + collide, one interior cell per thread. ODD: representation A -> B
// (reads F[i][x - c_i], writes F[inv i][x + c_i]); EVEN: B -> A (reads
// F[inv i][x], writes F[i][x]). Element indices are 32-bit (Q * dstride < 2^32).
// FUSED: the domain has fused no-slip links (p.mask is read); chosen on the
// host so domains without them run the unmasked code. A block walks
// kOnePlanes consecutive x planes; with fused links each thread loads the
// next plane's link words one iteration ahead (the population addresses
// depend on them, so they must not cost a second memory round trip).
constexpr int kOnePlanes = 4;
template <int Q, class S, int CL, bool ODD, bool FUSED>
__global__ void __launch_bounds__(256, StepOccupancy<Q, S, CL, FUSED>::blocks)
    k_stream_collide(S* __restrict__ F, const GridDesc g, const StepParams p,
                     typename MacroT<S>::T* __restrict__ rho_out, typename MacroT<S>::T* __restrict__ u_out) {
  using C = typename Store<S>::C;
  const int z = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int x0 = blockIdx.z * kOnePlanes + 1;
  const int x1 = min(g.nx, x0 + kOnePlanes - 1);
  if (z > g.nz || y > g.ny) return;
  const unsigned pl = (unsigned)g.plane;
  const unsigned s0 = (unsigned)sidx(g, x0, y, z);
  // fused no-slip links: a fluid cell reads bounce-back populations, a solid
  // cell skips the writes the condition would overwrite
  uint2 m = make_uint2(0u, 0u);
  if (FUSED) m = p.mask[s0];
  for (int x = x0; x <= x1; ++x) {
    const unsigned s = s0 + (unsigned)(x - x0) * pl;
    uint2 mn = make_uint2(0u, 0u);
    if (FUSED && x < x1) mn = p.mask[s + pl];
    int ox[3], oy[3], oz[3];
    nb_offsets(g, x, y, z, ox, oy, oz);
    C f[Q];
    cell_load<Q, S, ODD, FUSED>(F, (unsigned)g.dstride, s, ox, oy, oz, m.x, f);
    cell_finish<Q, S, CL, ODD, FUSED>(F, g, p, rho_out, u_out, x, y, z, s, ox, oy, oz, m.y, f, step_omega<C>(p));
    m = mn;
  }
}

// Two cells per thread, z and z + 32 of the same row: a warp covers 64
// consecutive cells, and each thread has the loads of both cells in flight
// before it collides the first, which doubles the bytes in flight per
// register-limited warp. Used for the plain (no closure) FP32 step of
// D3Q15/D3Q19 domains with fused links, at 768 threads (80 registers) per
// SM; without fused links the schedule hoists every address of both cells
// (over 128 registers), and with FP16 storage (fewer bytes, more
// instructions) the one-cell kernel is faster.
// M32: the links come from the one-word mask (p.mask32). A block walks
// kPairPlanes consecutive x planes; each thread loads the fused-link words of
// the next plane one iteration ahead, so that the population loads, whose
// addresses those words select, do not wait for a second memory round trip.
constexpr int kPairPlanes = 2;
// Blocks of 128 threads, six per SM (80 registers, the residency of three
// 256-thread blocks): the smaller blocks measured 0.8 % faster.
constexpr int kPairThreads = 128;
template <int Q, class S, bool ODD, bool FUSED, bool M32>
__global__ void __launch_bounds__(kPairThreads, 768 / kPairThreads)
    k_stream_collide_pair(S* __restrict__ F, const GridDesc g, const StepParams p,
                          typename MacroT<S>::T* __restrict__ rho_out, typename MacroT<S>::T* __restrict__ u_out) {
  using C = typename Store<S>::C;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int za = blockIdx.x * (2 * blockDim.x) + 64 * w + lane + 1;
  const int zb = za + 32;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int x0 = blockIdx.z * kPairPlanes + 1;
  const int x1 = min(g.nx, x0 + kPairPlanes - 1);
  if (za > g.nz || y > g.ny) return;
  const bool has_b = zb <= g.nz;
  const unsigned ds = (unsigned)g.dstride;
  const unsigned pl = (unsigned)g.plane;
  const unsigned s0 = (unsigned)sidx(g, x0, y, za);
  const C om0 = step_omega<C>(p);
  // the fused-link words of the next plane are loaded one plane ahead, so the
  // population loads (whose addresses they select) never wait for them
  uint2 wa = make_uint2(0u, 0u), wb = make_uint2(0u, 0u);
  if (FUSED && M32) {
    wa.x = p.mask32[s0];
    if (has_b) wb.x = p.mask32[s0 + 32u];
  } else if (FUSED) {
    wa = p.mask[s0];
    if (has_b) wb = p.mask[s0 + 32u];
  }
  for (int x = x0; x <= x1; ++x) {
    const unsigned sa = s0 + (unsigned)(x - x0) * pl;
    const unsigned sb = sa + 32u;
    uint2 na = make_uint2(0u, 0u), nb = make_uint2(0u, 0u);
    if (FUSED && x < x1) {
      if (M32) {
        na.x = p.mask32[sa + pl];
        if (has_b) nb.x = p.mask32[sb + pl];
      } else {
        na = p.mask[sa + pl];
        if (has_b) nb = p.mask[sb + pl];
      }
    }
    uint2 ma = wa, mb = wb;
    if (FUSED && M32) {
      ma = (wa.x >> 31) ? make_uint2(0u, wa.x & 0x7fffffffu) : make_uint2(wa.x, 0u);
      mb = (wb.x >> 31) ? make_uint2(0u, wb.x & 0x7fffffffu) : make_uint2(wb.x, 0u);
    }
    int ox[3], oy[3], oza[3], ozb[3];
    nb_offsets(g, x, y, za, ox, oy, oza);
    ozb[0] = -1;  // zb >= 33: the lower neighbour never wraps
    ozb[1] = 0;
    ozb[2] = ((g.periodic & 4) && zb == g.nz) ? -(g.nz - 1) : 1;
    C fa[Q], fb[Q];
    cell_load<Q, S, ODD, FUSED>(F, ds, sa, ox, oy, oza, ma.x, fa);
    if (has_b) cell_load<Q, S, ODD, FUSED>(F, ds, sb, ox, oy, ozb, mb.x, fb);
    cell_finish<Q, S, CL_NONE, ODD, FUSED>(F, g, p, rho_out, u_out, x, y, za, sa, ox, oy, oza, ma.y, fa, om0);
    if (has_b) cell_finish<Q, S, CL_NONE, ODD, FUSED>(F, g, p, rho_out, u_out, x, y, zb, sb, ox, oy, ozb, mb.y, fb, om0);
    wa = na;
    wb = nb;
  }
}

inline void step_launch_shape(const GridDesc& g, dim3& grid, dim3& block) {
  int tz = ((g.nz + 31) / 32) * 32;
  if (tz > 256) tz = 256;
  int ty = 256 / tz;
  block = dim3(tz, ty, 1);
  grid = dim3((g.nz + tz - 1) / tz, (g.ny + ty - 1) / ty, g.nx);
}

// The one-cell stream-collide: the same blocks, kOnePlanes x planes each.
inline void plane_launch_shape(const GridDesc& g, dim3& grid, dim3& block) {
  step_launch_shape(g, grid, block);
  grid.z = (g.nx + kOnePlanes - 1) / kOnePlanes;
}

// Launch of the TMA-staged variant (stream_collide_tma.cuh).
template <int Q, class S, int CL>
cudaError_t step_tma(const DomainDev& d, const StepParams& p, int parity_in, cudaStream_t st);

// Two-cells-per-thread shape: 32-thread groups cover 64 cells of a row.
inline void pair_launch_shape(const GridDesc& g, dim3& grid, dim3& block) {
  int tz = ((g.nz + 63) / 64) * 32;
  if (tz > kPairThreads) tz = kPairThreads;
  int ty = kPairThreads / tz;
  block = dim3(tz, ty, 1);
  grid = dim3((g.nz + 2 * tz - 1) / (2 * tz), (g.ny + ty - 1) / ty, (g.nx + kPairPlanes - 1) / kPairPlanes);
}

template <int Q, class S, int CL>
cudaError_t step_q_s_cl(const DomainDev& d, const StepParams& p, int parity_in, cudaStream_t st) {
  if (d.variant == 1) return step_tma<Q, S, CL>(d, p, parity_in, st);
  dim3 grid, block;
  using M = typename MacroT<S>::T;
  const bool fused = p.mask != nullptr;
  if constexpr (CL == CL_NONE && Q != 27 && std::is_same<S, float>::value) {
    if (d.variant == 0 && fused) {
      pair_launch_shape(d.g, grid, block);
      const bool m32 = p.mask32 != nullptr;
      if (parity_in == 0) {
        if (m32) k_stream_collide_pair<Q, S, true, true, true><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
        else k_stream_collide_pair<Q, S, true, true, false><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
      } else {
        if (m32) k_stream_collide_pair<Q, S, false, true, true><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
        else k_stream_collide_pair<Q, S, false, true, false><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
      }
      return cudaGetLastError();
    }
  }
  plane_launch_shape(d.g, grid, block);
  if (parity_in == 0) {
    if (fused)
      k_stream_collide<Q, S, CL, true, true><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
    else
      k_stream_collide<Q, S, CL, true, false><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
  } else {
    if (fused)
      k_stream_collide<Q, S, CL, false, true><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
    else
      k_stream_collide<Q, S, CL, false, false><<<grid, block, 0, st>>>((S*)d.F, d.g, p, (M*)d.rho, (M*)d.u);
  }
  return cudaGetLastError();
}

template <int Q, class S>
cudaError_t step_q_s(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st) {
  switch (closure) {
    case CL_NONE: return step_q_s_cl<Q, S, CL_NONE>(d, p, parity_in, st);
    case CL_ASL_INTENT: return step_q_s_cl<Q, S, CL_ASL_INTENT>(d, p, parity_in, st);
    case CL_SMAGORINSKY: return step_q_s_cl<Q, S, CL_SMAGORINSKY>(d, p, parity_in, st);
    case CL_MLP:
      // The learned closure is built for the lattices and storages it is trained for.
      if constexpr ((Q == 19 || Q == 27) && !std::is_same<S, double>::value)
        return step_q_s_cl<Q, S, CL_MLP>(d, p, parity_in, st);
      else
        return cudaErrorNotSupported;
  }
  return cudaErrorInvalidValue;
}

template <int Q>
cudaError_t step_q(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st) {
  switch (d.storage) {
    case ST_F32: return step_q_s<Q, float>(d, p, closure, parity_in, st);
    case ST_F16: return step_q_s<Q, __half>(d, p, closure, parity_in, st);
    case ST_F64: return step_q_s<Q, double>(d, p, closure, parity_in, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace aslb
