// Fused AA-pattern stream-collide kernel (one interior cell per thread) and its
// launch helpers. Instantiated per lattice and storage in step_q<Q>_<type>.cu
// so the instantiations compile in parallel.
#pragma once
#include <algorithm>
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

// Store one outgoing population unless its slot is elided (the slot keeps its
// bits). In the AA pattern a cell writes exactly the slots it read moments
// before, so the lines are still in L2 and a warp's partial store merges there
// without an HBM read.
template <class S>
__device__ __forceinline__ void store_slot(S* __restrict__ slot, typename Store<S>::C v, bool elided,
                                           const StepParams& p) {
  if (!elided) *slot = Store<S>::encode(v, p);
}

// Gather the Q incoming populations of cell s. MASKED: bounce bits select
// the bounce-back slot (this cell's own outgoing population: the upstream and
// own slots swap roles between representations). Offsets from the periodic
// wrap (nb_offsets): the slow path of cells on a periodic face.
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

// The same gather for a cell whose neighbours do not wrap: every slot is the
// cell's index plus a precomputed offset (p.slot).
template <int Q, class S, bool ODD, bool MASKED>
__device__ __forceinline__ void cell_load_flat(const S* __restrict__ F, unsigned s, const StepParams& p,
                                               uint32_t bounce, typename Store<S>::C (&f)[Q]) {
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const bool b = MASKED && ((bounce >> i) & 1u);
    // ODD: pull, or the opposite own slot when bounced; EVEN: the reverse
    const unsigned off = (ODD != b) ? p.slot[0][i] : p.slot[3][i];
    f[i] = Store<S>::load_c(F + (s + off));
  }
}

// Collide cell (x, y, z) at storage index s and write rho / u when asked;
// f becomes the outgoing populations.
template <int Q, class S, int CL>
__device__ __forceinline__ void cell_collide(const GridDesc& g, const StepParams& p,
                                             typename MacroT<S>::T* __restrict__ rho_out,
                                             typename MacroT<S>::T* __restrict__ u_out, int x, int y, int z,
                                             unsigned s, typename Store<S>::C (&f)[Q], typename Store<S>::C om0) {
  using C = typename Store<S>::C;
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
}

// Store the outgoing populations (elide bits keep the slot), wrap-aware.
template <int Q, class S, bool ODD, bool MASKED>
__device__ __forceinline__ void cell_store(S* __restrict__ F, const StepParams& p, unsigned ds, unsigned s,
                                           const int (&ox)[3], const int (&oy)[3], const int (&oz)[3],
                                           uint32_t elide, const typename Store<S>::C (&f)[Q]) {
  using Lt = Lattice<Q>;
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

// s, seen by the compiler as computed after v: addresses derived from the
// result cannot be hoisted above the collision that produced v (hoisted, the
// Q store addresses of a cell would stay live across it and spill).
__device__ __forceinline__ unsigned after(unsigned s, float v) {
  asm volatile("" : "+r"(s) : "f"(v));
  return s;
}
__device__ __forceinline__ unsigned after(unsigned s, double v) {
  asm volatile("" : "+r"(s) : "d"(v));
  return s;
}

// The same stores for a cell whose neighbours do not wrap (p.slot).
template <int Q, class S, bool ODD, bool MASKED>
__device__ __forceinline__ void cell_store_flat(S* __restrict__ F, const StepParams& p, unsigned s, uint32_t elide,
                                                const typename Store<S>::C (&f)[Q]) {
  const unsigned sl = after(s, f[0]);
#pragma unroll
  for (int i = 0; i < Q; ++i)
    store_slot<S>(F + (sl + (ODD ? p.slot[2][i] : p.slot[1][i])), f[i], MASKED && ((elide >> i) & 1u), p);
}

// Collision and wrap-aware stores of one cell (the batched step's form).
template <int Q, class S, int CL, bool ODD, bool MASKED>
__device__ __forceinline__ void cell_finish(S* __restrict__ F, const GridDesc& g, const StepParams& p,
                                            typename MacroT<S>::T* __restrict__ rho_out,
                                            typename MacroT<S>::T* __restrict__ u_out, int x, int y, int z,
                                            unsigned s, const int (&ox)[3], const int (&oy)[3], const int (&oz)[3],
                                            uint32_t elide, typename Store<S>::C (&f)[Q],
                                            typename Store<S>::C om0) {
  cell_collide<Q, S, CL>(g, p, rho_out, u_out, x, y, z, s, f, om0);
  cell_store<Q, S, ODD, MASKED>(F, p, (unsigned)g.dstride, s, ox, oy, oz, elide, f);
}

// Whether any neighbour of a cell with coordinate v on a periodic axis of n
// interior cells wraps to the opposite face.
__device__ __forceinline__ bool wraps(int periodic_bit, int v, int n) { return periodic_bit && (v == 1 || v == n); }

// ---------------------------------------------------------------------------
// Cells on periodic faces, whose neighbours wrap to the opposite face, are
// skipped by the main blocks of a stream-collide launch (by their loop range,
// so the main loop has no branch) and advanced by extra blocks of the same
// launch, one cell per thread with the wrap-aware offsets (disjoint cells:
// the AA update of a cell touches only its own slots). The face cells lie on
// up to eight planes: the two faces of every periodic axis and, with the
// two-cells-per-thread kernel (which skips both cells of a pair when either
// wraps), the planes of the z partners of the skipped pairs. A cell on
// several planes belongs to the first that holds it. The face blocks come
// first in the grid (blockIdx.z < fz), so they run alongside the main blocks
// instead of after them.
struct FaceWork {
  int n;          // planes
  int axis[8];
  int coord[8];
  int start[9];   // prefix sums of the planes' cell counts
  int fz;         // grid z-slices of face blocks
};

template <int Q, class S, int CL, bool ODD, bool FUSED>
__device__ __forceinline__ void face_cell(S* __restrict__ F, const GridDesc& g, const StepParams& p,
                                          const FaceWork& fw, typename MacroT<S>::T* __restrict__ rho_out,
                                          typename MacroT<S>::T* __restrict__ u_out) {
  using C = typename Store<S>::C;
  const int threads = blockDim.x * blockDim.y;
  const long long blk = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const long long c = blk * threads + threadIdx.y * blockDim.x + threadIdx.x;
  if (c >= fw.start[fw.n]) return;
  int k = 0;
  while (c >= fw.start[k + 1]) ++k;
  const int r = (int)(c - fw.start[k]);
  const int axis = fw.axis[k];
  // in-plane coordinates: the two other axes in order
  const int nu = axis == 0 ? g.ny : g.nx;
  const int nv = axis == 2 ? g.ny : g.nz;
  (void)nu;
  const int u = r / nv + 1, v = r % nv + 1;
  const int x = axis == 0 ? fw.coord[k] : u;
  const int y = axis == 1 ? fw.coord[k] : (axis == 0 ? u : v);
  const int z = axis == 2 ? fw.coord[k] : v;
  for (int j = 0; j < k; ++j)
    if ((fw.axis[j] == 0 ? x : (fw.axis[j] == 1 ? y : z)) == fw.coord[j]) return;
  const unsigned s = (unsigned)sidx(g, x, y, z);
  uint2 m = make_uint2(0u, 0u);
  if (FUSED) m = p.mask[s];
  int ox[3], oy[3], oz[3];
  nb_offsets(g, x, y, z, ox, oy, oz);
  C f[Q];
  cell_load<Q, S, ODD, FUSED>(F, (unsigned)g.dstride, s, ox, oy, oz, m.x, f);
  cell_collide<Q, S, CL>(g, p, rho_out, u_out, x, y, z, s, f, step_omega<C>(p));
  cell_store<Q, S, ODD, FUSED>(F, p, (unsigned)g.dstride, s, ox, oy, oz, m.y, f);
}

// The face planes of a domain and the grid z-slices their cells need with
// blocks of `threads` threads on a gx x gy grid face. paired: the main
// kernel is the two-cells-per-thread kernel, whose pairs are (z, z + 32) for
// z - 1 mod 64 < 32: with a periodic z it also skips cell 33 (partner of
// z = 1) and, when nz is the second cell of its pair, cell nz - 32.
inline FaceWork face_work(const GridDesc& g, bool paired, int threads, int gx, int gy) {
  FaceWork fw{};
  const int n[3] = {g.nx, g.ny, g.nz};
  auto add = [&](int a, int c) {
    for (int j = 0; j < fw.n; ++j)
      if (fw.axis[j] == a && fw.coord[j] == c) return;
    fw.axis[fw.n] = a;
    fw.coord[fw.n] = c;
    const int cells = (a == 0 ? g.ny * g.nz : (a == 1 ? g.nx * g.nz : g.nx * g.ny));
    fw.start[fw.n + 1] = fw.start[fw.n] + cells;
    ++fw.n;
  };
  for (int a = 0; a < 3; ++a)
    if ((g.periodic >> a) & 1) {
      add(a, 1);
      add(a, n[a]);
    }
  if (paired && (g.periodic & 4)) {
    if (g.nz >= 33) add(2, 33);
    if ((g.nz - 1) % 64 >= 32) add(2, g.nz - 32);
  }
  const long long per_slice = (long long)threads * gx * gy;
  fw.fz = (int)((fw.start[fw.n] + per_slice - 1) / per_slice);
  return fw;
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
    k_stream_collide(S* __restrict__ F, const __grid_constant__ GridDesc g, const __grid_constant__ StepParams p,
                     const __grid_constant__ FaceWork fw, typename MacroT<S>::T* __restrict__ rho_out,
                     typename MacroT<S>::T* __restrict__ u_out) {
  using C = typename Store<S>::C;
  if ((int)blockIdx.z < fw.fz) {
    face_cell<Q, S, CL, ODD, FUSED>(F, g, p, fw, rho_out, u_out);
    return;
  }
  const int z = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  int x0 = (blockIdx.z - fw.fz) * kOnePlanes + 1;
  int x1 = min(g.nx, x0 + kOnePlanes - 1);
  if (z > g.nz || y > g.ny) return;
  // cells whose neighbours wrap across a periodic face belong to the face
  // kernel; skipped by the loop's range, the loop body has no branch
  if (wraps(g.periodic & 2, y, g.ny) || wraps(g.periodic & 4, z, g.nz)) return;
  if (g.periodic & 1) {
    x0 = max(x0, 2);
    x1 = min(x1, g.nx - 1);
    if (x0 > x1) return;
  }
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
    C f[Q];
    cell_load_flat<Q, S, ODD, FUSED>(F, s, p, m.x, f);
    cell_collide<Q, S, CL>(g, p, rho_out, u_out, x, y, z, s, f, step_omega<C>(p));
    cell_store_flat<Q, S, ODD, FUSED>(F, p, s, m.y, f);
    m = mn;
  }
}

// Two cells per thread, z and z + 32 of the same row: a warp covers 64
// consecutive cells, and each thread has the loads of both cells in flight
// before it collides the first, which doubles the bytes in flight per
// register-limited warp. Used for the plain (no closure) FP32 and FP16 steps
// of D3Q15/D3Q19 domains with fused links, at 768 threads (80 registers) per
// SM (FP16 porous channel: 0.704 ms against 0.786 ms with one cell per
// thread).
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
    k_stream_collide_pair(S* __restrict__ F, const __grid_constant__ GridDesc g,
                          const __grid_constant__ StepParams p, const __grid_constant__ FaceWork fw,
                          typename MacroT<S>::T* __restrict__ rho_out, typename MacroT<S>::T* __restrict__ u_out) {
  using C = typename Store<S>::C;
  if ((int)blockIdx.z < fw.fz) {
    face_cell<Q, S, CL_NONE, ODD, FUSED>(F, g, p, fw, rho_out, u_out);
    return;
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int za = blockIdx.x * (2 * blockDim.x) + 64 * w + lane + 1;
  const int zb = za + 32;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  int x0 = (blockIdx.z - fw.fz) * kPairPlanes + 1;
  int x1 = min(g.nx, x0 + kPairPlanes - 1);
  if (za > g.nz || y > g.ny) return;
  const bool has_b = zb <= g.nz;
  // A pair with a cell whose neighbours wrap across a periodic face is left to
  // the face kernel (both cells; face_planes lists the partners). Skipping
  // by the loop's range keeps the loop body free of branches.
  if (wraps(g.periodic & 2, y, g.ny) || wraps(g.periodic & 4, za, g.nz) || (has_b && (g.periodic & 4) && zb == g.nz))
    return;
  if (g.periodic & 1) {
    x0 = max(x0, 2);
    x1 = min(x1, g.nx - 1);
    if (x0 > x1) return;
  }
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
    C fa[Q], fb[Q];
    cell_load_flat<Q, S, ODD, FUSED>(F, sa, p, ma.x, fa);
    if (has_b) cell_load_flat<Q, S, ODD, FUSED>(F, sb, p, mb.x, fb);
    cell_collide<Q, S, CL_NONE>(g, p, rho_out, u_out, x, y, za, sa, fa, om0);
    cell_store_flat<Q, S, ODD, FUSED>(F, p, sa, ma.y, fa);
    if (has_b) {
      cell_collide<Q, S, CL_NONE>(g, p, rho_out, u_out, x, y, zb, sb, fb, om0);
      cell_store_flat<Q, S, ODD, FUSED>(F, p, sb, mb.y, fb);
    }
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
  S* F = (S*)d.F;
  M* rho = (M*)d.rho;
  M* u = (M*)d.u;
  if constexpr (CL == CL_NONE && Q != 27 && !std::is_same<S, double>::value) {
    if (d.variant == 0 && fused) {
      pair_launch_shape(d.g, grid, block);
      const FaceWork fw = face_work(d.g, true, block.x * block.y, grid.x, grid.y);
      grid.z += fw.fz;
      const bool m32 = p.mask32 != nullptr;
      if (parity_in == 0) {
        if (m32) k_stream_collide_pair<Q, S, true, true, true><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
        else k_stream_collide_pair<Q, S, true, true, false><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
      } else {
        if (m32) k_stream_collide_pair<Q, S, false, true, true><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
        else k_stream_collide_pair<Q, S, false, true, false><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
      }
      return cudaGetLastError();
    }
  }
  plane_launch_shape(d.g, grid, block);
  const FaceWork fw = face_work(d.g, false, block.x * block.y, grid.x, grid.y);
  grid.z += fw.fz;
  if (parity_in == 0) {
    if (fused) k_stream_collide<Q, S, CL, true, true><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
    else k_stream_collide<Q, S, CL, true, false><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
  } else {
    if (fused) k_stream_collide<Q, S, CL, false, true><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
    else k_stream_collide<Q, S, CL, false, false><<<grid, block, 0, st>>>(F, d.g, p, fw, rho, u);
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
