// Finite-difference advection-diffusion coupled to the LBGK velocity field:
// ASL's FDAdvectionDiffusion (src/num/aslFDAdvectionDiffusion.cxx:88-180,
// 209-226) for one component with a constant diffusion coefficient D,
//   c' = D lap(c) + c - divProduct(u, c)
//   (compressibility correction: c' /= 1 - div(u); c' += lap(c) |u(x)|^2 / 2)
// and, with setElectricFieldParameters (:66-74, 166-172), c' -= divAgradB(c q / k, phi),
// with the stencil operators of src/math/aslTemplateVE.cxx:164-280 on the
// templates d3q7 / d3q15 / d3q19 (laplacian and gradient coefficients of
// src/math/aslTemplates.cxx:134-186):
//   lap(c)            = sum_i LC_i c(x + e_i)
//   div(u)            = sum_d sum_i GC_i e_i,d u_d(x + e_i)
//   divProduct(u, c)  = sum_d sum_i GC_i e_i,d (u_d(x + e_i) + u_d(x)) (c(x + e_i) + c(x)) / 2
//   divAgradB(a, b)   = sum_i GC_i (a(x + e_i) + a(x)) (b(x + e_i) - b(x))
// The update writes the interior of a second buffer and the buffers swap
// (postProcessing), so ghost values persist in both: they are the
// boundary values (BCConstantValue on faces, src/num/aslBasicBC.cxx:51-57).
// The velocity is the bound LBGK's device velocity field (ASL layout, FP32,
// FP64 for FP64 storage), read on that domain's stream after its step.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>
#include <nvtx3/nvToolsExt.h>
#include "aslb.h"
#include "kernels.h"
#include "lattice.cuh"

namespace aslb {
namespace {

// Template vectors: d3q7, d3q15 and d3q19 list their vectors in the order of
// the lattice tables (d3q7 is the first seven of d3q19). Coefficients by
// vector class: rest, axis, diagonal.
template <int Q>
struct FdTemplate {
  __host__ __device__ static constexpr int e(int i, int d) { return Q == 15 ? lat_c15(i, d) : lat_c27(i, d); }
  __host__ __device__ static constexpr double lc(int i) {
    return i == 0 ? (Q == 7 ? -6.0 : Q == 15 ? -14.0 / 3.0 : -4.0)
                  : (i <= 6 ? (Q == 7 ? 1.0 : Q == 15 ? 2.0 / 3.0 : 1.0 / 3.0) : (Q == 15 ? 1.0 / 12.0 : 1.0 / 6.0));
  }
  __host__ __device__ static constexpr double gc(int i) {
    return i == 0 ? 0.0
                  : (i <= 6 ? (Q == 7 ? 0.5 : Q == 15 ? 1.0 / 3.0 : 1.0 / 6.0) : (Q == 15 ? 1.0 / 24.0 : 1.0 / 12.0));
  }
};

struct FdGrid {
  int nx, ny, nz, gx, gy, gz;
  long long L;
};

// The update of one cell from its stencil values: cv(i) = c(x + e_i),
// uv(d, i) = u_d(x + e_i).
template <int Q, class T, bool U, bool E, class CV, class UV, class EV>
__device__ __forceinline__ T fd_cell(CV cvf, UV uvf, EV evf, T D, int cc) {
  using Tp = FdTemplate<Q>;
  T cv[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) cv[i] = cvf(i);
  T lap = T(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) lap += T(Tp::lc(i)) * cv[i];
  T cnew = D * lap + cv[0];
  if (U) {
    T dp[3], dv[3], u0[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) u0[d] = uvf(d, 0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T s = T(0), v = T(0);
#pragma unroll
      for (int i = 1; i < Q; ++i) {
        if (Tp::e(i, d) == 0) continue;
        const T ui = uvf(d, i);
        const T coef = T(Tp::gc(i) * Tp::e(i, d));
        s += T(0.5) * ((ui + u0[d]) * (cv[i] + cv[0])) * coef;
        v += coef * ui;
      }
      dp[d] = s;
      dv[d] = v;
    }
    cnew -= dp[0] + dp[1] + dp[2];
    if (cc) {
      cnew /= T(1) - (dv[0] + dv[1] + dv[2]);
      cnew += lap * (u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2]) * T(0.5);
    }
  }
  if (E) {
    // electric term: - divAgradB(c q / k, phi) = - sum_i GC_i (a_i + a_0) (phi_i - phi_0),
    // a = c q / k (evf(0, i) = phi, evf(1, i) = k, evf(2, i) = q at x + e_i)
    const T a0 = cv[0] * evf(2, 0) / evf(1, 0), p0 = evf(0, 0);
    T s = T(0);
#pragma unroll
    for (int i = 1; i < Q; ++i) s += T(Tp::gc(i)) * (cv[i] * evf(2, i) / evf(1, i) + a0) * (evf(0, i) - p0);
    cnew -= s;
  }
  return cnew;
}

// First nonzero component's sign of e_i (pairs i, opp(i) share |q_i|).
template <int Q>
__host__ __device__ constexpr int fd_lead_sign(int i) {
  return FdTemplate<Q>::e(i, 0) != 0 ? FdTemplate<Q>::e(i, 0)
                                     : (FdTemplate<Q>::e(i, 1) != 0 ? FdTemplate<Q>::e(i, 1) : FdTemplate<Q>::e(i, 2));
}

// The update without the electric term, regrouped per link i of the
// template (the same sums as fd_cell, in another order; fewer additions,
// which the register-blocked kernel needs, while the 2.5-D kernel's d3q7
// step ran 1.4 % slower with it):
//   divProduct = sum_i GC_i / 2 (c_i + c_0) (p_i + q_i),
//   p_i = e_i . u(x + e_i), q_i = e_i . u(x), div(u) = sum_i GC_i p_i,
// with the laplacian and both sums accumulated per coefficient class (axis,
// edge or corner vectors) and scaled once; q_i = -q_opp(i) is formed once
// per pair. cvf(i) = c(x + e_i), uvf(d, i) = u_d(x + e_i).
template <int Q, class T, bool U, bool CC, class CV, class UV>
__device__ __forceinline__ T fd_cell_links(CV cvf, UV uvf, T D) {
  using Tp = FdTemplate<Q>;
  const T c0 = cvf(0);
  T q0[3] = {T(0), T(0), T(0)};
  if constexpr (U) {
    q0[0] = uvf(0, 0);
    q0[1] = uvf(1, 0);
    q0[2] = uvf(2, 0);
  }
  T la = T(0), ld = T(0), aa = T(0), ad = T(0), va = T(0), vd = T(0);
#pragma unroll
  for (int i = 1; i < Q; ++i) {
    const T ci = cvf(i);
    const bool axis = i <= 6, first = i == 1 || i == 7;
    if (axis) la = first ? ci : la + ci; else ld = first ? ci : ld + ci;
    if constexpr (U) {
      // p = e_i . u(x + e_i); q = s e_i . u(x) with s the sign that makes
      // the leading component positive (the same sum for i and opp(i))
      const int sg = fd_lead_sign<Q>(i);
      T p = T(0), qc = T(0);
      bool fp = true;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int ed = Tp::e(i, d);
        if (ed == 0) continue;
        const T ud = uvf(d, i);
        p = fp ? (ed > 0 ? ud : -ud) : (ed > 0 ? p + ud : p - ud);
        qc = fp ? q0[d] : (ed * sg > 0 ? qc + q0[d] : qc - q0[d]);
        fp = false;
      }
      const T pq = sg > 0 ? p + qc : p - qc;
      const T m = ci + c0;
      if (axis) aa = first ? m * pq : fma(m, pq, aa); else ad = first ? m * pq : fma(m, pq, ad);
      if constexpr (CC) {
        if (axis) va = first ? p : va + p; else vd = first ? p : vd + p;
      }
    }
  }
  const T lap = T(Tp::lc(0)) * c0 + T(Tp::lc(1)) * la + (Q > 7 ? T(Tp::lc(7)) * ld : T(0));
  T cnew = D * lap + c0;
  if constexpr (U) {
    cnew -= T(0.5 * Tp::gc(1)) * aa + (Q > 7 ? T(0.5 * Tp::gc(7)) * ad : T(0));
    if constexpr (CC) {
      cnew /= T(1) - (T(Tp::gc(1)) * va + (Q > 7 ? T(Tp::gc(7)) * vd : T(0)));
      cnew += lap * (q0[0] * q0[0] + q0[1] * q0[1] + q0[2] * q0[2]) * T(0.5);
    }
  }
  return cnew;
}

// 2.5-D tiling: a block of 32 x 8 threads owns a 32 (z) x 8 (y) column of
// cells and walks kFdPlanes x planes, keeping three planes of c (and u) with
// a one-cell halo in shared memory, so every value is read from HBM about
// once (the y/z halos of neighbouring tiles come from L2) and every
// neighbour read of the stencil is a shared-memory load. (32 x 8 tiles step
// the d3q7 stencil 5 % faster than 64 x 4 ones.)
constexpr int kFdTZ = 32, kFdTY = 8, kFdPlanes = 32;

template <int Q, class T, bool U, bool E>
__global__ void __launch_bounds__(kFdTZ * kFdTY) k_fd_step(const T* __restrict__ c, T* __restrict__ cn,
                                                          const T* __restrict__ u, const T* __restrict__ ef,
                                                          FdGrid g, T D, int cc) {
  using Tp = FdTemplate<Q>;
  // fields per plane: c, then u (3) with a velocity, then phi, k, q with the electric term
  constexpr int UB = 1, EB = U ? 4 : 1;
  constexpr int W = kFdTZ + 2, H = kFdTY + 2, P = W * H, NF = 1 + (U ? 3 : 0) + (E ? 3 : 0);
  // three planes of the tile (dynamic: FP64 with velocity and electric fields
  // needs 56 KB)
  extern __shared__ __align__(16) unsigned char fd_smem[];
  auto sm = reinterpret_cast<T(*)[NF][P]>(fd_smem);
  const int tz = threadIdx.x, ty = threadIdx.y, t = ty * kFdTZ + tz;
  const int z0 = blockIdx.x * kFdTZ, y0 = blockIdx.y * kFdTY;  // ghosted origin of the tile
  const int x0 = blockIdx.z * kFdPlanes + 1, x1 = min(g.nx, x0 + kFdPlanes - 1);
  const int z = z0 + tz + 1, y = y0 + ty + 1;
  const bool active = z <= g.nz && y <= g.ny;
  // each thread owns tile entries t and t + 256 (P <= 512): a plane is
  // fetched into registers one iteration ahead, so its HBM latency overlaps
  // the arithmetic of the current plane
  constexpr int NT = kFdTZ * kFdTY;
  static_assert(P <= 2 * NT, "two tile entries per thread");
  T r[2][NF];
  auto fetch = [&](int xp) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int e = t + k * NT;
      const int yy = y0 + e / W, zz = z0 + e % W;
      if (e < P && yy < g.gy && zz < g.gz) {
        const long long a = ((long long)xp * g.gy + yy) * g.gz + zz;
        r[k][0] = c[a];
        if (U) {
          r[k][UB % NF] = u[a];
          r[k][(UB + 1) % NF] = u[g.L + a];
          r[k][(UB + 2) % NF] = u[2 * g.L + a];
        }
        if (E) {
          r[k][EB % NF] = ef[a];
          r[k][(EB + 1) % NF] = ef[g.L + a];
          r[k][(EB + 2) % NF] = ef[2 * g.L + a];
        }
      }
    }
  };
  auto stash = [&](int xp) {
    const int slot = xp % 3;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int e = t + k * NT;
      if (e < P)
#pragma unroll
        for (int f = 0; f < NF; ++f) sm[slot][f][e] = r[k][f];
    }
  };
  fetch(x0 - 1);
  stash(x0 - 1);
  fetch(x0);
  stash(x0);
  fetch(x0 + 1);
  for (int x = x0; x <= x1; ++x) {
    stash(x + 1);  // into the slot plane x - 2 used; everyone passed the barrier below
    __syncthreads();
    if (x < x1) fetch(x + 2);
    if (active) {
      const int sl[3] = {(x + 2) % 3, x % 3, (x + 1) % 3};
      const int base = (ty + 1) * W + tz + 1;
      auto cvf = [&](int i) { return sm[sl[1 + Tp::e(i, 0)]][0][base + Tp::e(i, 1) * W + Tp::e(i, 2)]; };
      auto uvf = [&](int d, int i) { return sm[sl[1 + Tp::e(i, 0)]][U ? UB + d : 0][base + Tp::e(i, 1) * W + Tp::e(i, 2)]; };
      auto evf = [&](int f, int i) { return sm[sl[1 + Tp::e(i, 0)]][E ? EB + f : 0][base + Tp::e(i, 1) * W + Tp::e(i, 2)]; };
      cn[((long long)x * g.gy + y) * g.gz + z] = fd_cell<Q, T, U, E>(cvf, uvf, evf, D, cc);
    }
    __syncthreads();
  }
}

// Register-blocked FP32 step (no electric term) for the d3q15 / d3q19
// templates: a block of 32 (z) x 4 (y) threads owns a 64 x 16 tile of a
// plane, each thread a 4 x 2 block of cells (two consecutive z, four
// consecutive y). Three planes of the tile with its one-cell halo sit in a
// ring of four shared-memory slots; plane x + 2 is loaded into registers
// during plane x and stored to its slot at the top of the next iteration.
// The stencil reads of a thread's cells overlap, the unrolled cells read each
// shared value once, and a thread's two middle columns are one 8-byte load
// (about 19 shared loads per d3q19 cell instead of 52). The update is
// fd_cell_links (ASL's sums regrouped per link). Work: the tiles' planes in
// tile-major order, an equal run of them per resident block (a run that
// crosses into the next tile restarts the ring there).
constexpr int kRbTZ = 32;

// The tile and its ring (two resident blocks of 128 threads per SM: eight
// cells per thread outweigh the lower occupancy; 198 registers). KZ
// consecutive z cells per thread: with two, a row's columns are shifted by
// one (column c holds z0 - 1 + c) so each thread's pair sits on an 8-byte
// boundary and is one shared load.
struct RbConf {
  static constexpr int TY = 4, KY = 4, KZ = 2, MINB = 2;
  static constexpr int CO = KZ == 2 ? 1 : 0;       // column of ghosted z0
  static constexpr int TZ = kRbTZ * KZ;            // tile cells along z
  static constexpr int H = TY * KY + 2;            // tile rows with the halo
  static constexpr int W = TZ + 2 + 2 * CO;        // tile columns with the halo
  static constexpr int P = H * W;                  // entries of one field plane
  static constexpr int NT = kRbTZ * TY;            // threads
  static constexpr int E = (P + NT - 1) / NT;      // entries per thread
  static constexpr int S = 4;                      // ring slots
  static_assert(KZ == 1 || KZ == 2, "one or two z cells per thread");
};

template <bool U>
constexpr size_t fd_rb_smem() {
  return (size_t)RbConf::S * (U ? 4 : 1) * RbConf::P * sizeof(float);
}

template <int Q, bool U, bool CC>
__global__ void __launch_bounds__(RbConf::NT, RbConf::MINB)
    k_fd_step_rb(const float* __restrict__ c, float* __restrict__ cn, const float* __restrict__ u, FdGrid g,
                 float D, int ntz, long long units, long long per_block) {
  using Tp = FdTemplate<Q>;
  using R = RbConf;
  constexpr int NF = U ? 4 : 1, P = R::P, W = R::W, NT = R::NT, KY = R::KY, S = R::S;
  extern __shared__ __align__(16) float rb_smem[];  // [S slots][NF][H][W]
  const int lane = threadIdx.x, w = threadIdx.y, t = w * kRbTZ + lane;
  long long u0 = (long long)blockIdx.x * per_block;
  const long long uend = min(units, u0 + per_block);
  const unsigned plane = (unsigned)(g.gy * g.gz);
  while (u0 < uend) {
    const int tile = (int)(u0 / g.nx);
    const int xa = (int)(u0 - (long long)tile * g.nx) + 1;
    const int xb = (int)min((long long)g.nx, (long long)xa + (uend - u0) - 1);
    u0 += xb - xa + 1;
    const int z0 = (tile % ntz) * R::TZ, y0 = (tile / ntz) * (R::TY * KY);  // ghosted origin
    // this thread's tile entries: offset within a plane, or ~0u off the grid
    unsigned off[R::E];
#pragma unroll
    for (int k = 0; k < R::E; ++k) {
      const int e = t + k * NT;
      const int yy = y0 + e / W, zz = z0 - R::CO + e % W;
      off[k] = (e < P && yy < g.gy && zz >= 0 && zz < g.gz) ? (unsigned)(yy * g.gz + zz) : ~0u;
    }
    const int col = R::KZ * lane + 1 + R::CO;  // tile column of the thread's first cell
    const int z = z0 + R::KZ * lane + 1;
    auto compute = [&](int x) {
      const float* sl[3] = {rb_smem + ((x - 1) % S) * NF * P, rb_smem + (x % S) * NF * P,
                            rb_smem + ((x + 1) % S) * NF * P};
#pragma unroll
      for (int rc = 0; rc < KY * R::KZ; ++rc) {
        const int r = rc / R::KZ, kz = rc % R::KZ;
        const int ry = w * KY + r + 1;  // tile row of the cell
        const int y = y0 + ry;
        // the value of field f at x + e_i; a pair's two middle columns are
        // one 8-byte load, which the unrolled rows and cells share
        auto at = [&](int f, int i) -> float {
          const float* b = sl[1 + Tp::e(i, 0)] + f * P + (ry + Tp::e(i, 1)) * W + col;
          const int k = kz + Tp::e(i, 2);
          if (R::KZ == 2 && (k == 0 || k == 1)) {
            const float2 v = *reinterpret_cast<const float2*>(b);
            return k == 0 ? v.x : v.y;
          }
          return b[k];
        };
        const float cnew = fd_cell_links<Q, float, U, CC>([&](int i) { return at(0, i); },
                                                          [&](int d, int i) { return at(1 + d, i); }, D);
        if (z + kz <= g.nz && y <= g.ny) cn[(unsigned)x * plane + (unsigned)(y * g.gz + z + kz)] = cnew;
      }
    };
    // planes through registers: plane x + 2 is loaded during plane x and
    // stored to its slot at the top of the next iteration
    float r[R::E][NF];
    auto fetch = [&](int xp) {
      const unsigned pb = (unsigned)xp * plane;
#pragma unroll
      for (int k = 0; k < R::E; ++k) {
        if (off[k] == ~0u) continue;
        const unsigned a = pb + off[k];
        r[k][0] = __ldg(c + a);
        if constexpr (U) {
          r[k][1] = __ldg(u + a);
          r[k][2] = __ldg(u + g.L + a);
          r[k][3] = __ldg(u + 2 * g.L + a);
        }
      }
    };
    auto stash = [&](int xp) {
      float* sp = rb_smem + (xp % S) * NF * P;
#pragma unroll
      for (int k = 0; k < R::E; ++k) {
        if (off[k] == ~0u) continue;
#pragma unroll
        for (int f = 0; f < NF; ++f) sp[f * P + t + k * NT] = r[k][f];
      }
    };
    __syncthreads();  // every thread is done with the ring's previous run
    fetch(xa - 1);
    stash(xa - 1);
    fetch(xa);
    stash(xa);
    fetch(xa + 1);
    for (int x = xa; x <= xb; ++x) {
      stash(x + 1);     // slot of plane x - 3: nobody reads it any more
      __syncthreads();  // planes x - 1 .. x + 1 are in
      if (x < xb) fetch(x + 2);
      compute(x);
    }
  }
}

// Face ghost layers (cells of the face with interior tangential indices).
template <class T>
__global__ void k_fd_face_value(T* __restrict__ c, FdGrid g, int axis, int layer, T value) {
  const int n1 = axis == 0 ? g.ny : g.nx, n2 = axis == 2 ? g.ny : g.nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n1 * n2) return;
  const int i = t / n2 + 1, j = t % n2 + 1;
  int x, y, z;
  if (axis == 0) { x = layer; y = i; z = j; }
  else if (axis == 1) { x = i; y = layer; z = j; }
  else { x = i; y = j; z = layer; }
  c[((long long)x * g.gy + y) * g.gz + z] = value;
}

// Conditions on c at a map (aslBasicBC.cxx:71-108, 271-350), thread t per
// guard cell (x, y, z, mask of fluid-neighbour directions of the template):
//   VALUE     c(x) = value
//   GRADIENT  c(x) = sum_k W_k (c(x + e_k) - (n . e_k / |e_k|) value) / sum_k W_k
//             when sum_k W_k > 0.1; W_k = (n . e_k / |e_k| + 1)^2 and
//             n . e_k / |e_k| precomputed per cell and direction (wt, nd).
template <int Q, class T>
__global__ void k_fd_map_bc(T* __restrict__ c, FdGrid g, const int4* __restrict__ cells, int n,
                            const double* __restrict__ wt, const double* __restrict__ nd, int gradient, T value) {
  using Tp = FdTemplate<Q>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 an = cells[t];
  const long long a = ((long long)an.x * g.gy + an.y) * g.gz + an.z;
  if (!gradient) {
    c[a] = value;
    return;
  }
  T sum = T(0), counter = T(0);
#pragma unroll
  for (int k = 1; k < Q; ++k) {
    if (!((unsigned)an.w >> k & 1u)) continue;
    const long long q = ((long long)(an.x + Tp::e(k, 0)) * g.gy + an.y + Tp::e(k, 1)) * g.gz + an.z + Tp::e(k, 2);
    const T w = T(wt[(size_t)t * Q + k]);
    sum += (c[q] - T(nd[(size_t)t * Q + k]) * value) * w;
    counter += w;
  }
  if (counter > T(0.1)) c[a] = sum / counter;
}

}  // namespace
}  // namespace aslb

using namespace aslb;

struct aslb_fd_bc;

struct aslb_fd {
  FdGrid g{};
  int q = 7;
  int dtype = ASLB_F32;
  double D = 0;
  void* c[2] = {nullptr, nullptr};
  int cur = 0;
  const void* u = nullptr;  // bound velocity field (device), or none
  int cc = 0;
  cudaStream_t stream = nullptr, own = nullptr;
  aslb_lbgk* bound = nullptr;  // domain whose velocity and stream are used
  void* ef = nullptr;           // electric term: phi, k, q (3 L values), or none
  long long steps = 0;
  std::vector<aslb_fd_bc*> bcs;  // map conditions on c (detached on destroy)
};

struct aslb_fd_bc {
  aslb_fd* fd = nullptr;
  int gradient = 0;
  double value = 0;
  int n = 0;
  int4* cells = nullptr;
  double* wt = nullptr;
  double* nd = nullptr;
};

namespace aslb {
// The bound domain is being destroyed: fall back to no velocity.
void fd_detached(aslb_fd* f) {
  f->u = nullptr;
  f->stream = f->own;
  f->cc = 0;
  f->bound = nullptr;
}
}  // namespace aslb

namespace {
int fd_err(const char* what, cudaError_t e) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return ASLB_ERR_CUDA;
}
int fd_arg(const char* what) {
  set_last_error(std::string(what));
  return ASLB_ERR_ARG;
}
size_t fd_elem(const aslb_fd* f) { return f->dtype == ASLB_F64 ? 8 : 4; }

// Launch one instantiation with its dynamic shared memory (three tile planes
// of every field it stages), raising the limit once where above 48 KB.
template <int Q, class T, bool U, bool E>
cudaError_t fd_launch_one(aslb_fd* f, dim3 grid, dim3 block, const T* c, T* cn, const T* u, const T* ef) {
  constexpr int NF = 1 + (U ? 3 : 0) + (E ? 3 : 0);
  constexpr size_t bytes = 3u * NF * (kFdTZ + 2) * (kFdTY + 2) * sizeof(T);
  static bool raised = false;
  if (bytes > 48 * 1024 && !raised) {
    cudaError_t e = cudaFuncSetAttribute(k_fd_step<Q, T, U, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    raised = true;
  }
  k_fd_step<Q, T, U, E><<<grid, block, bytes, f->stream>>>(c, cn, u, ef, f->g, T(f->D), U ? f->cc : 0);
  return cudaGetLastError();
}

// The register-blocked FP32 kernel: one block per resident slot, each with
// an equal run of the tiles' planes.
template <int Q, bool U, bool CC>
cudaError_t fd_launch_rb(aslb_fd* f) {
  using R = RbConf;
  constexpr size_t bytes = fd_rb_smem<U>();
  auto kern = k_fd_step_rb<Q, U, CC>;
  static int resident = 0;  // blocks per SM
  if (!resident) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, R::NT, bytes);
    if (e != cudaSuccess) return e;
    if (resident < 1) return cudaErrorInvalidConfiguration;
  }
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int ntz = (f->g.nz + R::TZ - 1) / R::TZ, nty = (f->g.ny + R::TY * R::KY - 1) / (R::TY * R::KY);
  const long long units = (long long)ntz * nty * f->g.nx;
  const long long blocks = std::min<long long>(units, (long long)resident * sms);
  const long long per_block = (units + blocks - 1) / blocks;
  kern<<<(unsigned)((units + per_block - 1) / per_block), dim3(kRbTZ, R::TY), bytes, f->stream>>>(
      (const float*)f->c[f->cur], (float*)f->c[1 - f->cur], (const float*)f->u, f->g, (float)f->D, ntz, units,
      per_block);
  return cudaGetLastError();
}

template <int Q, class T>
cudaError_t fd_launch(aslb_fd* f) {
  // d3q15 / d3q19 in FP32 without the electric term: the register-blocked
  // kernel; d3q7 (whose update is short and whose step is bound by the
  // plane fetches, which the smaller tiles below keep more of in flight),
  // FP64 and the electric term: the 32 x 8 tiles
  if constexpr (std::is_same<T, float>::value && Q != 7) {
    if (!f->ef) {
      if (!f->u) return fd_launch_rb<Q, false, false>(f);
      return f->cc ? fd_launch_rb<Q, true, true>(f) : fd_launch_rb<Q, true, false>(f);
    }
  }
  dim3 block(kFdTZ, kFdTY),
      grid((f->g.nz + kFdTZ - 1) / kFdTZ, (f->g.ny + kFdTY - 1) / kFdTY, (f->g.nx + kFdPlanes - 1) / kFdPlanes);
  const T* c = (const T*)f->c[f->cur];
  T* cn = (T*)f->c[1 - f->cur];
  const T* ef = (const T*)f->ef;
  const T* u = (const T*)f->u;
  if (u && ef) return fd_launch_one<Q, T, true, true>(f, grid, block, c, cn, u, ef);
  if (u) return fd_launch_one<Q, T, true, false>(f, grid, block, c, cn, u, nullptr);
  if (ef) return fd_launch_one<Q, T, false, true>(f, grid, block, c, cn, nullptr, ef);
  return fd_launch_one<Q, T, false, false>(f, grid, block, c, cn, nullptr, nullptr);
}

template <class T>
cudaError_t fd_step_t(aslb_fd* f) {
  switch (f->q) {
    case 7: return fd_launch<7, T>(f);
    case 15: return fd_launch<15, T>(f);
    case 19: return fd_launch<19, T>(f);
  }
  return cudaErrorInvalidValue;
}
}  // namespace

extern "C" {

int aslb_fd_create(int nx, int ny, int nz, int q, int dtype, double D, aslb_fd** out) {
  if (!out) return fd_arg("aslb_fd_create: null argument");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1) return fd_arg("aslb_fd_create: sizes must be positive");
  if (q != 7 && q != 15 && q != 19) return fd_arg("aslb_fd_create: template must be d3q7, d3q15 or d3q19");
  if (dtype != ASLB_F32 && dtype != ASLB_F64) return fd_arg("aslb_fd_create: dtype must be F32 or F64");
  auto* f = new aslb_fd();
  f->g = FdGrid{nx, ny, nz, nx + 2, ny + 2, nz + 2, (long long)(nx + 2) * (ny + 2) * (nz + 2)};
  f->q = q;
  f->dtype = dtype;
  f->D = D;
  cudaError_t e = cudaStreamCreateWithFlags(&f->own, cudaStreamNonBlocking);
  f->stream = f->own;
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaMalloc(&f->c[b], f->g.L * fd_elem(f));
    if (e == cudaSuccess) e = cudaMemsetAsync(f->c[b], 0, f->g.L * fd_elem(f), f->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) {
    aslb_fd_destroy(f);
    return fd_err("aslb_fd_create", e);
  }
  *out = f;
  return ASLB_OK;
}

int aslb_fd_set_velocity(aslb_fd* f, aslb_lbgk* h, int compressibility_correction) {
  if (!f) return fd_arg("aslb_fd_set_velocity: null argument");
  if (f->bound) {
    cudaStreamSynchronize(f->stream);
    lbgk_detach_fd(f->bound, f);
    fd_detached(f);
  }
  if (!h) return ASLB_OK;
  int n[3], storage;
  void* u;
  cudaStream_t st;
  int r = lbgk_velocity_binding(h, n, &storage, &u, &st);
  if (r) return r;
  if (n[0] != f->g.nx || n[1] != f->g.ny || n[2] != f->g.nz)
    return fd_arg("aslb_fd_set_velocity: the domain has another size");
  if ((storage == ASLB_F64) != (f->dtype == ASLB_F64))
    return fd_arg("aslb_fd_set_velocity: the velocity field is FP64 only for FP64 storage; match the FD dtype");
  cudaStreamSynchronize(f->stream);
  f->u = u;
  f->stream = st;  // after the domain's step, in order
  f->cc = compressibility_correction ? 1 : 0;
  f->bound = h;
  lbgk_attach_fd(h, f);
  return ASLB_OK;
}

int aslb_fd_set_electric_field(aslb_fd* f, int dtype, const void* phi, const void* k, const void* q) {
  if (!f) return fd_arg("aslb_fd_set_electric_field: null argument");
  if (!phi && !k && !q) {
    if (f->ef) {
      cudaStreamSynchronize(f->stream);
      cudaFree(f->ef);
      f->ef = nullptr;
    }
    return ASLB_OK;
  }
  if (!phi || !k || !q || dtype != f->dtype)
    return fd_arg("aslb_fd_set_electric_field: phi, k and q are all needed, in the FD's dtype");
  const size_t bytes = (size_t)f->g.L * fd_elem(f);
  cudaError_t e = cudaSuccess;
  if (!f->ef) e = cudaMalloc(&f->ef, 3 * bytes);
  const void* src[3] = {phi, k, q};
  for (int i = 0; i < 3 && e == cudaSuccess; ++i)
    e = cudaMemcpyAsync((char*)f->ef + i * bytes, src[i], bytes, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) return fd_err("aslb_fd_set_electric_field", e);
  return ASLB_OK;
}

int aslb_fd_set_diffusion(aslb_fd* f, double D) {
  if (!f) return fd_arg("aslb_fd_set_diffusion: null argument");
  f->D = D;
  return ASLB_OK;
}

int aslb_fd_write(aslb_fd* f, int dtype, const void* host) {
  if (!f || !host || dtype != f->dtype) return fd_arg("aslb_fd_write: null argument or dtype differs from the FD's");
  const size_t bytes = f->g.L * fd_elem(f);
  cudaError_t e = cudaMemcpyAsync(f->c[0], host, bytes, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(f->c[1], f->c[0], bytes, cudaMemcpyDeviceToDevice, f->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) return fd_err("aslb_fd_write", e);
  f->cur = 0;
  return ASLB_OK;
}

int aslb_fd_read(aslb_fd* f, int dtype, void* host) {
  if (!f || !host || dtype != f->dtype) return fd_arg("aslb_fd_read: null argument or dtype differs from the FD's");
  cudaError_t e = cudaMemcpyAsync(host, f->c[f->cur], f->g.L * fd_elem(f), cudaMemcpyDeviceToHost, f->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) return fd_err("aslb_fd_read", e);
  return ASLB_OK;
}

int aslb_fd_set_face_value(aslb_fd* f, unsigned wallmask, double value) {
  if (!f) return fd_arg("aslb_fd_set_face_value: null argument");
  cudaError_t e = cudaSuccess;
  for (int w = 0; w < 6 && e == cudaSuccess; ++w) {
    if (!(wallmask >> w & 1u)) continue;
    const int axis = w / 2;
    const int n[3] = {f->g.nx, f->g.ny, f->g.nz};
    const int layer = (w & 1) ? n[axis] + 1 : 0;
    const int cnt = (axis == 0 ? f->g.ny * f->g.nz : axis == 1 ? f->g.nx * f->g.nz : f->g.nx * f->g.ny);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
      if (f->dtype == ASLB_F64)
        k_fd_face_value<double><<<(cnt + 255) / 256, 256, 0, f->stream>>>((double*)f->c[b], f->g, axis, layer, value);
      else
        k_fd_face_value<float><<<(cnt + 255) / 256, 256, 0, f->stream>>>((float*)f->c[b], f->g, axis, layer,
                                                                         (float)value);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) return fd_err("aslb_fd_set_face_value", e);
  return ASLB_OK;
}

int aslb_fd_step(aslb_fd* f, int n) {
  nvtxRangePushA("aslb_fd_step");
  struct Pop { ~Pop() { nvtxRangePop(); } } pop;
  if (!f || n < 0) return fd_arg("aslb_fd_step: null argument or negative count");
  for (int s = 0; s < n; ++s) {
    cudaError_t e = f->dtype == ASLB_F64 ? fd_step_t<double>(f) : fd_step_t<float>(f);
    if (e != cudaSuccess) return fd_err("aslb_fd_step", e);
    f->cur = 1 - f->cur;
    f->steps++;
  }
  return ASLB_OK;
}

int aslb_fd_sync(aslb_fd* f) {
  if (!f) return fd_arg("aslb_fd_sync: null argument");
  cudaError_t e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) return fd_err("aslb_fd_sync", e);
  return ASLB_OK;
}

void* aslb_fd_device_field(aslb_fd* f) { return f ? f->c[f->cur] : nullptr; }

int aslb_fd_bc_create(aslb_fd* f, int kind, const float* map, double value, aslb_fd_bc** out) {
  if (!f || !map || !out) return fd_arg("aslb_fd_bc_create: null argument");
  *out = nullptr;
  if (kind != ASLB_FD_BC_VALUE_MAP && kind != ASLB_FD_BC_GRADIENT_MAP)
    return fd_arg("aslb_fd_bc_create: kind must be ASLB_FD_BC_VALUE_MAP or ASLB_FD_BC_GRADIENT_MAP");
  const FdGrid& g = f->g;
  const int q = f->q;
  auto e = [&](int k, int d) { return q == 15 ? lat_c15(k, d) : lat_c27(k, d); };
  auto gc = [&](int k) {
    return q == 7 ? FdTemplate<7>::gc(k) : q == 15 ? FdTemplate<15>::gc(k) : FdTemplate<19>::gc(k);
  };
  auto mat = [&](int x, int y, int z) -> double {  // the map, -0.9 off the grid (generateDCFullSafe)
    if (x < 0 || y < 0 || z < 0 || x >= g.gx || y >= g.gy || z >= g.gz) return -0.9;
    return map[((long long)x * g.gy + y) * g.gz + z];
  };
  std::vector<int4> cells;
  std::vector<double> wt, nd;
  for (int x = 0; x < g.gx; ++x)
    for (int y = 0; y < g.gy; ++y)
      for (int z = 0; z < g.gz; ++z) {
        const float m0 = map[((long long)x * g.gy + y) * g.gz + z];
        if (!(m0 <= 0.f && m0 > -0.9999f)) continue;
        unsigned mask = 0;
        double nrm[3] = {0, 0, 0};
        for (int k = 1; k < q; ++k) {
          const int qx = x + e(k, 0), qy = y + e(k, 1), qz = z + e(k, 2);
          const double mk = mat(qx, qy, qz);
          const bool in = qx >= 1 && qx <= g.nx && qy >= 1 && qy <= g.ny && qz >= 1 && qz <= g.nz;
          if (mk > 0.0 && in) mask |= 1u << k;
          for (int d = 0; d < 3; ++d) nrm[d] += gc(k) * e(k, d) * (float)mk;
        }
        if (kind == ASLB_FD_BC_GRADIENT_MAP) {
          const double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
          if (!(len > 0.0) || !mask) continue;  // no normal or no fluid neighbour: c stays
          for (int k = 0; k < q; ++k) {
            double w = 0, dn = 0;
            if (k > 0 && (mask >> k & 1u)) {
              const double cl = std::sqrt((double)(e(k, 0) * e(k, 0) + e(k, 1) * e(k, 1) + e(k, 2) * e(k, 2)));
              dn = (nrm[0] * e(k, 0) + nrm[1] * e(k, 1) + nrm[2] * e(k, 2)) / len / cl;
              w = (dn + 1.0) * (dn + 1.0);
            }
            wt.push_back(w);
            nd.push_back(dn);
          }
        }
        cells.push_back(make_int4(x, y, z, (int)mask));
      }
  auto* b = new aslb_fd_bc();
  b->fd = f;
  b->gradient = kind == ASLB_FD_BC_GRADIENT_MAP;
  b->value = value;
  b->n = (int)cells.size();
  cudaError_t err = cudaSuccess;
  if (b->n) {
    err = cudaMalloc((void**)&b->cells, cells.size() * sizeof(int4));
    if (err == cudaSuccess)
      err = cudaMemcpy(b->cells, cells.data(), cells.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && !wt.empty()) {
      err = cudaMalloc((void**)&b->wt, wt.size() * sizeof(double));
      if (err == cudaSuccess) err = cudaMalloc((void**)&b->nd, nd.size() * sizeof(double));
      if (err == cudaSuccess) err = cudaMemcpy(b->wt, wt.data(), wt.size() * sizeof(double), cudaMemcpyHostToDevice);
      if (err == cudaSuccess) err = cudaMemcpy(b->nd, nd.data(), nd.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
  }
  if (err != cudaSuccess) {
    aslb_fd_bc_destroy(b);
    return fd_err("aslb_fd_bc_create", err);
  }
  f->bcs.push_back(b);
  *out = b;
  return ASLB_OK;
}

int aslb_fd_bc_execute(aslb_fd_bc* b) {
  if (!b) return fd_arg("aslb_fd_bc_execute: null argument");
  if (!b->fd) {
    set_last_error("aslb_fd_bc_execute: its FD solver was destroyed");
    return ASLB_ERR_STATE;
  }
  aslb_fd* f = b->fd;
  if (!b->n) return ASLB_OK;
  const unsigned blocks = (unsigned)((b->n + 255) / 256);
  const int q = f->q;
  if (f->dtype == ASLB_F64) {
    double* c = (double*)f->c[f->cur];
    if (q == 7) k_fd_map_bc<7, double><<<blocks, 256, 0, f->stream>>>(c, f->g, b->cells, b->n, b->wt, b->nd, b->gradient, b->value);
    else if (q == 15) k_fd_map_bc<15, double><<<blocks, 256, 0, f->stream>>>(c, f->g, b->cells, b->n, b->wt, b->nd, b->gradient, b->value);
    else k_fd_map_bc<19, double><<<blocks, 256, 0, f->stream>>>(c, f->g, b->cells, b->n, b->wt, b->nd, b->gradient, b->value);
  } else {
    float* c = (float*)f->c[f->cur];
    const float v = (float)b->value;
    if (q == 7) k_fd_map_bc<7, float><<<blocks, 256, 0, f->stream>>>(c, f->g, b->cells, b->n, b->wt, b->nd, b->gradient, v);
    else if (q == 15) k_fd_map_bc<15, float><<<blocks, 256, 0, f->stream>>>(c, f->g, b->cells, b->n, b->wt, b->nd, b->gradient, v);
    else k_fd_map_bc<19, float><<<blocks, 256, 0, f->stream>>>(c, f->g, b->cells, b->n, b->wt, b->nd, b->gradient, v);
  }
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return fd_err("aslb_fd_bc_execute", err);
  return ASLB_OK;
}

long long aslb_fd_bc_cells(aslb_fd_bc* b) { return b ? b->n : -1; }

int aslb_fd_bc_destroy(aslb_fd_bc* b) {
  if (!b) return ASLB_OK;
  if (b->fd) {
    cudaStreamSynchronize(b->fd->stream);
    auto& v = b->fd->bcs;
    v.erase(std::remove(v.begin(), v.end(), b), v.end());
  }
  cudaFree(b->cells);
  cudaFree(b->wt);
  cudaFree(b->nd);
  delete b;
  return ASLB_OK;
}

int aslb_fd_destroy(aslb_fd* f) {
  if (!f) return ASLB_OK;
  if (f->stream) cudaStreamSynchronize(f->stream);
  if (f->bound) lbgk_detach_fd(f->bound, f);
  for (aslb_fd_bc* b : f->bcs) b->fd = nullptr;
  if (f->ef) cudaFree(f->ef);
  for (void* p : f->c)
    if (p) cudaFree(p);
  if (f->own) cudaStreamDestroy(f->own);
  delete f;
  return ASLB_OK;
}

}  // extern "C"
