// CUDA kernels of the LBGK hot path for sm_100a: the fused AA-pattern
// stream-collide, field initialisation and population export/import, the
// boundary-link kernel shared by every boundary condition, the surface force
// with its FP64 reduction, and global moments.
#include <type_traits>
#include "kernels.h"
#include "bc_links.cuh"
#include "stream_collide.cuh"

namespace aslb {

cudaError_t step_q15_f32(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q15_f16(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q15_f64(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q19_f32(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q19_f16(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q19_f64(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q27_f32(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q27_f16(const DomainDev&, const StepParams&, int, int, cudaStream_t);
cudaError_t step_q27_f64(const DomainDev&, const StepParams&, int, int, cudaStream_t);

cudaError_t launch_step(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st) {
  switch (d.q * 8 + d.storage) {
    case 15 * 8 + ST_F32: return step_q15_f32(d, p, closure, parity_in, st);
    case 15 * 8 + ST_F16: return step_q15_f16(d, p, closure, parity_in, st);
    case 15 * 8 + ST_F64: return step_q15_f64(d, p, closure, parity_in, st);
    case 19 * 8 + ST_F32: return step_q19_f32(d, p, closure, parity_in, st);
    case 19 * 8 + ST_F16: return step_q19_f16(d, p, closure, parity_in, st);
    case 19 * 8 + ST_F64: return step_q19_f64(d, p, closure, parity_in, st);
    case 27 * 8 + ST_F32: return step_q27_f32(d, p, closure, parity_in, st);
    case 27 * 8 + ST_F16: return step_q27_f16(d, p, closure, parity_in, st);
    case 27 * 8 + ST_F64: return step_q27_f64(d, p, closure, parity_in, st);
  }
  return cudaErrorInvalidValue;
}

// Generic dispatch for the remaining kernels (lattice x storage).
#define ASLB_DISPATCH(d, FN, ...)                                                   \
  switch ((d).q * 8 + (d).storage) {                                                \
    case 15 * 8 + ST_F32: return FN<15, float>(__VA_ARGS__);                        \
    case 15 * 8 + ST_F16: return FN<15, __half>(__VA_ARGS__);                       \
    case 15 * 8 + ST_F64: return FN<15, double>(__VA_ARGS__);                       \
    case 19 * 8 + ST_F32: return FN<19, float>(__VA_ARGS__);                        \
    case 19 * 8 + ST_F16: return FN<19, __half>(__VA_ARGS__);                       \
    case 19 * 8 + ST_F64: return FN<19, double>(__VA_ARGS__);                       \
    case 27 * 8 + ST_F32: return FN<27, float>(__VA_ARGS__);                        \
    case 27 * 8 + ST_F16: return FN<27, __half>(__VA_ARGS__);                       \
    case 27 * 8 + ST_F64: return FN<27, double>(__VA_ARGS__);                       \
    default: return cudaErrorInvalidValue;                                          \
  }

// ---------------------------------------------------------------------------
// Storage index of f*_i(x), the post-collision population of cell x in
// direction i, for either representation. With fused no-slip links the
// incoming slot of a link is never written; its value is the fluid end's
// outgoing population, held by the other slot of the pair. Returns -1 where
// representation B would need a cell outside the block (ghost cells only).
template <int Q>
__device__ __forceinline__ long long fstar_index(const GridDesc& g, const uint2* __restrict__ mask, int parity,
                                                 int x, int y, int z, int i) {
  using Lt = Lattice<Q>;
  const bool inter = x >= 1 && x <= g.nx && y >= 1 && y <= g.ny && z >= 1 && z <= g.nz;
  int tx = x + Lt::c(i, 0), ty = y + Lt::c(i, 1), tz = z + Lt::c(i, 2);
  if (inter) {
    tx = wrap_axis(tx, g.nx, g.periodic & 1);
    ty = wrap_axis(ty, g.ny, g.periodic & 2);
    tz = wrap_axis(tz, g.nz, g.periodic & 4);
  }
  const bool tin = tx >= 0 && ty >= 0 && tz >= 0 && tx < g.gx && ty < g.gy && tz < g.gz;
  const long long sx = sidx(g, wrap_axis(x, g.nx, g.periodic & 1), wrap_axis(y, g.ny, g.periodic & 2),
                            wrap_axis(z, g.nz, g.periodic & 4));
  const long long sq = tin ? sidx(g, tx, ty, tz) : -1;
  bool fused = false;
  if (mask && tin && tx >= 1 && tx <= g.nx && ty >= 1 && ty <= g.ny && tz >= 1 && tz <= g.nz) {
    fused = (mask[sq].x >> i) & 1u;
  }
  const bool in_own = (parity == 0) != fused;  // slot F[i][x] (else F[inv i][x + c_i])
  if (in_own) return (long long)i * g.dstride + sx;
  if (!tin) return -1;
  return (long long)Lt::inv(i) * g.dstride + sq;
}

// ---------------------------------------------------------------------------
// initF: f_i = rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u) on every ghosted cell
// (src/num/aslLBGK.cxx:262-280), representation A.
template <int Q, class S>
__global__ void k_init_f(S* __restrict__ F, const GridDesc g, const StepParams p, double rho0, double u0x,
                         double u0y, double u0z, const double* __restrict__ rho_field,
                         const double* __restrict__ u_field, typename MacroT<S>::T* __restrict__ rho_out,
                         typename MacroT<S>::T* __restrict__ u_out) {
  using Lt = Lattice<Q>;
  using C = typename Store<S>::C;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int x = blockIdx.z;
  if (z >= g.gz) return;
  const long long a = aidx(g, x, y, z);
  const long long s = sidx(g, x, y, z);
  const C r = rho_field ? C(rho_field[a]) : C(rho0);
  const C ux = u_field ? C(u_field[a]) : C(u0x);
  const C uy = u_field ? C(u_field[g.L + a]) : C(u0y);
  const C uz = u_field ? C(u_field[2 * g.L + a]) : C(u0z);
  const C vv = ux * ux + uy * uy + uz * uz;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const C cu = ux * C(Lt::c(i, 0)) + uy * C(Lt::c(i, 1)) + uz * C(Lt::c(i, 2));
    const C fi = r * (C(1) + C(3) * cu + C(4.5) * (cu * cu) - C(1.5) * vv);
    Store<S>::store(F + (size_t)i * g.dstride + s, fi, p);
  }
  rho_out[a] = r;
  u_out[a] = ux;
  u_out[g.L + a] = uy;
  u_out[2 * g.L + a] = uz;
}

template <int Q, class S>
static cudaError_t init_impl(const DomainDev& d, const StepParams& p, double rho0, const double* u0,
                             const double* rho_field, const double* u_field, cudaStream_t st) {
  using M = typename MacroT<S>::T;
  dim3 block(128), grid((d.g.gz + 127) / 128, d.g.gy, d.g.gx);
  k_init_f<Q, S><<<grid, block, 0, st>>>((S*)d.F, d.g, p, rho0, u0[0], u0[1], u0[2], rho_field, u_field,
                                         (M*)d.rho, (M*)d.u);
  return cudaGetLastError();
}

cudaError_t launch_init_f(const DomainDev& d, const StepParams& p, double rho0, const double* u0,
                          const double* rho_field, const double* u_field, cudaStream_t st) {
  ASLB_DISPATCH(d, init_impl, d, p, rho0, u0, rho_field, u_field, st)
}

// ---------------------------------------------------------------------------
// Export f*_i(x) in ASL's layout. In representation B the value sits at the
// cell it was pushed to; ghost cells whose target leaves the block read NaN.
// Population transfers between the storage and ASL's layout (a = the ghosted
// index, z fastest), directions [i0, i1): a grid-stride loop over the cells,
// so a one-direction transfer is one small launch.
inline unsigned transfer_blocks(long long L) {
  const long long b = (L + 255) / 256;
  return (unsigned)(b < 148 * 16 ? b : 148 * 16);
}

template <int Q, class S>
__global__ void __launch_bounds__(256) k_export_f(const S* __restrict__ F, const GridDesc g, const StepParams p,
                                                  int parity, int i0, int i1,
                                                  typename MacroT<S>::T* __restrict__ out) {
  using M = typename MacroT<S>::T;
  // 32-bit index arithmetic (L < 2^32): 64-bit divisions cost a slow subroutine per cell
  const unsigned L = (unsigned)g.L, gz = (unsigned)g.gz, gy = (unsigned)g.gy;
  for (unsigned a = blockIdx.x * blockDim.x + threadIdx.x; a < L; a += gridDim.x * blockDim.x) {
    const unsigned r = a / gz;
    const int z = (int)(a - r * gz);
    const int x = (int)(r / gy), y = (int)(r - (unsigned)x * gy);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      if (i < i0 || i >= i1) continue;
      const long long k = fstar_index<Q>(g, p.mask, parity, x, y, z, i);
      out[(long long)(i - i0) * g.L + a] = k < 0 ? M(NAN) : M(Store<S>::val(F + k, p.inv_scale));
    }
  }
}

template <int Q, class S>
static cudaError_t export_impl(const DomainDev& d, const StepParams& p, int parity, int i0, int i1, void* out,
                               cudaStream_t st) {
  using M = typename MacroT<S>::T;
  k_export_f<Q, S><<<transfer_blocks(d.g.L), 256, 0, st>>>((const S*)d.F, d.g, p, parity, i0, i1, (M*)out);
  return cudaGetLastError();
}

cudaError_t launch_export_f(const DomainDev& d, const StepParams& p, int parity, int i0, int i1, void* out,
                            cudaStream_t st) {
  ASLB_DISPATCH(d, export_impl, d, p, parity, i0, i1, out, st)
}

template <int Q, class S>
__global__ void __launch_bounds__(256) k_import_f(S* __restrict__ F, const GridDesc g, const StepParams p, int i0,
                                                  int i1, const typename MacroT<S>::T* __restrict__ in) {
  const unsigned L = (unsigned)g.L, gz = (unsigned)g.gz;
  for (unsigned a = blockIdx.x * blockDim.x + threadIdx.x; a < L; a += gridDim.x * blockDim.x) {
    // storage index: the rows (x, y) are in the same order in both layouts
    const unsigned r = a / gz;
    const long long s = (long long)r * g.pitch + g.zoff + (a - r * gz);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      if (i < i0 || i >= i1) continue;
      Store<S>::set_val(F + (size_t)i * g.dstride + s, typename Store<S>::C(in[(long long)(i - i0) * g.L + a]),
                        p.scale);
    }
  }
}

template <int Q, class S>
static cudaError_t import_impl(const DomainDev& d, const StepParams& p, int i0, int i1, const void* in,
                               cudaStream_t st) {
  using M = typename MacroT<S>::T;
  k_import_f<Q, S><<<transfer_blocks(d.g.L), 256, 0, st>>>((S*)d.F, d.g, p, i0, i1, (const M*)in);
  return cudaGetLastError();
}

cudaError_t launch_import_f(const DomainDev& d, const StepParams& p, int i0, int i1, const void* in,
                            cudaStream_t st) {
  ASLB_DISPATCH(d, import_impl, d, p, i0, i1, in, st)
}

// ---------------------------------------------------------------------------
// Boundary links. An anchor a (ghost or solid cell) with mask bit k stands for
// the link into the interior fluid cell q = a + c_k along c_k. Two slots are
// involved: IN, holding f*_k(a) that q pulls next step, and OUT, holding
// f*_inv(k)(q) that leaves q towards a:
//   representation A: IN = F[k][a],      OUT = F[inv k][q]
//   representation B: IN = F[inv k][q],  OUT = F[k][a]
// Within one boundary condition no OUT slot is an IN slot (IN belongs to a
// ghost/solid cell, OUT to a fluid cell), so links run in parallel; separate
// boundary conditions run in the user's order, later writers winning as in ASL.
template <int Q, class S>
__global__ void __launch_bounds__(256) k_bc(S* __restrict__ F, const GridDesc g, const int4* __restrict__ anchors,
                                            int n, const BcParams bp, int parity) {
  using Lt = Lattice<Q>;
  using C = typename Store<S>::C;
  using A = BcArith<S>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 an = anchors[t];
  const unsigned mask = (unsigned)an.w;
  const bool px = g.periodic & 1, py = g.periodic & 2, pz = g.periodic & 4;
  const long long sa = sidx(g, wrap_axis(an.x, g.nx, px), wrap_axis(an.y, g.ny, py), wrap_axis(an.z, g.nz, pz));
  long long sq[Q];
#pragma unroll
  for (int k = 1; k < Q; ++k)
    sq[k] = sidx(g, wrap_axis(an.x + Lt::c(k, 0), g.nx, px), wrap_axis(an.y + Lt::c(k, 1), g.ny, py),
                 wrap_axis(an.z + Lt::c(k, 2), g.nz, pz));

  const int kind = bp.kind;
  C rb = C(0), vel[3] = {C(bp.u[0]), C(bp.u[1]), C(bp.u[2])};
  if (kind == BCK_MAP_VELOCITY || kind == BCK_MAP_VELOCITY_ROTATION) {
    // rho_b = sum_k w_k f_inv(k)(a + c_k) / sum_k w_k over fluid neighbours (aslLBGKBC.cxx:312-326)
    C coef = C(0);
#pragma unroll
    for (int k = 1; k < Q; ++k)
      if (mask >> k & 1u) {
        const S* out = parity == 0 ? F + (size_t)Lt::inv(k) * g.dstride + sq[k] : F + (size_t)k * g.dstride + sa;
        coef += C(Lt::w(k));
        rb += A::get(out, bp) * C(Lt::w(k));
      }
    rb /= coef;
    if (A::kDev) rb += C(1);  // deviations averaged; rb is now absolute
    if (kind == BCK_MAP_VELOCITY_ROTATION) {
      const double r0 = bp.pos0[0] + (an.x - 1) * bp.dx - bp.cen[0];
      const double r1 = bp.pos0[1] + (an.y - 1) * bp.dx - bp.cen[1];
      const double r2 = bp.pos0[2] + (an.z - 1) * bp.dx - bp.cen[2];
      vel[0] = C(bp.om[1] * r2 - bp.om[2] * r1);
      vel[1] = C(bp.om[2] * r0 - bp.om[0] * r2);
      vel[2] = C(bp.om[0] * r1 - bp.om[1] * r0);
    }
  }
  C dep = C(0);
  if (kind == BCK_MAP_TRANSPORT_DEPOSITION || kind == BCK_MAP_KINETICS_DEPOSITION) {
    // rho = sum_k w_k f_inv(k)(a + c_k), coef = sum_k w_k over fluid neighbours;
    // transport limited j = rho - (rho - coef p0) / (1 + coef lF), kinetics
    // limited j = rho - beta (rho / coef - p0) / (1 + lF); every link of the
    // anchor gets j / coef (aslLBGKBC.cxx:477-500, 546-569)
    C coef = C(0), rs = C(0);
#pragma unroll
    for (int k = 1; k < Q; ++k)
      if (mask >> k & 1u) {
        const S* out = parity == 0 ? F + (size_t)Lt::inv(k) * g.dstride + sq[k] : F + (size_t)k * g.dstride + sa;
        coef += C(Lt::w(k));
        rs += A::get(out, bp) * C(Lt::w(k));
      }
    const C rho = A::kDev ? rs + coef : rs;  // deviations summed: add sum_k w_k * 1
    const C p0 = C(bp.p), lf = C(bp.lf);
    const C j = kind == BCK_MAP_TRANSPORT_DEPOSITION ? rho - (rho - coef * p0) / (C(1) + coef * lf)
                                                     : rho - C(bp.beta) * (rho / coef - p0) / (C(1) + lf);
    dep = j / coef;
  }
  const C P = C(bp.p);
  const C vv = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
#pragma unroll
  for (int k = 1; k < Q; ++k) {
    if (!(mask >> k & 1u)) continue;
    S* in;
    S* out;
    if (parity == 0) {
      in = F + (size_t)k * g.dstride + sa;
      out = F + (size_t)Lt::inv(k) * g.dstride + sq[k];
    } else {
      in = F + (size_t)Lt::inv(k) * g.dstride + sq[k];
      out = F + (size_t)k * g.dstride + sa;
    }
    const C cu = vel[0] * C(Lt::c(k, 0)) + vel[1] * C(Lt::c(k, 1)) + vel[2] * C(Lt::c(k, 2));
    switch (kind) {
      case BCK_NOSLIP:
      case BCK_MAP_NOSLIP:
        *in = *out;  // f_k(a) = f_inv(k)(a + c_k)   (aslLBGKBC.cxx:106-108, 243-244)
        break;
      case BCK_VELOCITY:  // + 6 u.c_k  (aslLBGKBC.cxx:164-167)
        A::put(in, A::get(out, bp) + C(6) * cu, bp);
        break;
      case BCK_PRESSURE:  // = p  (aslLBGKBC.cxx:135-137)
        A::put(in, A::rep(P), bp);
        break;
      case BCK_PRESSURE_VELOCITY:  // = p + 3 u.c_k  (aslLBGKBC.cxx:195-197)
        A::put(in, A::rep(P) + C(3) * cu, bp);
        break;
      case BCK_MAP_VELOCITY:
      case BCK_MAP_VELOCITY_ROTATION: {  // rho_b + 3 rho_b u.c_k  (aslLBGKBC.cxx:327-338)
        const C mc = (vel[0] * rb) * C(Lt::c(k, 0)) + (vel[1] * rb) * C(Lt::c(k, 1)) + (vel[2] * rb) * C(Lt::c(k, 2));
        A::put(in, A::rep(rb) + mc * C(3), bp);
        break;
      }
      case BCK_MAP_PRESSURE_VELOCITY: {  // f_eq(p, u)  (aslLBGKBC.cxx:404-415)
        C fe;
        if (bp.compressible)
          fe = P + C(3) * P * cu + C(4.5) * P * cu * cu - C(1.5) * P * vv;
        else
          fe = P + C(3) * cu + C(4.5) * cu * cu - C(1.5) * vv;
        A::put(in, A::rep(fe), bp);
        break;
      }
      case BCK_MAP_TRANSPORT_DEPOSITION:
      case BCK_MAP_KINETICS_DEPOSITION:
        A::put(in, A::rep(dep), bp);
        break;
    }
  }
}

template <int Q, class S>
static cudaError_t bc_impl(const DomainDev& d, const int4* anchors, int n, const BcParams& bp, int parity,
                           cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_bc<Q, S><<<(n + 255) / 256, 256, 0, st>>>((S*)d.F, d.g, anchors, n, bp, parity);
  return cudaGetLastError();
}

cudaError_t launch_bc(const DomainDev& d, const int4* anchors, int n, const BcParams& bp, int parity,
                      cudaStream_t st) {
  ASLB_DISPATCH(d, bc_impl, d, anchors, n, bp, parity, st)
}

// Conditions on the output fields near a map (aslBasicBC.cxx:152-230, 300-350
// through generateBCNoSlipVel / NoSlipRho / VelocityVel, aslLBGKBC.cxx:808-852).
// Thread t takes guard cell t (x, y, z, mask of fluid-neighbour directions):
//   NOSLIP_VEL   u(x) = sum_k LC_k (0 - u(x + c_k)) / max(sum_k LC_k, 0.01)
//                (the middle-point value 0 between the cell and each fluid neighbour)
//   NOSLIP_RHO   rho(x) = sum_k W_k rho(x + c_k) / sum_k W_k when sum_k W_k > 0.1,
//                W_k = (n . c_k / |c_k| + 1)^2 from the map's unit normal n (the
//                weights come precomputed per cell, wt[t * Q + k]; zero gradient)
//   VELOCITY_VEL u(x) = v(position of x): constant, or omega x (r - center)
// LC_k: laplacian coefficients of the lattice's template (D3Q15: 2/3 axis,
// 1/12 diagonal; D3Q19: 1/3 axis, 1/6 diagonal).
template <int Q, class S>
__global__ void __launch_bounds__(256) k_field_bc(typename MacroT<S>::T* __restrict__ rho,
                                                  typename MacroT<S>::T* __restrict__ u, const GridDesc g,
                                                  const int4* __restrict__ cells, int n,
                                                  const double* __restrict__ wt, const BcParams bp) {
  using Lt = Lattice<Q>;
  using M = typename MacroT<S>::T;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 an = cells[t];
  const unsigned mask = (unsigned)an.w;
  const bool px = g.periodic & 1, py = g.periodic & 2, pz = g.periodic & 4;
  const long long a = aidx(g, an.x, an.y, an.z);
  auto nb = [&](int k) {
    return aidx(g, wrap_axis(an.x + Lt::c(k, 0), g.nx, px), wrap_axis(an.y + Lt::c(k, 1), g.ny, py),
                wrap_axis(an.z + Lt::c(k, 2), g.nz, pz));
  };
  if (bp.kind == BCK_FIELD_NOSLIP_VEL) {
    M v[3] = {M(0), M(0), M(0)}, counter = M(0);
#pragma unroll
    for (int k = 1; k < Q; ++k) {
      if (!(mask >> k & 1u)) continue;
      const M lc = M(Lt::norm2(k) == 1 ? (Q == 15 ? 2.0 / 3.0 : 1.0 / 3.0) : (Q == 15 ? 1.0 / 12.0 : 1.0 / 6.0));
      const long long q = nb(k);
#pragma unroll
      for (int d = 0; d < 3; ++d) v[d] += (M(0) - u[d * g.L + q]) * lc;
      counter += lc;
    }
    const M c = counter > M(0.01) ? counter : M(0.01);
#pragma unroll
    for (int d = 0; d < 3; ++d) u[d * g.L + a] = v[d] / c;
  } else if (bp.kind == BCK_FIELD_NOSLIP_RHO) {
    M s = M(0), counter = M(0);
#pragma unroll
    for (int k = 1; k < Q; ++k) {
      if (!(mask >> k & 1u)) continue;
      const M w = M(wt[(size_t)t * Q + k]);
      s += rho[nb(k)] * w;
      counter += w;
    }
    if (counter > M(0.1)) rho[a] = s / counter;
  } else {
    M v[3] = {M(bp.u[0]), M(bp.u[1]), M(bp.u[2])};
    if (bp.kind == BCK_FIELD_VELOCITY_VEL_ROTATION) {
      const double r0 = bp.pos0[0] + (an.x - 1) * bp.dx - bp.cen[0];
      const double r1 = bp.pos0[1] + (an.y - 1) * bp.dx - bp.cen[1];
      const double r2 = bp.pos0[2] + (an.z - 1) * bp.dx - bp.cen[2];
      v[0] = M(bp.om[1] * r2 - bp.om[2] * r1);
      v[1] = M(bp.om[2] * r0 - bp.om[0] * r2);
      v[2] = M(bp.om[0] * r1 - bp.om[1] * r0);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) u[d * g.L + a] = v[d];
  }
}

template <int Q, class S>
static cudaError_t field_bc_impl(const DomainDev& d, const int4* cells, int n, const double* wt, const BcParams& bp,
                                 cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  if constexpr (Q == 27) {
    return cudaErrorNotSupported;
  } else {
    using M = typename MacroT<S>::T;
    k_field_bc<Q, S><<<(n + 255) / 256, 256, 0, st>>>((M*)d.rho, (M*)d.u, d.g, cells, n, wt, bp);
    return cudaGetLastError();
  }
}

cudaError_t launch_field_bc(const DomainDev& d, const int4* cells, int n, const double* wt, const BcParams& bp,
                            cudaStream_t st) {
  ASLB_DISPATCH(d, field_bc_impl, d, cells, n, wt, bp, st)
}

// Direction-sorted links: thread t handles link t, whose direction k comes from
// the segment table (warp-uniform except at segment ends). IN and OUT slots as
// above; the fluid end is anchor + off[k].
template <int Q, class S>
__global__ void __launch_bounds__(256) k_bc_links(S* __restrict__ F, const GridDesc g, const int* __restrict__ links,
                                                  int n, const LinkSet ls, const BcParams bp, int parity) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  link_apply<Q, S>(F, g.dstride, links, t, ls, bp, parity);
}

template <int Q, class S>
static cudaError_t bc_links_impl(const DomainDev& d, const int* links, int n, const LinkSet& ls, const BcParams& bp,
                                 int parity, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_bc_links<Q, S><<<(n + 255) / 256, 256, 0, st>>>((S*)d.F, d.g, links, n, ls, bp, parity);
  return cudaGetLastError();
}

cudaError_t launch_bc_links(const DomainDev& d, const int* links, int n, const LinkSet& ls, const BcParams& bp,
                            int parity, cudaStream_t st) {
  ASLB_DISPATCH(d, bc_links_impl, d, links, n, ls, bp, parity, st)
}

// ---------------------------------------------------------------------------
// Reductions: warp shuffle, then one row of partial sums per block.
template <int W>
__device__ __forceinline__ void block_reduce_rows(double (&v)[W], double* __restrict__ partials) {
  __shared__ double sh[32][W];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < W; ++j)
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < W; ++j) sh[warp][j] = v[j];
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < W; ++j) {
      double a = lane < nw ? sh[lane][j] : 0.0;
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      if (lane == 0) partials[(size_t)blockIdx.x * W + j] = a;
    }
  }
}

// ComputeSurfaceForceMap (aslLBGKBC.cxx:691-736): per listed cell x,
//   F(x) = sum_k s_k (f_k(x) + f_inv(k)(x + c_k) - 2) w_k c_k
// with s_k = +1 for links from a solid x (mask0) and -1 from a fluid x (mask_in).
// f_k(x) + f_inv(k)(x + c_k) is the same pair of slots in both representations.
constexpr int kForceThreads = 256;
int force_blocks(int n) { return n > 0 ? (n + kForceThreads - 1) / kForceThreads : 1; }

template <int Q, class S>
__global__ void __launch_bounds__(kForceThreads)
    k_force(const S* __restrict__ F, const GridDesc g, const int4* __restrict__ cells,
            const uint32_t* __restrict__ mask_in, int n, float* __restrict__ field, double r00, double r01,
            double r02, double p00, double p01, double p02, double dx, float inv_scale,
            const uint2* __restrict__ fused, int parity, double* __restrict__ partials) {
  using Lt = Lattice<Q>;
  using C = typename Store<S>::C;
  constexpr bool kDev = std::is_same<S, __half>::value;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (t < n) {
    const int4 an = cells[t];
    const unsigned m0 = (unsigned)an.w, mi = mask_in[t];
    const bool px = g.periodic & 1, py = g.periodic & 2, pz = g.periodic & 4;
    const long long sa = sidx(g, an.x, an.y, an.z);
    C Fx = C(0), Fy = C(0), Fz = C(0);
#pragma unroll
    for (int k = 1; k < Q; ++k) {
      const bool b0 = m0 >> k & 1u, bi = mi >> k & 1u;
      if (!(b0 || bi)) continue;
      const long long sq = sidx(g, wrap_axis(an.x + Lt::c(k, 0), g.nx, px), wrap_axis(an.y + Lt::c(k, 1), g.ny, py),
                                wrap_axis(an.z + Lt::c(k, 2), g.nz, pz));
      const S* pa = F + (size_t)k * g.dstride + sa;           // f_k(x) in representation A
      const S* pq = F + (size_t)Lt::inv(k) * g.dstride + sq;  // f_inv(k)(x + c_k) in representation A
      // A fused no-slip link never writes the solid end's incoming slot:
      // bounce-back makes it equal to the fluid end's outgoing population. The
      // fluid end carries the link's bit (direction k into q for mask0 links,
      // direction inv(k) into the anchor for mask_in links).
      bool solid_fused = false;
      if (fused) solid_fused = ((b0 ? fused[sq].x : fused[sa].x) >> (b0 ? k : Lt::inv(k))) & 1u;
      C a;
      if (solid_fused) {
        // outgoing slot of the fluid end: the anchor's neighbour q for mask0
        // links, the anchor itself for mask_in links; representation B holds
        // it in the other slot of the pair.
        const S* out = (b0 != (parity != 0)) ? pq : pa;
        a = kDev ? C(2) * Store<S>::dev(out, inv_scale) : C(2) * Store<S>::val(out, inv_scale) - C(2);
      } else if (kDev) {
        a = Store<S>::dev(pa, inv_scale) + Store<S>::dev(pq, inv_scale);
      } else {
        a = Store<S>::val(pa, inv_scale) + Store<S>::val(pq, inv_scale) - C(2);
      }
      if (bi) a = -a;
      const C wa = a * C(Lt::w(k));
      if (Lt::c(k, 0)) Fx += Lt::c(k, 0) > 0 ? wa : -wa;
      if (Lt::c(k, 1)) Fy += Lt::c(k, 1) > 0 ? wa : -wa;
      if (Lt::c(k, 2)) Fz += Lt::c(k, 2) > 0 ? wa : -wa;
    }
    if (field) {
      const long long a = aidx(g, an.x, an.y, an.z);
      field[a] = float(Fx);
      field[g.L + a] = float(Fy);
      field[2 * g.L + a] = float(Fz);
    }
    const double r0 = p00 + (an.x - 1) * dx - r00;
    const double r1 = p01 + (an.y - 1) * dx - r01;
    const double r2 = p02 + (an.z - 1) * dx - r02;
    const double F0 = double(Fx), F1 = double(Fy), F2 = double(Fz);
    v[0] = F0;
    v[1] = F1;
    v[2] = F2;
    v[3] = r1 * F2 - r2 * F1;
    v[4] = r2 * F0 - r0 * F2;
    v[5] = r0 * F1 - r1 * F0;
  }
  block_reduce_rows<6>(v, partials);
}

__global__ void k_reduce_rows(const double* __restrict__ partials, int nrows, int width, double* __restrict__ out) {
  __shared__ double sh[256];
  for (int j = 0; j < width; ++j) {
    double a = 0.0;
    for (int r = threadIdx.x; r < nrows; r += blockDim.x) a += partials[(size_t)r * width + j];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = sh[0];
    __syncthreads();
  }
}

cudaError_t launch_reduce_rows(const double* partials, int nblocks, int width, double* out, cudaStream_t st) {
  k_reduce_rows<<<1, 256, 0, st>>>(partials, nblocks, width, out);
  return cudaGetLastError();
}

template <int Q, class S>
static cudaError_t force_impl(const DomainDev& d, const int4* cells, const uint32_t* mask_in, int n, float* field,
                              const double* r0, const double* pos0, double dx, float inv_scale,
                              const uint2* fused, int parity, double* partials, double* out6, cudaStream_t st) {
  const int nb = force_blocks(n);
  k_force<Q, S><<<nb, kForceThreads, 0, st>>>((const S*)d.F, d.g, cells, mask_in, n, field, r0[0], r0[1], r0[2],
                                              pos0[0], pos0[1], pos0[2], dx, inv_scale, fused, parity, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_rows(partials, nb, 6, out6, st);
}

// ComputeSurfaceFluxMap (aslLBGKBC.cxx:623-665): per cell with |map| < 0.9999,
// flux = sum_k w_k s_k (f*_k(x) - f*_inv(k)(x + c_k)), s_k = +1 for links from a
// solid x (mask0), -1 from a fluid x (mask_in). The two populations of a link
// swap slots between the AA representations. A fused no-slip link carries no
// flux: bounce-back makes its two populations equal, as the separate
// condition does before the flux is taken.
template <int Q, class S>
__global__ void __launch_bounds__(kForceThreads)
    k_flux(const S* __restrict__ F, const GridDesc g, const int4* __restrict__ cells,
           const uint32_t* __restrict__ mask_in, int n, float* __restrict__ field, float inv_scale,
           const uint2* __restrict__ fused, int parity, double* __restrict__ partials) {
  using Lt = Lattice<Q>;
  using C = typename Store<S>::C;
  constexpr bool kDev = std::is_same<S, __half>::value;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0};
  if (t < n) {
    const int4 an = cells[t];
    const unsigned m0 = (unsigned)an.w, mi = mask_in[t];
    const bool px = g.periodic & 1, py = g.periodic & 2, pz = g.periodic & 4;
    const long long sa = sidx(g, an.x, an.y, an.z);
    C flux = C(0);
#pragma unroll
    for (int k = 1; k < Q; ++k) {
      const bool b0 = m0 >> k & 1u, bi = mi >> k & 1u;
      if (!(b0 || bi)) continue;
      const long long sq = sidx(g, wrap_axis(an.x + Lt::c(k, 0), g.nx, px), wrap_axis(an.y + Lt::c(k, 1), g.ny, py),
                                wrap_axis(an.z + Lt::c(k, 2), g.nz, pz));
      if (fused && (((b0 ? fused[sq].x : fused[sa].x) >> (b0 ? k : Lt::inv(k))) & 1u)) continue;
      const S* pa = F + (size_t)k * g.dstride + sa;
      const S* pq = F + (size_t)Lt::inv(k) * g.dstride + sq;
      const S* p0 = parity == 0 ? pa : pq;  // f*_k(x)
      const S* pI = parity == 0 ? pq : pa;  // f*_inv(k)(x + c_k)
      C d = kDev ? Store<S>::dev(p0, inv_scale) - Store<S>::dev(pI, inv_scale)
                 : Store<S>::val(p0, inv_scale) - Store<S>::val(pI, inv_scale);
      if (bi) d = -d;
      flux += d * C(Lt::w(k));
    }
    if (field) field[aidx(g, an.x, an.y, an.z)] = float(flux);
    v[0] = double(flux);
  }
  block_reduce_rows<1>(v, partials);
}

template <int Q, class S>
static cudaError_t flux_impl(const DomainDev& d, const int4* cells, const uint32_t* mask_in, int n, float* field,
                             float inv_scale, const uint2* fused, int parity, double* partials, double* out1,
                             cudaStream_t st) {
  const int nb = force_blocks(n);
  k_flux<Q, S><<<nb, kForceThreads, 0, st>>>((const S*)d.F, d.g, cells, mask_in, n, field, inv_scale, fused, parity,
                                             partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_rows(partials, nb, 1, out1, st);
}

cudaError_t launch_flux(const DomainDev& d, const int4* cells, const uint32_t* mask_in, int n, float* field,
                        float inv_scale, const uint2* fused, int parity, double* partials, double* out1,
                        cudaStream_t st) {
  ASLB_DISPATCH(d, flux_impl, d, cells, mask_in, n, field, inv_scale, fused, parity, partials, out1, st)
}

cudaError_t launch_force(const DomainDev& d, const int4* cells, const uint32_t* mask_in, int n, float* field,
                         const double* r0, const double* pos0, double dx, float inv_scale, const uint2* fused,
                         int parity, double* partials, double* out6, cudaStream_t st) {
  ASLB_DISPATCH(d, force_impl, d, cells, mask_in, n, field, r0, pos0, dx, inv_scale, fused, parity, partials, out6, st)
}

// ---------------------------------------------------------------------------
// Mass and momentum of the post-collision populations over interior cells.
constexpr int kMomentThreads = 256;
int moments_blocks(const GridDesc& g) {
  long long cells = (long long)g.nx * g.ny * g.nz;
  long long b = (cells + kMomentThreads * 8 - 1) / (kMomentThreads * 8);
  if (b > 4096) b = 4096;
  return (int)(b < 1 ? 1 : b);
}

template <int Q, class S>
__global__ void __launch_bounds__(kMomentThreads)
    k_moments(const S* __restrict__ F, const GridDesc g, const StepParams p, int parity,
              double* __restrict__ partials) {
  using Lt = Lattice<Q>;
  double v[4] = {0, 0, 0, 0};
  const long long total = (long long)g.nx * g.ny * g.nz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const int z = int(c % g.nz) + 1;
    const long long r = c / g.nz;
    const int y = int(r % g.ny) + 1;
    const int x = int(r / g.ny) + 1;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const double fi = double(Store<S>::val(F + fstar_index<Q>(g, p.mask, parity, x, y, z, i), p.inv_scale));
      const double wf = Lt::w(i) * fi;
      v[0] += wf;
      v[1] += Lt::c(i, 0) * wf;
      v[2] += Lt::c(i, 1) * wf;
      v[3] += Lt::c(i, 2) * wf;
    }
  }
  block_reduce_rows<4>(v, partials);
}

template <int Q, class S>
static cudaError_t moments_impl(const DomainDev& d, const StepParams& p, int parity, double* partials, double* out4,
                                cudaStream_t st) {
  const int nb = moments_blocks(d.g);
  k_moments<Q, S><<<nb, kMomentThreads, 0, st>>>((const S*)d.F, d.g, p, parity, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_rows(partials, nb, 4, out4, st);
}

cudaError_t launch_moments(const DomainDev& d, const StepParams& p, int parity, double* partials, double* out4,
                           cudaStream_t st) {
  ASLB_DISPATCH(d, moments_impl, d, p, parity, partials, out4, st)
}

// Blow-up watchdog: per block, the largest |u|^2 and smallest rho over its
// interior cells (u = m / rho, or m for the incompressible equilibrium) and
// the number of cells with a non-finite rho or u; rows [max u^2, min rho,
// count], reduced on the host.
template <int Q, class S>
__global__ void __launch_bounds__(kMomentThreads)
    k_watchdog(const S* __restrict__ F, const GridDesc g, const StepParams p, int parity,
               double* __restrict__ partials) {
  using Lt = Lattice<Q>;
  double umax = 0.0, rmin = 1e300, bad = 0.0;
  const long long total = (long long)g.nx * g.ny * g.nz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const int z = int(c % g.nz) + 1;
    const long long r = c / g.nz;
    const int y = int(r % g.ny) + 1;
    const int x = int(r / g.ny) + 1;
    double rho = 0, m[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      // stored populations are f_i / w_i (ASL's layout): rho = sum w f, m = sum w c f
      const double wf =
          Lt::w(i) * double(Store<S>::val(F + fstar_index<Q>(g, p.mask, parity, x, y, z, i), p.inv_scale));
      rho += wf;
      m[0] += Lt::c(i, 0) * wf;
      m[1] += Lt::c(i, 1) * wf;
      m[2] += Lt::c(i, 2) * wf;
    }
    const double inv = p.compressible ? 1.0 / rho : 1.0;
    const double u2 = (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) * inv * inv;
    if (!isfinite(u2) || !isfinite(rho)) {
      bad += 1.0;
    } else {
      umax = fmax(umax, u2);
      rmin = fmin(rmin, rho);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    umax = fmax(umax, __shfl_down_sync(0xffffffffu, umax, o));
    rmin = fmin(rmin, __shfl_down_sync(0xffffffffu, rmin, o));
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  __shared__ double sh[32][3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sh[warp][0] = umax;
    sh[warp][1] = rmin;
    sh[warp][2] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      umax = fmax(umax, sh[w][0]);
      rmin = fmin(rmin, sh[w][1]);
      bad += sh[w][2];
    }
    partials[(size_t)blockIdx.x * 3 + 0] = umax;
    partials[(size_t)blockIdx.x * 3 + 1] = rmin;
    partials[(size_t)blockIdx.x * 3 + 2] = bad;
  }
}

template <int Q, class S>
static cudaError_t watchdog_impl(const DomainDev& d, const StepParams& p, int parity, double* partials,
                                 cudaStream_t st) {
  k_watchdog<Q, S><<<moments_blocks(d.g), kMomentThreads, 0, st>>>((const S*)d.F, d.g, p, parity, partials);
  return cudaGetLastError();
}

cudaError_t launch_watchdog(const DomainDev& d, const StepParams& p, int parity, double* partials, cudaStream_t st) {
  ASLB_DISPATCH(d, watchdog_impl, d, p, parity, partials, st)
}

// Density and velocity of every interior cell from the populations as they
// stand (the post-collision values of the last step), into the domain's rho /
// u fields in ASL's ghosted layout: rho = sum w f, u = m / rho (m for the
// incompressible equilibrium), m = sum w c f, accumulated in the macro type.
template <int Q, class S>
__global__ void __launch_bounds__(256) k_compute_macro(const S* __restrict__ F, const GridDesc g, const StepParams p,
                                                       int parity, int comp_rho, int comp_vel,
                                                       typename MacroT<S>::T* __restrict__ rho_out,
                                                       typename MacroT<S>::T* __restrict__ u_out) {
  using Lt = Lattice<Q>;
  using M = typename MacroT<S>::T;
  const int z = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y + 1;
  const int x = blockIdx.z + 1;
  if (z > g.nz) return;
  M rho = M(0), m0 = M(0), m1 = M(0), m2 = M(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const M wf = M(Lt::w(i)) * M(Store<S>::val(F + fstar_index<Q>(g, p.mask, parity, x, y, z, i), p.inv_scale));
    rho += wf;
    if (Lt::c(i, 0)) m0 += Lt::c(i, 0) > 0 ? wf : -wf;
    if (Lt::c(i, 1)) m1 += Lt::c(i, 1) > 0 ? wf : -wf;
    if (Lt::c(i, 2)) m2 += Lt::c(i, 2) > 0 ? wf : -wf;
  }
  const long long a = aidx(g, x, y, z);
  if (comp_rho) rho_out[a] = rho;
  if (comp_vel) {
    const M inv = p.compressible ? M(1) / rho : M(1);
    u_out[a] = m0 * inv;
    u_out[g.L + a] = m1 * inv;
    u_out[2 * g.L + a] = m2 * inv;
  }
}

template <int Q, class S>
static cudaError_t compute_macro_impl(const DomainDev& d, const StepParams& p, int parity, int comp_rho,
                                      int comp_vel, cudaStream_t st) {
  using M = typename MacroT<S>::T;
  dim3 block(128), grid((d.g.nz + 127) / 128, d.g.ny, d.g.nx);
  k_compute_macro<Q, S><<<grid, block, 0, st>>>((const S*)d.F, d.g, p, parity, comp_rho, comp_vel, (M*)d.rho,
                                                (M*)d.u);
  return cudaGetLastError();
}

cudaError_t launch_compute_macro(const DomainDev& d, const StepParams& p, int parity, int comp_rho, int comp_vel,
                                 cudaStream_t st) {
  ASLB_DISPATCH(d, compute_macro_impl, d, p, parity, comp_rho, comp_vel, st)
}

}  // namespace aslb
