// Per-cell LBGK collision in ASL's formulation (src/num/aslLBGK.cxx:187-235,
// 298-355 of the reference project), ASL-normalised populations:
//   m = sum_i w_i c_i f_i,  rho = sum_i w_i f_i
//   f_eq,i = rho + 3 c_i.m + 4.5 (c_i.m)^2 / rho - 1.5 m.m / rho   (compressible)
//   f_eq,i = rho + 3 c_i.m + 4.5 (c_i.m)^2       - 1.5 m.m         (incompressible)
//   f_i   <- (1 - omega) f_i + omega f_eq,i,  omega = 1 / (3 nu + 1/2)
// plus the optional Coriolis term (component-sequential like ASL's generated
// code), Guo forcing for a body force, and the closures that replace omega.
#pragma once
#include <type_traits>
#include "internal.cuh"
#include "mlp.cuh"

namespace aslb {

// Arithmetic the compiler may neither re-associate nor fuse into other
// multiply-adds: every kernel variant that computes a cell produces the same
// bits, whatever code surrounds the collision.
__device__ __forceinline__ float mul_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float div_(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_(double a, double b) { return __ddiv_rn(a, b); }

// c_i . v with the lattice vector known at compile time: only the nonzero
// components are added (0 * v cannot be dropped by the compiler under IEEE
// rules), the same value as the full dot product for finite v.
template <int Q, class C>
__device__ __forceinline__ C cdot(int i, C v0, C v1, C v2) {
  using Lt = Lattice<Q>;
  C r = C(0);
  bool first = true;
  if (Lt::c(i, 0)) { r = Lt::c(i, 0) > 0 ? v0 : -v0; first = false; }
  if (Lt::c(i, 1)) { r = first ? (Lt::c(i, 1) > 0 ? v1 : -v1) : (Lt::c(i, 1) > 0 ? add_(r, v1) : sub_(r, v1)); first = false; }
  if (Lt::c(i, 2)) { r = first ? (Lt::c(i, 2) > 0 ? v2 : -v2) : (Lt::c(i, 2) > 0 ? add_(r, v2) : sub_(r, v2)); }
  return r;
}

template <int Q, class C, int CL>
__device__ __forceinline__ void collide_cell(C (&f)[Q], const StepParams& p, C& rho_out, C (&u_out)[3]) {
  using Lt = Lattice<Q>;
  C m0 = C(0), m1 = C(0), m2 = C(0), rho = C(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const C wf = mul_(C(Lt::w(i)), f[i]);
    rho = add_(rho, wf);
    if (Lt::c(i, 0) > 0) m0 = add_(m0, wf);
    if (Lt::c(i, 0) < 0) m0 = sub_(m0, wf);
    if (Lt::c(i, 1) > 0) m1 = add_(m1, wf);
    if (Lt::c(i, 1) < 0) m1 = sub_(m1, wf);
    if (Lt::c(i, 2) > 0) m2 = add_(m2, wf);
    if (Lt::c(i, 2) < 0) m2 = sub_(m2, wf);
  }
  // omega = 1 / (3 nu + 1/2), evaluated on the host in the storage's arithmetic
  const C om0 = std::is_same<C, double>::value ? C(p.om0d) : C(p.om0f);
  C om = om0;
  if (p.has_coriolis) {
    // component-sequential, as ACL emits `momentum += (2/w) Omega x momentum`
    const C k = div_(C(2), om);
    const C O0 = C(p.Om[0]), O1 = C(p.Om[1]), O2 = C(p.Om[2]);
    m0 = fma_(k, sub_(mul_(O1, m2), mul_(O2, m1)), m0);
    m1 = fma_(k, sub_(mul_(O2, m0), mul_(O0, m2)), m1);
    m2 = fma_(k, sub_(mul_(O0, m1), mul_(O1, m0)), m2);
  }
  if (p.has_force) {
    const C hr = mul_(C(0.5), rho);
    m0 = fma_(hr, C(p.g[0]), m0);
    m1 = fma_(hr, C(p.g[1]), m1);
    m2 = fma_(hr, C(p.g[2]), m2);
  }
  const C inv_rho = div_(C(1), rho);
  rho_out = rho;
  if (p.compressible) {
    u_out[0] = mul_(m0, inv_rho);
    u_out[1] = mul_(m1, inv_rho);
    u_out[2] = mul_(m2, inv_rho);
  } else {
    u_out[0] = m0;
    u_out[1] = m1;
    u_out[2] = m2;
  }
  const C mm = fma_(m2, m2, fma_(m1, m1, mul_(m0, m0)));
  const C a2 = p.compressible ? mul_(C(4.5), inv_rho) : C(4.5);
  const C a0 = p.compressible ? sub_(rho, mul_(mul_(C(1.5), mm), inv_rho)) : sub_(rho, mul_(C(1.5), mm));

  if (CL == CL_ASL_INTENT || CL == CL_SMAGORINSKY || CL == CL_MLP) {
    // Non-equilibrium quantities need f_eq first.
    C sn = C(0), sf = C(0);
    C P00 = C(0), P11 = C(0), P22 = C(0), P01 = C(0), P12 = C(0), P02 = C(0);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const C cm = cdot<Q, C>(i, m0, m1, m2);
      const C feq = fma_(a2, mul_(cm, cm), fma_(C(3), cm, a0));
      const C d = sub_(f[i], feq);
      if (CL == CL_ASL_INTENT) {
        sn = fma_(d, d, sn);
        sf = fma_(f[i], f[i], sf);
      } else {
        const C wd = mul_(C(Lt::w(i)), d);
        if (Lt::c(i, 0) != 0) P00 += wd;
        if (Lt::c(i, 1) != 0) P11 += wd;
        if (Lt::c(i, 2) != 0) P22 += wd;
        if (Lt::c(i, 0) * Lt::c(i, 1) > 0) P01 += wd;
        if (Lt::c(i, 0) * Lt::c(i, 1) < 0) P01 -= wd;
        if (Lt::c(i, 1) * Lt::c(i, 2) > 0) P12 += wd;
        if (Lt::c(i, 1) * Lt::c(i, 2) < 0) P12 -= wd;
        if (Lt::c(i, 0) * Lt::c(i, 2) > 0) P02 += wd;
        if (Lt::c(i, 0) * Lt::c(i, 2) < 0) P02 -= wd;
      }
    }
    if (CL == CL_ASL_INTENT) {
      // LBGKTurbulence's limiter: w = 4 |f - f_eq|^2 / |f|^2
      const C wl = mul_(C(4), div_(sn, sf));
      if (wl > C(1)) om = div_(C(1), add_(mul_(C(3), fmin(mul_(C(p.nu), wl), C(0.5))), C(0.5)));
    } else if (CL == CL_SMAGORINSKY) {
      // Hou, Sterling, Chen & Doolen (1996): tau = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 |Pi_neq| / rho)) / 2
      const C q2 = add_(fma_(P22, P22, fma_(P11, P11, mul_(P00, P00))),
                        mul_(C(2), fma_(P02, P02, fma_(P12, P12, mul_(P01, P01)))));
      const C tau0 = div_(C(1), om0);
      const C cs2 = mul_(C(p.cs), C(p.cs));
      const C tau = mul_(C(0.5), add_(tau0, sqrt(fma_(tau0, tau0, mul_(mul_(mul_(C(25.455844122715710), cs2),
                                                                            sqrt(q2)), inv_rho)))));
      om = div_(C(1), tau);
    } else {
      // Learned closure: tau_eff from invariants of Pi_neq and the strain.
      om = mlp_omega<C>(p.mlp, om0, rho, m0 * inv_rho, m1 * inv_rho, m2 * inv_rho, P00, P11, P22, P01, P12, P02);
    }
  }

  // Relaxation folded into three multiply-adds per direction:
  //   (1 - om) f + om f_eq = (1 - om) f + om a0 + cm (3 om + om a2 cm)
  const C one_m = sub_(C(1), om);
  const C oa0 = mul_(om, a0), o3 = mul_(C(3), om), oa2 = mul_(om, a2);
  // Guo source (1 - om/2) rho [3 (c - u).g + 9 (c.u)(c.g)] with u = m / rho:
  //   c.g (hs3 + hs9 c.m) + sA,  hs9 = 9 hs / rho,  sA = -hs3 u.g
  C gx = C(0), gy = C(0), gz = C(0), hs3 = C(0), hs9 = C(0), sA = C(0);
  if (p.has_force) {
    gx = C(p.g[0]);
    gy = C(p.g[1]);
    gz = C(p.g[2]);
    const C hs = mul_(sub_(C(1), mul_(C(0.5), om)), rho);
    hs3 = mul_(C(3), hs);
    hs9 = mul_(mul_(C(9), hs), inv_rho);
    sA = -mul_(hs3, mul_(fma_(m2, gz, fma_(m1, gy, mul_(m0, gx))), inv_rho));
  }
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const C cm = cdot<Q, C>(i, m0, m1, m2);
    C fn = fma_(one_m, f[i], fma_(fma_(oa2, cm, o3), cm, oa0));
    if (p.has_force) {
      const C cg = cdot<Q, C>(i, gx, gy, gz);
      fn = add_(fn, fma_(cg, fma_(hs9, cm, hs3), sA));
    }
    f[i] = fn;
  }
}

}  // namespace aslb
