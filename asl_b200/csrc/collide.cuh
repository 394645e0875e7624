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

// c_i . v with the lattice vector known at compile time: only the nonzero
// components are added (0 * v cannot be dropped by the compiler under IEEE
// rules), the same value as the full dot product for finite v.
template <int Q, class C>
__device__ __forceinline__ C cdot(int i, C v0, C v1, C v2) {
  using Lt = Lattice<Q>;
  C r = C(0);
  bool first = true;
  if (Lt::c(i, 0)) { r = Lt::c(i, 0) > 0 ? v0 : -v0; first = false; }
  if (Lt::c(i, 1)) { r = first ? (Lt::c(i, 1) > 0 ? v1 : -v1) : (Lt::c(i, 1) > 0 ? r + v1 : r - v1); first = false; }
  if (Lt::c(i, 2)) { r = first ? (Lt::c(i, 2) > 0 ? v2 : -v2) : (Lt::c(i, 2) > 0 ? r + v2 : r - v2); }
  return r;
}

template <int Q, class C, int CL>
__device__ __forceinline__ void collide_cell(C (&f)[Q], const StepParams& p, C& rho_out, C (&u_out)[3]) {
  using Lt = Lattice<Q>;
  C m0 = C(0), m1 = C(0), m2 = C(0), rho = C(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const C wf = C(Lt::w(i)) * f[i];
    rho += wf;
    if (Lt::c(i, 0) > 0) m0 += wf;
    if (Lt::c(i, 0) < 0) m0 -= wf;
    if (Lt::c(i, 1) > 0) m1 += wf;
    if (Lt::c(i, 1) < 0) m1 -= wf;
    if (Lt::c(i, 2) > 0) m2 += wf;
    if (Lt::c(i, 2) < 0) m2 -= wf;
  }
  // omega = 1 / (3 nu + 1/2), evaluated on the host in the storage's arithmetic
  const C om0 = std::is_same<C, double>::value ? C(p.om0d) : C(p.om0f);
  C om = om0;
  if (p.has_coriolis) {
    const C k = C(2) / om;
    m0 = m0 + k * (C(p.Om[1]) * m2 - C(p.Om[2]) * m1);
    m1 = m1 + k * (C(p.Om[2]) * m0 - C(p.Om[0]) * m2);
    m2 = m2 + k * (C(p.Om[0]) * m1 - C(p.Om[1]) * m0);
  }
  if (p.has_force) {
    const C hr = C(0.5) * rho;
    m0 += hr * C(p.g[0]);
    m1 += hr * C(p.g[1]);
    m2 += hr * C(p.g[2]);
  }
  const C inv_rho = C(1) / rho;
  rho_out = rho;
  if (p.compressible) {
    u_out[0] = m0 * inv_rho;
    u_out[1] = m1 * inv_rho;
    u_out[2] = m2 * inv_rho;
  } else {
    u_out[0] = m0;
    u_out[1] = m1;
    u_out[2] = m2;
  }
  const C mm = m0 * m0 + m1 * m1 + m2 * m2;
  const C a2 = p.compressible ? C(4.5) * inv_rho : C(4.5);
  const C a0 = p.compressible ? rho - C(1.5) * mm * inv_rho : rho - C(1.5) * mm;

  if (CL == CL_ASL_INTENT || CL == CL_SMAGORINSKY || CL == CL_MLP) {
    // Non-equilibrium quantities need f_eq first.
    C sn = C(0), sf = C(0);
    C P00 = C(0), P11 = C(0), P22 = C(0), P01 = C(0), P12 = C(0), P02 = C(0);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const C cm = cdot<Q, C>(i, m0, m1, m2);
      const C feq = a0 + C(3) * cm + a2 * (cm * cm);
      const C d = f[i] - feq;
      if (CL == CL_ASL_INTENT) {
        sn += d * d;
        sf += f[i] * f[i];
      } else {
        const C wd = C(Lt::w(i)) * d;
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
      const C wl = C(4) * (sn / sf);
      if (wl > C(1)) om = C(1) / (C(3) * fmin(C(p.nu) * wl, C(0.5)) + C(0.5));
    } else if (CL == CL_SMAGORINSKY) {
      // Hou, Sterling, Chen & Doolen (1996): tau = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 |Pi_neq| / rho)) / 2
      const C q2 = P00 * P00 + P11 * P11 + P22 * P22 + C(2) * (P01 * P01 + P12 * P12 + P02 * P02);
      const C tau0 = C(1) / om0;
      const C cs2 = C(p.cs) * C(p.cs);
      const C tau = C(0.5) * (tau0 + sqrt(tau0 * tau0 + C(25.455844122715710) * cs2 * sqrt(q2) * inv_rho));
      om = C(1) / tau;
    } else {
      // Learned closure: tau_eff from invariants of Pi_neq and the strain.
      om = mlp_omega<C>(p.mlp, om0, rho, m0 * inv_rho, m1 * inv_rho, m2 * inv_rho, P00, P11, P22, P01, P12, P02);
    }
  }

  // Relaxation folded into three multiply-adds per direction:
  //   (1 - om) f + om f_eq = (1 - om) f + om a0 + cm (3 om + om a2 cm)
  const C one_m = C(1) - om;
  const C oa0 = om * a0, o3 = C(3) * om, oa2 = om * a2;
  // Guo source (1 - om/2) rho [3 (c - u).g + 9 (c.u)(c.g)] with u = m / rho:
  //   hs3 c.g + hs9 (c.m / rho)(c.g) - hs3 u.g
  C gx = C(0), gy = C(0), gz = C(0), hs3 = C(0), hs9 = C(0), sA = C(0);
  if (p.has_force) {
    gx = C(p.g[0]);
    gy = C(p.g[1]);
    gz = C(p.g[2]);
    const C hs = (C(1) - C(0.5) * om) * rho;
    hs3 = C(3) * hs;
    hs9 = C(9) * hs * inv_rho;
    sA = -hs3 * ((m0 * gx + m1 * gy + m2 * gz) * inv_rho);
  }
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const C cm = cdot<Q, C>(i, m0, m1, m2);
    C t = oa2 * cm + o3;
    t = t * cm + oa0;
    C fn = one_m * f[i] + t;
    if (p.has_force) {
      const C cg = cdot<Q, C>(i, gx, gy, gz);
      fn += cg * (hs3 + hs9 * cm) + sA;
    }
    f[i] = fn;
  }
}

}  // namespace aslb
