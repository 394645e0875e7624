// Per-cell LBGK collision in ASL's formulation (src/num/aslLBGK.cxx:187-235,
// 298-355 of the reference project), ASL-normalised populations:
//   m = sum_i w_i c_i f_i,  rho = sum_i w_i f_i
//   f_eq,i = rho + 3 c_i.m + 4.5 (c_i.m)^2 / rho - 1.5 m.m / rho   (compressible)
//   f_eq,i = rho + 3 c_i.m + 4.5 (c_i.m)^2       - 1.5 m.m         (incompressible)
//   f_i   <- (1 - omega) f_i + omega f_eq,i,  omega = 1 / (3 nu + 1/2)
// plus the optional Coriolis term (component-sequential like ASL's generated
// code), Guo forcing for a body force, and the closures that replace omega.
//
// Evaluation. Opposite directions i, i' = inv(i) share |c|^2 and weight, and
// c_i.v = -c_i'.v, so the kernel works on pairs:
//   moments   s = f_i + f_i', d = f_i - f_i', summed per weight class first
//             (rho = w_0 f_0 + sum_k w_k S_k, m = sum_k w_k M_k),
//   update    f_i  <- (1 - om) f_i  + (P + A)
//             f_i' <- (1 - om) f_i' + (P - A)
//   with the even part P = om (a0 + a2 cm^2) + Guo's even part and the odd
//   part A = 3 om cm + Guo's odd part (cm = c_i.m). The result is the same
//   expression as ASL's, evaluated in another order (rounding differences only).
//
// Collision representation. FP32/FP64 storage hands the collision f itself.
// FP16 storage holds D = (f - 1) * sigma and the collision works on D
// directly: with V = sum w D = sigma (rho - 1) and M = sum w c D = sigma m,
//   sigma (f_eq,i - 1) = V + 3 c.M + 4.5 (c.M)^2 / (sigma rho) - 1.5 M.M / (sigma rho)
// i.e. the same update with a0, a2 rescaled, and rho = 1 + V / sigma.
#pragma once
#include <type_traits>
#include <utility>
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

// Compile-time loop: f(std::integral_constant<int, I>) for I = 0 .. N-1.
template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// Opposite pairs of a lattice, grouped by |c|^2 (the weight class).
template <int Q>
struct Pairs {
  using Lt = Lattice<Q>;
  // i represents the pair (i, inv i)
  __host__ __device__ static constexpr bool rep(int i) { return i > 0 && i < Lt::inv(i); }
  __host__ __device__ static constexpr bool present(int k) {
    for (int j = 1; j < Q; ++j)
      if (Lt::norm2(j) == k) return true;
    return false;
  }
  __host__ __device__ static constexpr int first_of(int k) {
    for (int j = 1; j < Q; ++j)
      if (Lt::norm2(j) == k) return j;
    return 0;
  }
  // first representative of its class (with c_a != 0 when a >= 0)
  __host__ __device__ static constexpr bool first(int i, int a) {
    for (int j = 1; j < i; ++j)
      if (rep(j) && Lt::norm2(j) == Lt::norm2(i) && (a < 0 || Lt::c(j, a) != 0)) return false;
    return true;
  }
  // smallest class present
  __host__ __device__ static constexpr int kmin() { return present(1) ? 1 : (present(2) ? 2 : 3); }
};

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

// Step parameters in the collision's arithmetic (FP32 copies for float).
template <class C>
__device__ __forceinline__ C par_g(const StepParams& p, int a) {
  if constexpr (std::is_same<C, double>::value) return p.g[a]; else return p.gf[a];
}
template <class C>
__device__ __forceinline__ C par_Om(const StepParams& p, int a) {
  if constexpr (std::is_same<C, double>::value) return p.Om[a]; else return p.Omf[a];
}
template <class C>
__device__ __forceinline__ C par_cg(const StepParams& p, int i) {
  if constexpr (std::is_same<C, double>::value) return p.cgd[i]; else return p.cgf[i];
}
template <class C>
__device__ __forceinline__ C par_nu(const StepParams& p) {
  if constexpr (std::is_same<C, double>::value) return p.nu; else return p.nuf;
}
template <class C>
__device__ __forceinline__ C par_cs(const StepParams& p) {
  if constexpr (std::is_same<C, double>::value) return p.cs; else return p.csf;
}

// omega = 1 / (3 nu + 1/2), evaluated on the host in the storage's arithmetic
template <class C>
__device__ __forceinline__ C step_omega(const StepParams& p) {
  if constexpr (std::is_same<C, double>::value) return p.om0d; else return p.om0f;
}

// Moments of one cell and the equilibrium coefficients,
//   f_eq,i = a0 + 3 c_i.m + a2 (c_i.m)^2,
// in the collision representation (m and a0 scaled by sigma with DEV).
template <class C>
struct Moments {
  C V, rho, inv_rho, m0, m1, m2, ium, a0, a2;
};

template <int Q, class C, bool DEV>
__device__ __forceinline__ Moments<C> cell_moments(const C (&f)[Q], const StepParams& p, const C om0) {
  using Lt = Lattice<Q>;
  using Pr = Pairs<Q>;
  // pair sums and differences, per weight class
  C S[4], M[4][3];
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    if constexpr (Pr::rep(i)) {
      constexpr int j = Lt::inv(i);
      constexpr int k = Lt::norm2(i);
      const C s = add_(f[i], f[j]);
      const C d = sub_(f[i], f[j]);
      if constexpr (Pr::first(i, -1)) S[k] = s; else S[k] = add_(S[k], s);
      static_for<3>([&](auto ac) {
        constexpr int a = decltype(ac)::value;
        if constexpr (Lt::c(i, a) != 0) {
          if constexpr (Pr::first(i, a)) M[k][a] = Lt::c(i, a) > 0 ? d : -d;
          else M[k][a] = Lt::c(i, a) > 0 ? add_(M[k][a], d) : sub_(M[k][a], d);
        }
      });
    }
  });
  Moments<C> r;
  C V = mul_(C(Lt::w(0)), f[0]);
  C m0 = C(0), m1 = C(0), m2 = C(0);
  static_for<4>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    if constexpr (k > 0 && Pr::present(k)) {
      const C wk = C(Lt::w(Pr::first_of(k)));
      V = fma_(wk, S[k], V);
      if constexpr (k == Pr::kmin()) {
        m0 = mul_(wk, M[k][0]);
        m1 = mul_(wk, M[k][1]);
        m2 = mul_(wk, M[k][2]);
      } else {
        m0 = fma_(wk, M[k][0], m0);
        m1 = fma_(wk, M[k][1], m1);
        m2 = fma_(wk, M[k][2], m2);
      }
    }
  });
  // rho; with DEV, V = sigma (rho - 1) and m = sigma * momentum
  const C sig = DEV ? C(p.scale) : C(1);
  const C isig = DEV ? C(p.inv_scale) : C(1);
  const C rho = DEV ? fma_(V, isig, C(1)) : V;
  if (p.has_coriolis) {
    // component-sequential, as ACL emits `momentum += (2/w) Omega x momentum`
    const C k = div_(C(2), om0);
    const C O0 = par_Om<C>(p, 0), O1 = par_Om<C>(p, 1), O2 = par_Om<C>(p, 2);
    m0 = fma_(k, sub_(mul_(O1, m2), mul_(O2, m1)), m0);
    m1 = fma_(k, sub_(mul_(O2, m0), mul_(O0, m2)), m1);
    m2 = fma_(k, sub_(mul_(O0, m1), mul_(O1, m0)), m2);
  }
  if (p.has_force) {
    const C hr = DEV ? mul_(mul_(C(0.5), rho), sig) : mul_(C(0.5), rho);
    m0 = fma_(hr, par_g<C>(p, 0), m0);
    m1 = fma_(hr, par_g<C>(p, 1), m1);
    m2 = fma_(hr, par_g<C>(p, 2), m2);
  }
  const C inv_rho = div_(C(1), rho);
  // factor taking the stored momentum to velocity (u = m / rho, or m when
  // incompressible), with the 1 / sigma of DEV folded in
  const C ium = p.compressible ? (DEV ? mul_(isig, inv_rho) : inv_rho) : isig;
  const C mm = fma_(m2, m2, fma_(m1, m1, mul_(m0, m0)));
  r.a2 = (DEV || p.compressible) ? mul_(C(4.5), ium) : C(4.5);
  r.a0 = (DEV || p.compressible) ? sub_(V, mul_(mul_(C(1.5), mm), ium)) : sub_(V, mul_(C(1.5), mm));
  r.V = V;
  r.rho = rho;
  r.inv_rho = inv_rho;
  r.m0 = m0;
  r.m1 = m1;
  r.m2 = m2;
  r.ium = ium;
  return r;
}

// Non-equilibrium stress Pi_ab = sum_i w_i c_ia c_ib (f_i - f_eq,i) in ASL's
// normalisation, order (00, 11, 22, 01, 12, 02).
template <int Q, class C, bool DEV>
__device__ __forceinline__ void cell_pneq(const C (&f)[Q], const Moments<C>& mo, const StepParams& p, C (&P)[6]) {
  using Lt = Lattice<Q>;
  C P00 = C(0), P11 = C(0), P22 = C(0), P01 = C(0), P12 = C(0), P02 = C(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const C cm = cdot<Q, C>(i, mo.m0, mo.m1, mo.m2);
    const C feq = fma_(mo.a2, mul_(cm, cm), fma_(C(3), cm, mo.a0));
    const C wd = mul_(C(Lt::w(i)), sub_(f[i], feq));
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
  if (DEV) {
    const C isig = C(p.inv_scale);
    P00 = mul_(P00, isig); P11 = mul_(P11, isig); P22 = mul_(P22, isig);
    P01 = mul_(P01, isig); P12 = mul_(P12, isig); P02 = mul_(P02, isig);
  }
  P[0] = P00; P[1] = P11; P[2] = P22; P[3] = P01; P[4] = P12; P[5] = P02;
}

// f: the Q values of one cell in the collision representation (f, or
// D = (f - 1) sigma when DEV), replaced by the post-collision values.
// om0: the BGK relaxation rate (step_omega, or a batch domain's own).
// cs2_cell: the cell's Smagorinsky coefficient Cs^2 for the learned closure
// (CL_MLP, from the closure field); unused otherwise.
// rho_out / u_out: density and velocity (ASL's compRho / compVel fields).
template <int Q, class C, int CL, bool DEV = false>
__device__ __forceinline__ void collide_cell(C (&f)[Q], const StepParams& p, const C om0, const C cs2_cell,
                                             C& rho_out, C (&u_out)[3]) {
  using Lt = Lattice<Q>;
  using Pr = Pairs<Q>;
  const Moments<C> mo = cell_moments<Q, C, DEV>(f, p, om0);
  const C rho = mo.rho, inv_rho = mo.inv_rho, m0 = mo.m0, m1 = mo.m1, m2 = mo.m2, a0 = mo.a0, a2 = mo.a2;
  const C sig = DEV ? C(p.scale) : C(1);
  const C isig = DEV ? C(p.inv_scale) : C(1);
  rho_out = rho;
  if (DEV || p.compressible) {
    u_out[0] = mul_(m0, mo.ium);
    u_out[1] = mul_(m1, mo.ium);
    u_out[2] = mul_(m2, mo.ium);
  } else {
    u_out[0] = m0;
    u_out[1] = m1;
    u_out[2] = m2;
  }

  C om = om0;
  if constexpr (CL == CL_ASL_INTENT) {
    // LBGKTurbulence's limiter: w = 4 |f - f_eq|^2 / |f|^2 (f_eq scaled by sigma with DEV)
    C sn = C(0), sf = C(0);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const C cm = cdot<Q, C>(i, m0, m1, m2);
      const C feq = fma_(a2, mul_(cm, cm), fma_(C(3), cm, a0));
      const C d = sub_(f[i], feq);
      const C fa = DEV ? fma_(f[i], isig, C(1)) : f[i];
      sn = fma_(d, d, sn);
      sf = fma_(fa, fa, sf);
    }
    if (DEV) sn = mul_(mul_(sn, isig), isig);
    const C wl = mul_(C(4), div_(sn, sf));
    if (wl > C(1)) om = div_(C(1), add_(mul_(C(3), fmin(mul_(par_nu<C>(p), wl), C(0.5))), C(0.5)));
  } else if constexpr (CL == CL_SMAGORINSKY || CL == CL_MLP) {
    // Hou, Sterling, Chen & Doolen (1996): tau = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 |Pi_neq| / rho)) / 2,
    // Cs^2 constant (Smagorinsky) or the network's per-cell value (learned closure)
    C P[6];
    cell_pneq<Q, C, DEV>(f, mo, p, P);
    const C q2 = add_(fma_(P[2], P[2], fma_(P[1], P[1], mul_(P[0], P[0]))),
                      mul_(C(2), fma_(P[5], P[5], fma_(P[4], P[4], mul_(P[3], P[3])))));
    const C tau0 = div_(C(1), om0);
    C cs2;
    if constexpr (CL == CL_SMAGORINSKY) {
      const C cs = par_cs<C>(p);
      cs2 = mul_(cs, cs);
    } else {
      cs2 = cs2_cell;
    }
    const C tau = mul_(C(0.5), add_(tau0, sqrt(fma_(tau0, tau0, mul_(mul_(mul_(C(25.455844122715710), cs2),
                                                                          sqrt(q2)), inv_rho)))));
    om = div_(C(1), tau);
  }

  // ---- relaxation, one opposite pair at a time:
  //   (1 - om) f + om f_eq = (1 - om) f + [om a0 + om a2 cm^2] +- [3 om cm]
  const C one_m = sub_(C(1), om);
  const C oa0 = mul_(om, a0), o3 = mul_(C(3), om), oa2 = mul_(om, a2);
  // Guo source (1 - om/2) rho [3 (c - u).g + 9 (c.u)(c.g)] with u = m / rho,
  // times sigma with DEV:  even part hs9 cm cg + sA, odd part hs3 cg, with
  // hs = (1 - om/2) rho, hs3 = 3 sigma hs, hs9 = 9 hs / rho, sA = -3 hs (m.g) / rho.
  C hs3 = C(0), hs9 = C(0), c0 = oa0;
  if (p.has_force) {
    const C gx = par_g<C>(p, 0), gy = par_g<C>(p, 1), gz = par_g<C>(p, 2);
    const C hs = mul_(sub_(C(1), mul_(C(0.5), om)), rho);
    const C h3 = mul_(C(3), hs);
    hs3 = DEV ? mul_(h3, sig) : h3;
    hs9 = mul_(mul_(C(9), hs), inv_rho);
    const C sA = -mul_(h3, mul_(fma_(m2, gz, fma_(m1, gy, mul_(m0, gx))), inv_rho));
    c0 = add_(oa0, sA);
  }
  f[0] = fma_(one_m, f[0], c0);
  static_for<Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    if constexpr (Pr::rep(i)) {
      constexpr int j = Lt::inv(i);
      const C cm = cdot<Q, C>(i, m0, m1, m2);
      C P = fma_(mul_(oa2, cm), cm, c0);
      C A = mul_(o3, cm);
      if (p.has_force) {
        const C cg = par_cg<C>(p, i);
        P = fma_(mul_(hs9, cg), cm, P);
        A = fma_(hs3, cg, A);
      }
      f[i] = fma_(one_m, f[i], add_(P, A));
      f[j] = fma_(one_m, f[j], sub_(P, A));
    }
  });
}

}  // namespace aslb
