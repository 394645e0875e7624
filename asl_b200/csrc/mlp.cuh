// Learned closure: a 9 -> 64 -> 64 -> 1 multilayer perceptron maps local
// invariants of the non-equilibrium stress Pi_neq (the strain-rate tensor up to
// a factor -1/(2 rho cs^2 tau)) to a local Smagorinsky coefficient Cs^2 >= 0,
// which sets the relaxation time through the Hou et al. (1996) closed form.
// Smagorinsky with a constant Cs is the special case of a constant network
// output, and tau_eff >= tau0 holds for every output, so the closure cannot
// make the scheme less dissipative than plain BGK.
#pragma once
#include <cuda_bf16.h>
#include "internal.cuh"

namespace aslb {

constexpr int kMlpIn = 9;
constexpr int kMlpInPad = 16;
constexpr int kMlpHidden = 64;

// Device-resident network. Weights are BF16, accumulation FP32.
struct MlpNet {
  float in_shift[kMlpInPad];               // feature normalisation x' = (x - shift) * scale
  float in_scale[kMlpInPad];
  __nv_bfloat16 w1[kMlpHidden][kMlpInPad]; // [out][in]
  float b1[kMlpHidden];
  __nv_bfloat16 w2[kMlpHidden][kMlpHidden];
  float b2[kMlpHidden];
  __nv_bfloat16 w3[kMlpHidden];
  float b3;
  float out_scale;                         // Cs^2 = out_scale * softplus(y)
  float pad[2];
};

// Features of a cell. p_ab = Pi_neq_ab / rho (standard normalisation).
// Cube root and logarithm of the features. The features are the network's
// inputs (the same function feeds training and inference), so in FP32 they
// use the hardware's fast base-2 exponential and logarithm (__expf, __logf):
// cbrt(v) = sign(v) 2^(log2|v| / 3).
template <class C>
__host__ __device__ inline C feat_cbrt(C v) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(C) == 4) return copysignf(__expf(__logf(fabsf(v)) * (1.0f / 3.0f)), v);
#endif
  return cbrt(v);
}
template <class C>
__host__ __device__ inline C feat_log(C v) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(C) == 4) return __logf(v);
#endif
  return log(v);
}

template <class C>
__host__ __device__ inline void mlp_features(C rho, C ux, C uy, C uz, C P00, C P11, C P22, C P01, C P12, C P02,
                                             float (&x)[kMlpIn]) {
  const C ir = C(1) / rho;
  const C a = P00 * ir, b = P11 * ir, c = P22 * ir, d = P01 * ir, e = P12 * ir, g = P02 * ir;
  const C tr = a + b + c;
  const C t3 = tr / C(3);
  const C da = a - t3, db = b - t3, dc = c - t3;
  const C off2 = d * d + e * e + g * g;
  const C n2 = a * a + b * b + c * c + C(2) * off2;
  const C dn2 = da * da + db * db + dc * dc + C(2) * off2;
  // tr(p_dev^3) and det(p)
  const C det = a * (b * c - e * e) - d * (d * c - e * g) + g * (d * e - b * g);
  const C ddet = da * (db * dc - e * e) - d * (d * dc - e * g) + g * (d * e - db * g);
  const C eps = C(1e-12);
  x[0] = float(tr);
  x[1] = float(sqrt(n2));
  x[2] = float(sqrt(dn2));
  x[3] = float(feat_cbrt(C(3) * ddet));  // tr(A^3) = 3 det(A) for traceless A
  x[4] = float(feat_cbrt(det));
  x[5] = float(feat_log(sqrt(dn2) + eps));
  x[6] = float(sqrt(a * a + b * b + c * c));
  x[7] = float(sqrt(C(2) * off2));
  x[8] = float(sqrt(ux * ux + uy * uy + uz * uz));
}

__host__ __device__ inline float mlp_softplus(float y) { return y > 20.f ? y : log1pf(expf(y)); }

}  // namespace aslb
