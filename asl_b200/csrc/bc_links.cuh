// Boundary-link arithmetic shared by the per-domain and the batched link
// kernels.
#pragma once
#include <type_traits>
#include "internal.cuh"

namespace aslb {

template <class S>
struct BcArith {
  using C = typename Store<S>::C;
  static constexpr bool kDev = std::is_same<S, __half>::value;
  // value of f, in the arithmetic the storage keeps exact (deviation for FP16)
  __device__ static __forceinline__ C get(const S* p, const BcParams& bp) {
    return kDev ? Store<S>::dev(p, bp.inv_scale) : Store<S>::val(p, bp.inv_scale);
  }
  __device__ static __forceinline__ void put(S* p, C v, const BcParams& bp) {
    if (kDev)
      Store<S>::set_dev(p, v, bp.scale);
    else
      Store<S>::set_val(p, v, bp.scale);
  }
  // representation of a constant population value P (absolute) in get/put arithmetic
  __device__ static __forceinline__ C rep(C v) { return kDev ? v - C(1) : v; }
};

// Apply link t of a direction-sorted link set: its direction k comes from the
// segment table (warp-uniform except at segment ends), the fluid end is
// anchor + off[k]. A link's IN slot (the population the fluid end streams in
// next) and OUT slot (that cell's outgoing population in the opposite
// direction) swap between the AA representations.
template <int Q, class S>
__device__ __forceinline__ void link_apply(S* __restrict__ F, long long dstride, const int* __restrict__ links, int t,
                                           const LinkSet& ls, const BcParams& bp, int parity) {
  using C = typename Store<S>::C;
  using A = BcArith<S>;
  int k = 1;
  while (t >= ls.seg[k + 1]) ++k;
  const int wa = links[t];
  const int wq = wa + ls.off[k];
  const int kb = ls.inv[k];
  S* in;
  S* out;
  if (parity == 0) {
    in = F + (size_t)k * dstride + wa;
    out = F + (size_t)kb * dstride + wq;
  } else {
    in = F + (size_t)kb * dstride + wq;
    out = F + (size_t)k * dstride + wa;
  }
  const C v = std::is_same<C, double>::value ? C(ls.vald[k]) : C(ls.val[k]);
  switch (bp.kind) {
    case BCK_NOSLIP:
    case BCK_MAP_NOSLIP:
      *in = *out;
      break;
    case BCK_VELOCITY:
      A::put(in, A::get(out, bp) + v, bp);
      break;
    default:  // pressure, pressure + velocity, equilibrium: a constant per direction
      A::put(in, A::rep(v), bp);
      break;
  }
}

}  // namespace aslb
