// Shared device-side definitions: the HBM layout of a domain, storage formats
// of the populations and the per-step parameters.
//
// Layout ("padded ghosted SoA"). A domain of Nx x Ny x Nz interior cells has,
// like ASL's DataWithGhostNodes (src/data/aslDataWithGhostNodes.h:97-145),
// one ghost layer: ghosted coordinates x in [0, Nx+1] etc. Direction i of the
// populations is one array; inside it cell (x, y, z) sits at
//     ((x * Gy + y) * pitch) + zoff + z
// with pitch a multiple of 128 bytes and zoff = 128 B / element - 1, so the
// first interior cell of every z-row (z = 1) starts on a 128-byte boundary
// (HBM is read in 64-byte pieces: a 32-byte aligned row would drag one extra
// piece per row). All Q arrays live in one allocation, `dstride` elements
// apart; Q * dstride < 2^32 so element indices are 32-bit.
//
// Streaming is the AA pattern: the populations are stored in one of two
// representations that alternate every step (parity 0 = "A", 1 = "B"):
//   A: F[i][x]          = f*_i(x)           (post-collision, not yet streamed)
//   B: F[inv(i)][x+c_i] = f*_i(x)           (post-collision, already pushed)
// An odd step (A -> B) reads F[i][x - c_i] and writes F[inv(i)][x + c_i]; an
// even step (B -> A) reads F[inv(i)][x] and writes F[i][x]. Each cell reads
// and writes exactly the same Q slots, so one array suffices and the update is
// in place and race-free.
#pragma once
#include <cuda_fp16.h>
#include <cstdint>
#include "lattice.cuh"

namespace aslb {

struct GridDesc {
  int nx, ny, nz;     // interior cells
  int gx, gy, gz;     // ghosted sizes (n + 2)
  int pitch;          // elements per z-row in storage
  int zoff;           // storage position of ghost z = 0 within a row
  int periodic;       // bit0 x, bit1 y, bit2 z
  long long plane;    // gy * pitch
  long long dstride;  // elements between direction arrays
  long long L;        // gx * gy * gz (ASL's flattened ghosted size)
};

__host__ __device__ inline long long sidx(const GridDesc& g, int x, int y, int z) {
  return ((long long)x * g.gy + y) * g.pitch + g.zoff + z;
}
// ASL's flattening of the ghosted block, z fastest (src/data/aslBlocks.h:118-130).
__host__ __device__ inline long long aidx(const GridDesc& g, int x, int y, int z) {
  return ((long long)x * g.gy + y) * g.gz + z;
}

// Periodic axes send a coordinate that left the interior to the opposite side.
__host__ __device__ inline int wrap_axis(int v, int n, bool periodic) {
  if (!periodic) return v;
  return v < 1 ? v + n : (v > n ? v - n : v);
}

struct StepParams {
  double nu;
  float om0f;   // 1 / (3 nu + 1/2) in FP32 (ASL's LBGK::init0 expression order)
  double om0d;  // the same in FP64
  double g[3];
  double Om[3];
  double cs;         // Smagorinsky constant
  // FP32 copies of the scalars above and c_i . g per direction, set on the
  // host before every launch so kernels convert nothing per cell.
  float nuf, csf, gf[3], Omf[3];
  float cgf[27];
  double cgd[27];
  int has_force;
  int has_coriolis;
  int compressible;
  int write_macro;   // write rho and u (ASL's compVel/compRho) this step
  int write_rho, write_vel;
  float scale, inv_scale;  // FP16 storage: d = (f - 1) * scale
  const float* cs2;        // learned closure (CL == 3): Cs^2 per storage cell
  // Fused no-slip conditions (null when none), two words per storage cell.
  // x (bounce): bit k = population k enters this cell through a fused link,
  // so it is read by bounce-back from the cell's own outgoing population.
  // y (elide): bit k = the cell's outgoing population k lands in the incoming
  // slot of a fused link, which the condition would overwrite: the slot keeps
  // its bits (the store is skipped).
  const uint2* mask;
  // The same links in one word per cell, when no cell has both kinds: bit 31
  // set = the low bits are elide bits, clear = bounce bits (or null).
  const uint32_t* mask32;
  // Element offsets of the population slots of direction i relative to a
  // cell's storage index s, for cells whose neighbours do not wrap across a
  // periodic face (with ds = dstride and t = (plane, pitch, 1)):
  //   slot[0][i] = i ds - c_i.t       F[i][x - c_i]      (pull)
  //   slot[1][i] = i ds                F[i][x]            (own)
  //   slot[2][i] = inv(i) ds + c_i.t   F[inv i][x + c_i]  (push)
  //   slot[3][i] = inv(i) ds           F[inv i][x]        (own, opposite)
  // Modulo 2^32: s + slot is the slot's index (Q * dstride < 2^32). Set on
  // the host from the domain's grid, so a population address is one add.
  unsigned slot[4][27];
};

// ---- storage formats -------------------------------------------------------
template <class S>
struct Store;

template <>
struct Store<float> {
  using C = float;
  __device__ static __forceinline__ C load(const float* p, const StepParams&) { return *p; }
  __device__ static __forceinline__ void store(float* p, C v, const StepParams&) { *p = v; }
  // Values in the collision's representation: f itself.
  static constexpr bool kDev = false;
  __device__ static __forceinline__ C load_c(const float* p) { return *p; }
  __device__ static __forceinline__ float encode(C v, const StepParams&) { return v; }
  // deviation from rest (f - 1)
  __device__ static __forceinline__ C dev(const float* p, float) { return *p - 1.0f; }
  __device__ static __forceinline__ void set_dev(float* p, C d, float) { *p = 1.0f + d; }
  __device__ static __forceinline__ C val(const float* p, float) { return *p; }
  __device__ static __forceinline__ void set_val(float* p, C v, float) { *p = v; }
};

template <>
struct Store<double> {
  using C = double;
  __device__ static __forceinline__ C load(const double* p, const StepParams&) { return *p; }
  __device__ static __forceinline__ void store(double* p, C v, const StepParams&) { *p = v; }
  static constexpr bool kDev = false;
  __device__ static __forceinline__ C load_c(const double* p) { return *p; }
  __device__ static __forceinline__ double encode(C v, const StepParams&) { return v; }
  __device__ static __forceinline__ C dev(const double* p, float) { return *p - 1.0; }
  __device__ static __forceinline__ void set_dev(double* p, C d, float) { *p = 1.0 + d; }
  __device__ static __forceinline__ C val(const double* p, float) { return *p; }
  __device__ static __forceinline__ void set_val(double* p, C v, float) { *p = v; }
};

// FP16 "shifted" storage: the half holds (f - 1) * scale, i.e. the deviation
// from the rest state (f_i^std - w_i in standard normalisation), scaled so that
// small deviations stay out of the half subnormal range. All arithmetic is FP32.
template <>
struct Store<__half> {
  using C = float;
  __device__ static __forceinline__ C load(const __half* p, const StepParams& sp) {
    return 1.0f + __half2float(*p) * sp.inv_scale;
  }
  __device__ static __forceinline__ void store(__half* p, C v, const StepParams& sp) {
    *p = __float2half_rn((v - 1.0f) * sp.scale);
  }
  // The collision works on the stored quantity D = (f - 1) * scale directly
  // (its moments and equilibrium are rescaled, see collide.cuh), so a load
  // and a store are one conversion each.
  static constexpr bool kDev = true;
  __device__ static __forceinline__ C load_c(const __half* p) { return __half2float(*p); }
  __device__ static __forceinline__ __half encode(C v, const StepParams&) { return __float2half_rn(v); }
  __device__ static __forceinline__ C dev(const __half* p, float inv_scale) { return __half2float(*p) * inv_scale; }
  __device__ static __forceinline__ void set_dev(__half* p, C d, float scale) { *p = __float2half_rn(d * scale); }
  __device__ static __forceinline__ C val(const __half* p, float inv_scale) { return 1.0f + __half2float(*p) * inv_scale; }
  __device__ static __forceinline__ void set_val(__half* p, C v, float scale) { *p = __float2half_rn((v - 1.0f) * scale); }
};

enum Closure { CL_NONE = 0, CL_ASL_INTENT = 1, CL_SMAGORINSKY = 2, CL_MLP = 3 };

// Boundary-condition kinds (the C-ABI exposes the same numbers).
enum BcKind {
  BCK_NOSLIP = 0,
  BCK_VELOCITY = 1,
  BCK_PRESSURE = 2,
  BCK_PRESSURE_VELOCITY = 3,
  BCK_MAP_NOSLIP = 10,
  BCK_MAP_VELOCITY = 11,
  BCK_MAP_VELOCITY_ROTATION = 12,
  BCK_MAP_PRESSURE_VELOCITY = 13,
  BCK_MAP_TRANSPORT_DEPOSITION = 14,
  BCK_MAP_KINETICS_DEPOSITION = 15,
  // conditions on the rho / u output fields (visualisation)
  BCK_FIELD_NOSLIP_VEL = 20,
  BCK_FIELD_NOSLIP_RHO = 21,
  BCK_FIELD_VELOCITY_VEL = 22,
  BCK_FIELD_VELOCITY_VEL_ROTATION = 23,
};

struct BcParams {
  int kind;
  int compressible;
  double p;
  double u[3];
  double om[3];
  double cen[3];
  double pos0[3];
  double dx;
  double lf, beta;  // deposition: limiting factor, kinetic coefficient
  float scale, inv_scale;
};

// Direction-sorted boundary links: links [seg[k], seg[k+1]) have direction k,
// each stored as the storage index of its anchor; the fluid end is
// anchor + off[k] (links that wrap across a periodic face go to the anchor
// form instead). val[k] is the per-direction constant of the condition:
// 6 c_k.u (velocity), p (pressure), p + 3 c_k.u, or f_eq,k(p, u).
struct LinkSet {
  int seg[28];
  int off[27];
  int inv[27];
  float val[27];
  double vald[27];
};

}  // namespace aslb
