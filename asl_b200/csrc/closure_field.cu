// Learned closure, inference side. Every `period` steps the closure-field
// kernel evaluates, for every interior cell, the invariants of the
// non-equilibrium stress that the next stream-collide step will see
// (mlp_features) and the 9 -> 64 -> 64 -> 1 network on the tensor cores
// (mma.sync m16n8k16, BF16 operands, FP32 accumulation): one warp runs the
// network for its 32 cells as two M = 16 tiles. The resulting Cs^2 field is
// read by the CL_MLP stream-collide, which applies the Hou et al. (1996)
// closed form with the step's own |Pi_neq|.
//
// The features kernel writes the same nine raw features (before
// normalisation) for training.
#include <cuda_bf16.h>
#include "kernels.h"
#include "mlp.cuh"
#include "stream_collide.cuh"

namespace aslb {

namespace {

// Features of cell (x, y, z) from the populations the next step reads.
template <int Q, class S, bool ODD, bool FUSED>
__device__ __forceinline__ void cell_features(const S* __restrict__ F, const GridDesc& g, const StepParams& p, int x,
                                              int y, int z, unsigned s, float (&feat)[kMlpIn]) {
  using C = typename Store<S>::C;
  constexpr bool DEV = Store<S>::kDev;
  uint32_t bounce = 0;
  if (FUSED) bounce = p.mask[s].x;
  int ox[3], oy[3], oz[3];
  nb_offsets(g, x, y, z, ox, oy, oz);
  C f[Q];
  cell_load<Q, S, ODD, FUSED>(F, (unsigned)g.dstride, s, ox, oy, oz, bounce, f);
  const Moments<C> mo = cell_moments<Q, C, DEV>(f, p, step_omega<C>(p));
  C P[6];
  cell_pneq<Q, C, DEV>(f, mo, p, P);
  const C iu = DEV ? mul_(C(p.inv_scale), mo.inv_rho) : mo.inv_rho;
  mlp_features<C>(mo.rho, mo.m0 * iu, mo.m1 * iu, mo.m2 * iu, P[0], P[1], P[2], P[3], P[4], P[5], feat);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// D = A (16x16, row-major) * B (16x8, column-major) + C, BF16 in, FP32 out.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int kFieldThreads = 256;
constexpr int kFieldWarps = kFieldThreads / 32;

template <int Q, class S, bool ODD, bool FUSED>
__global__ void __launch_bounds__(kFieldThreads, 3)
    k_closure_field(const S* __restrict__ F, const GridDesc g, const StepParams p, const MlpNet* __restrict__ net,
                    float* __restrict__ cs2) {
  // rows padded by 8 BF16 (16 bytes) so that the eight rows a fragment load
  // touches fall in different banks
  __shared__ __align__(16) __nv_bfloat16 w1[kMlpHidden][kMlpInPad + 8];
  __shared__ __align__(16) __nv_bfloat16 w2[kMlpHidden][kMlpHidden + 8];
  __shared__ __align__(16) __nv_bfloat16 xs[kFieldWarps][32][kMlpInPad + 8];
  __shared__ float ys[kFieldWarps][32];
  __shared__ float vb1[kMlpHidden], vb2[kMlpHidden], vw3[kMlpHidden], vin[2 * kMlpInPad];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  {
    const uint32_t* s1 = reinterpret_cast<const uint32_t*>(&net->w1[0][0]);
    const uint32_t* s2 = reinterpret_cast<const uint32_t*>(&net->w2[0][0]);
    const int nt = blockDim.x * blockDim.y;
    for (int i = tid; i < kMlpHidden * kMlpInPad / 2; i += nt) {
      const int r = i / (kMlpInPad / 2), c = i % (kMlpInPad / 2);
      *reinterpret_cast<uint32_t*>(&w1[r][2 * c]) = s1[i];
    }
    for (int i = tid; i < kMlpHidden * kMlpHidden / 2; i += nt) {
      const int r = i / (kMlpHidden / 2), c = i % (kMlpHidden / 2);
      *reinterpret_cast<uint32_t*>(&w2[r][2 * c]) = s2[i];
    }
    for (int i = tid; i < kMlpHidden; i += nt) {
      vb1[i] = net->b1[i];
      vb2[i] = net->b2[i];
      vw3[i] = __bfloat162float(net->w3[i]);
    }
    for (int i = tid; i < kMlpInPad; i += nt) {
      vin[i] = net->in_shift[i];
      vin[kMlpInPad + i] = net->in_scale[i];
    }
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const int z = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int x = blockIdx.z + 1;
  const bool valid = z <= g.nz && y <= g.ny;
  const unsigned s = valid ? (unsigned)sidx(g, x, y, z) : 0u;
  // this lane's row of the feature matrix, normalised, in BF16
  float feat[kMlpIn];
  if (valid) {
    cell_features<Q, S, ODD, FUSED>(F, g, p, x, y, z, s, feat);
  } else {
    for (int k = 0; k < kMlpIn; ++k) feat[k] = vin[k];
  }
#pragma unroll
  for (int k = 0; k < kMlpInPad; k += 2) {
    const float a = k < kMlpIn ? (feat[k] - vin[k]) * vin[kMlpInPad + k] : 0.f;
    const float b = k + 1 < kMlpIn ? (feat[k + 1] - vin[k + 1]) * vin[kMlpInPad + k + 1] : 0.f;
    *reinterpret_cast<uint32_t*>(&xs[warp][lane][k]) = pack_bf16(a, b);
  }
  __syncthreads();

  const int gr = lane >> 2, c0 = (lane & 3) * 2;
  // layer 1: H1 = relu(X W1^T + b1), 32 x 64, as 2 x 8 tiles of 16 x 8; each
  // m-tile's FP32 output becomes the BF16 A fragments of layer 2 (K = 64) in place
  uint32_t ha[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    uint32_t a[4];
    const int r0 = mt * 16 + gr;
    a[0] = *reinterpret_cast<const uint32_t*>(&xs[warp][r0][c0]);
    a[1] = *reinterpret_cast<const uint32_t*>(&xs[warp][r0 + 8][c0]);
    a[2] = *reinterpret_cast<const uint32_t*>(&xs[warp][r0][c0 + 8]);
    a[3] = *reinterpret_cast<const uint32_t*>(&xs[warp][r0 + 8][c0 + 8]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float h[2][4];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int nt = 2 * j + q;
        const int n = nt * 8 + gr;
        const float bb0 = vb1[nt * 8 + c0], bb1 = vb1[nt * 8 + c0 + 1];
        h[q][0] = bb0;
        h[q][1] = bb1;
        h[q][2] = bb0;
        h[q][3] = bb1;
        mma16816(h[q], a, *reinterpret_cast<const uint32_t*>(&w1[n][c0]),
                 *reinterpret_cast<const uint32_t*>(&w1[n][c0 + 8]));
      }
      ha[mt][j][0] = pack_bf16(fmaxf(h[0][0], 0.f), fmaxf(h[0][1], 0.f));
      ha[mt][j][1] = pack_bf16(fmaxf(h[0][2], 0.f), fmaxf(h[0][3], 0.f));
      ha[mt][j][2] = pack_bf16(fmaxf(h[1][0], 0.f), fmaxf(h[1][1], 0.f));
      ha[mt][j][3] = pack_bf16(fmaxf(h[1][2], 0.f), fmaxf(h[1][3], 0.f));
    }
  }
  float yp[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [mt][row g, row g + 8]
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int n = nt * 8 + gr;
    const float bb0 = vb2[nt * 8 + c0], bb1 = vb2[nt * 8 + c0 + 1];
    const float v0 = vw3[nt * 8 + c0], v1 = vw3[nt * 8 + c0 + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      float acc[4] = {bb0, bb1, bb0, bb1};
#pragma unroll
      for (int j = 0; j < 4; ++j)
        mma16816(acc, ha[mt][j], *reinterpret_cast<const uint32_t*>(&w2[n][16 * j + c0]),
                 *reinterpret_cast<const uint32_t*>(&w2[n][16 * j + c0 + 8]));
      yp[mt][0] += fmaxf(acc[0], 0.f) * v0 + fmaxf(acc[1], 0.f) * v1;
      yp[mt][1] += fmaxf(acc[2], 0.f) * v0 + fmaxf(acc[3], 0.f) * v1;
    }
  }
  // output layer: sum the four lanes of each row group
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      float v = yp[mt][r];
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      if ((lane & 3) == 0) ys[warp][mt * 16 + gr + 8 * r] = v;
    }
  __syncwarp();
  if (valid) cs2[s] = net->out_scale * mlp_softplus(ys[warp][lane] + net->b3);
}

template <int Q, class S, bool ODD, bool FUSED>
__global__ void __launch_bounds__(256)
    k_closure_features(const S* __restrict__ F, const GridDesc g, const StepParams p, float* __restrict__ out) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int x = blockIdx.z + 1;
  if (z > g.nz || y > g.ny) return;
  float feat[kMlpIn];
  cell_features<Q, S, ODD, FUSED>(F, g, p, x, y, z, (unsigned)sidx(g, x, y, z), feat);
  const long long n = (long long)g.nx * g.ny * g.nz;
  const long long c = ((long long)(x - 1) * g.ny + (y - 1)) * g.nz + (z - 1);
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k) out[k * n + c] = feat[k];
}

template <int Q, class S>
cudaError_t field_impl(const DomainDev& d, const StepParams& p, const MlpNet* net, float* cs2, int parity,
                       cudaStream_t st) {
  dim3 grid, block;
  step_launch_shape(d.g, grid, block);
  const bool odd = parity == 0, fused = p.mask != nullptr;
  const S* F = (const S*)d.F;
  if (odd && fused) k_closure_field<Q, S, true, true><<<grid, block, 0, st>>>(F, d.g, p, net, cs2);
  else if (odd) k_closure_field<Q, S, true, false><<<grid, block, 0, st>>>(F, d.g, p, net, cs2);
  else if (fused) k_closure_field<Q, S, false, true><<<grid, block, 0, st>>>(F, d.g, p, net, cs2);
  else k_closure_field<Q, S, false, false><<<grid, block, 0, st>>>(F, d.g, p, net, cs2);
  return cudaGetLastError();
}

template <int Q, class S>
cudaError_t features_impl(const DomainDev& d, const StepParams& p, float* out, int parity, cudaStream_t st) {
  dim3 grid, block;
  step_launch_shape(d.g, grid, block);
  const bool odd = parity == 0, fused = p.mask != nullptr;
  const S* F = (const S*)d.F;
  if (odd && fused) k_closure_features<Q, S, true, true><<<grid, block, 0, st>>>(F, d.g, p, out);
  else if (odd) k_closure_features<Q, S, true, false><<<grid, block, 0, st>>>(F, d.g, p, out);
  else if (fused) k_closure_features<Q, S, false, true><<<grid, block, 0, st>>>(F, d.g, p, out);
  else k_closure_features<Q, S, false, false><<<grid, block, 0, st>>>(F, d.g, p, out);
  return cudaGetLastError();
}

__global__ void k_gather_cells(const GridDesc g, const float* __restrict__ src, float* __restrict__ dst) {
  const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= g.L) return;
  const int z = (int)(a % g.gz);
  const int y = (int)((a / g.gz) % g.gy);
  const int x = (int)(a / ((long long)g.gz * g.gy));
  const bool in = x >= 1 && x <= g.nx && y >= 1 && y <= g.ny && z >= 1 && z <= g.nz;
  dst[a] = in ? src[sidx(g, x, y, z)] : 0.f;
}

}  // namespace

cudaError_t launch_gather_cells(const GridDesc& g, const float* src, float* dst_asl, cudaStream_t st) {
  k_gather_cells<<<(unsigned)((g.L + 255) / 256), 256, 0, st>>>(g, src, dst_asl);
  return cudaGetLastError();
}

cudaError_t launch_closure_field(const DomainDev& d, const StepParams& p, const void* net, float* cs2, int parity,
                                 cudaStream_t st) {
  const MlpNet* n = static_cast<const MlpNet*>(net);
  switch (d.q * 8 + d.storage) {
    case 19 * 8 + ST_F32: return field_impl<19, float>(d, p, n, cs2, parity, st);
    case 19 * 8 + ST_F16: return field_impl<19, __half>(d, p, n, cs2, parity, st);
    case 27 * 8 + ST_F32: return field_impl<27, float>(d, p, n, cs2, parity, st);
    case 27 * 8 + ST_F16: return field_impl<27, __half>(d, p, n, cs2, parity, st);
    default: return cudaErrorNotSupported;
  }
}

cudaError_t launch_closure_features(const DomainDev& d, const StepParams& p, float* out, int parity,
                                    cudaStream_t st) {
  switch (d.q * 8 + d.storage) {
    case 19 * 8 + ST_F32: return features_impl<19, float>(d, p, out, parity, st);
    case 19 * 8 + ST_F16: return features_impl<19, __half>(d, p, out, parity, st);
    case 27 * 8 + ST_F32: return features_impl<27, float>(d, p, out, parity, st);
    case 27 * 8 + ST_F16: return features_impl<27, __half>(d, p, out, parity, st);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace aslb
