// Velocity sets of the D3Q15 / D3Q19 / D3Q27 lattices in ASL's direction order
// (src/math/aslTemplates.cxx:146-200 of the reference project). Weights follow
// ASL's rule w_i = LaplaceCoef_i / 6 (+1 for the rest direction); D3Q27 uses the
// standard weights because ASL's d3q27() leaves them empty.
//
// Populations are ASL-normalised: rest state f_i == 1, rho = sum w_i f_i.
#pragma once

namespace aslb {

__host__ __device__ constexpr int lat_c27(int i, int d) {
  constexpr int t[27][3] = {
      {0, 0, 0},  {1, 0, 0},   {0, 1, 0},   {0, 0, 1},   {-1, 0, 0},  {0, -1, 0},  {0, 0, -1},
      {1, 1, 0},  {1, -1, 0},  {-1, -1, 0}, {-1, 1, 0},  {0, 1, 1},   {0, 1, -1},  {0, -1, -1},
      {0, -1, 1}, {1, 0, 1},   {1, 0, -1},  {-1, 0, -1}, {-1, 0, 1},  {1, 1, 1},   {1, 1, -1},
      {1, -1, 1}, {1, -1, -1}, {-1, 1, 1},  {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
  return t[i][d];
}

__host__ __device__ constexpr int lat_c15(int i, int d) {
  constexpr int t[15][3] = {{0, 0, 0},  {1, 0, 0},   {0, 1, 0},   {0, 0, 1},   {-1, 0, 0},
                            {0, -1, 0}, {0, 0, -1},  {1, 1, 1},   {1, 1, -1},  {1, -1, 1},
                            {1, -1, -1}, {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
  return t[i][d];
}

template <int Q>
struct Lattice {
  static constexpr int q = Q;
  __host__ __device__ static constexpr int c(int i, int d) { return Q == 15 ? lat_c15(i, d) : lat_c27(i, d); }
  __host__ __device__ static constexpr int norm2(int i) { return c(i, 0) * c(i, 0) + c(i, 1) * c(i, 1) + c(i, 2) * c(i, 2); }
  __host__ __device__ static constexpr double w(int i) {
    return Q == 15   ? (norm2(i) == 0 ? 2. / 9. : (norm2(i) == 1 ? 1. / 9. : 1. / 72.))
           : Q == 19 ? (norm2(i) == 0 ? 1. / 3. : (norm2(i) == 1 ? 1. / 18. : 1. / 36.))
                     : (norm2(i) == 0 ? 8. / 27.
                                      : (norm2(i) == 1 ? 2. / 27. : (norm2(i) == 2 ? 1. / 54. : 1. / 216.)));
  }
  // Runtime-index lookups (device code whose loop the compiler does not
  // unroll) read the constant-memory tables below.
  __device__ static int c_rt(int i, int d);
  __device__ static int inv_rt(int i);
  // Opposite direction (ASL's invertVectors).
  __host__ __device__ static constexpr int inv(int i) {
    int r = 0;
    for (int j = 0; j < Q; ++j)
      if (c(j, 0) == -c(i, 0) && c(j, 1) == -c(i, 1) && c(j, 2) == -c(i, 2)) r = j;
    return r;
  }
};

// Constant-memory copies of the velocity sets for runtime indexing in device
// code: [lattice: 0 = D3Q15, 1 = D3Q19/D3Q27 order][direction][axis], and the
// opposite-direction tables.
static __constant__ int kLatC[2][27][3] = {
    {{0, 0, 0},  {1, 0, 0},  {0, 1, 0},   {0, 0, 1},   {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {1, 1, 1},   {1, 1, -1},
     {1, -1, 1}, {1, -1, -1}, {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}},
    {{0, 0, 0},  {1, 0, 0},   {0, 1, 0},   {0, 0, 1},   {-1, 0, 0},  {0, -1, 0},  {0, 0, -1},
     {1, 1, 0},  {1, -1, 0},  {-1, -1, 0}, {-1, 1, 0},  {0, 1, 1},   {0, 1, -1},  {0, -1, -1},
     {0, -1, 1}, {1, 0, 1},   {1, 0, -1},  {-1, 0, -1}, {-1, 0, 1},  {1, 1, 1},   {1, 1, -1},
     {1, -1, 1}, {1, -1, -1}, {-1, 1, 1},  {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}}};
static __constant__ int kLatInv[3][27] = {
    {0, 4, 5, 6, 1, 2, 3, 14, 13, 12, 11, 10, 9, 8, 7},
    {0, 4, 5, 6, 1, 2, 3, 9, 10, 7, 8, 13, 14, 11, 12, 17, 18, 15, 16},
    {0, 4, 5, 6, 1, 2, 3, 9, 10, 7, 8, 13, 14, 11, 12, 17, 18, 15, 16, 26, 25, 24, 23, 22, 21, 20, 19}};

template <int Q>
__device__ inline int Lattice<Q>::c_rt(int i, int d) {
  return kLatC[Q == 15 ? 0 : 1][i][d];
}
template <int Q>
__device__ inline int Lattice<Q>::inv_rt(int i) {
  return kLatInv[Q == 15 ? 0 : (Q == 19 ? 1 : 2)][i];
}

// Runtime lookups for host code and for kernels that loop over a bitmask.
inline int lattice_c(int q, int i, int d) { return q == 15 ? lat_c15(i, d) : lat_c27(i, d); }
inline double lattice_w(int q, int i) {
  switch (q) {
    case 15: return Lattice<15>::w(i);
    case 19: return Lattice<19>::w(i);
    default: return Lattice<27>::w(i);
  }
}
inline int lattice_inv(int q, int i) {
  switch (q) {
    case 15: return Lattice<15>::inv(i);
    case 19: return Lattice<19>::inv(i);
    default: return Lattice<27>::inv(i);
  }
}

}  // namespace aslb
