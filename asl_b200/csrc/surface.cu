// Surfaces to distance maps: ASL's readSurface (src/readers/aslVTKFormatReaders.cxx:
// 136-210, 266-345) reads an STL/VTP surface, samples the unsigned distance to it
// on a grid through VTK's implicit modeller and maps it to (d - offset) / scale,
// so a shell of cells around the surface becomes solid. VTK is not part of this
// library: the STL reader and the distance sampling are written here.
//
// Distance: the grid is cut into bricks of 8 x 8 x 8 cells; on the host every
// triangle is listed in the bricks its bounding box, grown by the band width,
// overlaps (a CSR list). One CTA of 512 threads per brick stages its triangles
// in shared memory, 128 at a time, and each thread keeps the smallest squared
// distance of its cell (closest point on a triangle by the region tests of
// Ericson, Real-Time Collision Detection, 2005, section 5.1.5). A cell farther
// than the band from every triangle reads the band width; every cell within the
// band gets its exact distance, because its nearest triangle's grown bounding
// box contains it.
//
// Solid interior (an extension: ASL's maps keep only the shell): a cell is
// inside a closed surface when a ray from it towards -x crosses the surface an
// odd number of times. Triangles are listed per tile of 8 x 8 (y, z) columns;
// one thread per (column, triangle) pair intersects the column's line with the
// triangle (edge functions in double precision, a top-left rule so that a line
// through an edge shared by two triangles counts once) and marks the first
// cell past the crossing; a thread per column then walks x, flipping the
// inside flag at every mark, and writes the map.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "aslb.h"
#include "kernels.h"

namespace aslb {
namespace {

constexpr int kBrick = 8;       // cells per brick edge
constexpr int kStage = 128;     // triangles staged per pass
constexpr int kTile = 8;        // columns per tile edge (solid interior)

__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 axpy3(float s, float3 a, float3 b) {
  return make_float3(b.x + s * a.x, b.y + s * a.y, b.z + s * a.z);
}

// Squared distance from p to triangle (a, b, c): Voronoi regions of the
// vertices, then of the edges, else the face (distance to the plane).
__device__ float tri_dist2(float3 p, float3 a, float3 b, float3 c) {
  const float3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
  const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) return dot3(ap, ap);
  const float3 bp = sub3(p, b);
  const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.f && d4 <= d3) return dot3(bp, bp);
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    const float3 q = axpy3(-d1 / (d1 - d3), ab, ap);
    return dot3(q, q);
  }
  const float3 cp = sub3(p, c);
  const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.f && d5 <= d6) return dot3(cp, cp);
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    const float3 q = axpy3(-d2 / (d2 - d6), ac, ap);
    return dot3(q, q);
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.f && d4 - d3 >= 0.f && d5 - d6 >= 0.f) {
    const float3 q = axpy3(-(d4 - d3) / ((d4 - d3) + (d5 - d6)), sub3(c, b), bp);
    return dot3(q, q);
  }
  const float3 n = make_float3(ab.y * ac.z - ab.z * ac.y, ab.z * ac.x - ab.x * ac.z, ab.x * ac.y - ab.y * ac.x);
  const float nn = dot3(n, n);
  if (!(nn > 0.f)) return dot3(ap, ap);  // degenerate sliver: the region tests above bound it
  const float h = dot3(n, ap);
  return h * h / nn;
}

struct SurfGrid {
  int gx, gy, gz;          // cells
  int bx, by, bz;          // bricks
  float x0, y0, z0, dx;    // position of cell (0, 0, 0), spacing
};

// One CTA per brick, thread t -> cell (t / 64, t / 8 % 8, t % 8) of the brick.
__global__ void __launch_bounds__(512) k_surface_distance(const float* __restrict__ tri, const int* __restrict__ start,
                                                          const int* __restrict__ list, SurfGrid g, float band,
                                                          float* __restrict__ dist) {
  __shared__ float st[kStage * 9];
  const int b = blockIdx.x;
  const int bxi = b / (g.by * g.bz), byi = (b / g.bz) % g.by, bzi = b % g.bz;
  const int t = threadIdx.x;
  const int i = bxi * kBrick + t / 64, j = byi * kBrick + (t / 8) % 8, k = bzi * kBrick + t % 8;
  const float3 p = make_float3(g.x0 + i * g.dx, g.y0 + j * g.dx, g.z0 + k * g.dx);
  float best = band * band;
  const int s0 = start[b], s1 = start[b + 1];
  for (int s = s0; s < s1; s += kStage) {
    const int n = min(kStage, s1 - s);
    __syncthreads();
    for (int e = t; e < n * 9; e += blockDim.x) st[e] = tri[(size_t)list[s + e / 9] * 9 + e % 9];
    __syncthreads();
    for (int q = 0; q < n; ++q) {
      const float* v = st + q * 9;
      const float d2 = tri_dist2(p, make_float3(v[0], v[1], v[2]), make_float3(v[3], v[4], v[5]),
                                 make_float3(v[6], v[7], v[8]));
      best = fminf(best, d2);
    }
  }
  if (i < g.gx && j < g.gy && k < g.gz) dist[((size_t)i * g.gy + j) * g.gz + k] = sqrtf(best);
}

// Edge U -> V of a counter-clockwise triangle in the (y, z) plane owns the
// points on it when it points up, or exactly sideways towards -y.
__device__ __forceinline__ bool owns(double w, double ey, double ez) {
  return w > 0.0 || (w == 0.0 && (ez > 0.0 || (ez == 0.0 && ey < 0.0)));
}

// Edge function of U -> V at P (positive left of the edge). It is always
// evaluated from the lexicographically smaller end, so the two triangles that
// share an edge get exactly opposite values and a point on the edge is owned
// by one of them only.
__device__ __forceinline__ double edge_fn(double uy, double uz, double vy, double vz, double py, double pz) {
  const bool fwd = uy < vy || (uy == vy && uz < vz);
  if (!fwd) {
    double t = uy; uy = vy; vy = t;
    t = uz; uz = vz; vz = t;
  }
  const double w = (vy - uy) * (pz - uz) - (vz - uz) * (py - uy);
  return fwd ? w : -w;
}

// Work item e of tile b: triangle list[start[b] + e / 64] against column e % 64
// of the tile. A crossing at x_c marks the first cell whose x exceeds it.
__global__ void k_surface_crossings(const float* __restrict__ tri, const int* __restrict__ start,
                                    const int* __restrict__ list, SurfGrid g, int ty, int tz,
                                    int* __restrict__ marks) {
  const int b = blockIdx.y;
  const int s0 = start[b], n = start[b + 1] - s0;
  const int tyi = b / tz, tzi = b % tz;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)n * 64;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % 64);
    const int j = tyi * kTile + c / 8, k = tzi * kTile + c % 8;
    if (j >= g.gy || k >= g.gz) continue;
    const float* v = tri + (size_t)list[s0 + e / 64] * 9;
    const double py = (double)g.y0 + (double)j * g.dx, pz = (double)g.z0 + (double)k * g.dx;
    double ay = v[1], az = v[2], by = v[4], bz = v[5], cy = v[7], cz = v[8];
    double ax = v[0], bx = v[3], cx = v[6];
    double area = (by - ay) * (cz - az) - (bz - az) * (cy - ay);
    if (area == 0.0) continue;  // parallel to the line
    if (area < 0.0) {            // make it counter-clockwise in (y, z)
      double t;
      t = by; by = cy; cy = t;
      t = bz; bz = cz; cz = t;
      t = bx; bx = cx; cx = t;
      area = -area;
    }
    const double w0 = edge_fn(ay, az, by, bz, py, pz);  // edge a -> b
    const double w1 = edge_fn(by, bz, cy, cz, py, pz);  // edge b -> c
    const double w2 = edge_fn(cy, cz, ay, az, py, pz);  // edge c -> a
    if (!owns(w0, by - ay, bz - az) || !owns(w1, cy - by, cz - bz) || !owns(w2, ay - cy, az - cz)) continue;
    // barycentric weights of b and c are w2 / area and w0 / area
    const double wsum = w0 + w1 + w2;  // the area up to rounding
    const double xc = ax + (w2 * (bx - ax) + w0 * (cx - ax)) / wsum;
    const double r = (xc - (double)g.x0) / (double)g.dx;
    long long first = (long long)floor(r) + 1;  // first cell with x > xc
    if (first < 0) first = 0;
    if (first >= g.gx) continue;
    atomicAdd(marks + ((size_t)j * g.gz + k) * (g.gx + 1) + first, 1);
  }
}

// One thread per (y, z) column: walk x, sign the distance inside, write the map.
__global__ void k_surface_map(const float* __restrict__ dist, const int* __restrict__ marks, SurfGrid g,
                              int solid_interior, float offset, float inv_scale, float* __restrict__ map) {
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= (long long)g.gy * g.gz) return;
  int inside = 0;
  const size_t plane = (size_t)g.gy * g.gz;
  for (int i = 0; i < g.gx; ++i) {
    if (solid_interior) inside ^= marks[(size_t)col * (g.gx + 1) + i] & 1;
    const float d = dist[(size_t)i * plane + col];
    map[(size_t)i * plane + col] = ((inside ? -d : d) - offset) * inv_scale;
  }
}

int err_arg(const char* what) {
  set_last_error(std::string(what) + ": bad arguments");
  return ASLB_ERR_ARG;
}

int err_cuda(const char* what, cudaError_t e) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return ASLB_ERR_CUDA;
}

// CSR lists: items[start[c] .. start[c + 1]) of cell c, from (cell, item) pairs.
void csr(int ncells, const std::vector<std::pair<int, int>>& pairs, std::vector<int>& start, std::vector<int>& list) {
  start.assign(ncells + 1, 0);
  for (const auto& p : pairs) start[p.first + 1]++;
  for (int c = 0; c < ncells; ++c) start[c + 1] += start[c];
  list.resize(pairs.size());
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (const auto& p : pairs) list[fill[p.first]++] = p.second;
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

}  // namespace
}  // namespace aslb

using namespace aslb;

extern "C" {

int aslb_read_stl(const char* path, float* tri, long long cap, long long* ntri) {
  if (!path || !ntri) return err_arg("aslb_read_stl");
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_last_error(std::string("aslb_read_stl: cannot open ") + path);
    return ASLB_ERR_ARG;
  }
  std::vector<char> buf;
  char chunk[1 << 16];
  size_t r;
  while ((r = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + r);
  std::fclose(f);
  std::vector<float> out;
  bool binary = false;
  if (buf.size() >= 84) {
    uint32_t n;
    std::memcpy(&n, buf.data() + 80, 4);
    binary = buf.size() == 84 + 50ull * n;
    if (binary) {
      out.resize(9ull * n);
      for (uint32_t t = 0; t < n; ++t) std::memcpy(&out[9ull * t], buf.data() + 84 + 50ull * t + 12, 36);
    }
  }
  if (!binary) {
    // ASCII: every "vertex x y z" line, three per facet
    std::string s(buf.begin(), buf.end());
    if (s.compare(0, 5, "solid") != 0) {
      set_last_error("aslb_read_stl: neither binary STL nor ASCII STL");
      return ASLB_ERR_ARG;
    }
    size_t pos = 0;
    while ((pos = s.find("vertex", pos)) != std::string::npos) {
      pos += 6;
      const char* c = s.c_str() + pos;
      char* end = nullptr;
      for (int a = 0; a < 3; ++a) {
        const float v = std::strtof(c, &end);
        if (end == c) {
          set_last_error("aslb_read_stl: malformed vertex line");
          return ASLB_ERR_ARG;
        }
        out.push_back(v);
        c = end;
      }
    }
    if (out.size() % 9) {
      set_last_error("aslb_read_stl: vertex count is not a multiple of three");
      return ASLB_ERR_ARG;
    }
  }
  *ntri = (long long)(out.size() / 9);
  if (tri) {
    if (cap < *ntri) return err_arg("aslb_read_stl (capacity)");
    std::memcpy(tri, out.data(), out.size() * sizeof(float));
  }
  return ASLB_OK;
}

int aslb_surface_map(const float* tri, long long ntri, int gx, int gy, int gz, const double pos0[3], double dx,
                     double band, int solid_interior, double offset, double scale, float* map_host) {
  if ((!tri && ntri) || ntri < 0 || ntri > (1LL << 30) || gx < 1 || gy < 1 || gz < 1 || !pos0 || !(dx > 0) ||
      !(band > 0) || !(scale != 0) || !map_host)
    return err_arg("aslb_surface_map");
  SurfGrid g;
  g.gx = gx; g.gy = gy; g.gz = gz;
  g.bx = (gx + kBrick - 1) / kBrick; g.by = (gy + kBrick - 1) / kBrick; g.bz = (gz + kBrick - 1) / kBrick;
  g.x0 = (float)pos0[0]; g.y0 = (float)pos0[1]; g.z0 = (float)pos0[2]; g.dx = (float)dx;
  const long long nbricks = (long long)g.bx * g.by * g.bz;
  if (nbricks > (1LL << 30)) return err_arg("aslb_surface_map (grid too large)");
  // bricks (and, for the interior, column tiles) each triangle touches
  std::vector<std::pair<int, int>> pairs, tpairs;
  const int tyn = (gy + kTile - 1) / kTile, tzn = (gz + kTile - 1) / kTile;
  for (long long t = 0; t < ntri; ++t) {
    const float* v = tri + 9 * t;
    int lo[3], hi[3], tlo[3], thi[3];
    const int gn[3] = {gx, gy, gz};
    bool bad = false;
    for (int a = 0; a < 3; ++a) {
      const double mn = std::min({(double)v[a], (double)v[3 + a], (double)v[6 + a]});
      const double mx = std::max({(double)v[a], (double)v[3 + a], (double)v[6 + a]});
      if (!std::isfinite(mn) || !std::isfinite(mx)) bad = true;
      const double l = std::floor((mn - band - pos0[a]) / dx), h = std::ceil((mx + band - pos0[a]) / dx);
      lo[a] = (int)std::max(0.0, std::min(l, (double)gn[a]));
      hi[a] = (int)std::max(-1.0, std::min(h, (double)gn[a] - 1));
      const double tl = std::floor((mn - pos0[a]) / dx) - 1, th = std::ceil((mx - pos0[a]) / dx) + 1;
      tlo[a] = (int)std::max(0.0, std::min(tl, (double)gn[a]));
      thi[a] = (int)std::max(-1.0, std::min(th, (double)gn[a] - 1));
    }
    if (bad) {
      set_last_error("aslb_surface_map: a triangle has a non-finite vertex");
      return ASLB_ERR_ARG;
    }
    if (lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2])
      for (int bi = lo[0] / kBrick; bi <= hi[0] / kBrick; ++bi)
        for (int bj = lo[1] / kBrick; bj <= hi[1] / kBrick; ++bj)
          for (int bk = lo[2] / kBrick; bk <= hi[2] / kBrick; ++bk)
            pairs.emplace_back((bi * g.by + bj) * g.bz + bk, (int)t);
    if (solid_interior && tlo[1] <= thi[1] && tlo[2] <= thi[2])
      for (int tj = tlo[1] / kTile; tj <= thi[1] / kTile; ++tj)
        for (int tk = tlo[2] / kTile; tk <= thi[2] / kTile; ++tk) tpairs.emplace_back(tj * tzn + tk, (int)t);
  }
  std::vector<int> start, list, tstart, tlist;
  csr((int)nbricks, pairs, start, list);
  if (solid_interior) csr(tyn * tzn, tpairs, tstart, tlist);

  const size_t cells = (size_t)gx * gy * gz;
  DevBuf<float> d_tri, d_dist, d_map;
  DevBuf<int> d_start, d_list, d_tstart, d_tlist, d_marks;
  cudaError_t e = d_tri.alloc(9 * (size_t)ntri);
  if (e == cudaSuccess) e = d_dist.alloc(cells);
  if (e == cudaSuccess) e = d_map.alloc(cells);
  if (e == cudaSuccess) e = d_start.alloc(start.size());
  if (e == cudaSuccess) e = d_list.alloc(list.size());
  if (e == cudaSuccess && solid_interior) {
    e = d_tstart.alloc(tstart.size());
    if (e == cudaSuccess) e = d_tlist.alloc(tlist.size());
    if (e == cudaSuccess) e = d_marks.alloc((size_t)gy * gz * (gx + 1));
  }
  if (e != cudaSuccess) return err_cuda("aslb_surface_map", e);
  cudaStream_t st = 0;
  if (ntri) e = cudaMemcpyAsync(d_tri.p, tri, 9 * (size_t)ntri * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_start.p, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !list.empty())
    e = cudaMemcpyAsync(d_list.p, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_surface_distance<<<(unsigned)nbricks, 512, 0, st>>>(d_tri.p, d_start.p, d_list.p, g, (float)band, d_dist.p);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && solid_interior) {
    e = cudaMemsetAsync(d_marks.p, 0, (size_t)gy * gz * (gx + 1) * sizeof(int), st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_tstart.p, tstart.data(), tstart.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !tlist.empty())
      e = cudaMemcpyAsync(d_tlist.p, tlist.data(), tlist.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !tlist.empty()) {
      dim3 grid(64, (unsigned)(tyn * tzn));
      k_surface_crossings<<<grid, 256, 0, st>>>(d_tri.p, d_tstart.p, d_tlist.p, g, tyn, tzn, d_marks.p);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) {
    const long long cols = (long long)gy * gz;
    k_surface_map<<<(unsigned)((cols + 255) / 256), 256, 0, st>>>(d_dist.p, d_marks.p, g, solid_interior ? 1 : 0,
                                                                (float)offset, (float)(1.0 / scale), d_map.p);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(map_host, d_map.p, cells * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return err_cuda("aslb_surface_map", e);
  return ASLB_OK;
}

}  // extern "C"
