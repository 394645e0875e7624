// Host-side workload geometry: seeded random sequential addition of
// non-overlapping spheres (the porous-channel workload). Deterministic on
// every platform: a splitmix64 stream drives all random draws.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>
#include "aslb.h"

namespace {

struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  double uniform(double a, double b) { return a + (b - a) * (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

extern "C" int aslb_geom_pack_spheres(int nx, int ny, int nz, double rmin, double rmax, double solid_fraction,
                                      unsigned long long seed, int periodic_x, int attempts, int max_spheres,
                                      double* centers, double* radii, int* count) {
  if (!centers || !radii || !count || nx < 1 || ny < 1 || nz < 1 || !(rmin > 0) || rmax < rmin || max_spheres < 1)
    return ASLB_ERR_ARG;
  Rng rng{seed};
  const double box = double(nx) * ny * nz;
  const double target = solid_fraction * box;
  std::vector<double> rs;
  double vol = 0.0;
  while (vol < target * 1.25 && (int)rs.size() < 4 * max_spheres) {
    const double r = rng.uniform(rmin, rmax);
    rs.push_back(r);
    vol += 4.0 / 3.0 * M_PI * r * r * r;
  }
  std::sort(rs.begin(), rs.end(), [](double a, double b) { return a > b; });
  // Buckets at least 2 rmax wide, so every sphere that can overlap a
  // candidate sits in the candidate's bucket or an adjacent one. Along a
  // periodic x the buckets tile the period exactly (nbx whole buckets of
  // width nx / nbx), so the adjacency also holds across the seam.
  const double bucket = 2.0 * rmax;
  const int nbx = periodic_x ? std::max(1, (int)std::floor(nx / bucket)) : (int)std::ceil(nx / bucket);
  const double bwx = periodic_x ? double(nx) / nbx : bucket;
  const int nby = (int)std::ceil(ny / bucket), nbz = (int)std::ceil(nz / bucket);
  std::unordered_map<long long, std::vector<int>> grid;
  auto key = [&](int bx, int by, int bz) { return ((long long)bx * (nby + 2) + (by + 1)) * (nbz + 2) + (bz + 1); };
  int n = 0;
  double placed = 0.0;
  for (double r : rs) {
    if (placed >= target || n >= max_spheres) break;
    for (int a = 0; a < attempts; ++a) {
      const double cx = periodic_x ? rng.uniform(0, nx) : rng.uniform(r, nx - 1 - r);
      const double cy = rng.uniform(r, ny - 1 - r), cz = rng.uniform(r, nz - 1 - r);
      const int bx = std::min((int)std::floor(cx / bwx), nbx - 1);
      const int by = (int)std::floor(cy / bucket), bz = (int)std::floor(cz / bucket);
      bool ok = true;
      for (int ix = bx - 1; ix <= bx + 1 && ok; ++ix) {
        int jx = ix;
        // (with fewer than three buckets a wrapped bucket is checked twice)
        if (periodic_x) jx = ((ix % nbx) + nbx) % nbx;
        for (int iy = by - 1; iy <= by + 1 && ok; ++iy)
          for (int iz = bz - 1; iz <= bz + 1 && ok; ++iz) {
            auto it = grid.find(key(jx, iy, iz));
            if (it == grid.end()) continue;
            for (int k : it->second) {
              double dx = centers[3 * k] - cx;
              const double dy = centers[3 * k + 1] - cy, dz = centers[3 * k + 2] - cz;
              if (periodic_x) dx -= nx * std::nearbyint(dx / nx);
              const double rr = radii[k] + r;
              if (dx * dx + dy * dy + dz * dz < rr * rr) {
                ok = false;
                break;
              }
            }
          }
      }
      if (ok) {
        grid[key(bx, by, bz)].push_back(n);
        centers[3 * n] = cx;
        centers[3 * n + 1] = cy;
        centers[3 * n + 2] = cz;
        radii[n] = r;
        ++n;
        placed += 4.0 / 3.0 * M_PI * r * r * r;
        break;
      }
    }
  }
  *count = n;
  return ASLB_OK;
}
