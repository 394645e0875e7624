// lbgk_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A plain C++ CPU restatement of ASL's lattice-Boltzmann (LBGK) hot path. It
// is the checker for the CUDA library: tests, the smoke entry point and the
// CPU-baseline leg of bench.py may load it; product code never does.
//
// PARITY UNPINNED: the reference (AvtechScientific/ASL) has no tests, golden
// vectors or fixtures for LBGK, its boundary conditions or the surface force,
// and it cannot be built here (OpenCL, Boost and VTK are absent). This file
// restates the reference's algorithm from its sources; known-answer tests
// (rest state, conservation, Poiseuille, hand-computed single-cell collide,
// the reduction known answers of test/testMath/testReductionFunction.cc) pin
// it instead.
//
// What it follows (paths inside the reference project):
//   src/math/aslTemplates.cxx:30-83,146-200   lattices, weights = LC/6 + d_i0,
//                                             opposite-direction table
//   src/data/aslBlocks.h:118-130               z-fastest flattening, 1 ghost layer
//   src/num/aslLBGK.cxx:46-73                  rho = sum w f, m = sum w c f
//   src/num/aslLBGK.cxx:187-235                collide expression order
//   src/num/aslLBGK.cxx:237-250                pull streaming by window shift
//   src/num/aslLBGK.cxx:262-280                initF
//   src/num/aslLBGK.cxx:298-355                LBGKTurbulence (f_eq computed first:
//                                              the reference reads it before
//                                              assigning it)
//   src/num/aslBCond.cxx:373-510               slice point lists
//   src/num/aslLBGKBC.cxx:91-202               slice BC values
//   src/num/aslLBGKBC.cxx:219-432              map BCs and their guards
//   src/num/aslLBGKBC.cxx:440-598              deposition map BCs (transport
//                                              and kinetics limited)
//   src/num/aslLBGKBC.cxx:623-665              ComputeSurfaceFluxMap
//   src/num/aslLBGKBC.cxx:808-852 and           output-field conditions for
//   src/num/aslBasicBC.cxx:110-230, 300-350     visualisation (NoSlipVel/Rho,
//                                              VelocityVel)
//   src/num/aslLBGKBC.cxx:691-736              ComputeSurfaceForceMap
//   src/acl/aclMath/aclVectorOfElementsOperations.cxx:249-258
//                                              component-sequential `+=`
//                                              (matters for the Coriolis term)
//
// Documented restatement choices (the reference is undefined there):
//   * Ghost cells are neither streamed nor collided; their populations change
//     only when a boundary condition writes them. In the reference they are
//     collided from uninitialised pool memory; with every face covered by a
//     boundary condition (or periodic) that never reaches an interior cell.
//   * Map-BC and force links count only when the fluid end is an interior cell
//     (the reference reads ghost-layer populations, i.e. uninitialised data,
//     for the others).
//   * Extensions absent from the reference: periodic axes, a body force
//     (Guo et al. 2002 forcing), a Smagorinsky closure (Hou et al. 1996),
//     standard D3Q27 weights (the reference's d3q27() has none).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

struct Lattice {
  int q = 0;
  int c[27][3];
  double w[27];
  int inv[27];
};

// Direction order as listed in aslTemplates.cxx (d3q15/d3q19/d3q27).
Lattice make_lattice(int q) {
  static const int v27[27][3] = {
      {0, 0, 0},  {1, 0, 0},   {0, 1, 0},   {0, 0, 1},   {-1, 0, 0},  {0, -1, 0},  {0, 0, -1},
      {1, 1, 0},  {1, -1, 0},  {-1, -1, 0}, {-1, 1, 0},  {0, 1, 1},   {0, 1, -1},  {0, -1, -1},
      {0, -1, 1}, {1, 0, 1},   {1, 0, -1},  {-1, 0, -1}, {-1, 0, 1},  {1, 1, 1},   {1, 1, -1},
      {1, -1, 1}, {1, -1, -1}, {-1, 1, 1},  {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
  static const int v15[15][3] = {{0, 0, 0},  {1, 0, 0},   {0, 1, 0},  {0, 0, 1},   {-1, 0, 0},
                                 {0, -1, 0}, {0, 0, -1},  {1, 1, 1},  {1, 1, -1},  {1, -1, 1},
                                 {1, -1, -1}, {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
  Lattice L;
  L.q = q;
  // Laplace coefficients as in aslTemplates.cxx; weight = LC/6 (+1 for rest).
  for (int i = 0; i < q; ++i) {
    const int* v = (q == 15) ? v15[i] : v27[i];
    for (int d = 0; d < 3; ++d) L.c[i][d] = v[d];
    int n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    double lc;
    if (q == 15) {
      lc = (n2 == 0) ? -14. / 3. : (n2 == 1 ? 2. / 3. : 1. / 12.);
      L.w[i] = lc / 6. + (n2 == 0 ? 1. : 0.);
    } else if (q == 19) {
      lc = (n2 == 0) ? -4. : (n2 == 1 ? 1. / 3. : 1. / 6.);
      L.w[i] = lc / 6. + (n2 == 0 ? 1. : 0.);
    } else {
      // Standard D3Q27 weights (the reference defines none).
      L.w[i] = (n2 == 0) ? 8. / 27. : (n2 == 1 ? 2. / 27. : (n2 == 2 ? 1. / 54. : 1. / 216.));
    }
  }
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < q; ++j)
      if (L.c[i][0] == -L.c[j][0] && L.c[i][1] == -L.c[j][1] && L.c[i][2] == -L.c[j][2]) L.inv[i] = j;
  return L;
}

enum BcKind {
  BC_NOSLIP = 0,
  BC_VELOCITY = 1,
  BC_PRESSURE = 2,
  BC_PRESSURE_VELOCITY = 3,
  MAP_NOSLIP = 10,
  MAP_VELOCITY = 11,          // constant velocity field
  MAP_VELOCITY_ROTATION = 12, // u = Omega x (r - c)
  MAP_PRESSURE_VELOCITY = 13,
  MAP_TRANSPORT_DEPOSITION = 14,
  MAP_KINETICS_DEPOSITION = 15,
  FIELD_NOSLIP_VEL = 20,
  FIELD_NOSLIP_RHO = 21,
  FIELD_VELOCITY_VEL = 22,
  FIELD_VELOCITY_VEL_ROTATION = 23,
};

struct Bc {
  int kind;
  double p;
  double u[3];
  double om[3], cen[3];  // rotation field
  double lf = 0, beta = 0;  // deposition: limiting factor, kinetic coefficient
  // Slice: (point, direction) pairs in the reference's addSlice order.
  std::vector<long> pts;
  std::vector<int> dirs;
  // Map: cells passing the guard with their fluid-neighbour mask.
  std::vector<long> cells;
  std::vector<uint32_t> masks;
  // Output-field conditions: per-cell direction weights (rho), q per cell.
  std::vector<double> wts;
};

template <class T>
struct Sim {
  int N[3], G[3];
  long L;
  Lattice lat;
  double nu;
  bool compressible = true, comp_vel = true, comp_rho = true;
  int periodic[3] = {0, 0, 0};
  double g[3] = {0, 0, 0};
  bool has_g = false;
  double Om[3] = {0, 0, 0};
  bool has_om = false;
  int closure = 0;  // 0 none, 1 asl-intent, 2 smagorinsky
  double cs = 0.17;
  double pos0[3] = {0, 0, 0};  // physical position of interior cell (0,0,0)
  double dx = 1.0;
  std::vector<T> f, fin, rho, u;
  std::vector<Bc> bcs;

  long idx(int x, int y, int z) const { return ((long)x * G[1] + y) * G[2] + z; }
  bool interior(int x, int y, int z) const {
    return x >= 1 && x <= N[0] && y >= 1 && y <= N[1] && z >= 1 && z <= N[2];
  }
  // Periodic axes map their ghost layer onto the opposite interior layer.
  int wrapc(int v, int a) const {
    if (!periodic[a]) return v;
    if (v < 1) return v + N[a];
    if (v > N[a]) return v - N[a];
    return v;
  }
};

template <class T>
void init_f(Sim<T>& s, const double* rho_field, const double* u_field, double rho0, const double* u0) {
  const Lattice& lat = s.lat;
  // f_i = rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u) over every cell (aslLBGK.cxx:262-280).
#pragma omp parallel for schedule(static)
  for (long n = 0; n < s.L; ++n) {
    T r = rho_field ? T(rho_field[n]) : T(rho0);
    T v[3];
    for (int d = 0; d < 3; ++d) v[d] = u_field ? T(u_field[d * s.L + n]) : T(u0[d]);
    T vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    for (int i = 0; i < lat.q; ++i) {
      T cu = v[0] * T(lat.c[i][0]) + v[1] * T(lat.c[i][1]) + v[2] * T(lat.c[i][2]);
      s.f[(long)i * s.L + n] = r * (T(1) + T(3) * cu + T(4.5) * (cu * cu) - T(1.5) * vv);
    }
    s.rho[n] = r;
    for (int d = 0; d < 3; ++d) s.u[d * s.L + n] = v[d];
  }
}

template <class T>
void step(Sim<T>& s) {
  const Lattice& lat = s.lat;
  const int Q = lat.q;
  // Pull streaming: f_in_i(x) = f*_i(x - c_i)  (aslLBGK.cxx:237-250).
#pragma omp parallel for collapse(2) schedule(static)
  for (int x = 1; x <= s.N[0]; ++x)
    for (int y = 1; y <= s.N[1]; ++y)
      for (int z = 1; z <= s.N[2]; ++z) {
        long n = s.idx(x, y, z);
        for (int i = 0; i < Q; ++i) {
          int sx = s.wrapc(x - lat.c[i][0], 0), sy = s.wrapc(y - lat.c[i][1], 1),
              sz = s.wrapc(z - lat.c[i][2], 2);
          s.fin[(long)i * s.L + n] = s.f[(long)i * s.L + s.idx(sx, sy, sz)];
        }
      }
  const T om0 = T(1) / (T(3) * T(s.nu) + T(0.5));
  T wc[27][3], ww[27];
  for (int i = 0; i < Q; ++i) {
    ww[i] = T(lat.w[i]);
    for (int d = 0; d < 3; ++d) wc[i][d] = T(double(lat.c[i][d]) * lat.w[i]);
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int x = 1; x <= s.N[0]; ++x)
    for (int y = 1; y <= s.N[1]; ++y)
      for (int z = 1; z <= s.N[2]; ++z) {
        long n = s.idx(x, y, z);
        T fo[27], feq[27];
        for (int i = 0; i < Q; ++i) fo[i] = s.fin[(long)i * s.L + n];
        // momentum before density, as in aslLBGK.cxx:204-205
        T m[3];
        for (int d = 0; d < 3; ++d) {
          T a = T(0);
          for (int j = 0; j < Q; ++j) a += fo[j] * wc[j][d];
          m[d] = a;
        }
        T rho = T(0);
        for (int j = 0; j < Q; ++j) rho += fo[j] * ww[j];
        T om = om0;
        if (s.has_om) {
          // Component-sequential update, as ACL emits `momentum += ...`.
          T k = T(2) / om;
          m[0] = m[0] + k * (T(s.Om[1]) * m[2] - T(s.Om[2]) * m[1]);
          m[1] = m[1] + k * (T(s.Om[2]) * m[0] - T(s.Om[0]) * m[2]);
          m[2] = m[2] + k * (T(s.Om[0]) * m[1] - T(s.Om[1]) * m[0]);
        }
        // Guo forcing (extension): equilibrium momentum m + rho g / 2.
        T ueq[3];
        if (s.has_g)
          for (int d = 0; d < 3; ++d) m[d] = m[d] + T(0.5) * rho * T(s.g[d]);
        if (s.comp_rho) s.rho[n] = rho;
        if (s.comp_vel)
          for (int d = 0; d < 3; ++d) s.u[d * s.L + n] = s.compressible ? m[d] / rho : m[d];
        T mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
        for (int i = 0; i < Q; ++i) {
          T cm = T(lat.c[i][0]) * m[0] + T(lat.c[i][1]) * m[1] + T(lat.c[i][2]) * m[2];
          if (s.compressible)
            feq[i] = rho + T(3) * cm + T(4.5) * (cm * cm) / rho - T(1.5) * mm / rho;
          else
            feq[i] = rho + T(3) * cm + T(4.5) * (cm * cm) - T(1.5) * mm;
        }
        if (s.closure == 1) {
          // LBGKTurbulence with f_eq evaluated before use (aslLBGK.cxx:315-322).
          T a = T(0), b = T(0);
          for (int i = 0; i < Q; ++i) {
            a += (fo[i] - feq[i]) * (fo[i] - feq[i]);
            b += fo[i] * fo[i];
          }
          T wl = T(4) * (a / b);
          if (wl > T(1)) om = T(1) / (T(3) * std::min(T(s.nu) * wl, T(0.5)) + T(0.5));
        } else if (s.closure == 2) {
          // Smagorinsky (Hou et al. 1996): tau = (tau0 + sqrt(tau0^2 + 18 sqrt2 Cs^2 |Pi|/rho))/2,
          // Pi_ab = sum_i w_i c_ia c_ib (f_i - feq_i) in standard normalisation.
          double P[6] = {0, 0, 0, 0, 0, 0};
          for (int i = 0; i < Q; ++i) {
            double d = double(ww[i]) * double(fo[i] - feq[i]);
            const int* c = lat.c[i];
            P[0] += d * c[0] * c[0];
            P[1] += d * c[1] * c[1];
            P[2] += d * c[2] * c[2];
            P[3] += d * c[0] * c[1];
            P[4] += d * c[1] * c[2];
            P[5] += d * c[0] * c[2];
          }
          double q2 = P[0] * P[0] + P[1] * P[1] + P[2] * P[2] + 2 * (P[3] * P[3] + P[4] * P[4] + P[5] * P[5]);
          double tau0 = 1.0 / double(om0);
          double tau = 0.5 * (tau0 + std::sqrt(tau0 * tau0 + 18.0 * std::sqrt(2.0) * s.cs * s.cs *
                                                                 std::sqrt(q2) / double(rho)));
          om = T(1.0 / tau);
        }
        for (int i = 0; i < Q; ++i) {
          T fn = fo[i] * (T(1) - om) + om * feq[i];
          if (s.has_g) {
            // Guo source (1 - om/2) w_i [3 (c - u) + 9 (c.u) c] . (rho g), in ASL units (/w_i).
            T u[3] = {m[0] / rho, m[1] / rho, m[2] / rho};
            T cu = T(lat.c[i][0]) * u[0] + T(lat.c[i][1]) * u[1] + T(lat.c[i][2]) * u[2];
            T src = T(0);
            for (int d = 0; d < 3; ++d)
              src += (T(3) * (T(lat.c[i][d]) - u[d]) + T(9) * cu * T(lat.c[i][d])) * T(s.g[d]);
            fn += (T(1) - T(0.5) * om) * rho * src;
          }
          s.f[(long)i * s.L + n] = fn;
        }
      }
}

// ---- boundary conditions -------------------------------------------------

// addSlice* (aslBCond.cxx:373-493): for wall W with inward normal n_W, every
// direction k>=1 with c_k.n_W > 0 and every interior point a of the first
// interior layer (tangential coordinates 1..N'-2) gives ghost point a - c_k.
template <class T>
void add_slices(Sim<T>& s, Bc& bc, int wallmask) {
  const Lattice& lat = s.lat;
  // wall order X0, XE, Y0, YE, Z0, ZE; normal directions 1,4,2,5,3,6
  static const int normal_dir[6] = {1, 4, 2, 5, 3, 6};
  static const int axis[6] = {0, 0, 1, 1, 2, 2};
  for (int w = 0; w < 6; ++w) {
    if (!(wallmask & (1 << w))) continue;
    int ax = axis[w];
    int layer = (w % 2 == 0) ? 1 : s.G[ax] - 2;
    const int* nv = lat.c[normal_dir[w]];
    int t1 = (ax == 0) ? 1 : 0, t2 = (ax == 2) ? 1 : 2;
    for (int k = 1; k < lat.q; ++k) {
      int dot = lat.c[k][0] * nv[0] + lat.c[k][1] * nv[1] + lat.c[k][2] * nv[2];
      if (dot <= 0) continue;
      for (int i = 1; i < s.G[t1] - 1; ++i)
        for (int j = 1; j < s.G[t2] - 1; ++j) {
          int a[3];
          a[ax] = layer;
          a[t1] = i;
          a[t2] = j;
          int p[3] = {a[0] - lat.c[k][0], a[1] - lat.c[k][1], a[2] - lat.c[k][2]};
          bc.pts.push_back(s.idx(p[0], p[1], p[2]));
          bc.dirs.push_back(k);
        }
    }
  }
}

template <class T>
double map_at(const Sim<T>& s, const float* map, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= s.G[0] || y >= s.G[1] || z >= s.G[2]) return -0.9;  // generateDCFullSafe(map,-.9)
  return map[s.idx(x, y, z)];
}

// Map BC guard and links (aslLBGKBC.cxx:219-254): a cell x is processed iff
// -0.9999 < map(x) <= 0; link k iff map(x + c_k) > 0 (fluid end interior).
// With a computational-domain map cd, a neighbour also needs cd > 0
// (src/num/aslBCond.cxx:204-211).
template <class T>
void build_map_links(Sim<T>& s, Bc& bc, const float* map, const float* cd = nullptr) {
  const Lattice& lat = s.lat;
  for (int x = 0; x < s.G[0]; ++x)
    for (int y = 0; y < s.G[1]; ++y)
      for (int z = 0; z < s.G[2]; ++z) {
        if ((s.periodic[0] && (x < 1 || x > s.N[0])) || (s.periodic[1] && (y < 1 || y > s.N[1])) ||
            (s.periodic[2] && (z < 1 || z > s.N[2])))
          continue;
        float m0 = map[s.idx(x, y, z)];
        if (!(m0 <= 0.f && m0 > -0.9999f)) continue;
        uint32_t mask = 0;
        for (int k = 1; k < lat.q; ++k) {
          int q[3] = {s.wrapc(x + lat.c[k][0], 0), s.wrapc(y + lat.c[k][1], 1), s.wrapc(z + lat.c[k][2], 2)};
          if (!s.interior(q[0], q[1], q[2])) continue;
          if (map_at(s, map, q[0], q[1], q[2]) > 0.0 && (!cd || cd[s.idx(q[0], q[1], q[2])] > 0.f)) mask |= 1u << k;
        }
        if (mask) {
          bc.cells.push_back(s.idx(x, y, z));
          bc.masks.push_back(mask);
        }
      }
}

template <class T>
void decode(const Sim<T>& s, long n, int& x, int& y, int& z) {
  z = int(n % s.G[2]);
  long r = n / s.G[2];
  y = int(r % s.G[1]);
  x = int(r / s.G[1]);
}

template <class T>
void bc_execute(Sim<T>& s, Bc& bc) {
  const Lattice& lat = s.lat;
  const long L = s.L;
  std::vector<T>& f = s.f;
  if (bc.kind < 10) {
    // Slice BC values (aslLBGKBC.cxx:91-202). Target is the ghost slot that the
    // interior point a = p + c_k pulls (periodic axes wrap the ghost point).
    long np = (long)bc.pts.size();
    for (long t = 0; t < np; ++t) {
      int k = bc.dirs[t];
      int px, py, pz;
      decode(s, bc.pts[t], px, py, pz);
      int ax = px + lat.c[k][0], ay = py + lat.c[k][1], az = pz + lat.c[k][2];
      long tgt = (long)k * L + s.idx(s.wrapc(px, 0), s.wrapc(py, 1), s.wrapc(pz, 2));
      long src = (long)lat.inv[k] * L + s.idx(ax, ay, az);
      T cu = T(lat.c[k][0]) * T(bc.u[0]) + T(lat.c[k][1]) * T(bc.u[1]) + T(lat.c[k][2]) * T(bc.u[2]);
      switch (bc.kind) {
        case BC_NOSLIP: f[tgt] = f[src]; break;
        case BC_VELOCITY: f[tgt] = f[src] + T(6) * cu; break;
        case BC_PRESSURE: f[tgt] = T(bc.p); break;
        case BC_PRESSURE_VELOCITY: f[tgt] = T(bc.p) + T(3) * cu; break;
      }
    }
    return;
  }
  // Map BCs: writes go to ghost (solid) cells, reads come from fluid cells,
  // so the per-cell loop has no order dependence within one BC.
  long nc = (long)bc.cells.size();
#pragma omp parallel for schedule(static)
  for (long t = 0; t < nc; ++t) {
    long cell = bc.cells[t];
    uint32_t mask = bc.masks[t];
    int x, y, z;
    decode(s, cell, x, y, z);
    auto nb = [&](int k) {
      return s.idx(s.wrapc(x + lat.c[k][0], 0), s.wrapc(y + lat.c[k][1], 1), s.wrapc(z + lat.c[k][2], 2));
    };
    if (bc.kind == MAP_NOSLIP) {
      for (int k = 1; k < lat.q; ++k)
        if (mask >> k & 1u) f[(long)k * L + cell] = f[(long)lat.inv[k] * L + nb(k)];
    } else if (bc.kind == MAP_VELOCITY || bc.kind == MAP_VELOCITY_ROTATION) {
      // aslLBGKBC.cxx:312-339: rho_b = sum_k w_k f_kbar(x+c_k) / sum_k w_k, f_k = rho_b (1 + 3 u.c_k)
      T coef = T(0), rb = T(0);
      for (int k = 1; k < lat.q; ++k)
        if (mask >> k & 1u) {
          coef += T(lat.w[k]);
          rb += f[(long)lat.inv[k] * L + nb(k)] * T(lat.w[k]);
        }
      rb /= coef;
      T uu[3];
      if (bc.kind == MAP_VELOCITY) {
        for (int d = 0; d < 3; ++d) uu[d] = T(bc.u[d]);
      } else {
        double r[3] = {s.pos0[0] + (x - 1) * s.dx - bc.cen[0], s.pos0[1] + (y - 1) * s.dx - bc.cen[1],
                       s.pos0[2] + (z - 1) * s.dx - bc.cen[2]};
        uu[0] = T(bc.om[1] * r[2] - bc.om[2] * r[1]);
        uu[1] = T(bc.om[2] * r[0] - bc.om[0] * r[2]);
        uu[2] = T(bc.om[0] * r[1] - bc.om[1] * r[0]);
      }
      T mom[3] = {uu[0] * rb, uu[1] * rb, uu[2] * rb};
      for (int k = 1; k < lat.q; ++k)
        if (mask >> k & 1u) {
          T mc = mom[0] * T(lat.c[k][0]) + mom[1] * T(lat.c[k][1]) + mom[2] * T(lat.c[k][2]);
          f[(long)k * L + cell] = rb + mc * T(3);
        }
    } else if (bc.kind == MAP_TRANSPORT_DEPOSITION || bc.kind == MAP_KINETICS_DEPOSITION) {
      // aslLBGKBC.cxx:477-500, 546-569: rho = sum_k w_k f_kbar(x+c_k), coef = sum_k w_k,
      // transport: j = rho - (rho - coef p0) / (1 + coef lF); kinetics:
      // j = rho - beta (rho / coef - p0) / (1 + lF); f_k(x) = j / coef
      T coef = T(0), rho = T(0);
      for (int k = 1; k < lat.q; ++k)
        if (mask >> k & 1u) {
          coef += T(lat.w[k]);
          rho += f[(long)lat.inv[k] * L + nb(k)] * T(lat.w[k]);
        }
      const T p0 = T(bc.p), lf = T(bc.lf);
      const T j = bc.kind == MAP_TRANSPORT_DEPOSITION ? rho - (rho - coef * p0) / (T(1) + coef * lf)
                                                      : rho - T(bc.beta) * (rho / coef - p0) / (T(1) + lf);
      for (int k = 1; k < lat.q; ++k)
        if (mask >> k & 1u) f[(long)k * L + cell] = j / coef;
    } else if (bc.kind == MAP_PRESSURE_VELOCITY) {
      // aslLBGKBC.cxx:400-423
      T P = T(bc.p), uu[3] = {T(bc.u[0]), T(bc.u[1]), T(bc.u[2])};
      T vv = uu[0] * uu[0] + uu[1] * uu[1] + uu[2] * uu[2];
      for (int k = 1; k < lat.q; ++k)
        if (mask >> k & 1u) {
          T cu = uu[0] * T(lat.c[k][0]) + uu[1] * T(lat.c[k][1]) + uu[2] * T(lat.c[k][2]);
          T fe = s.compressible ? P + T(3) * P * cu + T(4.5) * P * cu * cu - T(1.5) * P * vv
                                : P + T(3) * cu + T(4.5) * cu * cu - T(1.5) * vv;
          f[(long)k * L + cell] = fe;
        }
    }
  }
}

// ComputeSurfaceForceMap (aslLBGKBC.cxx:691-736), per cell with |map| < 0.9999.
// out6 = (sum F, sum (r - r0) x F) in double, field (3L floats) optional.
template <class T>
void force(Sim<T>& s, const float* map, float* field, const double* r0, double* out6) {
  const Lattice& lat = s.lat;
  const long L = s.L;
  for (int i = 0; i < 6; ++i) out6[i] = 0;
  double F0 = 0, F1 = 0, F2 = 0, T0 = 0, T1 = 0, T2 = 0;
#pragma omp parallel for collapse(2) reduction(+ : F0, F1, F2, T0, T1, T2) schedule(static)
  for (int x = 0; x < s.G[0]; ++x)
    for (int y = 0; y < s.G[1]; ++y)
      for (int z = 0; z < s.G[2]; ++z) {
        if ((s.periodic[0] && (x < 1 || x > s.N[0])) || (s.periodic[1] && (y < 1 || y > s.N[1])) ||
            (s.periodic[2] && (z < 1 || z > s.N[2])))
          continue;
        long n = s.idx(x, y, z);
        float m0 = map[n];
        if (!(std::fabs(m0) < 0.9999f)) continue;
        T Fc[3] = {T(0), T(0), T(0)};
        bool in0 = s.interior(x, y, z);
        for (int k = 1; k < lat.q; ++k) {
          int q[3] = {s.wrapc(x + lat.c[k][0], 0), s.wrapc(y + lat.c[k][1], 1), s.wrapc(z + lat.c[k][2], 2)};
          double mk = map_at(s, map, q[0], q[1], q[2]);
          bool b0 = (m0 <= 0.f) && (mk > 0.0) && s.interior(q[0], q[1], q[2]);
          bool bI = (mk <= 0.0) && (m0 > 0.f) && in0;
          if (!b0 && !bI) continue;
          long nq = s.idx(q[0], q[1], q[2]);
          T f0 = s.f[(long)k * L + n];
          T fI = s.f[(long)lat.inv[k] * L + nq];
          T a = b0 ? (f0 + fI - T(2)) : (-f0 - fI + T(2));
          for (int d = 0; d < 3; ++d) Fc[d] += a * T(lat.w[k] * lat.c[k][d]);
        }
        if (field)
          for (int d = 0; d < 3; ++d) field[d * L + n] = float(Fc[d]);
        double r[3] = {s.pos0[0] + (x - 1) * s.dx - r0[0], s.pos0[1] + (y - 1) * s.dx - r0[1],
                       s.pos0[2] + (z - 1) * s.dx - r0[2]};
        double F[3] = {double(Fc[0]), double(Fc[1]), double(Fc[2])};
        F0 += F[0];
        F1 += F[1];
        F2 += F[2];
        T0 += r[1] * F[2] - r[2] * F[1];
        T1 += r[2] * F[0] - r[0] * F[2];
        T2 += r[0] * F[1] - r[1] * F[0];
      }
  out6[0] = F0; out6[1] = F1; out6[2] = F2;
  out6[3] = T0; out6[4] = T1; out6[5] = T2;
}

struct Handle {
  int prec;
  Sim<float>* sf = nullptr;
  Sim<double>* sd = nullptr;
};

template <class T>
Sim<T>* make_sim(int nx, int ny, int nz, int q, double nu, int flags) {
  auto* s = new Sim<T>();
  s->N[0] = nx; s->N[1] = ny; s->N[2] = nz;
  for (int a = 0; a < 3; ++a) s->G[a] = s->N[a] + 2;
  s->L = (long)s->G[0] * s->G[1] * s->G[2];
  s->lat = make_lattice(q);
  s->nu = nu;
  s->comp_vel = !(flags & 1);
  s->comp_rho = !(flags & 2);
  s->compressible = !(flags & 4);
  for (int a = 0; a < 3; ++a) s->periodic[a] = (flags >> (3 + a)) & 1;
  s->f.assign((size_t)q * s->L, T(1));
  s->fin.assign((size_t)q * s->L, T(1));
  s->rho.assign(s->L, T(1));
  s->u.assign(3 * s->L, T(0));
  return s;
}

}  // namespace

#define DISPATCH(h, call)            \
  do {                               \
    if ((h)->sf) { auto& S = *(h)->sf; call; } \
    else { auto& S = *(h)->sd; call; }         \
  } while (0)

// ComputeSurfaceFluxMap (aslLBGKBC.cxx:623-665), per cell with |map| < 0.9999:
// flux = sum_k w_k (f_k(x) - f_kbar(x + c_k)) over links from a solid x to a
// fluid interior neighbour, minus the same over links from a fluid interior x
// to a solid neighbour. field (L floats) optional; returns the FP64 total.
template <class T>
double flux(Sim<T>& s, const float* map, float* field) {
  const Lattice& lat = s.lat;
  const long L = s.L;
  double tot = 0;
#pragma omp parallel for collapse(2) reduction(+ : tot) schedule(static)
  for (int x = 0; x < s.G[0]; ++x)
    for (int y = 0; y < s.G[1]; ++y)
      for (int z = 0; z < s.G[2]; ++z) {
        if ((s.periodic[0] && (x < 1 || x > s.N[0])) || (s.periodic[1] && (y < 1 || y > s.N[1])) ||
            (s.periodic[2] && (z < 1 || z > s.N[2])))
          continue;
        long n = s.idx(x, y, z);
        float m0 = map[n];
        if (!(std::fabs(m0) < 0.9999f)) continue;
        T fl = T(0);
        bool in0 = s.interior(x, y, z), any = false;
        for (int k = 1; k < lat.q; ++k) {
          int q[3] = {s.wrapc(x + lat.c[k][0], 0), s.wrapc(y + lat.c[k][1], 1), s.wrapc(z + lat.c[k][2], 2)};
          double mk = map_at(s, map, q[0], q[1], q[2]);
          bool b0 = (m0 <= 0.f) && (mk > 0.0) && s.interior(q[0], q[1], q[2]);
          bool bI = (mk <= 0.0) && (m0 > 0.f) && in0;
          if (!b0 && !bI) continue;
          any = true;
          long nq = s.idx(q[0], q[1], q[2]);
          T f0 = s.f[(long)k * L + n];
          T fI = s.f[(long)lat.inv[k] * L + nq];
          fl += (b0 ? (f0 - fI) : (fI - f0)) * T(lat.w[k]);
        }
        if (!any) continue;
        if (field) field[n] = float(fl);
        tot += double(fl);
      }
  return tot;
}

// Output-field conditions (aslBasicBC.cxx): guard cells -0.9999 < map <= 0,
// fluid neighbours map > 0 and interior. NoSlipVel: u = sum LC_k (2*0 - u_nb) /
// max(sum LC_k, 0.01) (BCConstantValueMiddlePointMap, :171-230). NoSlipRho:
// rho = sum W_k rho_nb / sum W_k if sum W_k > 0.1, W_k = (n . c_k/|c_k| + 1)^2,
// n the unit map gradient with the template's gradient coefficients
// (BCConstantGradientMap, :300-350). VelocityVel: u = v(position) (BCValuePFMap,
// :123-145). Template coefficients of d3q15 / d3q19 (aslTemplates.cxx:146-185).
template <class T>
void build_field(Sim<T>& s, Bc& bc, const float* map) {
  const Lattice& lat = s.lat;
  const double gcax = lat.q == 15 ? 1.0 / 3.0 : 1.0 / 6.0, gcdg = lat.q == 15 ? 1.0 / 24.0 : 1.0 / 12.0;
  for (int x = 0; x < s.G[0]; ++x)
    for (int y = 0; y < s.G[1]; ++y)
      for (int z = 0; z < s.G[2]; ++z) {
        if ((s.periodic[0] && (x < 1 || x > s.N[0])) || (s.periodic[1] && (y < 1 || y > s.N[1])) ||
            (s.periodic[2] && (z < 1 || z > s.N[2])))
          continue;
        float m0 = map[s.idx(x, y, z)];
        if (!(m0 <= 0.f && m0 > -0.9999f)) continue;
        uint32_t mask = 0;
        double n[3] = {0, 0, 0};
        for (int k = 1; k < lat.q; ++k) {
          int q[3] = {s.wrapc(x + lat.c[k][0], 0), s.wrapc(y + lat.c[k][1], 1), s.wrapc(z + lat.c[k][2], 2)};
          double mk = map_at(s, map, q[0], q[1], q[2]);
          if (mk > 0.0 && s.interior(q[0], q[1], q[2])) mask |= 1u << k;
          int n2 = lat.c[k][0] * lat.c[k][0] + lat.c[k][1] * lat.c[k][1] + lat.c[k][2] * lat.c[k][2];
          for (int d = 0; d < 3; ++d) n[d] += (n2 == 1 ? gcax : gcdg) * lat.c[k][d] * mk;
        }
        if (bc.kind == FIELD_NOSLIP_RHO) {
          double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
          if (!(len > 0.0) || !mask) continue;
          for (int k = 0; k < lat.q; ++k) {
            double w = 0;
            if (k > 0 && (mask >> k & 1u)) {
              double cl = std::sqrt(double(lat.c[k][0] * lat.c[k][0] + lat.c[k][1] * lat.c[k][1] +
                                           lat.c[k][2] * lat.c[k][2]));
              double dc = (n[0] * lat.c[k][0] + n[1] * lat.c[k][1] + n[2] * lat.c[k][2]) / len / cl + 1.0;
              w = dc * dc;
            }
            bc.wts.push_back(w);
          }
        }
        bc.cells.push_back(s.idx(x, y, z));
        bc.masks.push_back(mask);
      }
}

template <class T>
void field_execute(Sim<T>& s, Bc& bc) {
  const Lattice& lat = s.lat;
  const long L = s.L;
  for (size_t t = 0; t < bc.cells.size(); ++t) {
    long cell = bc.cells[t];
    uint32_t mask = bc.masks[t];
    int x, y, z;
    decode(s, cell, x, y, z);
    auto nb = [&](int k) {
      return s.idx(s.wrapc(x + lat.c[k][0], 0), s.wrapc(y + lat.c[k][1], 1), s.wrapc(z + lat.c[k][2], 2));
    };
    if (bc.kind == FIELD_NOSLIP_VEL) {
      T v[3] = {T(0), T(0), T(0)}, counter = T(0);
      for (int k = 1; k < lat.q; ++k) {
        if (!(mask >> k & 1u)) continue;
        int n2 = lat.c[k][0] * lat.c[k][0] + lat.c[k][1] * lat.c[k][1] + lat.c[k][2] * lat.c[k][2];
        T lc = T(n2 == 1 ? (lat.q == 15 ? 2.0 / 3.0 : 1.0 / 3.0) : (lat.q == 15 ? 1.0 / 12.0 : 1.0 / 6.0));
        for (int d = 0; d < 3; ++d) v[d] += (T(0) - s.u[d * L + nb(k)]) * lc;
        counter += lc;
      }
      T c = counter > T(0.01) ? counter : T(0.01);
      for (int d = 0; d < 3; ++d) s.u[d * L + cell] = v[d] / c;
    } else if (bc.kind == FIELD_NOSLIP_RHO) {
      T sum = T(0), counter = T(0);
      for (int k = 1; k < lat.q; ++k) {
        if (!(mask >> k & 1u)) continue;
        T w = T(bc.wts[t * lat.q + k]);
        sum += s.rho[nb(k)] * w;
        counter += w;
      }
      if (counter > T(0.1)) s.rho[cell] = sum / counter;
    } else {
      T v[3] = {T(bc.u[0]), T(bc.u[1]), T(bc.u[2])};
      if (bc.kind == FIELD_VELOCITY_VEL_ROTATION) {
        double r[3] = {s.pos0[0] + (x - 1) * s.dx - bc.cen[0], s.pos0[1] + (y - 1) * s.dx - bc.cen[1],
                       s.pos0[2] + (z - 1) * s.dx - bc.cen[2]};
        v[0] = T(bc.om[1] * r[2] - bc.om[2] * r[1]);
        v[1] = T(bc.om[2] * r[0] - bc.om[0] * r[2]);
        v[2] = T(bc.om[0] * r[1] - bc.om[1] * r[0]);
      }
      for (int d = 0; d < 3; ++d) s.u[d * L + cell] = v[d];
    }
  }
}

extern "C" {

// flags: bit0 no velocity output, bit1 no density output, bit2 incompressible,
// bits3-5 periodic x/y/z.
void* orc_create(int nx, int ny, int nz, int q, int prec, double nu, int flags) {
  if (q != 15 && q != 19 && q != 27) return nullptr;
  auto* h = new Handle();
  h->prec = prec;
  if (prec == 4) h->sf = make_sim<float>(nx, ny, nz, q, nu, flags);
  else h->sd = make_sim<double>(nx, ny, nz, q, nu, flags);
  return h;
}

void orc_destroy(void* p) {
  auto* h = (Handle*)p;
  delete h->sf;
  delete h->sd;
  delete h;
}

void orc_set_threads(int n) { omp_set_num_threads(n); }
int orc_get_threads() { return omp_get_max_threads(); }

void orc_set_viscosity(void* p, double nu) { auto* h = (Handle*)p; DISPATCH(h, S.nu = nu); }
void orc_set_body_force(void* p, double gx, double gy, double gz) {
  auto* h = (Handle*)p;
  DISPATCH(h, { S.g[0] = gx; S.g[1] = gy; S.g[2] = gz; S.has_g = (gx != 0 || gy != 0 || gz != 0); });
}
void orc_set_omega(void* p, double wx, double wy, double wz) {
  auto* h = (Handle*)p;
  DISPATCH(h, { S.Om[0] = wx; S.Om[1] = wy; S.Om[2] = wz; S.has_om = true; });
}
void orc_set_closure(void* p, int mode, double cs) {
  auto* h = (Handle*)p;
  DISPATCH(h, { S.closure = mode; S.cs = cs; });
}
void orc_set_position(void* p, double x0, double y0, double z0, double dx) {
  auto* h = (Handle*)p;
  DISPATCH(h, { S.pos0[0] = x0; S.pos0[1] = y0; S.pos0[2] = z0; S.dx = dx; });
}

void orc_init_f(void* p, double rho, double ux, double uy, double uz) {
  auto* h = (Handle*)p;
  double u0[3] = {ux, uy, uz};
  DISPATCH(h, init_f(S, nullptr, nullptr, rho, u0));
}
void orc_init_f_fields(void* p, const double* rho, const double* u) {
  auto* h = (Handle*)p;
  double u0[3] = {0, 0, 0};
  DISPATCH(h, init_f(S, rho, u, 1.0, u0));
}

void orc_step(void* p, int n) {
  auto* h = (Handle*)p;
  for (int i = 0; i < n; ++i) DISPATCH(h, step(S));
}

int orc_bc_slice(void* p, int kind, int wallmask, double pr, double ux, double uy, double uz) {
  auto* h = (Handle*)p;
  int id = -1;
  DISPATCH(h, {
    Bc bc;
    bc.kind = kind;
    bc.p = pr;
    bc.u[0] = ux; bc.u[1] = uy; bc.u[2] = uz;
    add_slices(S, bc, wallmask);
    S.bcs.push_back(std::move(bc));
    id = (int)S.bcs.size() - 1;
  });
  return id;
}

int orc_bc_map_cd(void* p, int kind, const float* map, const float* cd, double pr, const double* u,
                  const double* om, const double* cen) {
  auto* h = (Handle*)p;
  int id = -1;
  DISPATCH(h, {
    Bc bc;
    bc.kind = kind;
    bc.p = pr;
    for (int d = 0; d < 3; ++d) {
      bc.u[d] = u ? u[d] : 0.0;
      bc.om[d] = om ? om[d] : 0.0;
      bc.cen[d] = cen ? cen[d] : 0.0;
    }
    build_map_links(S, bc, map, cd);
    S.bcs.push_back(std::move(bc));
    id = (int)S.bcs.size() - 1;
  });
  return id;
}

int orc_bc_map(void* p, int kind, const float* map, double pr, const double* u, const double* om,
               const double* cen) {
  auto* h = (Handle*)p;
  int id = -1;
  DISPATCH(h, {
    Bc bc;
    bc.kind = kind;
    bc.p = pr;
    for (int d = 0; d < 3; ++d) {
      bc.u[d] = u ? u[d] : 0.0;
      bc.om[d] = om ? om[d] : 0.0;
      bc.cen[d] = cen ? cen[d] : 0.0;
    }
    build_map_links(S, bc, map);
    S.bcs.push_back(std::move(bc));
    id = (int)S.bcs.size() - 1;
  });
  return id;
}

int orc_bc_deposition(void* p, int kind, const float* map, double p0, double lf, double beta) {
  auto* h = (Handle*)p;
  int id = -1;
  DISPATCH(h, {
    Bc bc;
    bc.kind = kind;
    bc.p = p0;
    bc.lf = lf;
    bc.beta = beta;
    for (int d = 0; d < 3; ++d) bc.u[d] = bc.om[d] = bc.cen[d] = 0.0;
    build_map_links(S, bc, map);
    S.bcs.push_back(std::move(bc));
    id = (int)S.bcs.size() - 1;
  });
  return id;
}

double orc_flux(void* p, const float* map, float* field) {
  auto* h = (Handle*)p;
  double t = 0;
  DISPATCH(h, t = flux(S, map, field));
  return t;
}

long orc_bc_size(void* p, int id) {
  auto* h = (Handle*)p;
  long n = 0;
  DISPATCH(h, { n = S.bcs[id].kind < 10 ? (long)S.bcs[id].pts.size() : (long)S.bcs[id].cells.size(); });
  return n;
}

void orc_bc_execute(void* p, int id) {
  auto* h = (Handle*)p;
  DISPATCH(h, {
    if (S.bcs[id].kind >= FIELD_NOSLIP_VEL)
      field_execute(S, S.bcs[id]);
    else
      bc_execute(S, S.bcs[id]);
  });
}

int orc_bc_field(void* p, int kind, const float* map, const double* u, const double* om, const double* cen) {
  auto* h = (Handle*)p;
  int id = -1;
  DISPATCH(h, {
    Bc bc;
    bc.kind = kind;
    bc.p = 0;
    for (int d = 0; d < 3; ++d) {
      bc.u[d] = u ? u[d] : 0.0;
      bc.om[d] = om ? om[d] : 0.0;
      bc.cen[d] = cen ? cen[d] : 0.0;
    }
    build_field(S, bc, map);
    S.bcs.push_back(std::move(bc));
    id = (int)S.bcs.size() - 1;
  });
  return id;
}

void orc_force(void* p, const float* map, float* field, const double* r0, double* out6) {
  auto* h = (Handle*)p;
  DISPATCH(h, force(S, map, field, r0, out6));
}

long orc_size(void* p) {
  auto* h = (Handle*)p;
  long n = 0;
  DISPATCH(h, n = S.L);
  return n;
}

void orc_get_f(void* p, double* out) {
  auto* h = (Handle*)p;
  DISPATCH(h, { for (size_t i = 0; i < S.f.size(); ++i) out[i] = double(S.f[i]); });
}
void orc_set_f(void* p, const double* in) {
  auto* h = (Handle*)p;
  DISPATCH(h, { for (size_t i = 0; i < S.f.size(); ++i) S.f[i] = decltype(S.f[0] + 0)(in[i]); });
}
void orc_get_rho(void* p, double* out) {
  auto* h = (Handle*)p;
  DISPATCH(h, { for (long i = 0; i < S.L; ++i) out[i] = double(S.rho[i]); });
}
void orc_get_u(void* p, double* out) {
  auto* h = (Handle*)p;
  DISPATCH(h, { for (long i = 0; i < 3 * S.L; ++i) out[i] = double(S.u[i]); });
}

// Lattice tables for cross-checks: c (3q ints), w (q doubles), inv (q ints).
void orc_lattice(int q, int* c, double* w, int* inv) {
  Lattice L = make_lattice(q);
  for (int i = 0; i < q; ++i) {
    for (int d = 0; d < 3; ++d) c[3 * i + d] = L.c[i][d];
    w[i] = L.w[i];
    inv[i] = L.inv[i];
  }
}

// Sum with FP64 accumulation; pinned against the reduction known answers of
// test/testMath/testReductionFunction.cc.
double orc_sum(const double* a, long n) {
  double s = 0;
  for (long i = 0; i < n; ++i) s += a[i];
  return s;
}

// Workload geometry for the CPU side of the benchmark: the porous channel's
// seeded random sequential addition of non-overlapping spheres, so that the
// CPU runs build their workload without the CUDA library. Same draws as the
// library's aslb_geom_pack_spheres (splitmix64 stream, uniform doubles from
// the top 53 bits, radii drawn until 1.25x the target volume and placed
// largest first, up to `attempts` centres per radius), with its own neighbour
// search: a dense grid of cells at least 2 rmax wide in every axis (the grid
// tiles a periodic x exactly), so the accept / reject decisions -- and the
// spheres -- are the same. A CPU test checks the two bit for bit.
int orc_pack_spheres(int nx, int ny, int nz, double rmin, double rmax, double solid_fraction,
                     unsigned long long seed, int periodic_x, int attempts, int max_spheres, double* centers,
                     double* radii, int* count) {
  if (!centers || !radii || !count || nx < 1 || ny < 1 || nz < 1 || !(rmin > 0) || rmax < rmin || max_spheres < 1)
    return -1;
  uint64_t state = seed;
  auto draw = [&](double a, double b) {
    state += 0x9e3779b97f4a7c15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return a + (b - a) * (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  const double target = solid_fraction * (double(nx) * ny * nz);
  std::vector<double> rs;
  double vol = 0.0;
  while (vol < target * 1.25 && (int)rs.size() < 4 * max_spheres) {
    const double r = draw(rmin, rmax);
    rs.push_back(r);
    vol += 4.0 / 3.0 * M_PI * r * r * r;
  }
  std::sort(rs.begin(), rs.end(), [](double a, double b) { return a > b; });
  const int N[3] = {nx, ny, nz};
  int nc[3];
  double cw[3];
  for (int a = 0; a < 3; ++a) {
    nc[a] = std::max(1, (int)std::floor(N[a] / (2.0 * rmax)));
    cw[a] = double(N[a]) / nc[a];
  }
  std::vector<std::vector<int>> cells((size_t)nc[0] * nc[1] * nc[2]);
  auto cell_of = [&](double v, int a) { return std::min(std::max((int)std::floor(v / cw[a]), 0), nc[a] - 1); };
  int n = 0;
  double placed = 0.0;
  for (double r : rs) {
    if (placed >= target || n >= max_spheres) break;
    for (int t = 0; t < attempts; ++t) {
      const double cx = periodic_x ? draw(0, nx) : draw(r, nx - 1 - r);
      const double cy = draw(r, ny - 1 - r), cz = draw(r, nz - 1 - r);
      const int c0[3] = {cell_of(cx, 0), cell_of(cy, 1), cell_of(cz, 2)};
      bool free = true;
      for (int i = -1; i <= 1 && free; ++i) {
        int ix = c0[0] + i;
        if (periodic_x) ix = (ix + nc[0]) % nc[0];
        else if (ix < 0 || ix >= nc[0]) continue;
        for (int j = -1; j <= 1 && free; ++j) {
          const int iy = c0[1] + j;
          if (iy < 0 || iy >= nc[1]) continue;
          for (int k = -1; k <= 1 && free; ++k) {
            const int iz = c0[2] + k;
            if (iz < 0 || iz >= nc[2]) continue;
            for (int o : cells[((size_t)ix * nc[1] + iy) * nc[2] + iz]) {
              double dx = centers[3 * o] - cx;
              const double dy = centers[3 * o + 1] - cy, dz = centers[3 * o + 2] - cz;
              if (periodic_x) dx -= nx * std::nearbyint(dx / nx);
              const double rr = radii[o] + r;
              if (dx * dx + dy * dy + dz * dz < rr * rr) {
                free = false;
                break;
              }
            }
          }
        }
      }
      if (!free) continue;
      cells[((size_t)c0[0] * nc[1] + c0[1]) * nc[2] + c0[2]].push_back(n);
      centers[3 * n] = cx;
      centers[3 * n + 1] = cy;
      centers[3 * n + 2] = cz;
      radii[n] = r;
      ++n;
      placed += 4.0 / 3.0 * M_PI * r * r * r;
      break;
    }
  }
  *count = n;
  return 0;
}

}  // extern "C"
