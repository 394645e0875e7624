// C ABI of libaslb.so (declared in include/aslb.h): domain handles, host-side
// construction of the compact boundary-link lists, and the time loop.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <nvtx3/nvToolsExt.h>
#include "aslb.h"
#include "kernels.h"
#include "mlp.cuh"

using namespace aslb;

namespace {
thread_local std::string g_err;
int g_device = 0;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace

void aslb::set_last_error(const std::string& msg) { g_err = msg; }

#define ASLB_CUDA(expr)                                                                              \
  do {                                                                                               \
    cudaError_t e_ = (expr);                                                                         \
    if (e_ != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define ASLB_CHECK_HANDLE(h) \
  if (!(h)) return fail(ASLB_ERR_ARG, std::string(__func__) + ": null handle")

// A named range on the profiler timeline (NVTX) for the duration of a call:
// nsys / ncu show the library's steps, conditions and batches by name. Without
// a tool attached the push and pop return at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

struct aslb_lbgk {
  DomainDev d{};
  StepParams p{};
  int closure = CL_NONE;
  int parity = 0;  // 0: representation A, 1: representation B
  unsigned flags = 0;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  long long steps = 0;
  bool comp_vel = true, comp_rho = true, macro_once = false;
  double pos0[3] = {0, 0, 0};
  double dx = 1.0;
  void* mlp_dev = nullptr;
  // learned closure: Cs^2 per storage cell, refreshed every mlp_period steps
  float* cs2_field = nullptr;
  int mlp_period = 32;
  long long mlp_last = -1;  // step at which the field was last computed
  void* stage = nullptr;            // one-direction transfer buffer (stage_buffer)
  void* u_own = nullptr;            // the domain's own velocity field (d.u may be a caller's)
  double* red_partials = nullptr;  // moments scratch
  double* red_out = nullptr;
  double* host_out = nullptr;      // pinned
  int* host_err = nullptr;         // pinned copy of the device error word
  // time-loop graph cache
  cudaGraphExec_t graph = nullptr;
  std::vector<aslb_bc*> graph_bcs;
  int graph_parity = -1;
  long long graph_version = -1;
  long long version = 0;  // bumped by every parameter change
  // fused no-slip conditions
  // fresh: populations were (re)initialised and no fused condition has run
  // since, so incoming slots still hold their initial values and the next
  // step must read them as they are (no bounce-back, no skipped writes).
  bool fresh = true;
  std::vector<uint2> mask_host;
  uint2* mask_dev = nullptr;
  // one word per cell when no cell has both bounce and elide bits (bit 31:
  // the low bits are elide bits), read by the two-cells-per-thread kernel
  uint32_t* mask32_dev = nullptr;
  // conditions and force objects made on this domain; destroying the domain
  // releases their device memory and detaches them (any destruction order)
  std::vector<aslb_bc*> bcs;
  std::vector<aslb_force*> forces;
  std::vector<aslb_batch*> batches;  // batches this domain belongs to
  std::vector<aslb_fd*> fds;         // FD solvers reading its velocity
};

namespace aslb {
int lbgk_velocity_binding(aslb_lbgk* h, int n[3], int* storage, void** u, cudaStream_t* st) {
  if (!h) {
    set_last_error("aslb_fd_set_velocity: null domain");
    return ASLB_ERR_ARG;
  }
  if (!h->comp_vel) {
    set_last_error("aslb_fd_set_velocity: the domain does not write its velocity (created with ASLB_NO_VELOCITY)");
    return ASLB_ERR_ARG;
  }
  n[0] = h->d.g.nx;
  n[1] = h->d.g.ny;
  n[2] = h->d.g.nz;
  *storage = h->d.storage;
  *u = h->d.u;
  *st = h->stream;
  return ASLB_OK;
}
void lbgk_attach_fd(aslb_lbgk* h, aslb_fd* f) { h->fds.push_back(f); }
void lbgk_detach_fd(aslb_lbgk* h, aslb_fd* f) { h->fds.erase(std::remove(h->fds.begin(), h->fds.end(), f), h->fds.end()); }
}  // namespace aslb

struct aslb_bc {
  aslb_lbgk* h = nullptr;
  int4* anchors = nullptr;  // anchor form: (x, y, z, direction mask)
  int n = 0;
  int* dlinks = nullptr;    // direction-sorted form: anchor storage index per link
  int nd = 0;
  LinkSet ls{};
  long long links = 0;
  bool fused = false;  // folded into the stream-collide kernel (execute is a no-op)
  BcParams bp{};
  std::vector<int> host_links;     // host copies, kept for fusing
  std::vector<int4> host_anchors;
  double* fweights = nullptr;      // field condition on rho: per-cell direction weights
  bool field() const { return bp.kind >= BCK_FIELD_NOSLIP_VEL; }
};

struct aslb_force {
  aslb_lbgk* h = nullptr;
  bool flux = false;  // ComputeSurfaceFlux object (one value per cell)
  int4* cells = nullptr;
  uint32_t* mask_in = nullptr;
  int n = 0;
  float* field = nullptr;
  double* partials = nullptr;
  double* out = nullptr;
  double* host_out = nullptr;
};

namespace {

void prepare_params(aslb_lbgk* h) {
  // omega = 1 / (3 nu + 1/2) (src/num/aslLBGK.cxx:203), once per step on the host
  h->p.om0f = 1.0f / (3.0f * (float)h->p.nu + 0.5f);
  h->p.om0d = 1.0 / (3.0 * h->p.nu + 0.5);
  h->p.nuf = (float)h->p.nu;
  h->p.csf = (float)h->p.cs;
  for (int a = 0; a < 3; ++a) {
    h->p.gf[a] = (float)h->p.g[a];
    h->p.Omf[a] = (float)h->p.Om[a];
  }
  for (int i = 0; i < 27; ++i) {
    double cg = 0.0;
    if (i < h->d.q)
      for (int a = 0; a < 3; ++a) cg += lattice_c(h->d.q, i, a) * h->p.g[a];
    h->p.cgd[i] = cg;
    h->p.cgf[i] = (float)cg;
  }
  h->p.write_rho = (h->comp_rho || h->macro_once) ? 1 : 0;
  h->p.write_vel = (h->comp_vel || h->macro_once) ? 1 : 0;
  h->p.write_macro = h->p.write_rho | h->p.write_vel;
  h->p.cs2 = h->cs2_field;
  h->p.mask = h->fresh ? nullptr : h->mask_dev;
  h->p.mask32 = h->fresh ? nullptr : h->mask32_dev;
  const GridDesc& g = h->d.g;
  for (int i = 0; i < h->d.q; ++i) {
    const int j = lattice_inv(h->d.q, i);
    const long long ct = lattice_c(h->d.q, i, 0) * g.plane + lattice_c(h->d.q, i, 1) * (long long)g.pitch +
                         lattice_c(h->d.q, i, 2);
    h->p.slot[0][i] = (unsigned)(i * g.dstride - ct);
    h->p.slot[1][i] = (unsigned)(i * g.dstride);
    h->p.slot[2][i] = (unsigned)(j * g.dstride + ct);
    h->p.slot[3][i] = (unsigned)(j * g.dstride);
  }
}

bool mlp_due(const aslb_lbgk* h) {
  return h->closure == CL_MLP && (h->mlp_last < 0 || h->steps - h->mlp_last >= h->mlp_period);
}

// Steps of one replayed time-loop graph: two (the AA parities), or a whole
// refresh period of the learned closure (even, so it starts on one parity).
int graph_cycle(const aslb_lbgk* h) {
  if (h->closure != CL_MLP) return 2;
  return h->mlp_period % 2 == 0 ? h->mlp_period : 2 * h->mlp_period;
}

int do_step(aslb_lbgk* h) {
  prepare_params(h);
  if (mlp_due(h)) {
    cudaError_t e = launch_closure_field(h->d, h->p, h->mlp_dev, h->cs2_field, h->parity, h->stream);
    if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("closure-field launch: ") + cudaGetErrorString(e));
    h->mlp_last = h->steps;
  }
  cudaError_t e = launch_step(h->d, h->p, h->closure, h->parity, h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("stream-collide launch: ") + cudaGetErrorString(e));
  h->parity ^= 1;
  h->steps += 1;
  if (h->macro_once) {
    h->macro_once = false;
    h->version++;
  }
  return ASLB_OK;
}

int do_bc(aslb_bc* bc) {
  aslb_lbgk* h = bc->h;
  if (bc->field()) {
    cudaError_t e = launch_field_bc(h->d, bc->anchors, bc->n, bc->fweights, bc->bp, h->stream);
    if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("field condition launch: ") + cudaGetErrorString(e));
    return ASLB_OK;
  }
  if (bc->fused) {
    // The condition takes effect inside the next steps (bounce-back reads).
    if (h->fresh) {
      h->fresh = false;
      h->version++;
    }
    return ASLB_OK;
  }
  cudaError_t e = cudaSuccess;
  if (bc->nd) e = launch_bc_links(h->d, bc->dlinks, bc->nd, bc->ls, bc->bp, h->parity, h->stream);
  if (e == cudaSuccess && bc->n) e = launch_bc(h->d, bc->anchors, bc->n, bc->bp, h->parity, h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("boundary launch: ") + cudaGetErrorString(e));
  return ASLB_OK;
}

void drop_graph(aslb_lbgk* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  h->graph_bcs.clear();
  h->graph_parity = -1;
}

template <class T>
int upload(T** dptr, const std::vector<T>& v) {
  *dptr = nullptr;
  if (v.empty()) return ASLB_OK;
  ASLB_CUDA(cudaMalloc((void**)dptr, v.size() * sizeof(T)));
  ASLB_CUDA(cudaMemcpy(*dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return ASLB_OK;
}

bool periodic_axis(const aslb_lbgk* h, int a) { return (h->d.g.periodic >> a) & 1; }

int wrapc(const aslb_lbgk* h, int v, int a) {
  const int n = a == 0 ? h->d.g.nx : (a == 1 ? h->d.g.ny : h->d.g.nz);
  return wrap_axis(v, n, periodic_axis(h, a));
}

bool on_periodic_ghost(const aslb_lbgk* h, int x, int y, int z) {
  const GridDesc& g = h->d.g;
  return (periodic_axis(h, 0) && (x < 1 || x > g.nx)) || (periodic_axis(h, 1) && (y < 1 || y > g.ny)) ||
         (periodic_axis(h, 2) && (z < 1 || z > g.nz));
}

bool interior(const GridDesc& g, int x, int y, int z) {
  return x >= 1 && x <= g.nx && y >= 1 && y <= g.ny && z >= 1 && z <= g.nz;
}

float map_at(const GridDesc& g, const float* map, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= g.gx || y >= g.gy || z >= g.gz) return -0.9f;  // generateDCFullSafe(map, -.9)
  return map[aidx(g, x, y, z)];
}


// Split candidate links (anchor a, direction k) into the direction-sorted form
// (fluid end at anchor + storage offset of c_k) and the anchor form (links
// that wrap across a periodic face, and every link of a velocity map, which
// needs all links of its anchor together).
struct Cand {
  int x, y, z, k;
};

int finalize_links(aslb_lbgk* h, aslb_bc* bc, const std::vector<Cand>& cand, bool anchor_form_only) {
  const GridDesc& g = h->d.g;
  const int q = h->d.q;
  std::vector<std::vector<int>> per_dir(q);
  std::vector<std::pair<long long, int>> rest;  // (ghosted linear index, k)
  for (const Cand& c : cand) {
    const long long wa = sidx(g, wrapc(h, c.x, 0), wrapc(h, c.y, 1), wrapc(h, c.z, 2));
    const long long wq = sidx(g, wrapc(h, c.x + lattice_c(q, c.k, 0), 0), wrapc(h, c.y + lattice_c(q, c.k, 1), 1),
                              wrapc(h, c.z + lattice_c(q, c.k, 2), 2));
    const long long off = lattice_c(q, c.k, 0) * g.plane + lattice_c(q, c.k, 1) * (long long)g.pitch + lattice_c(q, c.k, 2);
    if (!anchor_form_only && wq == wa + off)
      per_dir[c.k].push_back((int)wa);
    else
      rest.emplace_back(aidx(g, c.x, c.y, c.z), c.k);
  }
  std::vector<int> flat;
  bc->ls.seg[0] = 0;
  bc->ls.seg[1] = 0;
  for (int k = 1; k < 27; ++k) {
    if (k < q) {
      auto& v = per_dir[k];
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      flat.insert(flat.end(), v.begin(), v.end());
    }
    bc->ls.seg[k + 1] = (int)flat.size();
  }
  for (int k = 0; k < 27; ++k) {
    bc->ls.off[k] = k < q ? int(lattice_c(q, k, 0) * g.plane + lattice_c(q, k, 1) * (long long)g.pitch +
                                lattice_c(q, k, 2))
                          : 0;
    bc->ls.inv[k] = k < q ? lattice_inv(q, k) : 0;
  }
  std::sort(rest.begin(), rest.end());
  std::vector<int4> anchors;
  for (size_t i = 0; i < rest.size();) {
    const long long a = rest[i].first;
    unsigned mask = 0;
    while (i < rest.size() && rest[i].first == a) mask |= 1u << rest[i++].second;
    const int z = int(a % g.gz);
    const int y = int((a / g.gz) % g.gy);
    const int x = int(a / ((long long)g.gz * g.gy));
    anchors.push_back(make_int4(x, y, z, (int)mask));
  }
  bc->nd = (int)flat.size();
  bc->n = (int)anchors.size();
  bc->links = (long long)flat.size();
  for (auto& a : anchors) bc->links += __builtin_popcount((unsigned)a.w);
  int r = upload(&bc->dlinks, flat);
  if (!r) r = upload(&bc->anchors, anchors);
  bc->host_links.swap(flat);
  bc->host_anchors.swap(anchors);
  return r;
}

// Per-direction constants of a condition, evaluated in the arithmetic of the
// storage (float for FP32/FP16, double for FP64) like the per-link kernels.
void fill_link_values(aslb_lbgk* h, aslb_bc* bc) {
  const int q = h->d.q;
  const BcParams& bp = bc->bp;
  for (int k = 0; k < 27; ++k) {
    if (k >= q) {
      bc->ls.val[k] = 0.f;
      bc->ls.vald[k] = 0.0;
      continue;
    }
    const int c0 = lattice_c(q, k, 0), c1 = lattice_c(q, k, 1), c2 = lattice_c(q, k, 2);
    {
      const float u0 = (float)bp.u[0], u1 = (float)bp.u[1], u2 = (float)bp.u[2], P = (float)bp.p;
      const float cu = u0 * (float)c0 + u1 * (float)c1 + u2 * (float)c2;
      const float vv = u0 * u0 + u1 * u1 + u2 * u2;
      float v = 0.f;
      switch (bp.kind) {
        case BCK_VELOCITY: v = 6.0f * cu; break;
        case BCK_PRESSURE: v = P; break;
        case BCK_PRESSURE_VELOCITY: v = P + 3.0f * cu; break;
        case BCK_MAP_PRESSURE_VELOCITY:
          v = bp.compressible ? P + 3.0f * P * cu + 4.5f * P * cu * cu - 1.5f * P * vv
                              : P + 3.0f * cu + 4.5f * cu * cu - 1.5f * vv;
          break;
        default: break;
      }
      bc->ls.val[k] = v;
    }
    {
      const double u0 = bp.u[0], u1 = bp.u[1], u2 = bp.u[2], P = bp.p;
      const double cu = u0 * c0 + u1 * c1 + u2 * c2;
      const double vv = u0 * u0 + u1 * u1 + u2 * u2;
      double v = 0.0;
      switch (bp.kind) {
        case BCK_VELOCITY: v = 6.0 * cu; break;
        case BCK_PRESSURE: v = P; break;
        case BCK_PRESSURE_VELOCITY: v = P + 3.0 * cu; break;
        case BCK_MAP_PRESSURE_VELOCITY:
          v = bp.compressible ? P + 3.0 * P * cu + 4.5 * P * cu * cu - 1.5 * P * vv
                              : P + 3.0 * cu + 4.5 * cu * cu - 1.5 * vv;
          break;
        default: break;
      }
      bc->ls.vald[k] = v;
    }
  }
}

}  // namespace

extern "C" {

const char* aslb_last_error(void) { return g_err.c_str(); }
const char* aslb_version(void) { return "aslb 0.1 (sm_100a)"; }

int aslb_set_device(int device) {
  int n = 0;
  ASLB_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(ASLB_ERR_ARG, "aslb_set_device: no such device");
  g_device = device;
  ASLB_CUDA(cudaSetDevice(device));
  return ASLB_OK;
}

int aslb_synchronize(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(ASLB_ERR_CUDA, "aslb_synchronize: no CUDA device");
  }
  ASLB_CUDA(cudaSetDevice(g_device));
  ASLB_CUDA(cudaDeviceSynchronize());
  return ASLB_OK;
}

int aslb_lbgk_create(int nx, int ny, int nz, int q, int storage, double nu, unsigned flags, aslb_lbgk** out) {
  if (!out) return fail(ASLB_ERR_ARG, "aslb_lbgk_create: out is null");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1) return fail(ASLB_ERR_ARG, "aslb_lbgk_create: sizes must be >= 1");
  if (q != 15 && q != 19 && q != 27) return fail(ASLB_ERR_ARG, "aslb_lbgk_create: q must be 15, 19 or 27");
  if (storage != ASLB_F32 && storage != ASLB_F16 && storage != ASLB_F64)
    return fail(ASLB_ERR_ARG, "aslb_lbgk_create: unknown storage");
  if (!(nu > 0.0)) return fail(ASLB_ERR_ARG, "aslb_lbgk_create: viscosity must be positive");
  ASLB_CUDA(cudaSetDevice(g_device));
  auto* h = new aslb_lbgk();
  h->device = g_device;
  h->flags = flags;
  GridDesc& g = h->d.g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.gx = nx + 2; g.gy = ny + 2; g.gz = nz + 2;
  // Rows aligned to 128 bytes: the first interior cell (z = 1) of every row at
  // a multiple of `align` elements; or, with ASLB_PACKED_ROWS, rows back to
  // back (each direction array still starts on a 128-byte boundary).
  const int align = int(128 / storage_bytes(storage));
  if (flags & ASLB_PACKED_ROWS) {
    g.zoff = 0;
    g.pitch = g.gz;
  } else {
    g.zoff = align - 1;
    g.pitch = ((g.gz + g.zoff + align - 1) / align) * align;
  }
  g.periodic = int((flags >> 3) & 7u);
  g.plane = (long long)g.gy * g.pitch;
  g.dstride = (((long long)g.gx * g.plane + align - 1) / align) * align;
  g.L = (long long)g.gx * g.gy * g.gz;
  if ((long long)q * g.dstride >= (1ll << 32) || g.plane >= (1ll << 30)) {
    delete h;
    return fail(ASLB_ERR_ARG, "aslb_lbgk_create: domain too large for 32-bit element indexing on one GPU");
  }
  h->d.q = q;
  h->d.storage = storage;
  h->comp_vel = !(flags & ASLB_NO_VELOCITY);
  h->comp_rho = !(flags & ASLB_NO_RHO);
  h->p.nu = nu;
  h->p.compressible = (flags & ASLB_INCOMPRESSIBLE) ? 0 : 1;
  h->p.scale = 1024.0f;
  h->p.inv_scale = 1.0f / 1024.0f;
  h->p.cs = 0.17;
  // slack after the last direction: staged copies of a row segment may read a
  // little past the end of the final row
  const size_t fbytes = ((size_t)q * g.dstride + 4096) * storage_bytes(storage);
  const size_t mb = macro_bytes(storage);
  cudaError_t e = cudaMalloc(&h->d.F, fbytes);
  if (e == cudaSuccess) e = cudaMalloc(&h->d.rho, (size_t)g.L * mb);
  if (e == cudaSuccess) e = cudaMalloc(&h->d.u, 3 * (size_t)g.L * mb);
  h->u_own = h->d.u;
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->red_out, 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->d.err, sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h->host_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h->host_out, 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    std::string msg = std::string("aslb_lbgk_create: ") + cudaGetErrorString(e);
    aslb_lbgk_destroy(h);
    return fail(e == cudaErrorMemoryAllocation ? ASLB_ERR_NOMEM : ASLB_ERR_CUDA, msg);
  }
  h->stream = h->own_stream;
  h->d.variant = 0;  // direct-load stream-collide by default (measured faster)
  e = cudaMemsetAsync(h->d.F, 0, fbytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d.err, 0, sizeof(int), h->stream);
  if (e == cudaSuccess) {
    const double u0[3] = {0, 0, 0};
    e = launch_init_f(h->d, h->p, 1.0, u0, nullptr, nullptr, h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    std::string msg = std::string("aslb_lbgk_create: ") + cudaGetErrorString(e);
    aslb_lbgk_destroy(h);
    return fail(ASLB_ERR_CUDA, msg);
  }
  *out = h;
  return ASLB_OK;
}

void batch_detach(aslb_batch* b, aslb_lbgk* h);

int aslb_lbgk_destroy(aslb_lbgk* h) {
  if (!h) return ASLB_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graph(h);
  for (aslb_batch* b : std::vector<aslb_batch*>(h->batches)) batch_detach(b, h);
  for (aslb_fd* f : h->fds) fd_detached(f);
  h->fds.clear();
  for (aslb_bc* bc : h->bcs) {
    cudaFree(bc->anchors);
    cudaFree(bc->dlinks);
    bc->anchors = nullptr;
    bc->dlinks = nullptr;
    bc->h = nullptr;
  }
  for (aslb_force* fc : h->forces) {
    cudaFree(fc->cells);
    cudaFree(fc->mask_in);
    cudaFree(fc->field);
    cudaFree(fc->partials);
    cudaFree(fc->out);
    if (fc->host_out) cudaFreeHost(fc->host_out);
    fc->cells = nullptr;
    fc->mask_in = nullptr;
    fc->field = nullptr;
    fc->partials = nullptr;
    fc->out = nullptr;
    fc->host_out = nullptr;
    fc->h = nullptr;
  }
  cudaFree(h->d.F);
  cudaFree(h->d.rho);
  cudaFree(h->u_own);
  cudaFree(h->mlp_dev);
  cudaFree(h->cs2_field);
  cudaFree(h->mask_dev);
  cudaFree(h->mask32_dev);
  cudaFree(h->red_partials);
  cudaFree(h->stage);
  cudaFree(h->red_out);
  cudaFree(h->d.err);
  if (h->host_out) cudaFreeHost(h->host_out);
  if (h->host_err) cudaFreeHost(h->host_err);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return ASLB_OK;
}

void* aslb_lbgk_stream(aslb_lbgk* h) { return h ? (void*)h->stream : nullptr; }

int aslb_lbgk_set_stream(aslb_lbgk* h, void* stream) {
  ASLB_CHECK_HANDLE(h);
  ASLB_CUDA(cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  drop_graph(h);
  return ASLB_OK;
}

int aslb_lbgk_set_viscosity(aslb_lbgk* h, double nu) {
  ASLB_CHECK_HANDLE(h);
  if (!(nu > 0.0)) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_viscosity: viscosity must be positive");
  h->p.nu = nu;
  h->version++;
  return ASLB_OK;
}

double aslb_lbgk_get_viscosity(aslb_lbgk* h) { return h ? h->p.nu : 0.0; }

int aslb_lbgk_set_compressible(aslb_lbgk* h, int compressible) {
  ASLB_CHECK_HANDLE(h);
  h->p.compressible = compressible ? 1 : 0;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_set_omega(aslb_lbgk* h, const double omega[3]) {
  ASLB_CHECK_HANDLE(h);
  if (!omega) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_omega: null vector");
  for (int d = 0; d < 3; ++d) h->p.Om[d] = omega[d];
  h->p.has_coriolis = 1;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_set_macro_output(aslb_lbgk* h, int comp_vel, int comp_rho) {
  ASLB_CHECK_HANDLE(h);
  h->comp_vel = comp_vel != 0;
  h->comp_rho = comp_rho != 0;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_request_macro(aslb_lbgk* h) {
  ASLB_CHECK_HANDLE(h);
  h->macro_once = true;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_set_body_force(aslb_lbgk* h, const double g[3]) {
  ASLB_CHECK_HANDLE(h);
  if (!g) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_body_force: null vector");
  for (int d = 0; d < 3; ++d) h->p.g[d] = g[d];
  h->p.has_force = (g[0] != 0.0 || g[1] != 0.0 || g[2] != 0.0) ? 1 : 0;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_set_closure(aslb_lbgk* h, int closure, double cs) {
  ASLB_CHECK_HANDLE(h);
  if (closure < CL_NONE || closure > CL_MLP) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_closure: unknown closure");
  if (closure == CL_MLP && !h->mlp_dev)
    return fail(ASLB_ERR_STATE, "aslb_lbgk_set_closure: load a network with aslb_lbgk_set_mlp first");
  if (closure == CL_MLP && (h->d.q == 15 || h->d.storage == ST_F64))
    return fail(ASLB_ERR_ARG, "aslb_lbgk_set_closure: the learned closure runs on D3Q19 / D3Q27 with FP32 or FP16 storage");
  if (closure == CL_MLP && !h->cs2_field) {
    const size_t n = (size_t)h->d.g.dstride + 4096;
    ASLB_CUDA(cudaMalloc((void**)&h->cs2_field, n * sizeof(float)));
    ASLB_CUDA(cudaMemset(h->cs2_field, 0, n * sizeof(float)));
  }
  h->mlp_last = -1;
  h->closure = closure;
  h->p.cs = cs;
  h->version++;
  return ASLB_OK;
}

size_t aslb_mlp_layout_bytes(void) { return sizeof(MlpNet); }

int aslb_lbgk_set_mlp(aslb_lbgk* h, const void* net_host, size_t bytes) {
  ASLB_CHECK_HANDLE(h);
  if (!net_host || bytes != sizeof(MlpNet))
    return fail(ASLB_ERR_ARG, "aslb_lbgk_set_mlp: expected " + std::to_string(sizeof(MlpNet)) + " bytes");
  if (!h->mlp_dev) ASLB_CUDA(cudaMalloc(&h->mlp_dev, sizeof(MlpNet)));
  ASLB_CUDA(cudaMemcpyAsync(h->mlp_dev, net_host, sizeof(MlpNet), cudaMemcpyHostToDevice, h->stream));
  ASLB_CUDA(cudaStreamSynchronize(h->stream));
  h->mlp_last = -1;  // new weights: recompute the field before the next step
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_set_mlp_period(aslb_lbgk* h, int steps) {
  ASLB_CHECK_HANDLE(h);
  if (steps < 1) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_mlp_period: period must be >= 1");
  h->mlp_period = steps;
  h->mlp_last = -1;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_closure_features(aslb_lbgk* h, float* out_dev) {
  ASLB_CHECK_HANDLE(h);
  if (!out_dev) return fail(ASLB_ERR_ARG, "aslb_lbgk_closure_features: null output");
  prepare_params(h);
  cudaError_t e = launch_closure_features(h->d, h->p, out_dev, h->parity, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_closure_features: ") + cudaGetErrorString(e));
  return ASLB_OK;
}

int aslb_lbgk_set_fp16_scale(aslb_lbgk* h, double scale) {
  ASLB_CHECK_HANDLE(h);
  if (!(scale > 0.0)) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_fp16_scale: scale must be positive");
  if (h->d.storage == ASLB_F16 && h->steps > 0)
    return fail(ASLB_ERR_STATE, "aslb_lbgk_set_fp16_scale: set the scale before the first step");
  h->p.scale = (float)scale;
  h->p.inv_scale = (float)(1.0 / scale);
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_set_position(aslb_lbgk* h, const double pos0[3], double dx) {
  ASLB_CHECK_HANDLE(h);
  if (!pos0 || !(dx > 0)) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_position: bad arguments");
  for (int d = 0; d < 3; ++d) h->pos0[d] = pos0[d];
  h->dx = dx;
  return ASLB_OK;
}

int aslb_lbgk_shape(aslb_lbgk* h, int out[6]) {
  ASLB_CHECK_HANDLE(h);
  out[0] = h->d.g.nx; out[1] = h->d.g.ny; out[2] = h->d.g.nz;
  out[3] = h->d.q; out[4] = h->d.storage; out[5] = (int)h->flags;
  return ASLB_OK;
}

int aslb_lbgk_init_f(aslb_lbgk* h, double rho, const double u[3]) {
  ASLB_CHECK_HANDLE(h);
  const double z[3] = {0, 0, 0};
  cudaError_t e = launch_init_f(h->d, h->p, rho, u ? u : z, nullptr, nullptr, h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_init_f: ") + cudaGetErrorString(e));
  h->parity = 0;
  h->fresh = true;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_init_f_fields(aslb_lbgk* h, const double* rho, const double* u) {
  ASLB_CHECK_HANDLE(h);
  if (!u) return fail(ASLB_ERR_ARG, "aslb_lbgk_init_f_fields: velocity field required");
  const size_t L = (size_t)h->d.g.L;
  double *drho = nullptr, *du = nullptr;
  // every path below frees both buffers: errors are collected, not returned early
  cudaError_t e = cudaMalloc(&du, 3 * L * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(du, u, 3 * L * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && rho) e = cudaMalloc(&drho, L * sizeof(double));
  if (e == cudaSuccess && rho) e = cudaMemcpyAsync(drho, rho, L * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  const double z[3] = {0, 0, 0};
  if (e == cudaSuccess) e = launch_init_f(h->d, h->p, 1.0, z, drho, du, h->stream);
  cudaError_t e2 = cudaStreamSynchronize(h->stream);
  cudaFree(du);
  cudaFree(drho);
  if (e != cudaSuccess || e2 != cudaSuccess)
    return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_init_f_fields: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  h->parity = 0;
  h->fresh = true;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_bind_velocity(aslb_lbgk* h, void* u_dev) {
  ASLB_CHECK_HANDLE(h);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_bind_velocity: ") + cudaGetErrorString(e));
  h->d.u = u_dev ? u_dev : h->u_own;
  h->version++;  // recorded graphs hold the old pointer
  return ASLB_OK;
}

int aslb_lbgk_compute_macro(aslb_lbgk* h, int comp_rho, int comp_vel) {
  ASLB_CHECK_HANDLE(h);
  prepare_params(h);
  cudaError_t e = launch_compute_macro(h->d, h->p, h->parity, comp_rho ? 1 : 0, comp_vel ? 1 : 0, h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_compute_macro: ") + cudaGetErrorString(e));
  return ASLB_OK;
}

int aslb_lbgk_step(aslb_lbgk* h, int nsteps) {
  NvtxRange range("aslb_lbgk_step");
  ASLB_CHECK_HANDLE(h);
  if (nsteps < 0) return fail(ASLB_ERR_ARG, "aslb_lbgk_step: negative step count");
  for (int i = 0; i < nsteps; ++i) {
    int r = do_step(h);
    if (r) return r;
  }
  return ASLB_OK;
}

int aslb_lbgk_step_planes(aslb_lbgk* h, int x_first, int x_last, void* stream) {
  ASLB_CHECK_HANDLE(h);
  const GridDesc& g = h->d.g;
  if (x_first < 1 || x_last > g.nx || x_first > x_last)
    return fail(ASLB_ERR_ARG, "aslb_lbgk_step_planes: planes outside 1 .. nx");
  if (g.periodic & 1) return fail(ASLB_ERR_ARG, "aslb_lbgk_step_planes: the domain is periodic in x");
  if (h->closure == CL_MLP) return fail(ASLB_ERR_ARG, "aslb_lbgk_step_planes: not with the learned closure");
  prepare_params(h);
  // a view of planes x_first .. x_last as a domain of their own: every
  // per-cell array shifted by the planes before them (the slot offsets and
  // strides are relative, the component stride L of u stays the whole one)
  DomainDev v = h->d;
  StepParams q = h->p;
  const long long sh = (long long)(x_first - 1) * g.plane;
  const long long ash = (long long)(x_first - 1) * g.gy * g.gz;
  v.g.nx = x_last - x_first + 1;
  v.g.gx = v.g.nx + 2;
  v.F = (char*)h->d.F + sh * (long long)storage_bytes(h->d.storage);
  v.rho = (char*)h->d.rho + ash * (long long)macro_bytes(h->d.storage);
  v.u = (char*)h->d.u + ash * (long long)macro_bytes(h->d.storage);
  if (v.variant == 1) v.variant = 0;
  if (q.mask) q.mask += sh;
  if (q.mask32) q.mask32 += sh;
  if (q.cs2) q.cs2 += sh;
  cudaError_t e = launch_step(v, q, h->closure, h->parity, stream ? (cudaStream_t)stream : h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_step_planes: ") + cudaGetErrorString(e));
  return ASLB_OK;
}

int aslb_lbgk_step_commit(aslb_lbgk* h) {
  ASLB_CHECK_HANDLE(h);
  h->parity ^= 1;
  h->steps += 1;
  if (h->macro_once) {
    h->macro_once = false;
    h->version++;
  }
  return ASLB_OK;
}

int aslb_lbgk_run(aslb_lbgk* h, int nsteps, aslb_bc* const* bcs, int nbc, int use_graph) {
  NvtxRange range("aslb_lbgk_run");
  ASLB_CHECK_HANDLE(h);
  if (nsteps < 0 || nbc < 0 || (nbc > 0 && !bcs)) return fail(ASLB_ERR_ARG, "aslb_lbgk_run: bad arguments");
  for (int b = 0; b < nbc; ++b)
    if (!bcs[b] || bcs[b]->h != h) return fail(ASLB_ERR_ARG, "aslb_lbgk_run: boundary of another domain");
  // A fused condition takes effect inside the next step, after every separate
  // condition of this step: it must be the last writer of its links.
  for (int b = 1; b < nbc; ++b)
    if (bcs[b - 1]->fused && !bcs[b]->fused && !bcs[b]->field())
      return fail(ASLB_ERR_ARG, "aslb_lbgk_run: fused conditions must come after all separate ones");
  auto eager = [&](int n) -> int {
    for (int i = 0; i < n; ++i) {
      int r = do_step(h);
      if (r) return r;
      for (int b = 0; b < nbc; ++b) {
        r = do_bc(bcs[b]);
        if (r) return r;
      }
    }
    return ASLB_OK;
  };
  const int cycle = graph_cycle(h);
  if (!use_graph || h->stream == nullptr || nsteps < cycle) return eager(nsteps);
  int done = 0;
  if (h->macro_once || h->fresh) {
    int r = eager(1);
    if (r) return r;
    done = 1;
  }
  // the learned closure's graph starts where a field refresh is due
  if (h->closure == CL_MLP)
    while (done < nsteps && !mlp_due(h)) {
      int r = eager(1);
      if (r) return r;
      done += 1;
    }
  if (nsteps - done < cycle) return eager(nsteps - done);
  std::vector<aslb_bc*> key(bcs, bcs + nbc);
  const bool valid = h->graph && h->graph_version == h->version && h->graph_bcs == key;
  if (valid && h->graph_parity != h->parity && h->closure != CL_MLP && done < nsteps) {
    int r = eager(1);
    if (r) return r;
    done += 1;
  }
  if (!(h->graph && h->graph_version == h->version && h->graph_bcs == key && h->graph_parity == h->parity)) {
    drop_graph(h);
    const int start_parity = h->parity;
    const long long start_steps = h->steps;
    const long long start_mlp = h->mlp_last;
    cudaGraph_t graph = nullptr;
    ASLB_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int r = eager(cycle);
    cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
    h->parity = start_parity;  // capture enqueued nothing
    h->steps = start_steps;
    h->mlp_last = start_mlp;
    if (r) {
      if (graph) cudaGraphDestroy(graph);
      return r;
    }
    if (ce != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&h->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      h->graph = nullptr;
      return fail(ASLB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    }
    h->graph_bcs = key;
    h->graph_parity = start_parity;
    h->graph_version = h->version;
  }
  const int reps = (nsteps - done) / cycle;
  for (int i = 0; i < reps; ++i) ASLB_CUDA(cudaGraphLaunch(h->graph, h->stream));
  h->steps += (long long)cycle * reps;
  if (h->closure == CL_MLP && reps > 0) h->mlp_last = h->steps - cycle + (cycle - h->mlp_period);
  done += cycle * reps;
  return eager(nsteps - done);
}

int aslb_lbgk_sync(aslb_lbgk* h) {
  ASLB_CHECK_HANDLE(h);
  ASLB_CUDA(cudaMemcpyAsync(h->host_err, h->d.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  ASLB_CUDA(cudaStreamSynchronize(h->stream));
  if (*h->host_err)
    return fail(ASLB_ERR_STATE, "aslb_lbgk_sync: a bounded device wait gave up (asynchronous copy never completed)");
  return ASLB_OK;
}

int aslb_lbgk_set_kernel(aslb_lbgk* h, int variant) {
  ASLB_CHECK_HANDLE(h);
  if (variant < 0 || variant > 2) return fail(ASLB_ERR_ARG, "aslb_lbgk_set_kernel: variant must be 0, 1 or 2");
  if (variant == 1 && (h->flags & ASLB_PACKED_ROWS))
    return fail(ASLB_ERR_ARG, "aslb_lbgk_set_kernel: the TMA-staged kernel needs aligned rows (no ASLB_PACKED_ROWS)");
  h->d.variant = variant;
  h->version++;
  return ASLB_OK;
}

int aslb_lbgk_get_kernel(aslb_lbgk* h) { return h ? h->d.variant : -1; }

long long aslb_lbgk_steps(aslb_lbgk* h) { return h ? h->steps : -1; }

namespace {
// Staging buffer of one direction (L values of the macro type) for the
// population and Cs^2 transfers: allocated at the first such transfer, kept
// with the domain, so later reads and writes allocate nothing.
int stage_buffer(aslb_lbgk* h, void** out) {
  const size_t need = (size_t)h->d.g.L * macro_bytes(h->d.storage);
  if (!h->stage) ASLB_CUDA(cudaMalloc(&h->stage, need));
  *out = h->stage;
  return ASLB_OK;
}

// Device -> host copy of `count` values of `mb` bytes into host_out (dtype
// F32 / F64) at element offset `at`: straight into the caller's buffer when
// the types agree (a pinned buffer then transfers at full speed), else through
// a host copy and a conversion. Enqueued on the domain's stream; converting
// copies synchronise it.
cudaError_t copy_out(aslb_lbgk* h, const void* dev, size_t count, size_t mb, int dtype, void* host_out, size_t at,
                     std::vector<char>& tmp) {
  const bool direct = (mb == 4) == (dtype == ASLB_F32);
  if (direct) return cudaMemcpyAsync((char*)host_out + at * mb, dev, count * mb, cudaMemcpyDeviceToHost, h->stream);
  tmp.resize(count * mb);
  cudaError_t e = cudaMemcpyAsync(tmp.data(), dev, count * mb, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return e;
  if (mb == 4) {
    const float* src = (const float*)tmp.data();
    for (size_t i = 0; i < count; ++i) ((double*)host_out)[at + i] = src[i];
  } else {
    const double* src = (const double*)tmp.data();
    for (size_t i = 0; i < count; ++i) ((float*)host_out)[at + i] = (float)src[i];
  }
  return cudaSuccess;
}
}  // namespace

int aslb_lbgk_read(aslb_lbgk* h, int field, int dtype, void* host_out) {
  ASLB_CHECK_HANDLE(h);
  if (!host_out) return fail(ASLB_ERR_ARG, "aslb_lbgk_read: null output");
  if (dtype != ASLB_F32 && dtype != ASLB_F64) return fail(ASLB_ERR_ARG, "aslb_lbgk_read: dtype must be F32 or F64");
  if (field != ASLB_FIELD_CS2 && field != ASLB_FIELD_RHO && field != ASLB_FIELD_VELOCITY && field != ASLB_FIELD_F)
    return fail(ASLB_ERR_ARG, "aslb_lbgk_read: unknown field");
  const size_t L = (size_t)h->d.g.L;
  const size_t mb = field == ASLB_FIELD_CS2 ? sizeof(float) : macro_bytes(h->d.storage);
  std::vector<char> tmp;
  cudaError_t e = cudaSuccess;
  if (field == ASLB_FIELD_CS2) {
    if (h->closure != CL_MLP || !h->cs2_field)
      return fail(ASLB_ERR_STATE, "aslb_lbgk_read: the Cs^2 field exists with the learned closure only");
    void* stage = nullptr;
    if (int rc = stage_buffer(h, &stage)) return rc;
    if (mlp_due(h)) {  // the field the next step will use
      prepare_params(h);
      e = launch_closure_field(h->d, h->p, h->mlp_dev, h->cs2_field, h->parity, h->stream);
      if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_read: ") + cudaGetErrorString(e));
      h->mlp_last = h->steps;
    }
    e = launch_gather_cells(h->d.g, h->cs2_field, (float*)stage, h->stream);
    if (e == cudaSuccess) e = copy_out(h, stage, L, mb, dtype, host_out, 0, tmp);
  } else if (field == ASLB_FIELD_RHO) {
    e = copy_out(h, h->d.rho, L, mb, dtype, host_out, 0, tmp);
  } else if (field == ASLB_FIELD_VELOCITY) {
    e = copy_out(h, h->d.u, 3 * L, mb, dtype, host_out, 0, tmp);
  } else {
    // one direction at a time through the staging buffer (stream order keeps
    // each export behind the previous copy out of the same buffer)
    void* stage = nullptr;
    if (int rc = stage_buffer(h, &stage)) return rc;
    prepare_params(h);
    for (int i = 0; i < h->d.q && e == cudaSuccess; ++i) {
      e = launch_export_f(h->d, h->p, h->parity, i, i + 1, stage, h->stream);
      if (e == cudaSuccess) e = copy_out(h, stage, L, mb, dtype, host_out, (size_t)i * L, tmp);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_read: ") + cudaGetErrorString(e));
  return ASLB_OK;
}

int aslb_lbgk_write(aslb_lbgk* h, int field, int dtype, const void* host_in) {
  ASLB_CHECK_HANDLE(h);
  if (field != ASLB_FIELD_F || !host_in) return fail(ASLB_ERR_ARG, "aslb_lbgk_write: only the F field is writable");
  if (dtype != ASLB_F32 && dtype != ASLB_F64) return fail(ASLB_ERR_ARG, "aslb_lbgk_write: dtype must be F32 or F64");
  const size_t L = (size_t)h->d.g.L;
  const size_t mb = macro_bytes(h->d.storage);
  const bool direct = (mb == 4) == (dtype == ASLB_F32);
  void* stage = nullptr;
  if (int rc = stage_buffer(h, &stage)) return rc;
  std::vector<char> tmp(direct ? 0 : L * mb);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < h->d.q && e == cudaSuccess; ++i) {
    const void* src;
    if (direct) {
      src = (const char*)host_in + (size_t)i * L * mb;
    } else {
      // the previous direction's copy reads tmp: wait for it before refilling
      e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess) break;
      if (mb == 4)
        for (size_t k = 0; k < L; ++k) ((float*)tmp.data())[k] = (float)((const double*)host_in)[(size_t)i * L + k];
      else
        for (size_t k = 0; k < L; ++k) ((double*)tmp.data())[k] = ((const float*)host_in)[(size_t)i * L + k];
      src = tmp.data();
    }
    e = cudaMemcpyAsync(stage, src, L * mb, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = launch_import_f(h->d, h->p, i, i + 1, stage, h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_write: ") + cudaGetErrorString(e));
  h->parity = 0;
  h->fresh = true;
  h->version++;
  return ASLB_OK;
}

// ---- restart dump: the population array as stored ---------------------------
size_t aslb_lbgk_state_bytes(aslb_lbgk* h) {
  return h ? (size_t)h->d.q * h->d.g.dstride * storage_bytes(h->d.storage) : 0;
}

int aslb_lbgk_save_state(aslb_lbgk* h, void* host_out, size_t bytes, long long meta[4]) {
  ASLB_CHECK_HANDLE(h);
  if (!host_out || !meta || bytes != aslb_lbgk_state_bytes(h))
    return fail(ASLB_ERR_ARG, "aslb_lbgk_save_state: the buffer must hold aslb_lbgk_state_bytes() bytes");
  cudaError_t e = cudaMemcpyAsync(host_out, h->d.F, bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_save_state: ") + cudaGetErrorString(e));
  meta[0] = h->steps;
  meta[1] = h->parity;
  meta[2] = h->fresh ? 0 : 1;
  meta[3] = h->d.storage;
  return ASLB_OK;
}

int aslb_lbgk_load_state(aslb_lbgk* h, const void* host_in, size_t bytes, const long long meta[4]) {
  ASLB_CHECK_HANDLE(h);
  if (!host_in || !meta || bytes != aslb_lbgk_state_bytes(h))
    return fail(ASLB_ERR_ARG, "aslb_lbgk_load_state: the dump is of another domain size or lattice");
  if (meta[3] != h->d.storage || (meta[1] != 0 && meta[1] != 1) || meta[0] < 0)
    return fail(ASLB_ERR_ARG, "aslb_lbgk_load_state: the dump is of another storage or is damaged");
  cudaError_t e = cudaMemcpyAsync(h->d.F, host_in, bytes, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_load_state: ") + cudaGetErrorString(e));
  h->steps = meta[0];
  h->parity = (int)meta[1];
  h->fresh = meta[2] == 0;
  h->mlp_last = -1;
  h->macro_once = true;
  h->version++;
  return ASLB_OK;
}

void* aslb_lbgk_device_field(aslb_lbgk* h, int field) {
  if (!h) return nullptr;
  if (field == ASLB_FIELD_RHO) return h->d.rho;
  if (field == ASLB_FIELD_VELOCITY) return h->d.u;
  return nullptr;
}

// ---- x-slab decomposition: face buffers ------------------------------------
//
// A domain split into x slabs, one per GPU, exchanges after every step the
// populations that cross its two x faces; each direction's x plane is one
// contiguous run of `plane` elements, so a face buffer is (directions whose
// c_x points across the face) x plane, copied with one DMA per direction.
// After an odd step (representation B) the populations this slab's boundary
// cells pushed into its ghost plane belong to the neighbour's boundary cells;
// after an even step (A) this slab's ghost plane must receive the neighbour's
// boundary-plane populations that the next odd step pulls across the face.
//   pack   parity 0: low face  -> plane 1,      dirs c_x = -1
//                    high face -> plane nx,     dirs c_x = +1
//          parity 1: low face  -> plane 0,      dirs c_x = +1
//                    high face -> plane nx + 1, dirs c_x = -1
//   unpack parity 0: low face  -> plane 0,      dirs c_x = +1
//                    high face -> plane nx + 1, dirs c_x = -1
//          parity 1: low face  -> plane 1,      dirs c_x = -1
//                    high face -> plane nx,     dirs c_x = +1
// What one slab packs on its high face is what its high neighbour unpacks on
// its low face at the same parity.
namespace {
int halo_copy(aslb_lbgk* h, int face, void* buf, bool pack) {
  const GridDesc& g = h->d.g;
  const int q = h->d.q;
  const bool p0 = h->parity == 0;
  int x, sign;
  if (pack) {
    x = face == 0 ? (p0 ? 1 : 0) : (p0 ? g.nx : g.nx + 1);
    sign = face == 0 ? (p0 ? -1 : +1) : (p0 ? +1 : -1);
  } else {
    x = face == 0 ? (p0 ? 0 : 1) : (p0 ? g.nx + 1 : g.nx);
    sign = face == 0 ? (p0 ? +1 : -1) : (p0 ? -1 : +1);
  }
  const size_t eb = storage_bytes(h->d.storage);
  const size_t pb = (size_t)g.plane * eb;
  char* F = (char*)h->d.F;
  char* b = (char*)buf;
  int k = 0;
  for (int i = 1; i < q; ++i) {
    if (lattice_c(q, i, 0) != sign) continue;
    char* slab = F + ((size_t)i * g.dstride + (size_t)x * g.plane) * eb;
    char* dst = pack ? b + k * pb : slab;
    const char* src = pack ? slab : b + k * pb;
    ASLB_CUDA(cudaMemcpyAsync(dst, src, pb, cudaMemcpyDeviceToDevice, h->stream));
    ++k;
  }
  return ASLB_OK;
}
}  // namespace

size_t aslb_lbgk_halo_bytes(aslb_lbgk* h) {
  if (!h) return 0;
  int k = 0;
  for (int i = 1; i < h->d.q; ++i) k += lattice_c(h->d.q, i, 0) == 1;
  return (size_t)k * (size_t)h->d.g.plane * storage_bytes(h->d.storage);
}

int aslb_lbgk_halo_pack(aslb_lbgk* h, int face, void* dev_out) {
  ASLB_CHECK_HANDLE(h);
  if ((face != 0 && face != 1) || !dev_out) return fail(ASLB_ERR_ARG, "aslb_lbgk_halo_pack: bad arguments");
  if (h->flags & ASLB_PERIODIC_X)
    return fail(ASLB_ERR_STATE, "aslb_lbgk_halo_pack: a slab's x faces are exchanged, not periodic");
  return halo_copy(h, face, dev_out, true);
}

int aslb_lbgk_halo_unpack(aslb_lbgk* h, int face, const void* dev_in) {
  ASLB_CHECK_HANDLE(h);
  if ((face != 0 && face != 1) || !dev_in) return fail(ASLB_ERR_ARG, "aslb_lbgk_halo_unpack: bad arguments");
  if (h->flags & ASLB_PERIODIC_X)
    return fail(ASLB_ERR_STATE, "aslb_lbgk_halo_unpack: a slab's x faces are exchanged, not periodic");
  return halo_copy(h, face, const_cast<void*>(dev_in), false);
}

int aslb_lbgk_parity(aslb_lbgk* h) { return h ? h->parity : -1; }

int aslb_lbgk_moments(aslb_lbgk* h, double out[4]) {
  ASLB_CHECK_HANDLE(h);
  if (!out) return fail(ASLB_ERR_ARG, "aslb_lbgk_moments: null output");
  const int nb = moments_blocks(h->d.g);
  if (!h->red_partials) ASLB_CUDA(cudaMalloc((void**)&h->red_partials, (size_t)nb * 4 * sizeof(double)));
  prepare_params(h);
  cudaError_t e = launch_moments(h->d, h->p, h->parity, h->red_partials, h->red_out, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->host_out, h->red_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_moments: ") + cudaGetErrorString(e));
  for (int i = 0; i < 4; ++i) out[i] = h->host_out[i];
  return ASLB_OK;
}

int aslb_lbgk_watchdog(aslb_lbgk* h, double out[3]) {
  ASLB_CHECK_HANDLE(h);
  if (!out) return fail(ASLB_ERR_ARG, "aslb_lbgk_watchdog: null output");
  const int nb = moments_blocks(h->d.g);
  if (!h->red_partials) ASLB_CUDA(cudaMalloc((void**)&h->red_partials, (size_t)nb * 4 * sizeof(double)));
  prepare_params(h);
  std::vector<double> rows((size_t)nb * 3);
  cudaError_t e = launch_watchdog(h->d, h->p, h->parity, h->red_partials, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(rows.data(), h->red_partials, rows.size() * sizeof(double), cudaMemcpyDeviceToHost,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_lbgk_watchdog: ") + cudaGetErrorString(e));
  double umax = 0.0, rmin = 1e300, bad = 0.0;
  for (int b = 0; b < nb; ++b) {
    umax = std::max(umax, rows[(size_t)b * 3]);
    rmin = std::min(rmin, rows[(size_t)b * 3 + 1]);
    bad += rows[(size_t)b * 3 + 2];
  }
  out[0] = std::sqrt(umax);
  out[1] = rmin;
  out[2] = bad;
  return ASLB_OK;
}

// ---- boundary conditions ---------------------------------------------------

int aslb_bc_slice_create(aslb_lbgk* h, int kind, unsigned wallmask, double p, const double u[3], aslb_bc** out) {
  ASLB_CHECK_HANDLE(h);
  if (!out) return fail(ASLB_ERR_ARG, "aslb_bc_slice_create: out is null");
  *out = nullptr;
  if (kind < ASLB_BC_NOSLIP || kind > ASLB_BC_PRESSURE_VELOCITY)
    return fail(ASLB_ERR_ARG, "aslb_bc_slice_create: unknown slice kind");
  if (wallmask == 0 || wallmask > 63u) return fail(ASLB_ERR_ARG, "aslb_bc_slice_create: bad wall mask");
  const GridDesc& g = h->d.g;
  const int q = h->d.q;
  // Walls X0, XE, Y0, YE, Z0, ZE with inward normals c_1, c_4, c_2, c_5, c_3, c_6;
  // every direction k with c_k . n > 0 and every point a of the first interior
  // layer (tangential coordinates 1 .. N'-2) gives the ghost point a - c_k
  // (src/num/aslBCond.cxx:373-493).
  static const int normal_dir[6] = {1, 4, 2, 5, 3, 6};
  const int G[3] = {g.gx, g.gy, g.gz};
  std::vector<Cand> cand;
  for (int w = 0; w < 6; ++w) {
    if (!(wallmask >> w & 1u)) continue;
    const int ax = w / 2;
    if (periodic_axis(h, ax)) return fail(ASLB_ERR_ARG, "aslb_bc_slice_create: wall on a periodic axis");
    const int layer = (w % 2 == 0) ? 1 : G[ax] - 2;
    const int nd = normal_dir[w];
    const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
    for (int k = 1; k < q; ++k) {
      int dot = 0;
      for (int d = 0; d < 3; ++d) dot += lattice_c(q, k, d) * lattice_c(q, nd, d);
      if (dot <= 0) continue;
      for (int i = 1; i < G[t1] - 1; ++i)
        for (int j = 1; j < G[t2] - 1; ++j) {
          int a[3];
          a[ax] = layer;
          a[t1] = i;
          a[t2] = j;
          cand.push_back({a[0] - lattice_c(q, k, 0), a[1] - lattice_c(q, k, 1), a[2] - lattice_c(q, k, 2), k});
        }
    }
  }
  auto* bc = new aslb_bc();
  bc->h = h;
  bc->bp.kind = kind;
  bc->bp.compressible = h->p.compressible;
  bc->bp.p = p;
  for (int d = 0; d < 3; ++d) bc->bp.u[d] = u ? u[d] : 0.0;
  bc->bp.scale = h->p.scale;
  bc->bp.inv_scale = h->p.inv_scale;
  fill_link_values(h, bc);
  int r = finalize_links(h, bc, cand, false);
  if (r) {
    aslb_bc_destroy(bc);
    return r;
  }
  h->bcs.push_back(bc);
  *out = bc;
  return ASLB_OK;
}

namespace {
// Cell x is processed iff -0.9999 < map(x) <= 0; link k iff map(x + c_k) > 0
// (src/num/aslLBGKBC.cxx:235-251), counted when x + c_k is an interior cell.
// With a computational-domain map cd, a neighbour also needs cd > 0 to be a
// computation node (src/num/aslBCond.cxx:204-211; cd reads -1 off the grid).
void map_candidates(const aslb_lbgk* h, const float* map, std::vector<Cand>& cand, const float* cd = nullptr) {
  const GridDesc& g = h->d.g;
  const int q = h->d.q;
  for (int x = 0; x < g.gx; ++x)
    for (int y = 0; y < g.gy; ++y)
      for (int z = 0; z < g.gz; ++z) {
        if (on_periodic_ghost(h, x, y, z)) continue;
        const float m0 = map[aidx(g, x, y, z)];
        if (!(m0 <= 0.f && m0 > -0.9999f)) continue;
        for (int k = 1; k < q; ++k) {
          const int qx = wrapc(h, x + lattice_c(q, k, 0), 0), qy = wrapc(h, y + lattice_c(q, k, 1), 1),
                    qz = wrapc(h, z + lattice_c(q, k, 2), 2);
          if (!interior(g, qx, qy, qz)) continue;
          if (map_at(g, map, qx, qy, qz) > 0.f && (!cd || cd[aidx(g, qx, qy, qz)] > 0.f)) cand.push_back({x, y, z, k});
        }
      }
}
}  // namespace

int aslb_lattice(int q, int* c, double* w, int* inv) {
  if ((q != 15 && q != 19 && q != 27) || !c || !w || !inv) return fail(ASLB_ERR_ARG, "aslb_lattice: bad arguments");
  for (int i = 0; i < q; ++i) {
    for (int d = 0; d < 3; ++d) c[3 * i + d] = lattice_c(q, i, d);
    w[i] = q == 15 ? Lattice<15>::w(i) : q == 19 ? Lattice<19>::w(i) : Lattice<27>::w(i);
    inv[i] = lattice_inv(q, i);
  }
  return ASLB_OK;
}

int aslb_bc_field_create(aslb_lbgk* h, int kind, const float* map, const double u[3], const double omega[3],
                         const double center[3], aslb_bc** out) {
  ASLB_CHECK_HANDLE(h);
  if (!out || !map) return fail(ASLB_ERR_ARG, "aslb_bc_field_create: null argument");
  *out = nullptr;
  if (kind < ASLB_BC_FIELD_NOSLIP_VEL || kind > ASLB_BC_FIELD_VELOCITY_VEL_ROTATION)
    return fail(ASLB_ERR_ARG, "aslb_bc_field_create: unknown field condition kind");
  const int q = h->d.q;
  if (q == 27)
    return fail(ASLB_ERR_ARG,
                "aslb_bc_field_create: ASL's d3q27 template has no laplacian or gradient coefficients");
  const bool vel = kind == ASLB_BC_FIELD_NOSLIP_VEL || kind >= ASLB_BC_FIELD_VELOCITY_VEL;
  if ((vel && !h->comp_vel) || (kind == ASLB_BC_FIELD_NOSLIP_RHO && !h->comp_rho))
    return fail(ASLB_ERR_ARG, "aslb_bc_field_create: the domain does not write that output field");
  const GridDesc& g = h->d.g;
  // guard cells -0.9999 < map <= 0 (aslBasicBC.cxx:223-226, 343-346, 137-141);
  // fluid neighbours map > 0, interior (the same restatement as the map conditions)
  std::vector<int4> cells;
  std::vector<double> wts;
  const double gcax = q == 15 ? 1.0 / 3.0 : 1.0 / 6.0, gcdg = q == 15 ? 1.0 / 24.0 : 1.0 / 12.0;
  for (int x = 0; x < g.gx; ++x)
    for (int y = 0; y < g.gy; ++y)
      for (int z = 0; z < g.gz; ++z) {
        if (on_periodic_ghost(h, x, y, z)) continue;
        const float m0 = map[aidx(g, x, y, z)];
        if (!(m0 <= 0.f && m0 > -0.9999f)) continue;
        unsigned mask = 0;
        double nrm[3] = {0, 0, 0};
        for (int k = 1; k < q; ++k) {
          const int qx = wrapc(h, x + lattice_c(q, k, 0), 0), qy = wrapc(h, y + lattice_c(q, k, 1), 1),
                    qz = wrapc(h, z + lattice_c(q, k, 2), 2);
          const float mk = map_at(g, map, qx, qy, qz);
          if (mk > 0.f && interior(g, qx, qy, qz)) mask |= 1u << k;
          // map gradient with the template's gradient coefficients (aslTemplateVE.cxx:210-222)
          const int n2 = lattice_c(q, k, 0) * lattice_c(q, k, 0) + lattice_c(q, k, 1) * lattice_c(q, k, 1) +
                         lattice_c(q, k, 2) * lattice_c(q, k, 2);
          const double gc = n2 == 1 ? gcax : gcdg;
          for (int d = 0; d < 3; ++d) nrm[d] += gc * lattice_c(q, k, d) * (double)mk;
        }
        if (kind == ASLB_BC_FIELD_NOSLIP_RHO) {
          const double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
          if (!(len > 0.0) || !mask) continue;  // no normal or no fluid neighbour: the value stays
          std::vector<double> w(q, 0.0);
          for (int k = 1; k < q; ++k) {
            if (!(mask >> k & 1u)) continue;
            const int c0 = lattice_c(q, k, 0), c1 = lattice_c(q, k, 1), c2 = lattice_c(q, k, 2);
            const double cl = std::sqrt((double)(c0 * c0 + c1 * c1 + c2 * c2));
            const double dc = (nrm[0] * c0 + nrm[1] * c1 + nrm[2] * c2) / len / cl + 1.0;
            w[k] = dc * dc;
          }
          wts.insert(wts.end(), w.begin(), w.end());
        }
        cells.push_back(make_int4(x, y, z, (int)mask));
      }
  auto* bc = new aslb_bc();
  bc->h = h;
  bc->bp.kind = kind;
  for (int d = 0; d < 3; ++d) {
    bc->bp.u[d] = u ? u[d] : 0.0;
    bc->bp.om[d] = omega ? omega[d] : 0.0;
    bc->bp.cen[d] = center ? center[d] : 0.0;
    bc->bp.pos0[d] = h->pos0[d];
  }
  bc->bp.dx = h->dx;
  bc->n = (int)cells.size();
  bc->links = bc->n;
  int r = upload(&bc->anchors, cells);
  if (!r && !wts.empty()) r = upload(&bc->fweights, wts);
  if (r) {
    aslb_bc_destroy(bc);
    return r;
  }
  bc->host_anchors.swap(cells);
  h->bcs.push_back(bc);
  *out = bc;
  return ASLB_OK;
}

int aslb_bc_deposition_create(aslb_lbgk* h, int kind, const float* map, double p0, double limiting_factor,
                              double beta, aslb_bc** out) {
  ASLB_CHECK_HANDLE(h);
  if (!out || !map) return fail(ASLB_ERR_ARG, "aslb_bc_deposition_create: null argument");
  *out = nullptr;
  if (kind != ASLB_BC_MAP_TRANSPORT_DEPOSITION && kind != ASLB_BC_MAP_KINETICS_DEPOSITION)
    return fail(ASLB_ERR_ARG, "aslb_bc_deposition_create: unknown deposition kind");
  std::vector<Cand> cand;
  map_candidates(h, map, cand);
  if (cand.size() >= (size_t)(1u << 31))
    return fail(ASLB_ERR_ARG, "aslb_bc_deposition_create: too many boundary links");
  auto* bc = new aslb_bc();
  bc->h = h;
  bc->bp.kind = kind;
  bc->bp.compressible = h->p.compressible;
  bc->bp.p = p0;
  bc->bp.lf = limiting_factor;
  bc->bp.beta = beta;
  bc->bp.dx = h->dx;
  for (int d = 0; d < 3; ++d) bc->bp.pos0[d] = h->pos0[d];
  bc->bp.scale = h->p.scale;
  bc->bp.inv_scale = h->p.inv_scale;
  fill_link_values(h, bc);
  // every link of an anchor together: the value depends on all of them
  int r = finalize_links(h, bc, cand, true);
  if (r) {
    aslb_bc_destroy(bc);
    return r;
  }
  h->bcs.push_back(bc);
  *out = bc;
  return ASLB_OK;
}

int aslb_bc_map_create(aslb_lbgk* h, int kind, const float* map, double p, const double u[3], const double omega[3],
                       const double center[3], aslb_bc** out) {
  return aslb_bc_map_create_cd(h, kind, map, nullptr, p, u, omega, center, out);
}

int aslb_bc_map_create_cd(aslb_lbgk* h, int kind, const float* map, const float* cdomain, double p, const double u[3],
                          const double omega[3], const double center[3], aslb_bc** out) {
  ASLB_CHECK_HANDLE(h);
  if (!out || !map) return fail(ASLB_ERR_ARG, "aslb_bc_map_create: null argument");
  *out = nullptr;
  if (kind < ASLB_BC_MAP_NOSLIP || kind > ASLB_BC_MAP_PRESSURE_VELOCITY)
    return fail(ASLB_ERR_ARG, "aslb_bc_map_create: unknown map kind");
  std::vector<Cand> cand;
  map_candidates(h, map, cand, cdomain);
  if (cand.size() >= (size_t)(1u << 31)) return fail(ASLB_ERR_ARG, "aslb_bc_map_create: too many boundary links");
  auto* bc = new aslb_bc();
  bc->h = h;
  bc->bp.kind = kind;
  bc->bp.compressible = h->p.compressible;
  bc->bp.p = p;
  for (int d = 0; d < 3; ++d) {
    bc->bp.u[d] = u ? u[d] : 0.0;
    bc->bp.om[d] = omega ? omega[d] : 0.0;
    bc->bp.cen[d] = center ? center[d] : 0.0;
    bc->bp.pos0[d] = h->pos0[d];
  }
  bc->bp.dx = h->dx;
  bc->bp.scale = h->p.scale;
  bc->bp.inv_scale = h->p.inv_scale;
  fill_link_values(h, bc);
  const bool velocity_map = kind == ASLB_BC_MAP_VELOCITY || kind == ASLB_BC_MAP_VELOCITY_ROTATION;
  int r = finalize_links(h, bc, cand, velocity_map);
  if (r) {
    aslb_bc_destroy(bc);
    return r;
  }
  h->bcs.push_back(bc);
  *out = bc;
  return ASLB_OK;
}

int aslb_bc_fuse(aslb_bc* bc) {
  if (!bc) return fail(ASLB_ERR_ARG, "aslb_bc_fuse: null argument");
  if (!bc->h) return fail(ASLB_ERR_STATE, "aslb_bc_fuse: its domain was destroyed");
  if (bc->bp.kind != ASLB_BC_MAP_NOSLIP && bc->bp.kind != ASLB_BC_NOSLIP)
    return fail(ASLB_ERR_ARG, "aslb_bc_fuse: only no-slip conditions can be fused");
  if (bc->fused) return ASLB_OK;
  aslb_lbgk* h = bc->h;
  const GridDesc& g = h->d.g;
  const int q = h->d.q;
  std::vector<uint2> m = h->mask_host.empty() ? std::vector<uint2>((size_t)g.dstride, make_uint2(0u, 0u))
                                               : h->mask_host;
  // Link (anchor a, direction k) enters fluid cell f = a + c_k: f reads it by
  // bounce-back (bounce bit k), and an interior anchor, which the
  // stream-collide kernel advances, skips its write of direction k (elide bit k).
  auto add = [&](long long sa, bool anchor_interior, long long sf, int k) {
    m[sf].x |= 1u << k;
    if (anchor_interior) m[sa].y |= 1u << k;
  };
  for (int k = 1; k < q; ++k)
    for (int t = bc->ls.seg[k]; t < bc->ls.seg[k + 1]; ++t) {
      const long long sa = bc->host_links[t];
      const long long local = sa % ((long long)g.gx * g.plane);
      const int z = int(local % g.pitch) - g.zoff;
      const int y = int((local / g.pitch) % g.gy);
      const int x = int(local / g.plane);
      add(sa, interior(g, x, y, z), sa + bc->ls.off[k], k);
    }
  for (const int4& an : bc->host_anchors)
    for (int k = 1; k < q; ++k) {
      if (!((unsigned)an.w >> k & 1u)) continue;
      const int ax = wrapc(h, an.x, 0), ay = wrapc(h, an.y, 1), az = wrapc(h, an.z, 2);
      const long long sa = sidx(g, ax, ay, az);
      const long long sf = sidx(g, wrapc(h, an.x + lattice_c(q, k, 0), 0), wrapc(h, an.y + lattice_c(q, k, 1), 1),
                                wrapc(h, an.z + lattice_c(q, k, 2), 2));
      add(sa, interior(g, ax, ay, az), sf, k);
    }
  // the compact form exists when every cell is either a bounce-back reader or
  // a skipped writer
  bool compact = true;
  for (const uint2& w : m)
    if (w.x && w.y) {
      compact = false;
      break;
    }
  cudaFree(h->mask32_dev);
  h->mask32_dev = nullptr;
  if (compact) {
    std::vector<uint32_t> m32(m.size());
    for (size_t i = 0; i < m.size(); ++i) m32[i] = m[i].y ? (m[i].y | 0x80000000u) : m[i].x;
    ASLB_CUDA(cudaMalloc((void**)&h->mask32_dev, ((size_t)g.dstride + 4096) * sizeof(uint32_t)));
    ASLB_CUDA(cudaMemcpy(h->mask32_dev, m32.data(), m32.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  }
  if (!h->mask_dev) ASLB_CUDA(cudaMalloc((void**)&h->mask_dev, ((size_t)g.dstride + 4096) * sizeof(uint2)));
  ASLB_CUDA(cudaStreamSynchronize(h->stream));
  ASLB_CUDA(cudaMemcpy(h->mask_dev, m.data(), m.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  h->mask_host.swap(m);
  bc->fused = true;
  h->version++;
  drop_graph(h);
  return ASLB_OK;
}

int aslb_bc_is_fused(aslb_bc* bc) { return bc && bc->fused ? 1 : 0; }

int aslb_bc_execute(aslb_bc* bc) {
  NvtxRange range("aslb_bc_execute");
  if (!bc) return fail(ASLB_ERR_ARG, "aslb_bc_execute: null handle");
  if (!bc->h) return fail(ASLB_ERR_STATE, "aslb_bc_execute: its domain was destroyed");
  return do_bc(bc);
}

int aslb_bc_destroy(aslb_bc* bc) {
  if (!bc) return ASLB_OK;
  if (bc->h) {
    cudaStreamSynchronize(bc->h->stream);
    drop_graph(bc->h);
    auto& v = bc->h->bcs;
    v.erase(std::remove(v.begin(), v.end(), bc), v.end());
  }
  cudaFree(bc->anchors);
  cudaFree(bc->dlinks);
  cudaFree(bc->fweights);
  delete bc;
  return ASLB_OK;
}

long long aslb_bc_num_links(aslb_bc* bc) { return bc ? bc->links : -1; }

int aslb_bc_kernels(aslb_bc* bc) { return !bc || bc->fused ? 0 : (bc->nd > 0) + (bc->n > 0); }

// ---- surface force ---------------------------------------------------------

namespace {
// Cells with |map| < 0.9999 (src/num/aslLBGKBC.cxx:730-733, 659-661); mask0
// links from a solid cell to a fluid interior neighbour, mask_in links from a
// fluid interior cell to a solid neighbour (src/num/aslLBGKBC.cxx:713-726, 643-656).
void surface_cells(const aslb_lbgk* h, const float* map, std::vector<int4>& cells, std::vector<uint32_t>& mask_in) {
  const GridDesc& g = h->d.g;
  const int q = h->d.q;
  for (int x = 0; x < g.gx; ++x)
    for (int y = 0; y < g.gy; ++y)
      for (int z = 0; z < g.gz; ++z) {
        if (on_periodic_ghost(h, x, y, z)) continue;
        const float m0 = map[aidx(g, x, y, z)];
        if (!(std::fabs(m0) < 0.9999f)) continue;
        const bool in0 = interior(g, x, y, z);
        unsigned k0 = 0, ki = 0;
        for (int k = 1; k < q; ++k) {
          const int qx = wrapc(h, x + lattice_c(q, k, 0), 0), qy = wrapc(h, y + lattice_c(q, k, 1), 1),
                    qz = wrapc(h, z + lattice_c(q, k, 2), 2);
          const float mk = map_at(g, map, qx, qy, qz);
          if (m0 <= 0.f && mk > 0.f && interior(g, qx, qy, qz)) k0 |= 1u << k;
          if (mk <= 0.f && m0 > 0.f && in0) ki |= 1u << k;
        }
        if (k0 | ki) {
          cells.push_back(make_int4(x, y, z, (int)k0));
          mask_in.push_back(ki);
        }
      }
}

// A force (3 values per cell) or flux (1 value per cell) object on the
// surface of map.
int surface_object(aslb_lbgk* h, const float* map, bool flux, aslb_force** out, const char* what) {
  ASLB_CHECK_HANDLE(h);
  if (!out || !map) return fail(ASLB_ERR_ARG, std::string(what) + ": null argument");
  *out = nullptr;
  const GridDesc& g = h->d.g;
  std::vector<int4> cells;
  std::vector<uint32_t> mask_in;
  surface_cells(h, map, cells, mask_in);
  const int width = flux ? 1 : 6, comps = flux ? 1 : 3;
  auto* fc = new aslb_force();
  fc->h = h;
  fc->flux = flux;
  fc->n = (int)cells.size();
  int r = upload(&fc->cells, cells);
  if (!r) r = upload(&fc->mask_in, mask_in);
  if (r) {
    aslb_force_destroy(fc);
    return r;
  }
  cudaError_t e = cudaMalloc((void**)&fc->field, comps * (size_t)g.L * sizeof(float));
  if (e == cudaSuccess) e = cudaMemsetAsync(fc->field, 0, comps * (size_t)g.L * sizeof(float), h->stream);
  if (e == cudaSuccess) e = cudaMalloc((void**)&fc->partials, (size_t)force_blocks(fc->n) * width * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&fc->out, 6 * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&fc->host_out, 6 * sizeof(double));
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    aslb_force_destroy(fc);
    return fail(ASLB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
  h->forces.push_back(fc);
  *out = fc;
  return ASLB_OK;
}
}  // namespace

int aslb_force_create(aslb_lbgk* h, const float* map, aslb_force** out) {
  return surface_object(h, map, false, out, "aslb_force_create");
}

int aslb_flux_create(aslb_lbgk* h, const float* map, aslb_flux** out) {
  return surface_object(h, map, true, out, "aslb_flux_create");
}

int aslb_flux_compute(aslb_flux* fc, float* field_host, double* total) {
  if (!fc) return fail(ASLB_ERR_ARG, "aslb_flux_compute: null argument");
  if (!fc->flux) return fail(ASLB_ERR_ARG, "aslb_flux_compute: a force object, not a flux object");
  if (!fc->h) return fail(ASLB_ERR_STATE, "aslb_flux_compute: its domain was destroyed");
  aslb_lbgk* h = fc->h;
  cudaError_t e = launch_flux(h->d, fc->cells, fc->mask_in, fc->n, fc->field, h->p.inv_scale,
                              h->fresh ? nullptr : h->mask_dev, h->parity, fc->partials, fc->out, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(fc->host_out, fc->out, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess && field_host)
    e = cudaMemcpyAsync(field_host, fc->field, (size_t)h->d.g.L * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_flux_compute: ") + cudaGetErrorString(e));
  if (total) *total = fc->host_out[0];
  return ASLB_OK;
}

int aslb_flux_destroy(aslb_flux* fc) { return aslb_force_destroy(fc); }

int aslb_force_compute(aslb_force* fc, const double r0[3], float* field_host, double out6[6]) {
  NvtxRange range("aslb_force_compute");
  if (!fc || !out6) return fail(ASLB_ERR_ARG, "aslb_force_compute: null argument");
  if (fc->flux) return fail(ASLB_ERR_ARG, "aslb_force_compute: a flux object, not a force object");
  if (!fc->h) return fail(ASLB_ERR_STATE, "aslb_force_compute: its domain was destroyed");
  aslb_lbgk* h = fc->h;
  const double zero[3] = {0, 0, 0};
  cudaError_t e = launch_force(h->d, fc->cells, fc->mask_in, fc->n, fc->field, r0 ? r0 : zero, h->pos0, h->dx,
                               h->p.inv_scale, h->fresh ? nullptr : h->mask_dev, h->parity, fc->partials,
                               fc->out, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(fc->host_out, fc->out, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess && field_host)
    e = cudaMemcpyAsync(field_host, fc->field, 3 * (size_t)h->d.g.L * sizeof(float), cudaMemcpyDeviceToHost,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("aslb_force_compute: ") + cudaGetErrorString(e));
  for (int i = 0; i < 6; ++i) out6[i] = fc->host_out[i];
  return ASLB_OK;
}

int aslb_force_destroy(aslb_force* fc) {
  if (!fc) return ASLB_OK;
  if (fc->h) {
    cudaStreamSynchronize(fc->h->stream);
    auto& v = fc->h->forces;
    v.erase(std::remove(v.begin(), v.end(), fc), v.end());
  }
  cudaFree(fc->cells);
  cudaFree(fc->mask_in);
  cudaFree(fc->field);
  cudaFree(fc->partials);
  cudaFree(fc->out);
  if (fc->host_out) cudaFreeHost(fc->host_out);
  delete fc;
  return ASLB_OK;
}

// ---- surface force without any allocation ---------------------------------
//
// For callers that cannot allocate device memory at the moment they need a
// force: a host program whose allocator forbids new device allocations after
// set-up, or an embedding runtime that hands out all memory up front.
// aslb_force_compute allocates nothing per call either, but its scratch rows
// come from cudaMalloc at aslb_force_create; this variant takes the
// per-block partial sums and the final sums from one fixed array in the
// library's own device memory instead.

}  // extern "C"

namespace {
// Up to kNoAllocForceBlocks blocks of 256 listed force cells (1,048,576
// cells), six partial sums each, plus the six final sums: 196,672 bytes that
// every device which loads the library keeps until the process exits.
constexpr int kNoAllocForceBlocks = 4096;
constexpr int kNoAllocForceCells = kNoAllocForceBlocks * 256;
constexpr int kNoAllocScratch = kNoAllocForceBlocks * 6 + 8;
static __device__ __align__(256) double g_force_scratch[kNoAllocScratch];
// Device address of g_force_scratch per device (the name is only a host-side
// stand-in in host code), looked up on the first call on each device; the
// lock makes concurrent first calls from several host threads safe.
std::atomic<double*> g_force_scratch_dev[64];
std::mutex g_force_scratch_lock;
}  // namespace

extern "C" int aslb_force_compute_noalloc(aslb_force* fc, const double r0[3], double out6[6]) {
  if (!fc || !out6) return fail(ASLB_ERR_ARG, "aslb_force_compute_noalloc: null argument");
  if (fc->flux) return fail(ASLB_ERR_ARG, "aslb_force_compute_noalloc: a flux object, not a force object");
  if (!fc->h) return fail(ASLB_ERR_STATE, "aslb_force_compute_noalloc: its domain was destroyed");
  aslb_lbgk* h = fc->h;
  if (force_blocks(fc->n) > kNoAllocForceBlocks)
    return fail(ASLB_ERR_ARG, "aslb_force_compute_noalloc: " + std::to_string(fc->n) +
                                  " force cells exceed the fixed scratch limit of " +
                                  std::to_string(kNoAllocForceCells) + "; use aslb_force_compute");
  int dev = -1;
  ASLB_CUDA(cudaGetDevice(&dev));
  if (dev != h->device)
    return fail(ASLB_ERR_STATE, "aslb_force_compute_noalloc: make the domain's device current first");
  if (dev < 0 || dev >= 64) return fail(ASLB_ERR_ARG, "aslb_force_compute_noalloc: device index out of range");
  double* partials = g_force_scratch_dev[dev].load(std::memory_order_acquire);
  if (!partials) {
    std::lock_guard<std::mutex> lock(g_force_scratch_lock);
    partials = g_force_scratch_dev[dev].load(std::memory_order_relaxed);
    if (!partials) {
      ASLB_CUDA(cudaGetSymbolAddress((void**)&partials, g_force_scratch));
      g_force_scratch_dev[dev].store(partials, std::memory_order_release);
    }
  }
  double* sums = partials + (size_t)kNoAllocForceBlocks * 6;
  // Every block writes its whole row of partial sums and the final kernel
  // overwrites the six sums, so nothing left by an earlier call is read.
  const double zero[3] = {0, 0, 0};
  cudaError_t e = launch_force(h->d, fc->cells, fc->mask_in, fc->n, nullptr, r0 ? r0 : zero, h->pos0, h->dx,
                               h->p.inv_scale, h->fresh ? nullptr : h->mask_dev, h->parity, partials, sums,
                               h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out6, sums, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return fail(ASLB_ERR_CUDA, std::string("aslb_force_compute_noalloc: ") + cudaGetErrorString(e));
  return ASLB_OK;
}

// ---- batches of independent domains -----------------------------------------

struct aslb_batch {
  std::vector<aslb_lbgk*> doms;
  bool detached = false;  // a member domain was destroyed
  int q = 0, storage = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  // device tables
  std::vector<BatchDom> host_doms;
  BatchDom* dev_doms = nullptr;
  long long ntiles = 0;
  long long* dev_starts = nullptr;  // the work split's run tables (BatchWork)
  BatchWork work{};
  bool any_mask = false;
  int mask_mode = 0;  // 0 no fused links, 1 two-word masks, 2 one-word masks in every masked domain
  std::vector<BatchBc*> dev_pos;  // one table per condition position
  std::vector<int> pos_n;
  std::vector<long long> pos_links;
  std::vector<aslb_bc*> key;      // conditions the tables were built for
  std::vector<int> key_n;
  long long table_version = -1;   // sum of the domains' versions at build
  // time-loop graph
  cudaGraphExec_t graph = nullptr;
  int graph_parity = -1;
  long long graph_version = -1;
  // launch shape of the batched step (batch_shape_count() choices): fixed by
  // aslb_batch_set_shape, or chosen by timing (shape_auto) before the first
  // graph is recorded
  int shape = 0;
  bool shape_auto = true;
  std::vector<float> shape_ms;
};

void batch_detach(aslb_batch* b, aslb_lbgk* h) {
  for (auto& d : b->doms)
    if (d == h) d = nullptr;
  b->detached = true;
  auto& v = h->batches;
  v.erase(std::remove(v.begin(), v.end(), b), v.end());
}

namespace {

void batch_free_tables(aslb_batch* b) {
  cudaFree(b->dev_doms);
  b->dev_doms = nullptr;
  cudaFree(b->dev_starts);
  b->dev_starts = nullptr;
  b->work = BatchWork{};
  for (BatchBc* t : b->dev_pos) cudaFree(t);
  b->dev_pos.clear();
  b->pos_n.clear();
  b->pos_links.clear();
}

void batch_drop_graph(aslb_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_parity = -1;
}

long long batch_version(const aslb_batch* b) {
  long long v = 0;
  for (const aslb_lbgk* h : b->doms) v += h->version;
  return v;
}

// (Re)build the domain table and one link table per condition position.
int batch_tables(aslb_batch* b, aslb_bc* const* bcs, const int* nbc) {
  batch_free_tables(b);
  const int n = (int)b->doms.size();
  b->host_doms.assign(n, BatchDom{});
  b->ntiles = 0;
  b->any_mask = false;
  bool all_m32 = true;
  for (int i = 0; i < n; ++i) {
    aslb_lbgk* h = b->doms[i];
    BatchDom& D = b->host_doms[i];
    const GridDesc& g = h->d.g;
    D.g = g;
    D.F = h->d.F;
    D.mask = h->fresh ? nullptr : h->mask_dev;
    D.mask32 = h->fresh ? nullptr : h->mask32_dev;
    b->any_mask |= D.mask != nullptr;
    if (D.mask && !D.mask32) all_m32 = false;
    D.rho = h->d.rho;
    D.u = h->d.u;
    D.om0f = 1.0f / (3.0f * (float)h->p.nu + 0.5f);
    D.om0d = 1.0 / (3.0 * h->p.nu + 0.5);
    D.nz_inv = (unsigned)((0x100000000ULL + (unsigned long long)g.nz - 1) / (unsigned long long)g.nz);
    D.tile0 = b->ntiles;
    b->ntiles += g.nx;
  }
  // link-mask form of the launch: 0 none, 1 two words, 2 one word per cell
  b->mask_mode = b->any_mask ? (all_m32 ? 2 : 1) : 0;
  ASLB_CUDA(cudaMalloc((void**)&b->dev_doms, n * sizeof(BatchDom)));
  ASLB_CUDA(cudaMemcpy(b->dev_doms, b->host_doms.data(), n * sizeof(BatchDom), cudaMemcpyHostToDevice));
  // the work split: contiguous runs of tiles with equal shares of the cells
  {
    std::vector<long long> tile_cells;
    tile_cells.reserve((size_t)b->ntiles);
    for (const BatchDom& D : b->host_doms)
      for (int x = 0; x < D.g.nx; ++x) tile_cells.push_back((long long)D.g.ny * D.g.nz);
    int dev = 0, sms = 0;
    ASLB_CUDA(cudaGetDevice(&dev));
    ASLB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    std::vector<long long> starts;
    batch_work_tables(tile_cells, sms, starts, b->work.grid, b->work.group, b->work.off);
    ASLB_CUDA(cudaMalloc((void**)&b->dev_starts, starts.size() * sizeof(long long)));
    ASLB_CUDA(cudaMemcpy(b->dev_starts, starts.data(), starts.size() * sizeof(long long), cudaMemcpyHostToDevice));
    b->work.ntiles = b->ntiles;
    b->work.starts = b->dev_starts;
  }
  // condition positions: the j-th separate condition of every domain
  std::vector<std::vector<BatchBc>> pos;
  std::vector<long long> pos_total;
  int off = 0;
  for (int i = 0; i < n; ++i) {
    int j = 0;
    for (int c = 0; c < nbc[i]; ++c) {
      aslb_bc* bc = bcs[off + c];
      if (bc->fused) continue;
      if ((int)pos.size() <= j) {
        pos.resize(j + 1);
        pos_total.resize(j + 1, 0);
      }
      if (bc->nd > 0) {
        BatchBc e{};
        e.F = b->doms[i]->d.F;
        e.dstride = b->doms[i]->d.g.dstride;
        e.links = bc->dlinks;
        e.ls = bc->ls;
        e.bp = bc->bp;
        e.link0 = pos_total[j];
        pos_total[j] += bc->nd;
        pos[j].push_back(e);
      }
      ++j;
    }
    off += nbc[i];
  }
  for (size_t j = 0; j < pos.size(); ++j) {
    const auto& v = pos[j];
    BatchBc* t = nullptr;
    const long long links = pos_total[j];
    if (!v.empty()) {
      ASLB_CUDA(cudaMalloc((void**)&t, v.size() * sizeof(BatchBc)));
      ASLB_CUDA(cudaMemcpy(t, v.data(), v.size() * sizeof(BatchBc), cudaMemcpyHostToDevice));
    }
    b->dev_pos.push_back(t);
    b->pos_n.push_back((int)v.size());
    b->pos_links.push_back(links);
  }
  b->table_version = batch_version(b);
  return ASLB_OK;
}

// One step of every domain: the batched stream-collide, then each condition
// position in order (ASL's order within every domain).
int batch_step(aslb_batch* b) {
  aslb_lbgk* h0 = b->doms[0];
  prepare_params(h0);
  const int parity = h0->parity;
  cudaError_t e = launch_batch_step(b->q, b->storage, b->dev_doms, (int)b->doms.size(), b->work, b->mask_mode,
                                    h0->p, parity, b->shape, b->stream);
  for (size_t j = 0; e == cudaSuccess && j < b->dev_pos.size(); ++j)
    if (b->pos_n[j] > 0)
      e = launch_batch_links(b->q, b->storage, b->dev_pos[j], b->pos_n[j], b->pos_links[j], parity ^ 1, b->stream);
  if (e != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
  for (aslb_lbgk* h : b->doms) {
    h->parity ^= 1;
    h->steps += 1;
    if (h->macro_once) {
      h->macro_once = false;
      h->version++;
    }
  }
  return ASLB_OK;
}

}  // namespace

int aslb_batch_create(aslb_lbgk* const* domains, int n, aslb_batch** out) {
  if (!out || !domains || n <= 0) return fail(ASLB_ERR_ARG, "aslb_batch_create: bad arguments");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    aslb_lbgk* h = domains[i];
    if (!h) return fail(ASLB_ERR_ARG, "aslb_batch_create: null domain");
    for (int j = 0; j < i; ++j)
      if (domains[j] == h) return fail(ASLB_ERR_ARG, "aslb_batch_create: a domain appears twice");
    if (h->d.q != domains[0]->d.q || h->d.storage != domains[0]->d.storage)
      return fail(ASLB_ERR_ARG, "aslb_batch_create: domains differ in lattice or storage");
    if (h->device != domains[0]->device) return fail(ASLB_ERR_ARG, "aslb_batch_create: domains on different devices");
  }
  aslb_batch* b = new aslb_batch();
  b->doms.assign(domains, domains + n);
  b->q = domains[0]->d.q;
  b->storage = domains[0]->d.storage;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return fail(ASLB_ERR_CUDA, std::string("aslb_batch_create: ") + cudaGetErrorString(e));
  }
  for (aslb_lbgk* h : b->doms) h->batches.push_back(b);
  *out = b;
  return ASLB_OK;
}

int aslb_batch_run(aslb_batch* b, int nsteps, aslb_bc* const* bcs, const int* nbc, int use_graph) {
  NvtxRange range("aslb_batch_run");
  ASLB_CHECK_HANDLE(b);
  if (b->detached) return fail(ASLB_ERR_STATE, "aslb_batch_run: a domain of the batch was destroyed");
  const int n = (int)b->doms.size();
  if (nsteps < 0 || !nbc) return fail(ASLB_ERR_ARG, "aslb_batch_run: bad arguments");
  // every domain must step like the first one: same parity, closure and
  // batch-wide parameters (only the viscosity, geometry and conditions differ)
  aslb_lbgk* h0 = b->doms[0];
  int total = 0;
  for (int i = 0; i < n; ++i) {
    aslb_lbgk* h = b->doms[i];
    if (nbc[i] < 0) return fail(ASLB_ERR_ARG, "aslb_batch_run: negative condition count");
    if (h->parity != h0->parity) return fail(ASLB_ERR_STATE, "aslb_batch_run: domains are at different parities");
    if (h->closure != CL_NONE) return fail(ASLB_ERR_ARG, "aslb_batch_run: batches run the plain BGK collision only");
    if (h->p.compressible != h0->p.compressible || h->p.has_force != h0->p.has_force ||
        h->p.has_coriolis != h0->p.has_coriolis || h->p.scale != h0->p.scale || h->comp_vel != h0->comp_vel ||
        h->comp_rho != h0->comp_rho || h->macro_once != h0->macro_once ||
        std::memcmp(h->p.g, h0->p.g, sizeof(h->p.g)) != 0 || std::memcmp(h->p.Om, h0->p.Om, sizeof(h->p.Om)) != 0)
      return fail(ASLB_ERR_ARG, "aslb_batch_run: domains differ in a batch-wide parameter (body force, rotation, "
                                "compressibility, FP16 scale or output fields)");
    for (int c = 0; c < nbc[i]; ++c) {
      aslb_bc* bc = bcs ? bcs[total + c] : nullptr;
      if (!bc || bc->h != h) return fail(ASLB_ERR_ARG, "aslb_batch_run: condition of another domain");
      if (c > 0 && bcs[total + c - 1]->fused && !bc->fused)
        return fail(ASLB_ERR_ARG, "aslb_batch_run: fused conditions must come after all separate ones");
      if (!bc->fused && bc->n > 0)
        return fail(ASLB_ERR_ARG,
                    "aslb_batch_run: per-cell conditions (velocity, deposition and field maps, links across periodic "
                    "faces) are not batched");
    }
    total += nbc[i];
  }
  std::vector<aslb_bc*> key(bcs, bcs + total);
  std::vector<int> key_n(nbc, nbc + n);
  // the batch's stream follows every domain's pending work
  for (aslb_lbgk* h : b->doms) {
    ASLB_CUDA(cudaEventRecord(b->ev, h->stream));
    ASLB_CUDA(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  auto refresh = [&]() -> int {
    if (b->key == key && b->key_n == key_n && b->table_version == batch_version(b)) return ASLB_OK;
    ASLB_CUDA(cudaStreamSynchronize(b->stream));
    batch_drop_graph(b);
    int r = batch_tables(b, bcs, nbc);
    if (r) return r;
    b->key = key;
    b->key_n = key_n;
    return ASLB_OK;
  };
  // after the first step every fused condition has run: incoming slots are no
  // longer the initial values, the fused links take effect
  auto after_step = [&]() {
    int off = 0;
    for (int i = 0; i < n; ++i) {
      aslb_lbgk* h = b->doms[i];
      for (int c = 0; c < nbc[i]; ++c)
        if (bcs[off + c]->fused && h->fresh) {
          h->fresh = false;
          h->version++;
        }
      off += nbc[i];
    }
  };
  auto eager = [&](int k) -> int {
    for (int s = 0; s < k; ++s) {
      int r = refresh();
      if (r) return r;
      r = batch_step(b);
      if (r) return r;
      after_step();
    }
    return ASLB_OK;
  };
  int done = 0, r = ASLB_OK;
  bool fresh = false;
  for (aslb_lbgk* h : b->doms) fresh |= h->fresh || h->macro_once;
  if (!use_graph || nsteps < 2) {
    r = eager(nsteps);
    done = nsteps;
  } else {
    if (fresh) {
      r = eager(1);
      done = 1;
    }
    if (!r) r = refresh();
    // launch-shape tuner: two real steps (one of each parity) per shape,
    // timed on the batch's stream; the fastest is kept
    const int nshape = batch_shape_count();
    if (!r && b->shape_auto && b->shape_ms.empty() && nsteps - done >= 2 * nshape + 2) {
      cudaEvent_t t0 = nullptr, t1 = nullptr;
      ASLB_CUDA(cudaEventCreate(&t0));
      ASLB_CUDA(cudaEventCreate(&t1));
      int best = 0;
      for (int v = 0; v < nshape && !r; ++v) {
        b->shape = v;
        cudaEventRecord(t0, b->stream);
        r = eager(2);
        cudaEventRecord(t1, b->stream);
        cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        b->shape_ms.push_back(ms);
        if (ms < b->shape_ms[best]) best = v;
        done += 2;
      }
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      b->shape = best;
      batch_drop_graph(b);
    }
    if (!r && !(b->graph && b->graph_version == batch_version(b) && b->graph_parity == h0->parity)) {
      if (b->graph && b->graph_version == batch_version(b) && done < nsteps) {
        // graph of the other parity: one eager step realigns
        r = eager(1);
        done += 1;
      }
      if (!r && !(b->graph && b->graph_version == batch_version(b) && b->graph_parity == h0->parity)) {
        batch_drop_graph(b);
        std::vector<int> par(n);
        std::vector<long long> st(n);
        for (int i = 0; i < n; ++i) {
          par[i] = b->doms[i]->parity;
          st[i] = b->doms[i]->steps;
        }
        cudaGraph_t graph = nullptr;
        ASLB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rr = batch_step(b);
        if (!rr) rr = batch_step(b);
        cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
        for (int i = 0; i < n; ++i) {  // capture enqueued nothing
          b->doms[i]->parity = par[i];
          b->doms[i]->steps = st[i];
        }
        if (rr) {
          if (graph) cudaGraphDestroy(graph);
          return rr;
        }
        if (ce != cudaSuccess) return fail(ASLB_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&b->graph, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
          b->graph = nullptr;
          return fail(ASLB_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ce));
        }
        b->graph_parity = h0->parity;
        b->graph_version = batch_version(b);
      }
    }
    if (!r) {
      const int pairs = (nsteps - done) / 2;
      for (int i = 0; i < pairs; ++i) ASLB_CUDA(cudaGraphLaunch(b->graph, b->stream));
      for (aslb_lbgk* h : b->doms) h->steps += 2LL * pairs;
      done += 2 * pairs;
      r = eager(nsteps - done);
    }
  }
  // every domain's later work follows the batch
  ASLB_CUDA(cudaEventRecord(b->ev, b->stream));
  for (aslb_lbgk* h : b->doms) ASLB_CUDA(cudaStreamWaitEvent(h->stream, b->ev, 0));
  return r;
}

int aslb_batch_sync(aslb_batch* b) {
  ASLB_CHECK_HANDLE(b);
  ASLB_CUDA(cudaStreamSynchronize(b->stream));
  return ASLB_OK;
}

long long aslb_batch_tiles(aslb_batch* b) { return b ? b->ntiles : -1; }

int aslb_batch_set_shape(aslb_batch* b, int shape) {
  ASLB_CHECK_HANDLE(b);
  if (shape < -1 || shape >= batch_shape_count())
    return fail(ASLB_ERR_ARG, "aslb_batch_set_shape: shape must be -1 (tune) or 0 .. " +
                                  std::to_string(batch_shape_count() - 1));
  b->shape_auto = shape < 0;
  b->shape = shape < 0 ? 0 : shape;
  b->shape_ms.clear();
  batch_drop_graph(b);
  return ASLB_OK;
}

int aslb_batch_get_shape(aslb_batch* b) { return b ? b->shape : -1; }

int aslb_batch_shape_times(aslb_batch* b, float* ms_out, int n) {
  ASLB_CHECK_HANDLE(b);
  const int k = (int)b->shape_ms.size();
  for (int i = 0; i < k && i < n; ++i) ms_out[i] = b->shape_ms[i];
  return k;
}

int aslb_batch_destroy(aslb_batch* b) {
  if (!b) return ASLB_OK;
  cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  batch_free_tables(b);
  for (aslb_lbgk* h : b->doms)
    if (h) {
      auto& v = h->batches;
      v.erase(std::remove(v.begin(), v.end(), b), v.end());
    }
  cudaEventDestroy(b->ev);
  cudaStreamDestroy(b->stream);
  delete b;
  return ASLB_OK;
}
