// Host-side launch interface of the CUDA kernels (implemented in kernels.cu).
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include "internal.cuh"

struct aslb_lbgk;
struct aslb_fd;

namespace aslb {

enum StorageKind { ST_F32 = 0, ST_F16 = 1, ST_F64 = 2 };

// Message returned by aslb_last_error() on the calling thread.
void set_last_error(const std::string& msg);
// Velocity field of a domain for a coupled FD solver (fd.cu): interior
// sizes, storage, device pointer (ASL layout, 3 L values) and stream. Fails
// when the domain does not write its velocity every step.
int lbgk_velocity_binding(aslb_lbgk* h, int n[3], int* storage, void** u, cudaStream_t* st);
void lbgk_attach_fd(aslb_lbgk* h, aslb_fd* f);
void lbgk_detach_fd(aslb_lbgk* h, aslb_fd* f);
void fd_detached(aslb_fd* f);

struct DomainDev {
  GridDesc g;
  int q;
  int storage;
  void* F;     // populations (Q direction arrays)
  void* rho;   // density, ASL ghosted layout (float, or double for ST_F64)
  void* u;     // velocity, 3 components of L each
  int variant; // stream-collide kernel: 0 plain, 1 TMA-staged
  int* err;    // device error word (bounded waits that gave up)
};

inline size_t storage_bytes(int st) { return st == ST_F16 ? 2 : (st == ST_F64 ? 8 : 4); }
inline size_t macro_bytes(int st) { return st == ST_F64 ? 8 : 4; }

// One stream-collide step of the AA pattern. parity_in is the representation
// the populations are in before the step (0 = A, 1 = B).
cudaError_t launch_step(const DomainDev& d, const StepParams& p, int closure, int parity_in, cudaStream_t st);
// f = f_eq(rho, u) in representation A for every ghosted cell, rho/u written too.
// rho_field / u_field: device arrays in ASL layout (double) or null for constants.
cudaError_t launch_init_f(const DomainDev& d, const StepParams& p, double rho0, const double* u0,
                          const double* rho_field, const double* u_field, cudaStream_t st);
// Copy directions [i0, i1) of the populations to / from ASL's layout (f_i at
// (i - i0)*L + ghosted index), values in the macro type (float or double).
cudaError_t launch_export_f(const DomainDev& d, const StepParams& p, int parity, int i0, int i1, void* out,
                            cudaStream_t st);
cudaError_t launch_import_f(const DomainDev& d, const StepParams& p, int i0, int i1, const void* in,
                            cudaStream_t st);
// rho and / or u of every interior cell from the current populations.
cudaError_t launch_compute_macro(const DomainDev& d, const StepParams& p, int parity, int comp_rho, int comp_vel,
                                 cudaStream_t st);
// Boundary links: anchors (x, y, z, direction mask) in ghosted coordinates.
// Conditions on the rho / u output fields (visualisation): guard cells with
// their fluid-neighbour masks, per-cell weights for the rho condition.
cudaError_t launch_field_bc(const DomainDev& d, const int4* cells, int n, const double* wt, const BcParams& bp,
                            cudaStream_t st);
cudaError_t launch_bc(const DomainDev& d, const int4* anchors, int n, const BcParams& bp, int parity,
                      cudaStream_t st);
// Direction-sorted links (one thread per link), the common case of every
// condition except the velocity maps.
cudaError_t launch_bc_links(const DomainDev& d, const int* links, int n, const LinkSet& ls, const BcParams& bp,
                            int parity, cudaStream_t st);
// Surface force: per-cell field (ASL layout, optional) and per-block FP64
// partial sums of (F, (r - r0) x F), then a fixed-order final sum into out6.
int force_blocks(int n);
// Blow-up watchdog rows (moments_blocks(g) rows of [max |u|^2, min rho, non-finite cells]).
int moments_blocks(const GridDesc& g);
cudaError_t launch_watchdog(const DomainDev& d, const StepParams& p, int parity, double* partials, cudaStream_t st);
// Surface flux (ComputeSurfaceFluxMap): same cell lists as the force, one
// value per cell (field, optional) and its FP64 total (out1).
cudaError_t launch_flux(const DomainDev& d, const int4* cells, const uint32_t* mask_in, int n, float* field,
                        float inv_scale, const uint2* fused, int parity, double* partials, double* out1,
                        cudaStream_t st);
cudaError_t launch_force(const DomainDev& d, const int4* cells, const uint32_t* mask_in, int n, float* field,
                         const double* r0, const double* pos0, double dx, float inv_scale, const uint2* fused,
                         int parity, double* partials, double* out6, cudaStream_t st);
// Global diagnostics over interior cells (fluid cells in fused mode): (mass,
// momentum x, y, z) in FP64.
int moments_blocks(const GridDesc& g);
cudaError_t launch_moments(const DomainDev& d, const StepParams& p, int parity, double* partials, double* out4,
                           cudaStream_t st);
// Sum `nblocks` rows of `width` doubles into out (fixed order, one block).
cudaError_t launch_reduce_rows(const double* partials, int nblocks, int width, double* out, cudaStream_t st);


// Learned closure: Cs^2 per storage cell from the network (closure_field.cu),
// and the nine raw features per interior cell, out[k * cells + compact index]
// (x-major, z fastest), for training. D3Q19 / D3Q27, FP32 or FP16 storage.
cudaError_t launch_closure_field(const DomainDev& d, const StepParams& p, const void* net, float* cs2, int parity,
                                 cudaStream_t st);
cudaError_t launch_closure_features(const DomainDev& d, const StepParams& p, float* out, int parity,
                                    cudaStream_t st);
// One float per storage cell (interior) -> ASL's ghosted layout, 0 on ghosts.
cudaError_t launch_gather_cells(const GridDesc& g, const float* src, float* dst_asl, cudaStream_t st);

// ---- batches of independent domains ----------------------------------------
// One entry per domain of a batch (device table, ordered by tile0).
struct BatchDom {
  GridDesc g;
  void* F;
  const uint2* mask;  // fused links, or null
  const uint32_t* mask32;  // the same links in one word per cell (null when a cell has both kinds)
  void* rho;
  void* u;
  float om0f;
  double om0d;
  unsigned nz_inv;   // ceil(2^32 / nz): y = l / nz by a multiply-high
  long long tile0;   // first tile (x plane) of this domain in the batch
};
// One entry per (domain, condition) of a batched link launch (ordered by link0).
struct BatchBc {
  void* F;
  long long dstride;
  const int* links;
  long long link0;  // first link of this entry in the launch
  LinkSet ls;
  BcParams bp;
};
// The work split of a batched step: the tiles in order, each group of
// `group` blocks of the persistent grid a contiguous run of them holding an
// equal share of the cells (group g: tiles starts[g] .. starts[g + 1] - 1,
// block j of the group every group-th of them from the j-th), one table per
// residency (2, 3, 4 blocks per SM), back to back in device memory.
struct BatchWork {
  long long ntiles;
  const long long* starts;  // device
  int grid[3];              // blocks at 2, 3, 4 resident blocks per SM
  int group[3];             // blocks per group (the grid is a multiple)
  long long off[3];         // each residency's table in starts
};
// Host side of the split: the per-residency tables for tiles of the given
// cell counts on `sms` SMs (grid = min(tiles, sms x residency), in groups of
// four blocks where that divides it).
void batch_work_tables(const std::vector<long long>& tile_cells, int sms, std::vector<long long>& starts,
                       int (&grid)[3], int (&group)[3], long long (&off)[3]);
// One stream-collide step of every domain of a batch (same lattice, storage
// and parity; CL_NONE), a persistent grid over all domains' tiles; `shape`
// (0 .. batch_shape_count() - 1) picks the resident blocks per SM.
cudaError_t launch_batch_step(int q, int storage, const BatchDom* doms, int ndom, const BatchWork& w, int fused,
                              const StepParams& p, int parity_in, int shape, cudaStream_t st);
int batch_shape_count();
// Every link of the entries (one condition position across the batch).
cudaError_t launch_batch_links(int q, int storage, const BatchBc* bcs, int nbc, long long nlinks, int parity,
                               cudaStream_t st);

}  // namespace aslb
