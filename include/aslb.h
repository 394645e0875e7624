/*
 * aslb.h -- C ABI of the B200 lattice-Boltzmann library (libaslb.so).
 *
 * A drop-in compute layer for the LBGK hot path of the Advanced Simulation
 * Library (ASL). Every entry point takes plain pointers and sizes, returns
 * ASLB_OK (0) or a negative error code, and records a message retrievable with
 * aslb_last_error() (thread-local). Citations name the reference project's
 * interface each call replaces (paths inside AvtechScientific/ASL).
 *
 * Conventions shared with ASL:
 *  - A domain has nx x ny x nz interior cells and one ghost layer. Host arrays
 *    use ASL's flattening of the ghosted block, z fastest:
 *      idx = (x * (ny+2) + y) * (nz+2) + z,   x in [0, nx+1] ...
 *    (src/data/aslBlocks.h:118-130, src/data/aslDataWithGhostNodes.h:97-145).
 *    L = (nx+2)(ny+2)(nz+2). Vector fields store component c at c*L + idx.
 *  - Populations are ASL-normalised (rest state f_i = 1; rho = sum w_i f_i).
 *    Direction order is ASL's (src/math/aslTemplates.cxx:146-200).
 *  - Calls enqueue work on the domain's CUDA stream and return; calls that
 *    deliver data to the host synchronise that stream first, so a program sees
 *    the blocking semantics of ASL's acl::Kernel::compute()
 *    (src/acl/Kernels/aclKernel.cxx:289-313).
 *  - Not thread-safe per handle, as in the reference.
 */
#ifndef ASLB_H
#define ASLB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASLB_OK 0
#define ASLB_ERR_ARG (-1)
#define ASLB_ERR_CUDA (-2)
#define ASLB_ERR_NOMEM (-3)
#define ASLB_ERR_STATE (-4)

/* storage of the populations */
#define ASLB_F32 0 /* FP32 populations, FP32 arithmetic (ASL with FlT=float) */
#define ASLB_F16 1 /* FP16 shifted deviations (f-1)*scale, FP32 arithmetic */
#define ASLB_F64 2 /* FP64 populations and arithmetic (ASL with FlT=double) */

/* aslb_lbgk_create flags */
#define ASLB_NO_VELOCITY 1u    /* LBGK(..., compVel=false, ...)            */
#define ASLB_NO_RHO 2u         /* LBGK(..., compRho=false, ...)            */
#define ASLB_INCOMPRESSIBLE 4u /* LBGK::setCompressible(false)             */
#define ASLB_PERIODIC_X 8u     /* extension: periodic axes (no ASL analogue) */
#define ASLB_PERIODIC_Y 16u
#define ASLB_PERIODIC_Z 32u
/* extension: z rows stored back to back instead of each row's first interior
 * cell on a 128-byte boundary. Fewer HBM bytes when rows are short (below
 * about 100 FP32 cells: the +-1 z neighbours then share the fetched pieces
 * of the adjacent rows); results are identical. The TMA-staged kernel
 * (variant 1) needs aligned rows and is unavailable. */
#define ASLB_PACKED_ROWS 64u

/* closures (aslb_lbgk_set_closure) */
#define ASLB_CLOSURE_NONE 0        /* asl::LBGK                                        */
#define ASLB_CLOSURE_ASL_INTENT 1  /* asl::LBGKTurbulence, f_eq evaluated before use     */
#define ASLB_CLOSURE_SMAGORINSKY 2 /* extension: Smagorinsky, Hou et al. (1996)          */
#define ASLB_CLOSURE_MLP 3         /* extension: learned Cs^2 from a 9-64-64-1 network  */

/* boundary conditions (slice kinds 0-3, map kinds 10-13) */
#define ASLB_BC_NOSLIP 0
#define ASLB_BC_VELOCITY 1
#define ASLB_BC_PRESSURE 2
#define ASLB_BC_PRESSURE_VELOCITY 3
#define ASLB_BC_MAP_NOSLIP 10
#define ASLB_BC_MAP_VELOCITY 11
#define ASLB_BC_MAP_VELOCITY_ROTATION 12
#define ASLB_BC_MAP_PRESSURE_VELOCITY 13
#define ASLB_BC_MAP_TRANSPORT_DEPOSITION 14
#define ASLB_BC_MAP_KINETICS_DEPOSITION 15
#define ASLB_BC_FIELD_NOSLIP_VEL 20
#define ASLB_BC_FIELD_NOSLIP_RHO 21
#define ASLB_BC_FIELD_VELOCITY_VEL 22
#define ASLB_BC_FIELD_VELOCITY_VEL_ROTATION 23

/* walls for slice BCs: bit w for asl::SlicesNames {X0,XE,Y0,YE,Z0,ZE}
 * (src/num/aslBCond.h:309) */
#define ASLB_WALL(w) (1u << (w))

/* fields for aslb_lbgk_read / aslb_lbgk_write */
#define ASLB_FIELD_RHO 0
#define ASLB_FIELD_VELOCITY 1
#define ASLB_FIELD_F 2
#define ASLB_FIELD_CS2 3 /* learned closure: the Cs^2 field the next step uses */

typedef struct aslb_lbgk aslb_lbgk;
typedef struct aslb_bc aslb_bc;
typedef struct aslb_force aslb_force;
typedef struct aslb_force aslb_flux;
typedef struct aslb_fd aslb_fd;
typedef struct aslb_fd_bc aslb_fd_bc;
typedef struct aslb_batch aslb_batch;

/* Last error message of the calling thread ("" if none). */
const char* aslb_last_error(void);
/* Library version string. */
const char* aslb_version(void);
/* Select the CUDA device used by subsequent create calls
 * (ApplicationParametersManager --device, src/acl/aclHardware.cxx:98-120). */
int aslb_set_device(int device);
/* Wait until every launch and copy the library queued on the selected device
 * has finished. ASL's kernels block the host (src/acl/aclKernel.cxx:311), so
 * a program's Timer measures finished work; the C++ API's Timer::start/stop
 * call this so that it still does when steps are queued asynchronously. */
int aslb_synchronize(void);

/* ---- LBGK domain ------------------------------------------------------- */

/* asl::LBGK::LBGK(Block b, Param nu, const VectorTemplate* vT, bool compVel,
 *                 bool compRho, CommandQueue)  (src/num/aslLBGK.cxx:114-158).
 * q = 15, 19 or 27; storage = ASLB_F32/F16/F64 (ASL selects FP32/FP64 by the
 * type of nu). Allocates the populations once (AA pattern: one copy, not
 * ASL's 2L+4m pool), density and velocity fields, and a CUDA stream. */
int aslb_lbgk_create(int nx, int ny, int nz, int q, int storage, double nu, unsigned flags, aslb_lbgk** out);
int aslb_lbgk_destroy(aslb_lbgk* h);

/* CUDA stream the domain enqueues on (cudaStream_t as void*). set_stream
 * replaces it with a caller-owned stream (NULL restores the own stream). */
void* aslb_lbgk_stream(aslb_lbgk* h);
int aslb_lbgk_set_stream(aslb_lbgk* h, void* stream);

/* LBGK::setViscosity / getViscosity (declared, never defined in the reference:
 * src/num/aslLBGK.h:117-118). */
int aslb_lbgk_set_viscosity(aslb_lbgk* h, double nu);
double aslb_lbgk_get_viscosity(aslb_lbgk* h);
/* LBGK::setCompressible (src/num/aslLBGK.h:198-201). */
int aslb_lbgk_set_compressible(aslb_lbgk* h, int compressible);
/* LBGK::setOmega: angular velocity of the rotating frame (Coriolis term,
 * src/num/aslLBGK.cxx:207-208,252-255). */
int aslb_lbgk_set_omega(aslb_lbgk* h, const double omega[3]);
/* Which of rho / u the step writes (compVel/compRho of the constructor). */
int aslb_lbgk_set_macro_output(aslb_lbgk* h, int comp_vel, int comp_rho);
/* Write rho and u on the next step only, whatever the flags say. */
int aslb_lbgk_request_macro(aslb_lbgk* h);
/* Extension: body force per unit mass (Guo et al. 2002 forcing). */
int aslb_lbgk_set_body_force(aslb_lbgk* h, const double g[3]);
/* asl::LBGKTurbulence (src/num/aslLBGK.cxx:298-355) and extensions; cs is the
 * Smagorinsky constant (ignored otherwise). */
int aslb_lbgk_set_closure(aslb_lbgk* h, int closure, double cs);
/* Learned closure network (extension standing in for LBGKTurbulence's
 * limiter): `bytes` of the packed device layout produced by the training code
 * (see aslb_mlp_layout_bytes). Copied to the device. With closure
 * ASLB_CLOSURE_MLP, every `period` steps (aslb_lbgk_set_mlp_period, default
 * 32) a tensor-core kernel evaluates the network on the invariants of every
 * cell's non-equilibrium stress and stores a Cs^2 field; each step then
 * applies the Smagorinsky closed form with that cell's Cs^2. D3Q19 / D3Q27,
 * FP32 or FP16 storage. */
size_t aslb_mlp_layout_bytes(void);
int aslb_lbgk_set_mlp(aslb_lbgk* h, const void* net_host, size_t bytes);
int aslb_lbgk_set_mlp_period(aslb_lbgk* h, int steps);
/* The network's nine input features of every interior cell, before
 * normalisation, from the populations the next step reads: out_dev is DEVICE
 * memory of 9 * nx * ny * nz floats, feature-major, cells x-major with z
 * fastest. Training data for the closure. Synchronises. */
int aslb_lbgk_closure_features(aslb_lbgk* h, float* out_dev);
/* FP16 storage scale: stored half = (f - 1) * scale (default 1024). */
int aslb_lbgk_set_fp16_scale(aslb_lbgk* h, double scale);
/* Physical position of interior cell (0,0,0) and the spacing
 * (asl::Block::position / dx, src/data/aslBlocks.h:56-88). */
int aslb_lbgk_set_position(aslb_lbgk* h, const double pos0[3], double dx);
/* Domain shape: out[0..2] interior sizes, out[3] q, out[4] storage,
 * out[5] flags. */
int aslb_lbgk_shape(aslb_lbgk* h, int out[6]);

/* LBGKUtilities::initF(rho, vel) with constants (src/num/aslLBGK.cxx:262-280). */
int aslb_lbgk_init_f(aslb_lbgk* h, double rho, const double u[3]);
/* initF with fields: rho (L doubles, or NULL for 1) and u (3L doubles), host. */
int aslb_lbgk_init_f_fields(aslb_lbgk* h, const double* rho, const double* u);

/* asl::LBGK::LBGK(DataD v, Param nu, const VectorTemplate*) and
 * LBGKTurbulence(DataD v, ...) (src/num/aslLBGK.h:112,165; src/num/aslLBGK.cxx:
 * 95-112): the domain writes its velocity into the caller's container
 * instead of its own. u_dev is DEVICE memory of 3 * L values (float; double
 * for FP64 storage) in ASL's ghosted layout, owned by the caller and valid
 * until it is unbound (NULL restores the domain's own field). Every later
 * velocity write, read and FD binding uses it. Synchronises the domain's
 * stream. */
int aslb_lbgk_bind_velocity(aslb_lbgk* h, void* u_dev);
/* LBGKUtilities::computeRho / computeVelocity / computeRhoVelocity (declared,
 * never defined in the reference: src/num/aslLBGK.h:153-155): rho = sum w_i f_i
 * and u = m / rho (m for the incompressible equilibrium), m = sum w_i c_i f_i,
 * of every interior cell from the populations as they stand (the
 * post-collision values of the last step), into the domain's density and / or
 * velocity fields. Enqueued on the domain's stream. */
int aslb_lbgk_compute_macro(aslb_lbgk* h, int comp_rho, int comp_vel);

/* LBGK::execute(): one stream + collide step (src/num/aslLBGK.cxx:237-250,
 * src/num/aslSingleKernelNM.cxx:48-53), nsteps times. Boundary conditions are
 * separate objects, executed by the caller after each step as in ASL. */
int aslb_lbgk_step(aslb_lbgk* h, int nsteps);
/* The reference's time loop `for n: lbgk->execute(); executeAll(bc);`
 * (examples/flow/flow.cc:124-134) as one call. use_graph != 0 records two
 * steps into a CUDA graph once and replays it. */
int aslb_lbgk_run(aslb_lbgk* h, int nsteps, aslb_bc* const* bcs, int nbc, int use_graph);
/* Extension (no ASL analogue): one step split into parts, for overlapping
 * the face exchange of an x-slab decomposition with the interior.
 * aslb_lbgk_step_planes launches the stream-collide of interior x planes
 * x_first .. x_last (1-based) at the current AA parity on `stream` (NULL: the
 * domain's stream; the caller orders it against the domain's other work),
 * without advancing the step; aslb_lbgk_step_commit then advances the step
 * count and parity once every plane has been launched exactly once. Not for
 * x-periodic domains or the learned closure. Parts of one step touch disjoint
 * population slots, so they may run concurrently. */
int aslb_lbgk_step_planes(aslb_lbgk* h, int x_first, int x_last, void* stream);
int aslb_lbgk_step_commit(aslb_lbgk* h);
/* Wait for all work of the domain; fails with ASLB_ERR_STATE if a kernel's
 * bounded wait gave up. */
int aslb_lbgk_sync(aslb_lbgk* h);
/* Stream-collide kernel variant: 0 (default) loads directly, two cells per
 * thread for the plain FP32/FP16 D3Q15/D3Q19 step with fused no-slip links
 * (one cell per thread otherwise); 1 stages
 * every tile's population rows in shared memory with asynchronous bulk copies
 * (TMA) in a persistent, pipelined kernel; 2 loads directly, one cell per
 * thread. All give identical results. */
int aslb_lbgk_set_kernel(aslb_lbgk* h, int variant);
int aslb_lbgk_get_kernel(aslb_lbgk* h);
/* Steps taken so far. */
long long aslb_lbgk_steps(aslb_lbgk* h);

/* Host copies in ASL layout (they synchronise): RHO (L), VELOCITY (3L),
 * F (q*L, post-collision populations f*_i). dtype is ASLB_F32 (float) or
 * ASLB_F64 (double). getRho()/getVelocity()/getF() + acl::map
 * (src/acl/DataTypes/aclMemBlock.cxx:111-136). */
int aslb_lbgk_read(aslb_lbgk* h, int field, int dtype, void* host_out);
/* Load populations (field F only), ASL layout; used for restart. */
int aslb_lbgk_write(aslb_lbgk* h, int field, int dtype, const void* host_in);
/* Restart dump (the role of ASL's ABD dumps, src/writers/aslABDFormat.h:45-137;
 * ASL itself keeps the population pools protected): the population array
 * exactly as stored (storage format, current AA representation, padding),
 * aslb_lbgk_state_bytes(h) bytes, plus meta = {steps, parity, fused-links
 * active, storage}. Loading it into a domain of the same size, lattice,
 * storage and conditions continues bit for bit where the dumped domain
 * stood. A learned-closure domain recomputes its Cs^2 field at the first
 * step after a load. */
size_t aslb_lbgk_state_bytes(aslb_lbgk* h);
int aslb_lbgk_save_state(aslb_lbgk* h, void* host_out, size_t bytes, long long meta[4]);
int aslb_lbgk_load_state(aslb_lbgk* h, const void* host_in, size_t bytes, const long long meta[4]);
/* Device pointer of RHO or VELOCITY (ASL layout; float, double for F64). */
void* aslb_lbgk_device_field(aslb_lbgk* h, int field);
/* Extension (no ASL analogue): x-slab decomposition across GPUs. A domain
 * whose x range is split into slabs (one LBGK per slab, not x-periodic, its
 * ghost planes x = 0 and nx + 1 standing for the neighbours' boundary planes)
 * exchanges after every step, before that step's separate conditions, one
 * face buffer per neighbour: aslb_lbgk_halo_pack(h, face, buf) fills the
 * buffer the neighbour across `face` (0 = low x, 1 = high x) needs now, and
 * the neighbour passes it to aslb_lbgk_halo_unpack(h, its opposite face, buf).
 * Buffers are DEVICE memory of aslb_lbgk_halo_bytes(h) bytes (the directions
 * crossing the face, one x plane each); the copies are enqueued on the
 * domain's stream. Which plane and directions move depends on the parity
 * (aslb_lbgk_parity: 0 after an even number of steps). */
size_t aslb_lbgk_halo_bytes(aslb_lbgk* h);
int aslb_lbgk_halo_pack(aslb_lbgk* h, int face, void* dev_out);
int aslb_lbgk_halo_unpack(aslb_lbgk* h, int face, const void* dev_in);
int aslb_lbgk_parity(aslb_lbgk* h);
/* Global FP64 moments of the post-collision populations over interior cells:
 * out[0] mass, out[1..3] momentum (a blow-up watchdog). Synchronises. */
int aslb_lbgk_moments(aslb_lbgk* h, double out[4]);
/* Extension (no ASL analogue): blow-up watchdog over the interior cells
 * (solid ones included), from the post-collision populations in FP64:
 * out[0] the largest |u| (u = m / rho; m for the incompressible
 * equilibrium), out[1] the smallest rho, out[2] the number of cells whose
 * rho or u is not finite. Synchronises. */
int aslb_lbgk_watchdog(aslb_lbgk* h, double out[3]);

/* ---- boundary conditions ----------------------------------------------- */

/* generateBCNoSlip / generateBCConstantVelocity / generateBCConstantPressure /
 * generateBCConstantPressureVelocity on walls (src/num/aslLBGKBC.cxx:745-798,
 * point lists src/num/aslBCond.cxx:373-510). wallmask: ASLB_WALL bits. */
int aslb_bc_slice_create(aslb_lbgk* h, int kind, unsigned wallmask, double p, const double u[3], aslb_bc** out);
/* Map BCs on a distance map (L floats, host, ASL layout; map > 0 fluid):
 * generateBCNoSlip(map), generateBCVelocity(PF, map) with a constant field or
 * a rotation field u = omega x (r - center), generateBCConstantPressure(map) /
 * generateBCConstantPressureVelocity(map) (src/num/aslLBGKBC.cxx:205-438). */
int aslb_bc_map_create(aslb_lbgk* h, int kind, const float* map, double p, const double u[3], const double omega[3],
                       const double center[3], aslb_bc** out);
/* The same with a computational-domain map (L floats, host; NULL for none):
 * a neighbour is a fluid end only where map > 0 and cdomain > 0, as in
 * generateBCVelocity(nm, v, map, computationalDomain)
 * (src/num/aslLBGKBC.cxx:273-282, 837-844; src/num/aslBCond.cxx:204-211). */
int aslb_bc_map_create_cd(aslb_lbgk* h, int kind, const float* map, const float* cdomain, double p, const double u[3],
                          const double omega[3], const double center[3], aslb_bc** out);
/* The velocity set the kernels use (host copy, no device needed):
 * VectorTemplate::vectors, quasiparticlesCoefs and invertVectors of d3q15 /
 * d3q19 / d3q27 (src/math/aslTemplates.cxx:30-83, 146-200; D3Q27 with the
 * standard weights, the reference's d3q27 has none). c: 3q ints, w: q, inv: q. */
int aslb_lattice(int q, int* c, double* w, int* inv);
/* Conditions on the output fields near a map, for visualisation
 * (generateBCNoSlipVel / generateBCNoSlipRho / generateBCVelocityVel,
 * src/num/aslLBGKBC.cxx:808-852 -> src/num/aslBasicBC.cxx:110-230, 300-350),
 * on guard cells -0.9999 < map <= 0 of the domain's velocity / density
 * fields (the domain must write them): FIELD_NOSLIP_VEL sets u to the
 * middle-point zero value (laplacian-weighted 2*0 - u of fluid neighbours);
 * FIELD_NOSLIP_RHO gives rho a zero normal gradient (neighbours weighted by
 * (n . c/|c| + 1)^2, n the map's unit normal); FIELD_VELOCITY_VEL(_ROTATION)
 * sets u = v (constant u, or omega x (r - center)). Executed like any
 * condition, after the step that wrote the fields. D3Q15 and D3Q19 only
 * (ASL's d3q27 template has no laplacian or gradient coefficients). */
int aslb_bc_field_create(aslb_lbgk* h, int kind, const float* map, const double u[3], const double omega[3],
                         const double center[3], aslb_bc** out);
/* Deposition on a map surface (generateBCTransportLimitedDeposition(nm, p0,
 * limitingFactor, map) and generateBCKineticsLimitedDeposition(nm, p0,
 * limitingFactor, beta, map) in the argument order of their definitions,
 * src/num/aslLBGKBC.cxx:878-903; BCTransportLimitedDepositionMap /
 * BCKineticsLimitedDepositionMap :440-598). Per solid cell x with fluid
 * neighbours: rho = sum_k w_k f_inv(k)(x + c_k), coef = sum_k w_k; transport
 * limited j = rho - (rho - coef p0) / (1 + coef lF), kinetics limited
 * j = rho - beta (rho / coef - p0) / (1 + lF); f_k(x) = j / coef on every
 * link. kind: ASLB_BC_MAP_TRANSPORT_DEPOSITION (beta unused) or
 * ASLB_BC_MAP_KINETICS_DEPOSITION. */
int aslb_bc_deposition_create(aslb_lbgk* h, int kind, const float* map, double p0, double limiting_factor,
                              double beta, aslb_bc** out);
/* Extension (no ASL analogue): fold a no-slip condition (walls or map) into
 * the stream-collide kernel, removing its separate launch. Fluid cells read
 * bounce-back populations inline and solid cells skip the writes the
 * condition would overwrite; every cell evolves exactly as with the separate
 * condition (populations read back through aslb_lbgk_read are identical),
 * provided no condition executed after it writes the same links (ASL: later
 * writers win). aslb_lbgk_run enforces that fused conditions come last.
 * Like any condition it must be executed after every step (aslb_bc_execute
 * or aslb_lbgk_run): after initF or a population write, the steps read the
 * initial values until a fused condition has been executed, as in ASL. */
int aslb_bc_fuse(aslb_bc* bc);
int aslb_bc_is_fused(aslb_bc* bc);
/* BCond::execute() (src/num/aslLBGKBC.cxx:80-83, 257-260). */
int aslb_bc_execute(aslb_bc* bc);
int aslb_bc_destroy(aslb_bc* bc);
/* Number of boundary links (direction slots written per execute). */
long long aslb_bc_num_links(aslb_bc* bc);
/* Kernel launches one execute makes (0 for a fused condition). */
int aslb_bc_kernels(aslb_bc* bc);

/* ---- surface force ------------------------------------------------------- */

/* generateComputeSurfaceForce(lbgk, forceField, map)
 * (src/num/aslLBGKBC.cxx:674-742, 915-921). */
int aslb_force_create(aslb_lbgk* h, const float* map, aslb_force** out);
/* ComputeSurfaceForceMap::execute() plus the FP64 reduction the reference
 * lacks: out6 = (sum F, sum (r - r0) x F). field_host (3L floats, optional)
 * receives the per-cell force field. Synchronises. */
int aslb_force_compute(aslb_force* fc, const double r0[3], float* field_host, double out6[6]);
int aslb_force_destroy(aslb_force* fc);
/* No counterpart in the reference. The same totals as aslb_force_compute
 * (without the per-cell field) for callers that cannot allocate device memory
 * when they need them: a host program whose device memory is managed by an
 * allocator that forbids new allocations after set-up, or an embedding
 * runtime that hands out all device memory up front. It calls no cudaMalloc
 * or cudaFree and keeps its partial sums in a fixed array of the library's
 * device memory (196,672 bytes per device, held until exit). Lists of more
 * than 1,048,576 force cells are rejected with ASLB_ERR_ARG. The domain's
 * device must be current; the first call on each device looks up the
 * array's device address (a lookup, not an allocation; safe from several
 * host threads). All calls share the array and each call overwrites what the
 * previous one left there: calls whose work overlaps on the GPU (different
 * streams) race. Synchronises the domain's stream. */
int aslb_force_compute_noalloc(aslb_force* fc, const double r0[3], double out6[6]);

/* ---- surface flux -------------------------------------------------------- */

/* generateComputeSurfaceFlux(lbgk, fluxField, map) (src/num/aslLBGKBC.cxx:
 * 623-665, 906-912): per cell with |map| < 0.9999, flux = sum_k w_k
 * (f_k(x) - f_inv(k)(x + c_k)) over links from a solid x to fluid neighbours
 * minus the same over links from a fluid x to solid neighbours. field_host
 * (L floats, optional) receives the flux field (cells off the surface hold
 * 0), total (optional) its FP64 sum. Synchronises. */
int aslb_flux_create(aslb_lbgk* h, const float* map, aslb_flux** out);
int aslb_flux_compute(aslb_flux* fx, float* field_host, double* total);
int aslb_flux_destroy(aslb_flux* fx);

/* ---- learned closure: training (extension, no ASL analogue) ------------ */

/* The network's own training kernels. All pointers are DEVICE memory except
 * in aslb_mlp_pack; `stream` is a cudaStream_t (null: the default stream).
 * Parameters: aslb_mlp_param_count() FP32 values, W1[64][9], b1[64],
 * W2[64][64], b2[64], w3[64], b3. Model: x' = (x - norm[0:9]) * norm[9:18],
 * h1 = relu(W1 x' + b1), h2 = relu(W2 h1 + b2), y = w3.h2 + b3,
 * Cs^2 = out_scale * softplus(y); loss = mean over samples of (Cs^2 - t)^2. */
int aslb_mlp_param_count(void);
/* Scratch the gradient kernel needs, in floats. */
size_t aslb_mlp_grad_scratch_floats(void);
/* Gradient of the loss over n samples (x: 9 x n floats, feature-major; t: n
 * targets) into grad_loss[0 .. P-1], and the sum of squared errors into
 * grad_loss[P]. Deterministic (fixed reduction order). */
int aslb_mlp_grad(const float* params, const float* x, const float* t, long long n, const float* norm,
                  float out_scale, float* scratch, float* grad_loss, void* stream);
/* One Adam step (Kingma & Ba 2015) of the parameters; step counts from 1. */
int aslb_mlp_adam(float* params, const float* grad, float* m, float* v, int step, float lr, float beta1,
                  float beta2, float eps, void* stream);
/* HOST memory: the inference layout (aslb_mlp_layout_bytes() bytes, weights
 * rounded to BF16) from FP32 parameters and the input normalisation. */
int aslb_mlp_pack(const float* params_host, const float* norm_host, float out_scale, void* net_host);

/* ---- batches of independent domains ------------------------------------ */

/* Extension (no ASL analogue; an ASL program steps each LBGK object with its
 * own execute() and executeAll(bc), src/num/aslNumMethod.h:47-77): advance many
 * independent domains together. One persistent stream-collide launch per step
 * covers every domain, and the k-th separate condition of every domain is one
 * link launch; the whole step is replayed from a CUDA graph. The domains must
 * share lattice, storage and device; aslb_batch_run also requires the same
 * parity, the plain BGK collision (no closure) and equal batch-wide
 * parameters (body force, rotation, compressibility, FP16 scale, output
 * fields); viscosity, size, geometry and conditions are per domain. The batch
 * refers to its domains: destroying a domain detaches it and later runs fail
 * with ASLB_ERR_STATE. Each domain's pending work is waited for, and its later
 * work waits for the batch. */
int aslb_batch_create(aslb_lbgk* const* domains, int n, aslb_batch** out);
/* nsteps steps of every domain. bcs: the conditions of domain 0 in ASL's
 * order, then those of domain 1, ...; nbc[i] of them for domain i (fused
 * no-slip conditions last, as in aslb_lbgk_run). Velocity maps and links
 * across periodic faces are not batched (ASLB_ERR_ARG). use_graph as in
 * aslb_lbgk_run. */
int aslb_batch_run(aslb_batch* b, int nsteps, aslb_bc* const* bcs, const int* nbc, int use_graph);
int aslb_batch_sync(aslb_batch* b);
/* Tiles (x planes) of one batched step, over all domains. */
long long aslb_batch_tiles(aslb_batch* b);
/* Launch shape of the batched step: shape 0, 1, 2: one cell per thread at
 * 4, 3, 2 resident blocks of 256 threads per SM; 3, 4: two cells per thread
 * at 3, 2 blocks (D3Q15 / D3Q19, FP32 / FP16, one-word link masks; other
 * batches take the one-cell shape of the same residency). By default (or
 * after shape -1) the first
 * aslb_batch_run that records a graph first times two real steps with every
 * shape and keeps the fastest (all shapes give identical results);
 * aslb_batch_shape_times returns those timings (ms, up to n; the count). */
int aslb_batch_set_shape(aslb_batch* b, int shape);
int aslb_batch_get_shape(aslb_batch* b);
int aslb_batch_shape_times(aslb_batch* b, float* ms_out, int n);
int aslb_batch_destroy(aslb_batch* b);

/* ---- workload geometry (host) ----------------------------------------- */

/* Extension (no ASL analogue; ASL builds such media from user distance
 * functions): seeded random sequential addition of non-overlapping spheres in
 * an nx x ny x nz box, radii uniform in [rmin, rmax] placed largest first until
 * their volume reaches solid_fraction of the box. Spheres stay inside y and z;
 * x wraps when periodic_x. centers (3 * max_spheres doubles, interior-cell
 * coordinates) and radii (max_spheres) receive *count spheres. */
int aslb_geom_pack_spheres(int nx, int ny, int nz, double rmin, double rmax, double solid_fraction,
                           unsigned long long seed, int periodic_x, int attempts, int max_spheres, double* centers,
                           double* radii, int* count);

/* ---- FD advection-diffusion coupled to the flow -------------------------- */

/* generateFDAdvectionDiffusion(c, D, v, template[, compressibilityCorrection])
 * (src/num/aslFDAdvectionDiffusion.cxx:88-180, 209-226), one component, no
 * electric field: per interior cell
 *   c' = D lap(c) + c - divProduct(v, c)
 * and, with the correction, c' /= 1 - div(v); c' += lap(c) |v(x)|^2 / 2,
 * with the template operators of src/math/aslTemplateVE.cxx:164-267 on
 * q = 7, 15 or 19 (d3q7 / d3q15 / d3q19). c is an (nx+2)(ny+2)(nz+2) field
 * in ASL layout (dtype ASLB_F32 or ASLB_F64); ghost values are never
 * written by a step, so they act as fixed boundary values. */
int aslb_fd_create(int nx, int ny, int nz, int q, int dtype, double D, aslb_fd** out);
/* setVelocity(lbgk->getVelocity(), compressibilityCorrection): reads the
 * domain's device velocity field and runs on the domain's stream (after its
 * steps, in order). Same size; dtype ASLB_F64 for FP64 storage, ASLB_F32
 * otherwise. NULL unbinds. Destroying the domain unbinds it. */
int aslb_fd_set_velocity(aslb_fd* fd, aslb_lbgk* h, int compressibility_correction);
int aslb_fd_set_diffusion(aslb_fd* fd, double D);
/* setElectricFieldParameters(phi, k, f2, q) (src/num/aslFDAdvectionDiffusion.cxx:
 * 66-74, 166-172; f2 is unused there): each step also subtracts
 * divAgradB(c q / k, phi) = sum_i GC_i (a_i + a_0) (phi_i - phi_0), a = c q / k.
 * phi, k, q: host arrays of L values in the FD's dtype, copied to the device;
 * all three NULL removes the term. */
int aslb_fd_set_electric_field(aslb_fd* fd, int dtype, const void* phi, const void* k, const void* q);
/* Host copies of c (ghosted, L values of dtype); writing resets both buffers. */
int aslb_fd_write(aslb_fd* fd, int dtype, const void* host_in);
int aslb_fd_read(aslb_fd* fd, int dtype, void* host_out);
/* generateBCConstantValue(c, value, {faces}) (src/num/aslBasicBC.cxx:51-57;
 * faces as ASLB_WALL bits): the face ghost layers (interior tangential
 * indices) hold value from now on. */
int aslb_fd_set_face_value(aslb_fd* fd, unsigned wallmask, double value);
/* Conditions on c at a map surface, executed like ASL's (after each FD step,
 * asynchronous on the FD's stream), on guard cells -0.9999 < map <= 0 (map:
 * host floats in the FD's ghosted layout): ASLB_FD_BC_VALUE_MAP sets
 * c = value (generateBCConstantValue(c, v, map): BCConstantValueMap,
 * src/num/aslBasicBC.cxx:71-108); ASLB_FD_BC_GRADIENT_MAP sets a normal
 * gradient `value` (generateBCConstantGradient(c, v, map, template):
 * BCConstantGradientMap, :271-350): c = sum_k W_k (c(x + e_k) - (n.e_k/|e_k|)
 * value) / sum_k W_k over fluid neighbours (map > 0, interior) of the FD's
 * template, W_k = (n.e_k/|e_k| + 1)^2, n the unit map gradient. */
#define ASLB_FD_BC_VALUE_MAP 0
#define ASLB_FD_BC_GRADIENT_MAP 1
int aslb_fd_bc_create(aslb_fd* fd, int kind, const float* map, double value, aslb_fd_bc** out);
int aslb_fd_bc_execute(aslb_fd_bc* bc);
long long aslb_fd_bc_cells(aslb_fd_bc* bc);
int aslb_fd_bc_destroy(aslb_fd_bc* bc);
/* execute() n times (asynchronous on the FD's stream). */
int aslb_fd_step(aslb_fd* fd, int n);
int aslb_fd_sync(aslb_fd* fd);
/* Device pointer of the current c (valid until the next step). */
void* aslb_fd_device_field(aslb_fd* fd);
int aslb_fd_destroy(aslb_fd* fd);

/* ---- surfaces (readSurface) -------------------------------------------- */

/* Triangles of an STL file, binary or ASCII (the STL branch of ASL's
 * readSurface, src/readers/aslVTKFormatReaders.cxx:266-345, which reads it with
 * vtkSTLReader): *ntri triangles of 9 floats (x0 y0 z0 x1 ... z2, file
 * coordinates) into tri when tri is not NULL and cap >= *ntri. */
int aslb_read_stl(const char* path, float* tri, long long cap, long long* ntri);
/* Distance map of a triangle surface on a gx x gy x gz grid whose cell
 * (i, j, k) sits at pos0 + (i, j, k) dx (x slowest, z fastest): d = distance
 * to the nearest triangle, exact within `band` of the surface, `band` beyond;
 * with solid_interior, cells inside the closed surface take -d. Writes
 * map = (d - offset) / scale (FP32, gx*gy*gz). ASL's surfaceToData
 * (src/readers/aslVTKFormatReaders.cxx:136-210, VTK's implicit modeller)
 * samples the unsigned distance and maps it with offset 1.2 dx, scale 1.8 dx
 * (block overload) or 1.8 dx, 1.8 dx (spacing overloads): solid_interior = 0.
 * Runs on the current device. */
int aslb_surface_map(const float* tri, long long ntri, int gx, int gy, int gz, const double pos0[3], double dx,
                     double band, int solid_interior, double offset, double scale, float* map_host);

#ifdef __cplusplus
}
#endif
#endif /* ASLB_H */
