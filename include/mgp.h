/*
 * mgp.h -- C ABI of the B200-native geometric multigrid Poisson engine (libmgp.so).
 *
 * Plain C: pointers, sizes and status codes only.  This is the drop-in boundary under the
 * reference's public solver API, Poisson::PoissonSolver<T,Restriction,Prolongation,Relaxation>
 * of eljens/multigrid-poisson (include/libpoisson.h:28-67).  Each entry point names the
 * reference interface it replaces.  The C++ header facade in
 * multigrid-poisson_b200/poisson/libpoisson.h rebuilds that class on top of these calls.
 *
 * Conventions
 *  - Every function returns an int status (mgp_status).  On failure a message is kept per
 *    thread and returned by mgp_last_error().
 *  - Host arrays exchanged with the engine use the reference's own halo-padded layout
 *    (include/array.h:20-30,70-77):
 *        idx(i,j,k) = (i+halo.west)*stride[0] + (j+halo.south)*stride[1] + (k+halo.bottom)
 *        stride = {pad[1]*pad[2], pad[2], 1}, pad = shape + halo
 *    mgp_level_info() returns shape, halo, pad, stride and size for every level.
 *    Element type is double for MGP_F64 solvers and float for MGP_F32 solvers.
 *  - Face (boundary-condition) arrays have no halo and the reference's face shapes
 *    (include/domain.h:125-192): north/south (nx,1,nz), east/west (1,ny,nz),
 *    top/bottom (nx,ny,1), k unit-stride.
 *  - A solver owns all device memory of its level hierarchy, one CUDA stream and its cached
 *    CUDA graphs.  A solver is not thread-safe; use one solver per host thread (the
 *    reference's solver is not thread-safe either: GaussSeidel::alternate is mutable state).
 */
#ifndef MGP_H
#define MGP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGP_ABI_VERSION 1

/* Status codes.  The C++ facade maps INVALID_ARG to std::invalid_argument (reference:
 * bad solver name include/libpoisson.h:242-244, bad dims src/domainsettings.cpp:20-27) and
 * NO_DEVICE to std::runtime_error (include/devicearray.h:117-119). */
typedef enum {
    MGP_OK = 0,
    MGP_ERR_INVALID_ARG = 1,
    MGP_ERR_OOM = 2,
    MGP_ERR_NO_DEVICE = 3,
    MGP_ERR_CUDA = 4,
    MGP_ERR_TIMEOUT = 5,
    MGP_ERR_DIVERGED = 6,
    MGP_ERR_UNSUPPORTED = 7,
    MGP_ERR_STATE = 8
} mgp_status;

/* Boundary_t (include/boundary.h:14). */
typedef enum { MGP_DIRICHLET = 0, MGP_NEUMANN = 1 } mgp_bc;
/* Location_t order (include/boundary.h:12) -- also the field order of BoundaryCondition
 * (include/boundary.h:23-30). */
typedef enum { MGP_NORTH = 0, MGP_SOUTH = 1, MGP_EAST = 2, MGP_WEST = 3, MGP_TOP = 4, MGP_BOTTOM = 5 } mgp_face;
/* Template plug-ins R, P, S of PoissonSolver<T,R,P,S>. */
typedef enum { MGP_INJECTION = 0, MGP_FULLWEIGHTING = 1 } mgp_restriction;
typedef enum { MGP_TRILINEAR = 0 } mgp_prolongation;
typedef enum { MGP_JACOBI = 0, MGP_GAUSSSEIDEL = 1 } mgp_relaxation;
/* T of PoissonSolver<T,...>. */
typedef enum { MGP_F64 = 0, MGP_F32 = 1 } mgp_dtype;
/* DeviceArray members of Domain<T> (include/domain.h:62-65). */
typedef enum { MGP_FIELD_U = 0, MGP_FIELD_UPREV = 1, MGP_FIELD_F = 2, MGP_FIELD_R = 3 } mgp_field;
/* solve("relaxation"|"Vcycle"|"Fcycle") (include/libpoisson.h:239-244). */
typedef enum { MGP_CYCLE_RELAXATION = 0, MGP_CYCLE_V = 1, MGP_CYCLE_F = 2 } mgp_cycle;

/* mgp_desc.flags */
#define MGP_FLAG_STRICT_BC 1u /* honour the requested north/south/bottom kinds instead of the
                                 reference's resolution to Dirichlet (include/domain.h:140-145,191-192) */
#define MGP_FLAG_REFINE_F32 16u /* iterative refinement, FP32 correction hierarchy (see mgp_solve) */
#define MGP_FLAG_REFINE_F64 32u /* iterative refinement, FP64 correction hierarchy */
#define MGP_FLAG_WAVE 256u /* Jacobi levels of >= 2^20 points relax with the TMA-fed wavefront pass: two
                             sweeps, and the residual that follows them, in one march over HBM (same
                             results; one more level-sized buffer per such level).  Off by default: on
                             B200 the pass is bound by instruction issue, not HBM, and takes longer
                             than the separate passes (513x257x129 FP64: two sweeps 234 us against
                             2 x 85 us) */
#define MGP_FLAG_FUSED_SETUP 8u /* cycles form the residual inside the restriction kernel (one
                                   launch, r never stored) on every level; without the flag only
                                   levels of at most 2^20 points do */

/* Settings (include/settings.h:14-39) plus the BoundaryCondition and the template choice. */
typedef struct mgp_desc {
    int64_t dims[3];   /* Settings::dims */
    int64_t levels;    /* Settings::levels */
    int64_t maxiter;   /* Settings::maxiter */
    int64_t miniter;   /* Settings::miniter (reference default 1) */
    double tolerance;  /* Settings::tolerance */
    double h;          /* Settings::h, uniform spacing */
    double origin[3];  /* Settings::origin */
    int32_t bc[6];     /* requested mgp_bc per face, mgp_face order */
    int32_t restriction;
    int32_t prolongation;
    int32_t relaxation;
    int32_t dtype;
    int32_t device;    /* CUDA device ordinal */
    uint32_t flags;
} mgp_desc;

/* Geometry of one level: DomainSettings(l) (src/domainsettings.cpp:12-29) and the
 * host array layout of Domain<T>'s arrays (include/domain.h:102-121). */
typedef struct mgp_level_info {
    int64_t shape[3];
    int64_t halo[6]; /* east, west, north, south, top, bottom (Halo, include/halo.h:6-34) */
    int64_t pad[3];
    int64_t stride[3];
    int64_t size;    /* elements of one host field array */
    double h;
    double origin[3];
    int32_t face_kind[6];      /* resolved mgp_bc per face, mgp_face order */
    int64_t face_shape[6][3];
} mgp_level_info;

/* Results of PoissonSolver::solve: relative_residual(), solve_iterations(), solve_time()
 * (include/libpoisson.h:377-393). */
typedef struct mgp_stats {
    double rel_res;
    double iterations;  /* loop index at exit, as the reference reports it */
    double seconds;
    int64_t cycles_run; /* cycles actually executed */
    double first_rel_res;   /* relative residual before the first cycle */
    int64_t kernel_launches; /* CUDA kernels this call launched (graph nodes included) */
} mgp_stats;

/* mgp_solve flags */
#define MGP_SOLVE_VERBOSE 1u          /* PoissonSolver::verbose(true) prints (:286-288, :337-339) */
#define MGP_SOLVE_PRINT_CYCLE_TIME 2u /* the reference's unconditional "Vcycle took ..." line (:297,:302) */

typedef struct mgp_solver mgp_solver;

const char* mgp_status_string(int status);
/* Last error message of the calling thread ("" if none). */
const char* mgp_last_error(void);
int mgp_abi_version(void);
/* Number of visible CUDA devices (omp_get_num_devices() in the reference drivers). */
int mgp_device_count(int* n);

/* PoissonSolver(Settings&, BoundaryCondition&) (include/libpoisson.h:80-87) with
 * PoissonSolver::alloc (:112-156): builds the level hierarchy (Grid, src/grid.cpp:6-13)
 * and allocates every level's arrays on the device, zero-initialised.
 * Errors: INVALID_ARG for non-coarsenable dims (src/domainsettings.cpp:20-27) or a bad
 * descriptor; UNSUPPORTED for red-black Gauss-Seidel on a layout whose padded z extent is
 * even (the reference's colouring degenerates and its result depends on thread timing);
 * NO_DEVICE; OOM. */
int mgp_create(const mgp_desc* desc, mgp_solver** out);
/* ~PoissonSolver (include/libpoisson.h:100-110). */
int mgp_destroy(mgp_solver* s);
int mgp_level_info_get(const mgp_solver* s, int level, mgp_level_info* out);
/* The same geometry from a descriptor alone, without a device: validates `desc` exactly as
 * mgp_create does (INVALID_ARG for bad dims/levels/kinds, UNSUPPORTED for a degenerate
 * red-black colouring) and fills the host layout of `level` (DomainSettings(l) and the
 * Domain<T> halo widths and face kinds, include/domain.h:100-193). */
int mgp_plan_level(const mgp_desc* desc, int level, mgp_level_info* out);
int mgp_num_levels(const mgp_solver* s);

/* DeviceArray<T>::to_device / to_host (include/devicearray.h:71-110) of one field of one
 * level.  host points to `count` elements in the reference layout of that level
 * (count must equal mgp_level_info.size).  Only shape points are transferred; the halo
 * entries of a host array are left untouched by downloads and ignored by uploads. */
int mgp_upload_field(mgp_solver* s, int field, int level, const void* host, int64_t count);
int mgp_download_field(mgp_solver* s, int field, int level, void* host, int64_t count);
/* Boundary<T>::arr to_device (dirichlet.h:232-235, neumann.h:511-514) and back. */
int mgp_upload_face(mgp_solver* s, int face, int level, const void* host, int64_t count);
int mgp_download_face(mgp_solver* s, int face, int level, void* host, int64_t count);
/* External coupling on the device (the role DeviceArray::devptr plays for codes such as
 * include/poisson_helpers.h:8-34, which fill get_rhs / get_*_bc between init_zero and
 * to_device): the device buffer that holds `field` of `level`, so a caller's own kernels can
 * write or read it without a host round trip.  The layout is the engine's, not the
 * reference's padded host layout: shape points only, k unit-stride,
 *   element (i,j,k) at ptr[i*layout[3] + j*layout[4] + k],  layout = {nx, ny, nz, sx, sy}.
 * The pointer stays valid until the solver is destroyed, but for MGP_FIELD_U / UPREV of a
 * Jacobi solver it names the buffer that holds the field NOW: every sweep swaps the pair, so
 * ask again after relaxing or solving.  Work on the returned memory must be ordered with the
 * solver's stream (mgp_get_stream) by the caller. */
int mgp_field_device(mgp_solver* s, int field, int level, void** ptr, int64_t layout[5]);
/* The same for a face array of `level` (dense, the reference's face layout of shape
 * shape[0] x shape[1] x shape[2], k unit-stride). */
int mgp_face_device(mgp_solver* s, int face, int level, void** ptr, int64_t shape[3]);
/* Domain<T>::write_bc_to(u) and (u_prev) as done at the end of Domain::to_device
 * (include/domain.h:259-262, 318-326): Dirichlet face data into the boundary planes, in
 * the reference's face order so that later faces win on shared edges. */
int mgp_write_bc(mgp_solver* s, int level);

/* PoissonSolver::solve (include/libpoisson.h:237-357) on the device: initial norms, the
 * cycle loop (each iteration one CUDA-graph launch holding the whole cycle plus the fine
 * residual and its max-norm) and the reference's stopping rule.  omega < 0 selects the
 * relaxation's default (6/7 Jacobi, 8/9 Gauss-Seidel).  ofile may be NULL or "" (no log).
 * INVALID_ARG for an F-cycle with fewer than 2 levels (the reference indexes past its
 * hierarchy there). */
int mgp_solve(mgp_solver* s, int cycle, int64_t nsmooth, double omega, const char* ofile, double maxtime,
              uint32_t flags, mgp_stats* out);
/* Settings::maxiter / miniter / tolerance after construction. */
int mgp_set_iteration_limits(mgp_solver* s, int64_t maxiter, int64_t miniter, double tolerance);

/* ---- operator entry points (the reference's operator plug-ins, one level each) ---- */
/* Relaxation<T>::relax (include/relaxation.h:19-94): smoothing_multiplier()*nsmooth
 * half-sweeps (Jacobi ping-pong / red-black SOR) with the Neumann ghost values formed in
 * the kernel. */
int mgp_relax(mgp_solver* s, int level, double omega, int64_t nsmooth);
/* One red-black half-sweep of `level` over the points of colour `colour` (0 or 1: the parity
 * of the reference's padded linear index on this solver's level, the colour
 * GaussSeidel::relaxation_kernel updates in one call, include/gaussseidel.h:28-94), in place,
 * with the solver's alternate flag neither read nor changed.  For callers that order the
 * colours themselves: a domain split into slabs exchanges its halo planes between the two
 * half-sweeps.  UNSUPPORTED for Jacobi solvers. */
int mgp_relax_colour(mgp_solver* s, int level, double omega, int colour);
/* Failure detection of the wavefront passes (MGP_FLAG_WAVE): bound on the polls of a wait for a
 * plane copy (0 = the default, 2^22).  A wait that runs out marks the pass failed; the pass
 * still lets every copy it issued land before it exits, and the next norm read-back (the solve
 * loop's) returns MGP_ERR_TIMEOUT.  No counterpart in the reference (its target regions are
 * synchronous); a test sets a bound of 1 to drive the failure path without a GPU fault. */
int mgp_set_wait_polls(mgp_solver* s, int64_t polls);
/* Relaxation<T>::relax followed by residual<T> (include/relaxation.h:19-94,
 * include/residual.h:17-81) and, when norm != NULL, the max-norm of r over the shape
 * (DeviceArray<T>::infinity_norm, include/devicearray.h:198-240): the solve loop's step on a
 * single level (include/libpoisson.h:294-330).  Same results as mgp_relax, mgp_residual and
 * mgp_norm in turn; on large Jacobi levels the last sweeps and the residual share one pass. */
int mgp_relax_residual(mgp_solver* s, int level, double omega, int64_t nsmooth, double* norm);
/* residual<T>(Domain&) (include/residual.h:17-81). */
int mgp_residual(mgp_solver* s, int level);
/* Restriction<T>::restrict_to(r_l, f_{l+1}) (injection.h:29-67 / fullweighting.h:37-122). */
int mgp_restrict(mgp_solver* s, int level);
/* DeviceArray<T>::init_zero of u_{l} (include/devicearray.h:132-159). */
int mgp_zero_u(mgp_solver* s, int level);
/* The six Boundary<T>::restrict_to calls from level l to l+1 (include/vcycle.h:52-75). */
int mgp_restrict_bc(mgp_solver* s, int level);
/* TrilinearInterpolation::prolong(u_{l+1}, r_l) (include/trilinearinterpolation.h:29-134). */
int mgp_prolong(mgp_solver* s, int level);
/* DeviceArray<T>::add(r_l) into u_l (include/devicearray.h:161-196). */
int mgp_add(mgp_solver* s, int level);
/* prolong followed by add, fused: u_l += P u_{l+1} without materialising P u_{l+1}
 * in r_l's interior (the form the cycles use). */
int mgp_prolong_add(mgp_solver* s, int level);
/* Vcycle<T> / Fcycle<T> from `level` (include/vcycle.h:14-98, include/fcycle.h:13-97). */
int mgp_vcycle(mgp_solver* s, int level, double omega, int64_t nsmooth);
int mgp_fcycle(mgp_solver* s, int level, double omega, int64_t nsmooth);
/* DeviceArray<T>::infinity_norm (include/devicearray.h:198-240), returned as double. */
int mgp_norm(mgp_solver* s, int field, int level, double* out);
/* ---- launch-shape tuning (no counterpart in the reference, whose OpenMP target regions
 * take the runtime's teams) ----
 * Per level: how the kernels of that level cut their work.  None of these changes any
 * value a kernel computes or the order of its arithmetic: results stay bit-identical. */
#define MGP_TUNE_RELAX_PLANES 0 /* planes marched per block by the relaxation (0 = built-in choice) */
#define MGP_TUNE_RESID_PLANES 1 /* planes per block of the residual */
#define MGP_TUNE_NORM_PLANES 2  /* planes per block of the residual + max-norm (solve loop) */
#define MGP_TUNE_SETUP_FORM 3   /* coarse-grid set-up of this level: 0 built-in, 1 three kernels, 2 one kernel */
#define MGP_TUNE_SETUP_PLANES 4 /* coarse planes per block of the one-kernel set-up (0 = built-in) */
#define MGP_TUNE_WAVE 5         /* 0 built-in (wavefront passes where MGP_FLAG_WAVE prepared them), 1 off */
#define MGP_TUNE_TAIL 6         /* level 0 only: 1 runs each cycle visit of the coarsest levels that fit in one
                                   CTA's shared memory as one launch of one block; 0 (built-in) keeps the
                                   grid kernels, which are faster on B200 for the 513x257x129 hierarchy */
#define MGP_TUNE_PROLONG_SWEEP 7 /* prolongation + add fused with the first Jacobi sweep after it (levels >= 1,
                                    nsmooth even): 0 built-in (levels of at most 2^16 points), 1 separate
                                    passes, 2 fused */
#define MGP_TUNE_PARAMS 8
int mgp_set_tuning(mgp_solver* s, int level, int param, int64_t value);
int mgp_get_tuning(mgp_solver* s, int level, int param, int64_t* value);
#define MGP_AUTOTUNE_FORCE 1u /* search again even when the process cache holds this configuration */
/* Searches the parameters above, level by level (coordinate descent), for the fastest solve
 * iteration of (cycle, nsmooth, omega) -- the captured graph of mgp_solve's loop body, timed
 * with CUDA events -- and keeps them on the solver.  Refinement solvers tune their correction
 * hierarchy.  Every field is saved to a device copy first and restored afterwards (needs that
 * much free device memory; MGP_ERR_OOM otherwise).  Results are cached per process
 * by (device, dtype, geometry, boundary kinds, operators, cycle, nsmooth, flags); set
 * MGP_TUNE_CACHE to a file name to keep them across processes.  untuned_ms / tuned_ms (either
 * may be NULL): one iteration with the built-in choices and with the tuned ones, measured
 * after a search (0 when the cache answered). */
int mgp_autotune(mgp_solver* s, int cycle, int64_t nsmooth, double omega, uint32_t flags, double* untuned_ms,
                 double* tuned_ms);

/* Waits for all work queued on the solver's stream. */
int mgp_synchronize(mgp_solver* s);
/* The solver's CUDA stream (a cudaStream_t), for callers that time or order work on it. */
int mgp_get_stream(mgp_solver* s, void** stream);

/* ---- batches: many independent problems solved together ----------------------------
 * A batch holds refinement solvers (FP64 level 0, correction hierarchy in inner_dtype) of any
 * sizes and level counts.  One mgp_batch_step() is one refinement step (correction cycle,
 * u += e, FP64 residual) for every active problem; each level operation is ONE persistent
 * kernel launch over a (problem, tile) work list covering every problem that takes part in
 * it (problems are aligned by depth below their finest level).  No counterpart in the
 * reference, which solves one problem per PoissonSolver. */
typedef struct mgp_batch_desc {
    int32_t restriction;   /* mgp_restriction, shared by all problems */
    int32_t relaxation;    /* mgp_relaxation */
    int32_t inner_dtype;   /* MGP_F32 (mixed precision) or MGP_F64 */
    int32_t cycle;         /* MGP_CYCLE_F or MGP_CYCLE_V */
    int64_t nsmooth;
    double omega;          /* < 0: the relaxation's default */
    int64_t max_problems;  /* capacity (problems resident at once) */
    int32_t device;
    uint32_t flags;
} mgp_batch_desc;
typedef struct mgp_batch mgp_batch;
int mgp_batch_create(const mgp_batch_desc* desc, mgp_batch** out);
int mgp_batch_destroy(mgp_batch* b);
/* Device bytes one problem takes in a batch (for admission by free device memory). */
int mgp_batch_problem_bytes(const mgp_batch_desc* bdesc, const mgp_desc* problem, int64_t* bytes);
/* Allocates a problem (dims, levels, h, bc, origin of `problem`; the batch's operators and
 * precision).  Load its data through mgp_batch_problem() + mgp_upload_* + mgp_write_bc. */
int mgp_batch_add(mgp_batch* b, const mgp_desc* problem, int* id);
int mgp_batch_problem(mgp_batch* b, int id, mgp_solver** s);
int mgp_batch_remove(mgp_batch* b, int id);
int mgp_batch_set_active(mgp_batch* b, int id, int active);
/* One refinement step for every active problem (problems added since the last step first get
 * their initial residual).  n_active: problems stepped. */
int mgp_batch_step(mgp_batch* b, int* n_active);
/* rel_res / iterations / first_rel_res of one problem. */
int mgp_batch_status(mgp_batch* b, int id, mgp_stats* out);
/* Steps until every active problem has ||r||inf/||f||inf < tol (each problem stops when it
 * gets there) or maxiter steps; then stores every problem's FP64 residual. */
int mgp_batch_solve(mgp_batch* b, double tol, int64_t maxiter, int64_t* steps);
/* Kernel launches of one step for the current active set (for the latest non-empty active
 * set once every problem has converged). */
int mgp_batch_kernel_launches(const mgp_batch* b, int64_t* per_step);
/* Device memory available to this batch: cudaMemGetInfo's free bytes plus what the batch's
 * memory pool holds from retired problems (problems allocate from that pool, in the batch
 * stream's order, and give their memory back to it on removal).  No counterpart in the
 * reference, which has no batching. */
int mgp_batch_mem_info(mgp_batch* b, size_t* free_bytes, size_t* total_bytes);
/* Reserve `bytes` of device memory in the batch's memory pool up front (allocated once and
 * returned to the pool, which keeps it): problems added later are carved out of it without
 * the pool growing while the batch is serving.  No counterpart in the reference. */
int mgp_batch_reserve(mgp_batch* b, size_t bytes);

/* Free and total device memory (cudaMemGetInfo) of `device`, for admission control. */
int mgp_mem_info(int device, size_t* free_bytes, size_t* total_bytes);
/* Device-side right-hand side: level-0 f of an FP64 (or refinement) solver set to
 *   f(x,y,z) = sum_m amp[m] sin(kx[m] pi x/L[0]) sin(ky[m] pi y/L[1]) sin(kz[m] pi z/L[2])
 * at every shape point, (x,y,z) = (i,j,k)*h measured from the origin (n_modes <= 64).  The
 * host-side alternative is to sample f and mgp_upload_field it; this skips the host and
 * the PCIe copy.  No counterpart in the reference (its init() samples ffun on the host). */
int mgp_fill_sine_modes(mgp_solver* s, int n_modes, const double* amp, const double* kx, const double* ky,
                        const double* kz, const double L[3]);

/* Device-side right-hand side: level-0 f set to independent uniform values in [lo, hi):
 * value(n) = lo + (hi-lo) * (splitmix64(seed + n*0x9E3779B97F4A7C15) >> 11) * 2^-53, n the
 * point's linear index i*ny*nz + j*nz + k over the shape. */
int mgp_fill_uniform(mgp_solver* s, uint64_t seed, double lo, double hi);

/* Device-side PoissonSolver::init (include/libpoisson.h:158-171) for the reference's test
 * problems (src/problem_definition.cpp): problem 1 sin(3x)sin(5.3y)sin(-7.8z), 2 x^3y^2z,
 * 3 cos(xz^2)sin(y^3).  Level-0 f at every shape point, the level-0 face arrays (Dirichlet: u,
 * Neumann: the normal derivative, as Boundary::init_by_fun samples them), u = 0, then the
 * Dirichlet data written into u (mgp_write_bc).  Coordinates origin + index*h.  The values
 * come from the device's sin/cos, so they may differ from a host init() in the last bit. */
int mgp_fill_problem(mgp_solver* s, int problem);

/* Error of level-0 u over the shape against another solver's level-0 u (ref != NULL, same
 * shape) or, with ref == NULL, against the analytic solution of test problem `problem`
 * (1..3, see mgp_fill_problem).  out[0] = max |u - v|, out[1] = sqrt(sum (u-v)^2),
 * out[2] = sqrt(sum v^2), out[3] = max |v|. */
int mgp_u_error(mgp_solver* s, mgp_solver* ref, int problem, double out[4]);
/* Re-start a batch problem (after new data was loaded): active again, initial residual
 * recomputed at the next step. */
int mgp_batch_restart(mgp_batch* b, int id);

/* Max-norm (max |a|, as mgp_norm returns it) of a caller-owned device array of
 * shape[0] x shape[1] x shape[2] points of type dtype (MGP_F64 double, MGP_F32 float), point
 * (i,j,k) at a[i*stride[0] + j*stride[1] + k] (strides in elements), computed on `device`
 * on `stream` (a cudaStream_t, NULL = default stream); waits for the stream and writes the
 * norm to *out.  No counterpart in the reference: it is a variant of mgp_norm for callers
 * that must not allocate device memory.  It allocates nothing: its scratch is a static 256 KB
 * device array.  A non-NULL stream must belong to `device`.
 *  - At most 268435456 (2^28) points; larger shapes return MGP_ERR_INVALID_ARG.
 *  - The first call on a device looks up the scratch array's address
 *    (cudaGetSymbolAddress); make that first call (an empty shape does only this setup)
 *    before any stream capture on that device.
 *  - Nothing has to be zeroed first; every call rewrites the scratch it reads.
 *  - Calls on the same device share the scratch: calls that overlap in time (other host
 *    threads, or work still running on another stream) race and give wrong results.
 *    Order them on the host. */
int mgp_norm_device(int device, const void* a, int dtype, const int64_t shape[3], const int64_t stride[2],
                    void* stream, double* out);

/* Page-locked host memory for field buffers (faster uploads/downloads). */
int mgp_host_alloc(void** p, size_t bytes);
int mgp_host_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* MGP_H */
