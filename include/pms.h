/* pms.h -- C ABI of libpms_b200.so, the B200 (sm_100a) implementation of pmsim's implicit
 * solid hot path: von Mises radial return + consistent tangent at every integration point
 * (IP), per-element residual B^T.sigma and tangent B^T.D.B, and a deterministic scatter of
 * the element blocks into a global CSR matrix.  All arithmetic is FP64.
 *
 * Each entry point replaces one call of the reference (pmsim 0.3.0, paths inside that project):
 *   ElementTrait           src/fem/element_trait.rs:6-38     -> pms_elements_* (batched over cells)
 *   Elements loops         src/fem/elements.rs:132-205       -> pms_elements_* (one launch per call)
 *   StressStrainTrait      src/material/model_stress_strain.rs:8-43 -> pms_vm_*_batch
 *   assemble_vector/matrix src/base/assembly.rs:38-139       -> CSR/R gathers inside pms_elements_assemble_*
 * Errors: the reference returns Result<_, &'static str>; here every call returns an int status
 * (PMS_OK = 0) and pms_elements_last_error() returns the reference's message text.
 * No torch or CUDA types cross this boundary: pointers are plain, streams are void*.
 */
#ifndef PMS_B200_H
#define PMS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
enum pms_status_code {
    PMS_OK = 0,
    PMS_ERR_INVALID = 1,      /* invalid argument (message in pms_elements_last_error) */
    PMS_ERR_CUDA = 2,         /* CUDA runtime error */
    PMS_ERR_ZERO_SIGMA_D = 3, /* "von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)"
                                 src/material/von_mises.rs:212-216 */
    PMS_ERR_ZERO_NORM_S = 4,  /* "von Mises stiffness cannot be computed with zero deviatoric norm
                                 (norm_s < 1e-10)"  src/material/von_mises.rs:147-150 */
    PMS_ERR_JACOBIAN = 5,     /* non-positive Jacobian determinant at an IP (gemlab calc_gradient) */
    PMS_ERR_NOMEM = 6,        /* device allocation failed */
    PMS_ERR_UNSUPPORTED = 7,  /* idealization/kind not implemented (plane stress, axisymmetric) */
    PMS_ERR_TOO_LARGE = 8,    /* batch does not fit the fixed scratch of pms_element_calc_noalloc */
    PMS_ERR_DF_DSIGMA = 9,    /* "cannot compute df/dsigma due to singularity" (von_mises.rs:254-260) */
    PMS_ERR_NUMERATOR = 10,   /* "plastic numerator (df/dsigma : De : deps) is overly negative"
                                 (elastoplastic.rs:193-195) */
    PMS_ERR_ODE = 11,         /* the elastoplastic ODE took more than max_steps steps */
    PMS_ERR_INTERSECTION = 12, /* no crossing found although the trial point lies outside the yield
                                 surface (the reference asserts, elastoplastic.rs:484) */
    PMS_ERR_ORDER = 13        /* internal: a wait of the ordered CSR assembly timed out (no counterpart) */
};

/* ---- element kinds (gemlab GeoKind subset used by solids) ---------------------------------- */
enum pms_kind {
    PMS_TRI3 = 0, PMS_TRI6 = 1, PMS_QUA4 = 2, PMS_QUA8 = 3, PMS_QUA9 = 4,
    PMS_TET4 = 5, PMS_TET10 = 6, PMS_HEX8 = 7, PMS_HEX20 = 8,
    PMS_TRI10 = 9, PMS_TRI15 = 10  /* complete cubic / quartic triangles (default 6 / 12 IPs) */
};

/* ---- stress-strain models (src/base/parameters.rs:17-35) ---------------------------------- */
enum pms_model { PMS_LINEAR_ELASTIC = 0, PMS_VON_MISES = 1 };

/* where a caller's buffer lives */
enum pms_mem { PMS_MEM_HOST = 0, PMS_MEM_DEVICE = 1 };

/* StressStrain::VonMises { young, poisson, hh, z_ini } / LinearElastic { young, poisson } */
typedef struct pms_material {
    int32_t model;  /* enum pms_model */
    double young;
    double poisson;
    double hh;      /* hardening H (von Mises) */
    double z_ini;   /* initial yield-surface size (von Mises); must be > 1e-6 */
} pms_material;

/* Homogeneous mesh: ncell cells of one kind; coords[npoint*ndim]; cells[ncell*nnode] (point ids).
 * Global DOF numbering: eq = ndim*point + d (src/base/all_dofs.rs:87-116).
 * cell_material (nullable) selects materials[cell_material[c]] per cell (cell attribute). */
typedef struct pms_mesh {
    int32_t ndim;
    int32_t kind;          /* enum pms_kind */
    int64_t npoint;
    int64_t ncell;
    const double* coords;  /* host */
    const int64_t* cells;  /* host */
    const int32_t* cell_material; /* host, nullable */
} pms_mesh;

/* The Config fields the hot path reads (src/base/config.rs:19-229). */
typedef struct pms_config {
    int32_t ngauss;        /* 0 = default rule of the kind (ParamSolid::ngauss = None) */
    int32_t plane_stress;  /* Idealization::plane_stress: 2D linear-elastic materials only; with a von Mises
                              material the call returns PMS_ERR_UNSUPPORTED, as the reference refuses it
                              ("von Mises model does not work in plane-stress", von_mises.rs:60-62) */
    int32_t axisymmetric;  /* Idealization::axisymmetric: 2D kinds (x = radius), any material; 3D kinds
                              return PMS_ERR_UNSUPPORTED; cannot be combined with plane_stress */
    double thickness;      /* Idealization::thickness, default 1.0 (ignored when axisymmetric) */
} pms_config;

typedef struct pms_elements_info {
    int32_t ndim, kind, nnode, ngauss, ncomp;  /* ncomp = Mandel components (4 in 2D, 6 in 3D) */
    int64_t npoint, ncell, ndof, nip;          /* nip = ncell*ngauss */
    int64_t nnz;                               /* CSR nonzeros of K in the storage set by
                                                  pms_elements_set_symmetry (default: both triangles) */
    int64_t nblock_upper;                      /* node-pair blocks with A <= B */
    int64_t ncontrib;                          /* element blocks summed into them */
    int64_t device_bytes;                      /* device memory held by the handle so far */
} pms_elements_info;

typedef struct pms_elements pms_elements; /* opaque; not thread-safe; one CUDA stream per handle */

/* Elements::new + ElementSolid::new for all cells (src/fem/elements.rs:45-70,
 * src/fem/element_solid.rs:47-92): uploads the mesh, builds the CSR pattern of K and the
 * deterministic gather maps, allocates the device-resident IP state (SoA). */
int pms_elements_create(const pms_mesh* mesh, const pms_material* materials, int32_t nmaterial,
                        const pms_config* config, pms_elements** out);
void pms_elements_destroy(pms_elements* h);
int pms_elements_get_info(const pms_elements* h, pms_elements_info* out);
/* ElementTrait::symmetric_jacobian (src/fem/element_solid.rs:100-102): 1 when the Jacobian of every
 * cell is symmetric, i.e. every material's symmetric_stiffness() is true -- always, for the linear
 * elastic (src/material/linear_elastic.rs:26-28) and von Mises (src/material/von_mises.rs:92-94)
 * models.  A caller picks the storage of K from it as LinearSystem::new does
 * (src/fem/linear_system.rs:96-119; pms_elements_set_symmetry). */
int pms_elements_symmetric_jacobian(const pms_elements* h, int32_t* out);
/* stream: a cudaStream_t (or NULL for the handle's own stream) */
int pms_elements_set_stream(pms_elements* h, void* stream);
/* CSR pattern of K (sorted columns): indptr[ndof+1], indices[nnz] (host or device) */
int pms_elements_csr_pattern(pms_elements* h, int64_t* indptr, int32_t* indices, int32_t mem);

/* ElementTrait::initialize_internal_values (von_mises.rs:107-116): sigma = 0, z = z_ini,
 * lambda = 0, elastic = true at every IP */
int pms_elements_initialize(pms_elements* h);
/* ElementTrait::reset_algorithmic_variables (von_mises.rs:119-121): lambda = 0 */
int pms_elements_reset_algorithmic(pms_elements* h);
/* ElementTrait::backup_secondary_values / restore_secondary_values
 * (element_solid.rs:227-238; LocalState::mirror, local_state.rs:40-44) */
int pms_elements_backup(pms_elements* h);
int pms_elements_restore(pms_elements* h);

/* ElementTrait::update_secondary_values (element_solid.rs:190-224): per IP,
 * delta_eps = B.ddu, then update_stress in place on the current state (the Newton loop has
 * just backed it up or restored it).  ddu[ndof] is the cumulative step increment. */
int pms_elements_update_secondary(pms_elements* h, const double* ddu, int32_t mem);
/* Elements::assemble_f_int (elements.rs:132-138; element_solid.rs:124-138; assembly.rs:38-46):
 * ff_int[ndof] = sum_e sum_p B^T sigma |J| w t  (overwritten, not accumulated) */
int pms_elements_assemble_f_int(pms_elements* h, double* ff_int, int32_t mem);
/* Elements::assemble_kke (elements.rs:156-163; element_solid.rs:168-185; assembly.rs:70-139):
 * csr_values[nnz] = sum_e sum_p B^T D_ep B |J| w t in the pattern of pms_elements_csr_pattern.
 * Bit-reproducible: every entry sums its element contributions in a fixed order (pms_assembly). */
int pms_elements_assemble_kk(pms_elements* h, double* csr_values, int32_t mem);
/* Fused Newton-iteration call = restore + update_secondary(ddu) + assemble_f_int + assemble_kk
 * on the updated state, in one pass over the cells (ff_int/csr_values nullable).  Every IP starts
 * from the backed-up state (pms_elements_backup at iteration 0), as SolverImplicit::iterate does
 * (src/fem/solver_implicit.rs:254-263); the backup itself is not modified. */
int pms_elements_update_and_assemble(pms_elements* h, const double* ddu, double* ff_int, double* csr_values,
                                     int32_t mem);
/* Per-cell drop-ins for callers that loop over cells themselves (host output):
 * ElementTrait::calc_f_int -> f[nnode*ndim]; ElementTrait::calc_jacobian -> kk[ne*ne] row-major */
int pms_element_calc_f_int(pms_elements* h, int64_t cell, double* f);
int pms_element_calc_jacobian(pms_elements* h, int64_t cell, double* kk);

/* IP state in the reference's LocalState layout, cell-major (ip = cell*ngauss + p):
 * sig[nip*ncomp] (Mandel), ivs[nip*2] = [z, lambda], elastic[nip]; host buffers */
int pms_elements_get_state(pms_elements* h, double* sig, double* ivs, uint8_t* elastic);
int pms_elements_set_state(pms_elements* h, const double* sig, const double* ivs, const uint8_t* elastic);

/* How K and R are assembled (no counterpart in the reference, whose COO triplets are summed by the
 * sparse solver, src/base/assembly.rs:70-139).  Both are bit-reproducible run to run; they agree to
 * the last bits (their summation orders differ).
 *   PMS_ASSEMBLY_GATHER (default): the element kernel writes each cell's upper node-pair blocks of
 *     K_e (a <= b) and F_e, then gather kernels sum them row by row, every entry over its cells in
 *     ascending cell order (8*ncell*nnode*(nnode+1)/2*ndim^2 bytes more device memory).
 *   PMS_ASSEMBLY_DIRECT: the element kernel adds each cell's blocks straight into the CSR values
 *     and R (per-row tickets), every entry over its cells in the processing order of
 *     pms_mesh_assembly_maps; no element matrices are stored. */
enum pms_assembly { PMS_ASSEMBLY_DIRECT = 0, PMS_ASSEMBLY_GATHER = 1 };
int pms_elements_set_assembly(pms_elements* h, int32_t mode);

/* Storage of K in the CSR values, as russell_sparse's Sym that LinearSystem::new picks from the
 * linear solver when every element Jacobian is symmetric (src/fem/linear_system.rs:96-119), with the
 * entries kept as assemble_matrix keeps them (src/base/assembly.rs:92-136):
 *   PMS_SYM_FULL (default): both triangles (Sym::YesFull, Sym::No);
 *   PMS_SYM_LOWER: the entries with column <= row (Sym::YesLower, the choice for MUMPS);
 *   PMS_SYM_UPPER: the entries with column >= row (Sym::YesUpper).
 * It sets what pms_elements_get_info's nnz, pms_elements_csr_pattern and the CSR values of
 * pms_elements_assemble_kk / pms_elements_update_and_assemble hold; a kept entry has the bits of
 * the same entry of the full matrix.  The triangles need the gather assembly: PMS_ERR_UNSUPPORTED
 * when PMS_ASSEMBLY_DIRECT is set (either call refuses the other's combination).  The per-cell calls
 * always return full element matrices. */
enum pms_sym { PMS_SYM_FULL = 0, PMS_SYM_LOWER = 1, PMS_SYM_UPPER = 2 };
int pms_elements_set_symmetry(pms_elements* h, int32_t sym);

/* Instrumentation: when on, every batched call records CUDA events around its kernels on the
 * handle's stream; pms_elements_kernel_times waits for the stream and returns the summed device
 * time (ms) and launch count of [0] element kernel, [1] F_int gather, [2] CSR gather since the
 * previous query. */
int pms_elements_set_timing(pms_elements* h, int32_t on);
int pms_elements_kernel_times(pms_elements* h, double* ms, int64_t* counts);

/* Host-only (no GPU needed): the element tables pms_elements_create uploads for a kind and rule
 * (ngauss 0: the default), as gemlab's Scratchpad/Gauss provide them to ElementSolid::new
 * (src/fem/element_solid.rs:47-92): tab[ng*nnode*ndim] = dN_m/dksi_j at each IP, then the weights
 * w[ng], then N[ng*nnode].  tab NULL: only *ngauss_out (the number of IPs) is set. */
int pms_shape_table(int32_t kind, int32_t ngauss, double* tab, int32_t* ngauss_out);

/* Host-only (no GPU needed): the maps of the direct assembly pms_elements_create builds (no
 * counterpart in the reference, which sums COO triplets in the solver, src/base/assembly.rs:70-139).
 * The kernel takes the cells in a processing order: order[k] is the k-th cell, colour classes of a
 * greedy colouring (cells that share a node get different colours) within each segment of cells that
 * shares no node with the rest.  Every entry of K and R is summed over its cells in that order.
 * For cell c and local nodes a, b -- cslot[(c*nnode + a)*nnode + b] the column slot of node b in
 * block row conn[a]; crank[c*nnode + a] c's position, in the processing order, among the cells of
 * conn[a] (bits 0..29; bit 30 set for the last one); cfirst[c*nnode + a] bit b set when c is the
 * first of the cells holding both conn[a] and conn[b] (it stores the first contribution of that
 * block).  Any output may be NULL. */
int pms_mesh_assembly_maps(const pms_mesh* mesh, int16_t* cslot, int32_t* crank, uint32_t* cfirst,
                           int32_t* order);

/* Host-only (no GPU needed): the CSR pattern pms_elements_create would build for this mesh.
 * Call with indices = NULL to get nnz (indptr[ndof+1] may already be filled). */
int pms_mesh_csr_pattern(const pms_mesh* mesh, int64_t* indptr, int32_t* indices, int64_t* nnz);
/* Host-only (no GPU needed): the same in the storage sym of pms_elements_set_symmetry (enum pms_sym;
 * the full pattern's entries with column <= row, or >= row, in the same order). */
int pms_mesh_csr_pattern_sym(const pms_mesh* mesh, int32_t sym, int64_t* indptr, int32_t* indices, int64_t* nnz);

/* Waits for the handle's stream and returns the first device-side error (PMS_OK if none). */
int pms_elements_sync(pms_elements* h);
/* Message of the handle's last error; with h = NULL, the message of this thread's last refused
 * pms_elements_create (for example "von Mises initial size of the yield surface must > 1e-6",
 * src/material/von_mises.rs:68-70), empty if it succeeded. */
const char* pms_elements_last_error(const pms_elements* h);
/* cell and IP of the failing integration point that the reference would report (-1 if none): its
 * loops stop at the first error, and they run the stress update of every cell before the tangent of
 * any cell, each in ascending cell and IP order (src/fem/elements.rs:156-181) -- so an update error
 * is reported before a tangent error, and the lowest failing cell, then its lowest IP, is named. */
int pms_elements_error_location(const pms_elements* h, int64_t* cell, int32_t* ip);
/* Number of kernels this handle has launched since creation (instrumentation). */
int64_t pms_elements_launch_count(const pms_elements* h);

/* ---- batched Newton solver on the device --------------------------------------------------
 * Many independent problems share one pms_elements handle: problem p owns the points
 * [point_ptr[p], point_ptr[p+1]) and the cells [cell_ptr[p], cell_ptr[p+1]) (disjoint ranges, so
 * the handle's CSR matrix is block diagonal).  Every Newton iteration is one element launch for all
 * problems and one batched PCG solve; the sequencing, the Lagrange-multiplier treatment of the
 * prescribed equations and the convergence tests are those of SolverImplicit::iterate
 * (src/fem/solver_implicit.rs:187-272, src/fem/bc_prescribed.rs:99-134,
 * src/fem/convergence_control.rs:52-128).  The reference's direct solve (UMFPACK,
 * src/fem/linear_system.rs:185-201) is replaced by FP64 PCG with a node-block Jacobi preconditioner
 * on the system with the prescribed equations eliminated; it reproduces the augmented system's
 * iterates.  Each problem's arithmetic is independent of the other problems in the batch. */
typedef struct pms_batch_config {
    double tol_rr_abs;          /* max|R| < tol_rr_abs: converged (reference default 1e-10) */
    double tol_mdu_rel;         /* rel(mdu) < tol_mdu_rel (iteration > 0): converged (default 1e-8) */
    int32_t n_max_iterations;   /* Newton iterations per step (reference default 10) */
    double pcg_rtol;            /* PCG stops at |r|_2 <= pcg_rtol |r0|_2 (default 1e-12) */
    int32_t pcg_max_iterations; /* PCG iteration cap per solve (default 20000) */
    int32_t constant_tangent;   /* Config::constant_tangent (src/fem/solver_implicit.rs:216): K assembled (and
                                   the preconditioner formed) only at the first Newton iteration of each
                                   load step; later iterations update the IP state and R only */
} pms_batch_config;

typedef struct pms_batch pms_batch;

/* pres_eq[npres]: sorted, unique global equations with prescribed values (Essential);
 * ff_ext[ndof] (host, nullable): constant external forces (loading factor 1). */
int pms_batch_create(pms_elements* el, int32_t nproblem, const int64_t* point_ptr, const int64_t* cell_ptr,
                     int64_t npres, const int64_t* pres_eq, const double* ff_ext, const pms_batch_config* cfg,
                     pms_batch** out);
void pms_batch_destroy(pms_batch* b);
/* U = 0, multipliers = 0 and pms_elements_initialize of the handle */
int pms_batch_reset(pms_batch* b);
/* One load step for the problems with active[p] != 0: dU = 0, lambda = 0 at the IPs, then Newton
 * iterations until each problem converges.  c_values[npres] (host) are the prescribed values at the
 * new time of each problem.  Per problem (host, nullable): iterations (residual evaluations, as the
 * reference counts them), final max|R|, status (0 ok, 1 NaN/Inf in R, 2 NaN/Inf in mdu,
 * 3 "Newton-Raphson did not converge", 4/5/6 the stress-update, tangent or Jacobian error of the
 * element path -- a failing problem stops, the others go on) and the PCG iterations spent. */
int pms_batch_solve_step(pms_batch* b, const double* c_values, const uint8_t* active, int32_t* iterations,
                         double* norm_rr, int32_t* status, int32_t* pcg_iterations);
/* One Newton iteration of every problem with cmd[p] != 0, each at its own load step and iteration
 * (continuous batching): cmd 1 = start a new load step (dU = 0, lambda = 0 at the IPs; c_values hold
 * its prescribed values), cmd 2 = continue the step (stress update with the current dU, then the
 * next iteration).  result[p]: -1 idle, 0 still iterating (send cmd 2), 1 converged (state and U are
 * the step's solution), 100 + status on failure (status codes as for pms_batch_solve_step).
 * iteration[p] (0-based), norm_rr[p] and pcg_iterations[p] of this tick are optional outputs.
 * A tick advances each problem by one stage of its own iteration (element pass and residual test;
 * PCG iterations; completion of the iteration), so a problem never waits for another problem's
 * linear solve: result 2 = the problem's linear solve is still under way (send cmd 2 again; no
 * iteration is completed by this tick). */
int pms_batch_tick(pms_batch* b, const uint8_t* cmd, const double* c_values, int32_t* result, int32_t* iteration,
                   double* norm_rr, int32_t* pcg_iterations);
/* The same lock-step load step as pms_batch_solve_step (same arguments, same results bit for bit),
 * with the Newton loop resident on the device: one CUDA graph launch per load step, in which a
 * conditional WHILE node runs every active problem's Newton iterations -- element pass, residual
 * test, PCG start, a nested WHILE over PCG iterations, completion and update -- with the
 * per-problem sequencing of SolverImplicit::iterate (src/fem/solver_implicit.rs:187-272) done by
 * controller kernels; the host waits once per load step.  Every problem's PCG runs on the
 * batch-wide engine (the engines give the same bits).  The graph is built on the first call and
 * kept by the batch.  Not while a tick-driven linear solve is under way (PMS_ERR_INVALID). */
int pms_batch_solve_step_graph(pms_batch* b, const double* c_values, const uint8_t* active, int32_t* iterations,
                               double* norm_rr, int32_t* status, int32_t* pcg_iterations);
/* Host waits for the device made by pms_batch_tick / pms_batch_solve_step / _graph so far. */
int64_t pms_batch_host_syncs(const pms_batch* b);

/* Launch shapes of the PCG (they change speed only: every engine computes bit-identical iterates).
 * A problem with at most team_max_ndof DOFs runs its whole PCG on a thread-block cluster ("team")
 * of C = 1, 2, 4, 8 or 16 CTAs of team_threads threads (256, 512 or 1024), its vectors resident in
 * the CTAs' shared memory; C is the smallest team whose CTAs hold at most team_chunks 128-node
 * chunks each (0: as many as fit).  Other problems run the batch-wide kernels, graph_iters
 * iterations per CUDA-graph launch.  pcg_budget bounds the PCG iterations a problem gets per tick.
 * No counterpart in the reference (its solve is a direct factorisation,
 * src/fem/linear_system.rs:185-201). */
typedef struct pms_batch_tuning {
    int64_t team_max_ndof;
    int32_t team_threads;
    int32_t team_chunks;
    int32_t pcg_budget;
    int32_t graph_iters;
} pms_batch_tuning;
int pms_batch_set_tuning(pms_batch* b, const pms_batch_tuning* t);
int pms_batch_get_tuning(const pms_batch* b, pms_batch_tuning* t);
/* Autotuner: times 32 PCG iterations of every problem on its initial tangent (unit right-hand
 * side) for each candidate (batch-wide only; teams up to several sizes, CTA sizes and chunks per
 * CTA), keeps the fastest, then resets the batch (pms_batch_reset).  *out (nullable) receives the
 * choice. */
int pms_batch_autotune(pms_batch* b, pms_batch_tuning* out);
/* Instrumentation (the autotuner's measurement): device time in ms of `iterations` PCG iterations
 * of every problem, on its initial tangent, with the launch shapes *t; resets the batch and keeps
 * its own tuning. */
int pms_batch_time_pcg(pms_batch* b, const pms_batch_tuning* t, int32_t iterations, double* ms);
int pms_batch_get_u(pms_batch* b, double* u);                 /* host u[ndof] */
int pms_batch_get_multipliers(pms_batch* b, double* lam);     /* host lambda[npres] (reactions) */
/* kernels launched by the solver (PCG iterations captured in graphs count once per kernel) */
int64_t pms_batch_counters(const pms_batch* b, int64_t* pcg_iterations_total);
const char* pms_batch_last_error(const pms_batch* b);

/* ---- material batch (StressStrainTrait::update_stress + stiffness over n IPs) -------------
 * Device buffers, structure-of-arrays with component stride n:
 *   sig[ncomp*n] (in/out), z[n] (in/out), lambda[n] (out), elastic[n] (out), deps[ncomp*n] (in),
 *   hh[n] (nullable: per-IP hardening, else mat->hh), dd[nd*n] (out, nullable): upper triangle of
 *   the Mandel tangent, row-major (i <= j), nd = ncomp*(ncomp+1)/2 (21 in 3D, 10 in 2D).
 * VonMises::update_stress (von_mises.rs:170-226) then VonMises::stiffness (von_mises.rs:124-167)
 * on the updated state; LinearElastic (linear_elastic.rs:49-71) when mat->model == 0.
 * status (device int[4], nullable): {code, ip_lo, ip_hi, 0} of the first failing IP. */
int pms_vm_update_and_stiffness_batch(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                                      double* lambda, uint8_t* elastic, const double* deps, const double* hh,
                                      double* dd, int32_t* status, void* stream);
/* VonMises::stiffness alone, from a given state (sig, lambda, elastic) */
int pms_vm_stiffness_batch(const pms_material* mat, int32_t ndim, int64_t n, const double* sig,
                           const double* lambda, const uint8_t* elastic, const double* hh, double* dd,
                           int32_t* status, void* stream);
/* Same as pms_vm_update_and_stiffness_batch on HOST buffers: copies in, runs, copies out
 * (the library keeps a device staging area, grown on demand). */
int pms_vm_update_and_stiffness_host(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                                     double* lambda, uint8_t* elastic, const double* deps, const double* hh,
                                     double* dd);

/* ---- general elastoplastic update (Elastoplastic::update_stress over n IPs) ----------------
 * Replaces Elastoplastic::update_stress (src/material/elastoplastic.rs:539-641) with the von Mises
 * plasticity model (src/material/von_mises.rs:229-282), the only model Elastoplastic accepts:
 * yield-surface intersection along the elastic path, then the ODE dsigma/dt = Dep : deps,
 * dz/dt = Lambda_d H integrated from the crossing to the end of the increment.  mat->model must be
 * PMS_VON_MISES (else PMS_ERR_INVALID); mat->hh is the hardening H.  Device buffers as in
 * pms_vm_update_and_stiffness_batch: sig[ncomp*n], z[n], elastic[n] in/out, deps[ncomp*n] in.
 * cases[n] (nullable) receives the case of each IP (pms_ep_case; -1 where the IP failed) and
 * steps[n] (nullable) the ODE steps taken (accepted and rejected).  On an error the IP's state is
 * left as it was and status {code, ip_lo, ip_hi, 0} names the first failing IP.  No tangent: the
 * reference's Elastoplastic::stiffness is not implemented either (elastoplastic.rs:528-537). */
typedef struct pms_ep_settings {
    double tol_rel;     /* relative tolerance of the ODE error control (default 1e-10) */
    double tol_abs;     /* absolute tolerance (default 1e-10) */
    double h_ini;       /* first trial step in pseudo-time, clipped to the interval (default 1) */
    int32_t max_steps;  /* step limit per IP (default 1000); beyond it PMS_ERR_ODE */
    int32_t pad_;
} pms_ep_settings;
enum pms_ep_case { PMS_EP_AE = 0, PMS_EP_AXB = 1, PMS_EP_BE = 2, PMS_EP_BXP = 3, PMS_EP_BP = 4 };
int pms_ep_update_stress_batch(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                               uint8_t* elastic, const double* deps, const pms_ep_settings* settings,
                               int32_t* cases, int32_t* steps, int32_t* status, void* stream);
/* Same as pms_ep_update_stress_batch on HOST buffers (same layout): copies in, runs, copies out,
 * and returns the first failing IP's code (PMS_OK if none); the library keeps a device staging
 * area, grown on demand. */
int pms_ep_update_stress_host(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                              uint8_t* elastic, const double* deps, const pms_ep_settings* settings,
                              int32_t* cases, int32_t* steps);

/* Measures the FP64 FMA pipe: blocks x 256 threads, 8 independent FMA chains of `iters` each
 * (16*iters FLOP per thread); out[blocks*256] receives the chain sums.  Used as the FP64 peak. */
int pms_probe_fp64_fma(int64_t iters, int32_t blocks, double* out, void* stream);

/* ---- Distributed block-Jacobi PCG (one rank's part of a sharded linear solve) ----
 * No counterpart in the reference, which solves one problem in one process with a direct solver
 * (src/fem/solver_implicit.rs:187-272, LinSolver in src/fem/linear_system.rs).  The rank holds the
 * owned rows of its local K: indptr[n_owned+1] and indices (host arrays) give their pattern in
 * local DOF numbering (owned DOFs first, then ghosts, n_local in all); fixed_local[n_local] flags the
 * prescribed DOFs, whose rows and columns are replaced by the identity.  send_idx: the owned DOFs
 * the neighbours need, recv_idx: the ghost DOFs, each concatenated in ascending neighbour order.
 * Vectors are device memory bound once (pms_dpcg_bind): x, r, z, q hold n_owned entries, p
 * n_local, the send and receive buffers nsend and nrecv, scal 6 doubles (slot 0: r.z, slot 1: p.q,
 * the two slots the caller all-reduces across ranks; 2: r.z of the current iteration, 3: r0.z0,
 * 4: 1 once converged, 5: iterations).  One iteration, all on the handle's stream:
 *   pack; post the exchange of the send/receive buffers; spmv(0) (interior rows, overlapping the
 *   exchange); wait; unpack; spmv(1) (boundary rows); dot_pq; all-reduce slot 1; update;
 *   all-reduce slot 0; direction(rtol).
 * A solve starts with set_values (the local CSR values, device; every Newton iteration), start(b)
 * (b: owned right-hand side, device), the all-reduce of slot 0 and init.  Once slot 4 is set every
 * call leaves the iterates unchanged, so the host may read it every few iterations. */
typedef struct pms_dpcg pms_dpcg;
int pms_dpcg_create(int32_t ndim, int64_t n_owned, int64_t n_local, const int64_t* indptr, const int32_t* indices,
                    const uint8_t* fixed_local, int64_t nsend, const int64_t* send_idx, int64_t nrecv,
                    const int64_t* recv_idx, pms_dpcg** out);
void pms_dpcg_destroy(pms_dpcg* h);
const char* pms_dpcg_last_error(const pms_dpcg* h); /* NULL: the last refused pms_dpcg_create */
int pms_dpcg_set_stream(pms_dpcg* h, void* stream);
int pms_dpcg_bind(pms_dpcg* h, double* x, double* r, double* z, double* p, double* q, double* sendbuf,
                  double* recvbuf, double* scal);
int pms_dpcg_set_values(pms_dpcg* h, const double* values);
int pms_dpcg_start(pms_dpcg* h, const double* b);
int pms_dpcg_init(pms_dpcg* h);
int pms_dpcg_pack(pms_dpcg* h);
int pms_dpcg_unpack(pms_dpcg* h);
int pms_dpcg_spmv(pms_dpcg* h, int32_t boundary);
int pms_dpcg_dot_pq(pms_dpcg* h);
int pms_dpcg_update(pms_dpcg* h);
int pms_dpcg_direction(pms_dpcg* h, double rtol);
int pms_dpcg_info(const pms_dpcg* h, int64_t* counts); /* nnz, interior rows, boundary rows, reduction blocks */

/* Element vectors and matrices for a batch of cells WITHOUT ANY DEVICE ALLOCATION.
 * No counterpart in the reference: it exists for callers that cannot call cudaMalloc -- a program
 * running inside another framework that owns the whole device-memory budget, a real-time loop
 * where an allocation would stall or synchronise the GPU, or a foreign-language element loop (for
 * example Rust behind an FFI) that has no CUDA allocator.  For ncell independent cells given on
 * the host it returns each cell's internal-force vector f = sum_p B^T sigma |J| w t and its
 * tangent matrix K = sum_p B^T D B |J| w t (D the consistent tangent of the IP state: elastic
 * modulus where elastic[ip] != 0, the von Mises elastoplastic tangent otherwise).  2D cells are
 * always in plane strain: there is no plane-stress or axisymmetric option here.
 * Inputs: X[ncell][nnode][ndim] coordinates; the IP state structure-of-arrays with stride
 * nip = ncell*ngauss: sig[ncomp][nip] (Mandel), ivs[2][nip] (z then lambda), elastic[nip].
 * Outputs (host, nullable, at least one): f[ncell][nnode*ndim] and kk[ncell][ne][ne] row-major.
 * All device work uses one file-scope array of 16 MiB, held by every GPU that loads the library
 * until the process exits; *max_cells (nullable) receives the largest batch that fits for this
 * kind, rule and choice of outputs, and a larger batch returns PMS_ERR_TOO_LARGE (split it).
 * The array is shared by every call and keeps the last call's contents: calls that overlap on the
 * GPU (from two threads, or on two streams without ordering) race, so serialise them.  The first
 * call on a device looks up the array's address for that device; make that first call before any
 * stream capture.  stream: cudaStream_t or NULL; the call returns after its results are on the host. */
int pms_element_calc_noalloc(int32_t kind, int32_t ngauss, double thickness, const pms_material* mat,
                             int64_t ncell, const double* X, const double* sig, const double* ivs,
                             const uint8_t* elastic, double* f, double* kk, int64_t* max_cells, void* stream);

/* The calling host thread's CUDA device (no counterpart in the reference, which runs on the host):
 * every handle is created on, and must be used from, the device that is current in the creating
 * thread.  pms_device_count reports 0 when no device is visible. */
int pms_set_device(int32_t device);
int pms_device_count(int32_t* count);

/* Library version string and the number of kernels launched by the material entry points. */
const char* pms_version(void);
int64_t pms_material_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* PMS_B200_H */
