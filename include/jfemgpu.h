/*
 * jfemgpu.h -- C ABI of the B200 SOL101 linear-static library (libjfemgpu.so).
 *
 * The library replaces the device-side half of OpenJFEM's SOL101 parity path:
 * element stiffness (CQUAD4 / CQUAD8 / CTETRA10), assembly of the global
 * stiffness K, the sparse Cholesky factorisation of K_ff and the triangular
 * solves, residual and SPC-force recovery.  Parsing, SPC/AUTOSPC reduction
 * and result output stay with the caller (the Julia host in the reference).
 *
 * Conventions
 *   - Every pointer argument is a caller-owned HOST array; it is read (or
 *     written) during the call only.  No pointer is retained after return.
 *   - Indices are 0-based.  Node index n is the position of the GRID in the
 *     sorted list of GRID ids (reference: src/solver/assembly.jl:2653-2665).
 *     Global DOF d = 6*n + c, c in 0..5 = (T1,T2,T3,R1,R2,R3).
 *   - Dense matrices are column-major (Julia layout): A[r + nrow*c].
 *   - K is stored exactly like Julia's SparseMatrixCSC built by
 *     sparse(I,J,V,ndof,ndof): colptr (ndof+1), rowval (nnz), nzval (nnz),
 *     duplicates summed in triplet order, explicit zeros kept
 *     (reference: src/solver/assembly.jl:5942, 5963-5974).
 *   - Every function returns a jfg_status; on failure jfg_last_error()
 *     returns a thread-local message.
 */
#ifndef JFEMGPU_H
#define JFEMGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  JFG_OK = 0,
  JFG_NOT_SPD = 1,          /* non-positive pivot; detail = permuted DOF index     */
  JFG_IR_STALLED = 2,       /* iterative refinement did not reach the tolerance   */
  JFG_OOM_BUDGET = 3,       /* request exceeds the device-memory budget           */
  JFG_TIMEOUT = 4,          /* a bounded device wait expired                      */
  JFG_UNSUPPORTED = 5,      /* element flags/geometry outside the supported path  */
  JFG_BAD_INPUT = 6,        /* malformed arguments (sizes, indices, NaN, ...)     */
  JFG_CUDA_ERROR = 7,       /* CUDA runtime error                                 */
  JFG_NOT_READY = 8         /* call order violated (e.g. solve before factor)     */
} jfg_status;

typedef enum {
  JFG_PREC_FP64 = 0,        /* plain FP64 supernodal Cholesky                      */
  JFG_PREC_MIXED = 1        /* FP32-storage factor, FP64 iterative refinement on
                               the FP64 CSR matrix; front updates on the tensor
                               cores in 3xTF32 (JFG_TENSOR_CORES=0: SIMT FP32) */
} jfg_precision;

typedef struct jfg_ctx jfg_ctx;
typedef struct jfg_model jfg_model;

typedef struct {
  int32_t device;           /* CUDA device ordinal                                */
  int32_t flags;            /* reserved, 0                                        */
  int64_t hbm_budget_bytes; /* 0 = no budget                                      */
} jfg_config;

/* Per-element section records (doubles, column-major 3x3 / 2x2 blocks). */
#define JFG_Q4_SECT_STRIDE 26 /* Cm[9] Cb[9] Cs[4] h Eref k6rot flags              */
#define JFG_Q8_SECT_STRIDE 22 /* A[9] D[9] shear(=Gts, INF=rigid) Dref hasA hasD  */
#define JFG_T10_MAT_STRIDE 2  /* E nu                                             */

/* Q4 section flag bits (flags word): only 0 is the supported default path.   */
#define JFG_Q4_FLAG_DEFAULT 0

typedef struct {
  double rel_residual;      /* max over RHS of |K_ff u - F_ff| / |F_ff|            */
  double max_rel_update;    /* last IR correction |du|/|u|                         */
  int32_t ir_iters;         /* refinement steps taken                              */
  int32_t fallback_used;    /* 1 when the FP64 factor replaced the mixed factor   */
  int32_t precision;        /* precision of the factor that produced U            */
  int32_t reserved;
} jfg_solve_report;

typedef struct {
  int64_t n_supernodes;
  int64_t n_levels;
  int64_t nnz_L;            /* stored factor entries (lower, incl. diagonal)       */
  double flops;             /* sum_j c_j^2 over the symbolic factor                */
  int64_t factor_bytes;     /* device bytes of the factor                          */
  int64_t max_front;        /* largest front order                                */
} jfg_symbolic_info;

/* ---- context ------------------------------------------------------------ */
/* Replaces: nothing on the reference side (CPU); owns the CUDA stream.       */
jfg_status jfg_create(jfg_ctx** ctx, const jfg_config* cfg);
jfg_status jfg_destroy(jfg_ctx* ctx);
const char* jfg_last_error(void);
int64_t jfg_last_error_detail(void);

/* ---- model upload ------------------------------------------------------- */
/* Replaces the input side of Solver.assemble_stiffness
 * (src/solver/assembly.jl:2630-2675 node indexing / node_R,
 *  :3223-3480 per-element section arrays, :5806-5921 solid / CQUAD8 lists).
 * xyz: n_nodes*3 (row per node); node_R: n_nodes*9 (3x3 column-major, the
 * CD-frame rotation node_R of assembly.jl:2667-2675).
 * q4_nodes: n_q4*4, q8_nodes: n_q8*8, t10_nodes: n_t10*10 (0-based node idx). */
jfg_status jfg_model_upload(jfg_ctx* ctx, int64_t n_nodes, const double* xyz,
                            const double* node_R, int64_t n_q4,
                            const int32_t* q4_nodes, const double* q4_sect,
                            int64_t n_q8, const int32_t* q8_nodes,
                            const double* q8_sect, int64_t n_t10,
                            const int32_t* t10_nodes, const double* t10_mat,
                            jfg_model** out);
/* CTRIA3 shells of a model (src/solver/assembly.jl:3293-3480 section arrays,
 * :5386-5510 the TRIA3 loop; also the six triangles that replace a CQUAD8
 * without the native eight-node section, :3176-3196).  Called at most once,
 * after jfg_model_upload and before the first jfg_assemble.  t3_nodes: n_t3*3
 * (0-based node idx); t3_sect: n_t3 records of JFG_Q4_SECT_STRIDE doubles
 * laid out as for CQUAD4 (Cm Cb Cs h Eref k6rot flags; flags is ignored).
 * The triangles' triplets follow the CQUAD4 ones, as in the reference.      */
jfg_status jfg_model_add_tria3(jfg_model* model, int64_t n_t3, const int32_t* t3_nodes,
                               const double* t3_sect);
jfg_status jfg_model_free(jfg_model* model);

/* ---- assembly ------------------------------------------------------------ */
/* Replaces Solver.assemble_stiffness's element loops and sparse()
 * (src/solver/assembly.jl:3603-5335 Q4, :5806-5890 solids, :5893-5921 Q8,
 *  :5942 sparse).  The first call builds the CSC pattern and the
 * triplet->nzval slot map on the host; every call recomputes the values on
 * the device (element kernels + deterministic slot-map gather).          */
jfg_status jfg_assemble(jfg_model* model);
jfg_status jfg_get_sizes(jfg_model* model, int64_t* ndof, int64_t* nnz,
                         int64_t* n_triplets);
jfg_status jfg_get_pattern(jfg_model* model, int64_t* colptr, int32_t* rowval);
jfg_status jfg_get_values(jfg_model* model, double* nzval);
jfg_status jfg_get_slot_map(jfg_model* model, int64_t* slot);
/* max_elem_stiff and orig_diag of assembly.jl:5923-5936; diag has ndof entries. */
jfg_status jfg_get_diag(jfg_model* model, double* diag, double* max_elem_stiff);
/* 3x3 translational and rotational node blocks (column-major, 18 per node)
 * consumed by the host's grid-point-singularity AUTOSPC
 * (src/solver/boundary_conditions.jl:745-845).                            */
jfg_status jfg_get_node_blocks(jfg_model* model, double* blocks);
/* Element stiffness in the global frame, as captured by element_capture
 * (assembly.jl:5333, 5885, 5918, 5508).  kind: 0=Q4 (24x24), 1=Q8 (48x48),
 * 2=T10 (30x30), 3=T3 (18x18).                                            */
jfg_status jfg_get_element_matrix(jfg_model* model, int32_t kind, int64_t elem,
                                  double* Ke);

/* ---- partition + symbolic analysis ---------------------------------------- */
/* Replaces K_ff = K[free,free] (src/solver/boundary_conditions.jl:1591-1610)
 * and the symbolic half of cholesky(Symmetric(K_ff)) (:1660): nested-
 * dissection ordering, elimination tree, supernodes, front maps.  free_dofs
 * must be strictly ascending global DOF indices.                          */
jfg_status jfg_set_free_dofs(jfg_model* model, int64_t n_free,
                             const int32_t* free_dofs);
jfg_status jfg_get_symbolic_info(jfg_model* model, jfg_symbolic_info* info);
/* No counterpart in the reference, whose worker re-parses and re-analyses
 * every request (warm_model_session.jl:5-99 keeps one model warm).  For a
 * new model `dst` of the same mesh as a resident model `src` (same grid count
 * and CQUAD4 / CTETRA10 connectivity, no CQUAD8, whose pattern depends on the
 * element values): copies src's CSC pattern and slot map (device to device)
 * and keeps src's symbolic analysis, so that the first jfg_assemble on dst
 * skips the pattern build and jfg_set_free_dofs skips the ordering and
 * analysis when its free set equals src's.  Call before dst's first
 * jfg_assemble.  Different meshes give JFG_BAD_INPUT.                     */
jfg_status jfg_model_share_structure(jfg_model* dst, const jfg_model* src);
/* Fill-reducing permutation (F.p of the factor object, :1666): perm[k] = the
 * position in free_dofs of the k-th eliminated unknown.                   */
jfg_status jfg_get_perm(jfg_model* model, int32_t* perm);

/* ---- numeric factorisation and solves ------------------------------------ */
/* Replaces cholesky(Symmetric(K_ff)) numeric phase (:1656-1660).          */
jfg_status jfg_factor(jfg_model* model, int32_t precision);
/* diag(F) in permuted order (:1663): L_ii of the FP64 or mixed factor.     */
jfg_status jfg_get_factor_diag(jfg_model* model, double* Ldiag);
/* Replaces F \ F_ff (:1714, cached path :1442) for nrhs load cases at once.
 * F and U are ndof x nrhs column-major GLOBAL vectors; U is zero at fixed
 * DOFs.  tol is the relative residual target of iterative refinement
 * (<= 0: 1e-10), max_ir the refinement-step cap (<0: 10).                  */
jfg_status jfg_solve(jfg_model* model, int32_t nrhs, const double* F,
                     double* U, double tol, int32_t max_ir,
                     jfg_solve_report* report);
/* R = K*U - F over all ndof (solve_case.jl:1200); SPC forces are R at the
 * fixed DOFs (solve_case.jl:212-262).                                       */
jfg_status jfg_residual(jfg_model* model, int32_t nrhs, const double* U,
                        const double* F, double* R);

/* Element stresses and strains from displacement fields U (ndof x nrhs,
 * column-major, the node-frame displacements jfg_solve returns), the step
 * after the solve in _build_results_from_state (solve_case.jl:182-303).
 * kind 0 = CQUAD4, at the element centre in the element frame as
 * recover_shell_stresses! on the default isotropic PSHELL path
 * (src/solver/stress_recovery.jl:505-1237): out is nrhs x n_q4 records of
 * 31 doubles (load case major): forces fx fy fxy mx my mxy qx qy; stresses
 * at fibre -T/2 then +T/2, each sx sy txy von_mises major minor; membrane
 * strain ex ey gxy major minor; curvature (-kappa, the reference's sign)
 * kx ky kxy major minor; the major principal stress at -T/2.  The shear
 * resultant is the area-mean MacNeal resultant.  Elements whose stiffness
 * was refused get NaN records.  The bilinear corner forces are not
 * returned.
 * kind 2 = CTETRA10, at the element centroid as recover_solid_stresses!
 * (src/solver/stress_recovery.jl:1823-1960): out is nrhs x n_t10 records of
 * 13 doubles (load case major): sxx syy szz txy tyz tzx, exx eyy ezz gxy gyz
 * gzx (engineering shears), von Mises, in the basic frame.  Other kinds
 * return JFG_UNSUPPORTED.                                                  */
jfg_status jfg_recover_stresses(jfg_model* model, int32_t kind, int32_t nrhs,
                                const double* U, double* out);

/* Same as jfg_solve with F and U in DEVICE memory (ndof x nrhs, column-major). */
jfg_status jfg_solve_device(jfg_model* model, int32_t nrhs, const double* F_dev,
                            double* U_dev, double tol, int32_t max_ir,
                            jfg_solve_report* report);
/* No counterpart in the reference (for admission control in a server):
 * device bytes the model holds now, and the bytes it will hold once factored
 * at `precision` (with any factor it already has) and solved with `nrhs`
 * right-hand sides (work space of up to 32 at a time).  Needs the symbolic
 * analysis for the numeric part; before it only the inputs and pattern count. */
jfg_status jfg_get_memory(jfg_model* model, int32_t precision, int32_t nrhs, int64_t* now,
                          int64_t* peak);

/* ---- asynchronous calls ---------------------------------------------------- */
/* The reference's calls block (cholesky(Symmetric(K_ff)) and F \ b at
 * boundary_conditions.jl:1660, 1714); these variants only enqueue, so that a
 * caller overlaps the factorisation and its applications with its own work
 * on `stream` (a cudaStream_t; the library's stream waits for the work the
 * caller has already put there, and the caller's stream waits for the
 * library's).  jfg_factor_async enqueues the numeric factorisation (its first
 * call for a precision allocates and so synchronises); its device error
 * record -- a non-positive pivot, an expired tensor-core wait -- is read by
 * jfg_wait, which every synchronous call on the model also makes first.
 * jfg_apply_factor_async enqueues U = K_ff^{-1} F by one application of the
 * last enqueued (or, without one, the current) factor: forward and backward
 * sweeps with no refinement, F and U DEVICE arrays (ndof x nrhs, column-
 * major, U zero at fixed DOFs); a new right-hand-side count may allocate its
 * workspace.  jfg_wait blocks until the model's enqueued work is done.      */
jfg_status jfg_factor_async(jfg_model* model, int32_t precision, void* stream);
jfg_status jfg_apply_factor_async(jfg_model* model, int32_t nrhs, const double* F_dev,
                                  double* U_dev, void* stream);
jfg_status jfg_wait(jfg_model* model);

/* Device time of the last element, assembly, factor and solve calls (s). */
jfg_status jfg_get_timings(jfg_model* model, double* seconds4);

/* No counterpart in the reference.  Re-runs the element kernels and the
 * slot-map gather of jfg_assemble and writes K's nnz values (the order of
 * jfg_get_pattern) to nzval_dev, a DEVICE buffer the caller owns, without
 * allocating any device memory: for callers that cannot call cudaMalloc
 * between solves (device memory held by another framework's caching pool,
 * or other streams that a device-wide cudaMalloc/cudaFree would stall).
 * The element matrices live in one fixed 16 MiB device array of the
 * library, so models needing more element storage (about 2,600 CQUAD4 or
 * 2,300 CTETRA10) get JFG_BAD_INPUT.  jfg_assemble must have been called
 * once on the model (it builds the pattern).  All calls on a device share
 * that array: calls that overlap on the GPU race and must be serialised.
 * The first call on each device looks the array's address up; make it
 * before starting any stream capture on that device.  Returns after the
 * values are written (synchronises the model's stream).                  */
jfg_status jfg_assemble_values_noalloc(jfg_model* model, double* nzval_dev);

/* ---- instrumentation ----------------------------------------------------- */
/* Number of kernels this library has launched since load.                   */
int64_t jfg_launch_count(void);
/* When on (1), the library brackets the launches of its main kernels with
 * CUDA events on its stream and accumulates, per kernel class, launches,
 * device milliseconds and algorithmic work (which: 0 = Schur-complement
 * update, flops; 1 = CQUAD4 element kernel, bytes; 2 = assembly gather,
 * bytes; 3 = triangular solves, bytes; 4 = CTETRA10 element kernel, bytes).
 * Level 2 also brackets every factor and solve kernel class (5 = extend-add,
 * 6 = diagonal-block Cholesky and inverse, flops; 7 = panel triangular
 * solve, flops; 8 = panel updates, flops; 9..13 = solve sweeps).  While on,
 * the factor and solve loops run eagerly instead of as CUDA graphs.        */
jfg_status jfg_set_profiling(int32_t on);
jfg_status jfg_get_kernel_stats(int32_t which, double* out3);
jfg_status jfg_reset_kernel_stats(void);

/* ---- host-only analysis (no device needed) ----------------------------------- */
/* Runs the symbolic analysis of jfg_set_free_dofs on a given pattern and
 * returns its summary and permutation; used to check the ordering on hosts
 * without a GPU.  colptr/rowval: CSC pattern of K (ndof = 6*n_nodes).       */
jfg_status jfg_symbolic_dry_run(int64_t ndof, const int64_t* colptr,
                                const int32_t* rowval, int64_t n_free,
                                const int32_t* free_dofs, const double* xyz,
                                jfg_symbolic_info* info, int32_t* perm);

/* ---- re-solve fast paths --------------------------------------------------- */
/* New Q4 sections for a subset of elements (thickness change): element +
 * assembly values are recomputed on the next jfg_assemble; the symbolic
 * analysis is kept (warm_model_session.jl:39-99 re-solve without re-parse). */
jfg_status jfg_update_q4_sections(jfg_model* model, int64_t n,
                                  const int32_t* q4_elems,
                                  const double* q4_sect);

#ifdef __cplusplus
}
#endif
#endif /* JFEMGPU_H */
