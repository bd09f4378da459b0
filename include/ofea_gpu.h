/* ofea_gpu.h - C ABI of the B200 implicit-static hot path for OpenFEA models.
 *
 * One GPU, no CPU fallback: every compute entry point runs hand-written
 * sm_100a kernels and fails with OFEA_ERR_NO_DEVICE when no CUDA device is
 * present.  All functions return an int status (OFEA_OK = 0, negative codes
 * below); none calls exit() or throws across the boundary.  ofea_last_error()
 * gives a message for the calling thread's last failure.
 *
 * Threading: a context belongs to one host thread at a time; work on a context
 * is ordered on its CUDA stream.  Host arrays passed in are borrowed for the
 * duration of the call only.  The library owns all device memory it allocates.
 *
 * Conventions (those of the reference's data_management, so a host shim can
 * pass its vectors straight through):
 *   - node ids in `topo` are 1-based, 8 slots per element, C3D4 uses the first
 *     4 (node_topos_, src/include/data_management.h:49);
 *   - etype 0 = C3D4, 1 = C3D8 (ELE_TYPES, src/include/data_management.h:76);
 *   - free_map[node] = free-node index or -1 (resort_free_nodes_,
 *     src/set_bc.cpp:20-43); DOF d = 3*free_map[node] + component, n = 3*nfree;
 *   - K is symmetric; exported in CSR, which equals the reference's CSC arrays
 *     (col_idx_/row_idx_/nz_val_, src/include/assemble.h:41-43).
 */
#ifndef OFEA_GPU_H
#define OFEA_GPU_H

#if defined(__GNUC__)
#define OFEA_API __attribute__((visibility("default")))
#else
#define OFEA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define OFEA_OK 0
#define OFEA_ERR_INVALID_ARG (-1)   /* bad pointer, size, id or option */
#define OFEA_ERR_CUDA (-2)          /* a CUDA runtime call failed */
#define OFEA_ERR_OOM (-3)           /* device allocation failed */
#define OFEA_ERR_NOT_CONVERGED (-4) /* max_iter reached above rtol */
#define OFEA_ERR_TIMEOUT (-5)       /* time_budget_s exceeded */
#define OFEA_ERR_STATE (-6)         /* call out of order (e.g. solve before assemble) */
#define OFEA_ERR_CAPACITY (-7)      /* mesh exceeds a kernel limit (neighbour count) */
#define OFEA_ERR_BREAKDOWN (-8)     /* p.Kp <= 0 or NaN: K not SPD (e.g. no BCs) */
#define OFEA_ERR_NO_DEVICE (-9)     /* no CUDA device visible */
#define OFEA_ERR_IO (-10)           /* file cannot be read / parsed / written */
#define OFEA_ERR_UNKNOWN_SOLVER (-11)
#define OFEA_ERR_REJECTED (-12)     /* learned stage rejected by the FP64 residual check */

/* Solver methods (ofea_solve_opts.method). */
#define OFEA_SOLVER_PCG64 0   /* FP64 PCG, 3x3 block-Jacobi (the plain method) */
#define OFEA_SOLVER_MIXED 1   /* FP64 flexible PCG, FP32 two-level V-cycle preconditioner:
                                 block-Jacobi/Chebyshev smoothing with FP32 SpMV and a
                                 rigid-body coarse correction */
#define OFEA_SOLVER_LEARNED 2 /* MIXED + graph-network coarse correction (flexible PCG) */

typedef struct ofea_ctx ofea_ctx;

typedef struct {
    int method;           /* OFEA_SOLVER_* */
    double rtol;          /* stop when ||f - K u||_2 <= rtol ||f||_2 (FP64 true residual) */
    int max_iter;         /* inner iterations, summed over refinements */
    double time_budget_s; /* <= 0: unlimited */
    int check_every;      /* iterations between host convergence polls (0: 4 for MIXED and LEARNED, 16 for PCG64) */
    double ru_delta;      /* reserved (0) */
    int use_graph;        /* 1: replay iteration chunks as a captured CUDA graph; 0: plain launches */
} ofea_solve_opts;

typedef struct {
    int status;            /* OFEA_OK or an error code */
    int iterations;        /* inner iterations performed */
    int refinements;       /* restarts from a recomputed FP64 residual */
    double rel_residual;   /* final ||f - K u|| / ||f|| in FP64 */
    double seconds;        /* device time of the solve (CUDA events), setup included */
    double setup_seconds;  /* part of `seconds` spent building the preconditioner */
    int rejected_learned;  /* 1 when the learned stage was rejected and plain PCG finished */
    long long kernel_launches;
} ofea_solve_stats;

/* ---- library ---------------------------------------------------------- */
OFEA_API const char *ofea_version(void);
OFEA_API const char *ofea_status_string(int status);
OFEA_API const char *ofea_last_error(void);
/* Fills opts with defaults: PCG64, rtol 1e-8, max_iter 100000, check_every 0 (by method),
 * ru_delta 0.1, use_graph 1, no time budget. */
OFEA_API void ofea_solve_opts_default(ofea_solve_opts *opts);

/* ---- context ---------------------------------------------------------- */
OFEA_API int ofea_ctx_create(ofea_ctx **out, int device);
OFEA_API int ofea_ctx_destroy(ofea_ctx *ctx);
/* No counterpart in the reference.  Device memory the library frees is kept
 * per GPU (up to a quarter of its memory, at most 32 GB) and reused by later
 * allocations of a fitting size (a failed cudaMalloc returns the cached
 * blocks and retries), so
 * that a fresh context does not pay cudaMalloc for every buffer again; large
 * host blocks (the mesh's host copies, set-up scratch; up to 1 GB) are kept
 * the same way so that a new context does not fault in fresh pages.  This
 * returns both to the driver / the C allocator (e.g. before handing the GPU
 * to another allocator). */
OFEA_API int ofea_trim_device_memory(void);
/* Run this context's work on an existing cudaStream_t (NULL: library-owned stream). */
OFEA_API int ofea_ctx_set_stream(ofea_ctx *ctx, void *cuda_stream);

/* ---- mesh -------------------------------------------------------------- */
/* Replaces the data the reference's assemblers read from data_management
 * (src/include/data_management.h:48-62): coordinates nd x 3, topo ne x 8
 * (1-based), etype, per-element Young's modulus E_elem (NULL: E0 everywhere;
 * the reference has one material per element type, src/data_managrment.cpp:20-26),
 * Poisson ratio nu, and the DOF numbering free_map (nd).  Copies to the device. */
OFEA_API int ofea_mesh_upload(ofea_ctx *ctx, int nd, const double *xyz, int ne, const int *topo,
                     const int *etype, const double *E_elem, double E0, double nu,
                     const int *free_map);
/* Replace the per-element Young's modulus (same mesh and pattern). */
OFEA_API int ofea_mesh_set_modulus(ofea_ctx *ctx, const double *E_elem, double E0);

/* ---- assembly ----------------------------------------------------------- */
/* assamble_stiffness::build_CSR (src/assemble.cpp:19-77): the symmetric
 * sparsity pattern, built on the device, plus the element-to-slot map used by
 * the assembly kernels.  Returns n (free DOFs) and nnz (scalar non-zeros). */
OFEA_API int ofea_assemble_pattern(ofea_ctx *ctx, int *n, long long *nnz);
/* assamble_stiffness::fill_CSR_sparse_mat (src/assemble.cpp:95-151): FP64
 * element integration (C3D8 2x2x2 Gauss, C3D4 one point) and atomic-free
 * assembly into K on the device. */
OFEA_API int ofea_assemble_linear(ofea_ctx *ctx);
/* assamble_nl_stiffness::fill_CSR_sparse_mat (src/nl_assemble.cpp:94-166):
 * tangent K_T(u) replaces K on the device; f_int (n, host) receives the
 * internal force.  u: n free-DOF displacements (host). */
OFEA_API int ofea_assemble_nl(ofea_ctx *ctx, const double *u, double *f_int);
/* The matrix the reference has already assembled, as solution_api receives it
 * (src/linear_solution.cpp:17-64, reading item_ass.col_idx_ / row_idx_ /
 * nz_val_, src/include/assemble.h:41-43; solution_nl_api, :66-137, reads
 * assamble_nl_stiffness's col_idx / row_idx / nz_val): K in 0-based CSC, n
 * columns, col_ptr (n+1), row_idx (col_ptr[n], rows ascending in each column),
 * val.  K must be symmetric and 3x3-block structured in the reference's DOF
 * numbering 3*free_map[node]+c (build_CSR always stores every DOF pair of an
 * element, so its output is); a matrix that is not block structured returns
 * OFEA_ERR_INVALID_ARG.  The nd node coordinates (coords_) and free_map
 * (resort_free_nodes_) give the solver's coarse levels their rigid-body
 * modes.  Replaces any mesh or matrix of the context; then ofea_solve /
 * ofea_solve_device / ofea_spmv / ofea_get_csr work as after an assembly,
 * while the element-based calls (assembly, stress) return OFEA_ERR_STATE. */
OFEA_API int ofea_matrix_upload_csc(ofea_ctx *ctx, int nd, const double *xyz, const int *free_map, int n,
                                   const int *col_ptr, const int *row_idx, const double *val);
/* Copy K to the host as CSR: rowptr (n+1), col (nnz), val (nnz); any may be NULL. */
OFEA_API int ofea_get_csr(ofea_ctx *ctx, int *rowptr, int *col, double *val);
/* Element matrices of the last assembly, for checking: Ke of element e in the
 * caller's element order, (3 npe)^2 row-major.  first..first+count-1. */
OFEA_API int ofea_get_element_matrices(ofea_ctx *ctx, int first, int count, double *Ke);
/* y = K x on the device (n values, host arrays). */
OFEA_API int ofea_spmv(ofea_ctx *ctx, const double *x, double *y);

/* ---- solve -------------------------------------------------------------- */
/* solution_api (src/linear_solution.cpp:17-64) / solution_nl_api (:66-137):
 * solve K u = f for nrhs right-hand sides (column-major n x nrhs, host).
 * opts NULL: defaults.  stats may be NULL (one entry per rhs otherwise).
 * With 2..32 right-hand sides and PCG64 or MIXED, all of them are solved
 * together by one persistent launch of the batched solver (ofea_batch_*,
 * one variant), which reads K once per iteration for every load case; the
 * first such call on a problem class tunes its tiles (OFEA_TUNE_FILE).
 * LEARNED, and more than 32 right-hand sides, solve them one after another. */
OFEA_API int ofea_solve(ofea_ctx *ctx, const double *f, double *u, int nrhs, const ofea_solve_opts *opts,
               ofea_solve_stats *stats);
/* Drop the preconditioner built for the current K (coarse operator, smoother
 * bounds), so the next solve rebuilds it; a new assembly does this too. */
OFEA_API int ofea_precond_reset(ofea_ctx *ctx);
/* Same with device pointers (f, u of n doubles each), stream-ordered. */
OFEA_API int ofea_solve_device(ofea_ctx *ctx, const double *d_f, double *d_u, const ofea_solve_opts *opts,
                      ofea_solve_stats *stats);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (an application whose own pool allocator reserves the GPU up front, a
 * latency-critical loop that must not call cudaMalloc/cudaFree because they
 * can synchronize the device): norms[2k] = ||f_k - K u_k||_2 and
 * norms[2k+1] = ||f_k||_2 for load cases k < nrhs, with f, u device arrays of
 * n x nrhs (column-major) and norms a device array of 2 nrhs doubles.  K is
 * the context's assembled matrix.  Allocates nothing: its partial sums live
 * in a 512 KB static device array that every GPU loading this library holds
 * until the process exits.  At most 16 load cases per call; more returns
 * OFEA_ERR_CAPACITY.  ofea_ctx_create looks up that array's device address
 * and loads this entry point's kernels on the context's device (CUDA loads
 * code lazily, which allocates), so the entry point itself allocates nothing
 * from its first call on; create the context before the caller's allocator
 * reserves the GPU.  Calls
 * share the array: calls that overlap on one GPU race and must be ordered by
 * the caller.  Enqueued on the context's stream; returns without waiting. */
OFEA_API int ofea_residual_norms_noalloc(ofea_ctx *ctx, int nrhs, const double *d_f,
                                         const double *d_u, double *d_norms);

/* No counterpart in the reference: the target number of free nodes per
 * aggregate of the MIXED / LEARNED coarse level (default 1000; the learned
 * level's aggregates are 8 times smaller).  Larger aggregates make the
 * per-matrix set-up cheaper (its dense inverse is cubic in their count) and
 * the iterations more numerous.  Invalidates the coarse levels. */
OFEA_API int ofea_set_coarse_nodes(ofea_ctx *ctx, int nodes);

/* No counterpart in the reference: how the MIXED / LEARNED coarse level
 * solves with E = Z^T K Z.  0 (default): E is banded in aggregate order, and
 * where its block half-bandwidth is at most 8 blocks of 64 it is factored as
 * a block LDL^T by one thread-block cluster and applied as two FP32
 * triangular GEMVs; wider bands take the dense inverse.  1: always the dense
 * inverse (blocked Gauss-Jordan, one FP32 GEMV).  A direction whose pivot
 * vanishes (a degenerate aggregate) is dropped by both.  Invalidates the
 * preconditioner of the current K. */
OFEA_API int ofea_set_coarse_solver(ofea_ctx *ctx, int method);
/* The current coarse solve applied to a host vector: y = E^-1 c (m values
 * each, FP32 arithmetic as in the V-cycle); *m_out (if not NULL) = m and
 * *factored (if not NULL) = 1 for the block LDL^T form.  The coarse level
 * must exist (after a MIXED or LEARNED solve); c and y may be NULL to query. */
OFEA_API int ofea_coarse_apply(ofea_ctx *ctx, const double *c, double *y, int *m_out, int *factored);

/* No counterpart in the reference: how ofea_assemble_linear runs.  0
 * (default): C3D8 meshes whose nodes lie in at most 8 elements are integrated
 * and assembled in one pass that writes only the solver's copy of K (block
 * CSR values and element matrices are derived from it when ofea_get_csr or
 * ofea_get_element_matrices asks); other meshes take the two-pass assembly
 * (element matrices, then a gather).  1: always the two-pass assembly.  Both
 * give the same bits. */
OFEA_API int ofea_set_assembly_path(ofea_ctx *ctx, int path);

/* Which assembly produced the current K: 0 the one-pass C3D8 assembly, 1 the
 * two-pass assembly or K uploaded as CSC.  OFEA_ERR_STATE before an
 * assembly. */
OFEA_API int ofea_get_assembly_path(ofea_ctx *ctx, int *path);

/* ---- learned coarse-correction stage -------------------------------------- */
/* No counterpart in the reference.  OFEA_SOLVER_LEARNED adds a second coarse
 * stage to the mixed V-cycle, on nested aggregates (cells half as wide as the
 * exact coarse level's): the level's residual, with the exact coarse
 * correction taken out, is mapped to rigid-body-mode corrections by
 * y = s * M(s * x), M a degree-2 polynomial in the block-Jacobi-preconditioned
 * level operator with trainable coefficients, s per-aggregate scalings set by
 * a 4-layer message-passing network (hidden width 64, FP32 weights and
 * accumulation) from the aggregates' features.  The stage is linear and
 * symmetric.  Trained on the GPU by this library's forward/backward/Adam
 * kernels from the residuals of plain-PCG iterates on the current K, with the
 * energy loss whose minimiser is the level's exact Galerkin correction.  A
 * LEARNED solve whose FP64 true residual misses rtol is redone by plain
 * PCG64 (stats.rejected_learned = 1). */
#define OFEA_LEARN_NFEAT 8 /* features per aggregate */
typedef struct {
    int sample_iters;  /* plain-PCG iterations whose residuals are sampled (600) */
    int sample_every;  /* one sample every this many iterations (4) */
    int steps;         /* Adam steps (400) */
    int batch;         /* samples per step (16) */
    float lr;          /* learning rate (1e-3) */
    unsigned seed;     /* weight initialisation and batch order (1234) */
    int reset;         /* 1: re-initialise the weights before training (0) */
} ofea_learn_opts;

typedef struct {
    int samples;
    int steps;
    double loss_first; /* energy loss of the first batch before the first step */
    double loss_last;  /* ... and of the same batch after the last step */
    double seconds;    /* wall time of sampling + training */
} ofea_learn_stats;

OFEA_API void ofea_learn_opts_default(ofea_learn_opts *opts);
/* f: load of the sampling solves (n host values); NULL: a seeded random load. */
OFEA_API int ofea_learned_train(ofea_ctx *ctx, const double *f, const ofea_learn_opts *opts,
                                ofea_learn_stats *stats);
/* Flat FP32 weight vector: count in *count; w may be NULL to query the size. */
OFEA_API int ofea_learned_get_weights(ofea_ctx *ctx, float *w, long long *count);
OFEA_API int ofea_learned_set_weights(ofea_ctx *ctx, const float *w, long long count);
OFEA_API int ofea_learned_save(ofea_ctx *ctx, const char *path);
OFEA_API int ofea_learned_load(ofea_ctx *ctx, const char *path);
/* The nested level of the current K, for checking: na aggregates, the
 * 27-slot neighbour table (na x 27, -1 = none, slot (dx+1)*9+(dy+1)*3+(dz+1)),
 * the Jacobi-scaled coarse blocks Ehat (na x 27 x 6 x 6) and the network's
 * input features (na x OFEA_LEARN_NFEAT: centred log stiffness, neighbour
 * count / 26, log of the diagonal of the inverse diagonal blocks of Ehat).
 * Arrays may be NULL to query na. */
OFEA_API int ofea_learned_level(ofea_ctx *ctx, int *na, int *nbr, float *Ehat, float *feat);
/* Energy loss (sum over the batch) and its gradient w.r.t. every weight for
 * given stage inputs x (batch x na x 6, scaled level residuals). */
OFEA_API int ofea_learned_gradient(ofea_ctx *ctx, const float *x, int batch, double *loss,
                                   float *grad);

/* No counterpart in the reference.  The learned stage's dense layers run on
 * the tensor cores (tcgen05.mma, BF16 operands in shared memory, FP32
 * accumulation in tensor memory); this exposes that product on its own, for
 * checking: D = A B^T with A (M x K) and B (N x K) row-major FP32 host arrays,
 * each entry rounded to BF16 (nearest even), D (M x N) row-major FP32. */
OFEA_API int ofea_tc_matmul(int device, int M, int N, int K, const float *A, const float *B, float *D);

/* ---- batched reanalysis ---------------------------------------------------- */
/* Replaces the per-variant factor + per-load-case dgstrs loop of the
 * reference's reanalysis (src/solver/solver_superlu.cpp:31-94 SuperLU_class /
 * superlu_solution_next, driven by src/ca_analysis.cpp:148-248): many
 * assembled variants (one context each, all on one GPU) times up to 32 load
 * cases each, solved together by one persistent cooperative kernel launched
 * from a CUDA graph.  Methods OFEA_SOLVER_MIXED (FP64 flexible CG + FP32
 * two-level V-cycle per variant) and OFEA_SOLVER_PCG64.  Its tile sizes
 * (load cases per lane, hence the CTA size, and CTAs per SM) are chosen by
 * timing candidates on the first solve of a problem class and kept in a JSON
 * file (OFEA_TUNE_FILE, default ~/.cache/openfea_b200_tune.json).  The batch borrows the contexts:
 * keep them alive and unchanged until ofea_batch_destroy. */
typedef struct ofea_batch ofea_batch;
#define OFEA_BATCH_MAX_RHS 32
OFEA_API int ofea_batch_create(ofea_batch **out, ofea_ctx *const *ctxs, int n_variants, int nrhs);
OFEA_API int ofea_batch_destroy(ofea_batch *batch);
/* f[v]: the nrhs load cases of variant v, case j at f[v] + j * n_v (host). */
OFEA_API int ofea_batch_set_rhs(ofea_batch *batch, const double *const *f);
/* Solves on the load cases last set; the solution stays on the device.
 * stats: n_variants entries (worst load case of each variant). */
OFEA_API int ofea_batch_solve_resident(ofea_batch *batch, const ofea_solve_opts *opts,
                                       ofea_solve_stats *stats);
/* u[v]: nrhs * n_v host values, laid out like f. */
OFEA_API int ofea_batch_get_solution(ofea_batch *batch, double *const *u);
/* set_rhs + solve_resident + get_solution. */
OFEA_API int ofea_batch_solve(ofea_batch *batch, const double *const *f, double *const *u,
                              const ofea_solve_opts *opts, ofea_solve_stats *stats);
/* The tile configuration used for `method` (tuning it now if needed). */
OFEA_API int ofea_batch_tuning(ofea_batch *batch, int method, int *rhs_per_lane, int *threads,
                               int *ctas_per_sm, double *ms_per_iteration);
/* Phase trace (no counterpart in the reference, which prints clock() spans):
 * with max_phases > 0 every later solve launch records the device clock
 * (%globaltimer, CTA 0) at its start and after each of its grid barriers, at
 * most max_phases of them; 0 turns it off.  ofea_batch_phase_times returns
 * the durations in milliseconds between consecutive records of the last
 * launch, in barrier order (MIXED: init, init pairs, then the V-cycle's five
 * phases and its pair step, then per iteration A, pairs, B, pairs, the
 * V-cycle's five and its pair step; PCG64: init, init pairs, r.z, pairs,
 * then A, pairs, B, pairs per iteration); *count = how many exist, up to cap
 * are written (ms may be NULL to query). */
OFEA_API int ofea_batch_set_trace(ofea_batch *batch, int max_phases);
OFEA_API int ofea_batch_phase_times(ofea_batch *batch, double *ms, int cap, int *count);
/* One-call form: create, solve, destroy. */
OFEA_API int ofea_solve_batched(ofea_ctx *const *ctxs, int n_variants, const double *const *f,
                                double *const *u, int nrhs, const ofea_solve_opts *opts,
                                ofea_solve_stats *stats);
/* Checks the failure path of the batched solver's grid barrier: launches a
 * cooperative kernel whose barrier waits for one CTA more than exists; every
 * wait gives up after limit_ms and *released is set to 0 (1 would mean the
 * barrier opened).  The context stays usable. */
OFEA_API int ofea_check_barrier_timeout(ofea_ctx *ctx, int limit_ms, int *released);

/* ---- stress recovery ------------------------------------------------------ */
/* Replaces simulation_post::get_cauchy_stress_3d (src/post_process.cpp:79-167):
 * per element xx, yy, zz, xy, yz, xz and von Mises (the reference's expression,
 * :103-109), and per node the mean over its incident elements.  u: host [n]
 * (free DOF; fixed DOF are zero).  OFEA_STRESS_REFERENCE gives the reference's
 * numbers: for C3D4 the engineering strain B u that its get_stress_node_hammer
 * returns as stress (src/Elements/C3D4_hammer.cpp:219-226), for C3D8 zero (the
 * reference computes nothing there and leaves the values unset).
 * OFEA_STRESS_CAUCHY gives the Cauchy stress D B u (C3D8: the mean over its 8
 * Gauss points).  elem: host [ne x 7] in caller element order, node: host
 * [7 x nd] (component-major, as the reference's stress_node_mat_); either may
 * be NULL.  Needs the pattern (node-to-element incidence). */
#define OFEA_STRESS_REFERENCE 0
#define OFEA_STRESS_CAUCHY 1
OFEA_API int ofea_stress(ofea_ctx *ctx, const double *u, int mode, double *elem, double *node);

/* ---- CA reanalysis -------------------------------------------------------- */
/* Replaces the combined-approximations reanalysis of the reference:
 * ca_get_delt_stiffness / ca_build_rom / ca_SVD / ca_solve
 * (src/ca_analysis.cpp:18-30, 146-250), driven by CAE_process::CA_ReAnalysis
 * (src/cae.cpp:317-375).  base: the original model, K0 assembled.  modified:
 * the modified model on the SAME nodes, element list and free numbering, K
 * assembled: a deleted element has E = 0 there (an added one is in both
 * meshes, with E = 0 in the base), moved nodes carry their new coordinates.
 * Then ΔK x = K x - K0 x.  Basis r_0 = u0 (host [n], the base solution; NULL:
 * solved here), r_i = -K0^-1 ΔK r_(i-1) for 0 < i < n_basis (device solves
 * with opts), made orthonormal in FP64 (directions whose Gram eigenvalue is
 * below 1e-13 of the largest are dropped); the reduced system
 * V^T K V y = V^T f is solved on the host and u = V y.  f: the load (host
 * [n]; the reference uses the original model's), u: host [n] out.
 * Differences from the reference: its basis SVD runs in FP32 (here FP64, the
 * same span), and its moved-element branch reads the old coordinates into
 * the wrong row (src/ca_analysis.cpp:103-105); here a moved node changes
 * every element on it, through the modified model's assembly. */
#define OFEA_CA_MAX_BASIS 32
typedef struct {
    int status;
    int basis_requested;
    int basis_used;        /* after dropping dependent directions */
    int solve_iterations;  /* summed over the solves with K0 */
    double rel_residual;   /* ||f - K u|| / ||f|| of the CA solution on the modified K */
    double seconds;        /* wall time of the call */
} ofea_ca_stats;
OFEA_API int ofea_ca_reanalysis(ofea_ctx *base, ofea_ctx *modified, const double *f, const double *u0,
                                int n_basis, const ofea_solve_opts *opts, double *u, ofea_ca_stats *stats);

/* ---- measurement ------------------------------------------------------- */
/* No counterpart in the reference (it only prints clock() spans): times the
 * solver's two per-iteration kernels (A: p update + SpMV + p.q, B: vector
 * updates + block-Jacobi + dots) of `method` in isolation, `reps` launches
 * each between CUDA events on the context's stream, on the current K and
 * solver vectors (call after a solve).  ms[0], ms[1] = average milliseconds
 * per launch of A and B; bytes[0], bytes[1] = algorithmic bytes per launch
 * (every array the kernel must touch, counted once). */
OFEA_API int ofea_profile_solver_kernels(ofea_ctx *ctx, int method, int reps, double *ms,
                                         double *bytes);
/* Set-up trace (no counterpart in the reference): with on != 0 every later
 * MIXED or LEARNED solve records CUDA events on the context's stream at the
 * phase boundaries of its preconditioner set-up (the coarse levels' Galerkin
 * blocks, the coarse inverse, the smoother interval, the network).
 * ofea_setup_phase_times returns the last set-up's phases: ms[i] = device
 * milliseconds of phase i, names = the phase names separated by ',' (NUL
 * terminated, cut at names_len); *count = how many exist, up to cap are
 * written (ms and names may be NULL to query). */
OFEA_API int ofea_set_setup_trace(ofea_ctx *ctx, int on);
OFEA_API int ofea_setup_phase_times(ofea_ctx *ctx, double *ms, int cap, int *count, char *names,
                                    int names_len);

#ifdef __cplusplus
}
#endif
#endif /* OFEA_GPU_H */
