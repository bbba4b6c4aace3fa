/*
 * b200ldl: B200 (sm_100a) supernodal multifrontal LDL^T / Cholesky for
 * Amigo's interior-point KKT systems  K = [[H + Sigma, A^T], [A, -delta I]].
 *
 * C ABI. Plain pointers and sizes only. Every call returns an int status:
 *   0   success
 *   >0  numerical condition (see b200ldl_last_error)
 *   <0  argument, allocation or CUDA error (the handle stays usable)
 * Nothing aborts the process.
 *
 * Matrix convention (same as the reference's CSRMat input to SparseLDL):
 * one CSR over all n variables holding the FULL symmetric pattern, 0-based
 * int32 indices, double values, every row containing its diagonal. The
 * optional diagonal vector `diag` is added to the diagonal during the
 * factorization (Amigo passes Sigma + delta_w on primal rows and -delta_c on
 * constraint rows this way).
 *
 * Each entry point names the reference interface it replaces
 * (Mersoltane/amigo, paths relative to the repository root).
 */
#ifndef B200LDL_H
#define B200LDL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b200ldl_handle* b200ldl_t;

/* Solver type, as amigo::SparseLDL<T>::SolverType (include/sparse_ldl.h:23). */
#define B200LDL_LDL 0
#define B200LDL_CHOLESKY 1

/* Orderings, numbered as amigo::OrderingType (include/ordering_utils.h:21).
 * NESTED_DISSECTION is the identity (the reference without METIS,
 * include/ordering_utils.h:189-194); MULTI_COLOR is rejected. */
#define B200LDL_ORDER_NESTED_DISSECTION 0
#define B200LDL_ORDER_AMD 1
#define B200LDL_ORDER_MULTI_COLOR 2
#define B200LDL_ORDER_NATURAL 3
/* Our own nested dissection without METIS (no counterpart in the reference,
 * whose nested dissection needs METIS): dense rows last, recursive
 * separators from breadth-first level structures, AMD on small parts. */
#define B200LDL_ORDER_GRAPH_ND 4

/* Create a solver for a fixed sparsity pattern and run the symbolic phase on
 * the host (ordering, elimination tree, supernodes, contribution rows), then
 * upload the assembly and extend-add maps to the current CUDA device.
 * rowp/cols are host arrays. Replaces SparseLDL::SparseLDL
 * (include/sparse_ldl.h:65-118); defaults there are ustab = 0.01,
 * pivot_tol = 1e-14, delay_growth = 2.0. */
int b200ldl_create(b200ldl_t* out, int n, int nnz, const int* rowp,
                   const int* cols, int solver_type, double ustab,
                   double pivot_tol, double delay_growth, int order);

/* Release the handle and its device memory. */
void b200ldl_destroy(b200ldl_t h);

/* Run subsequent work on this cudaStream_t (0 = the legacy default stream). */
int b200ldl_set_stream(b200ldl_t h, void* stream);

/* Numeric factorization of the CSR values `vals` [nnz] plus the optional
 * diagonal `diag` [n] (NULL for none); both are DEVICE pointers. Threshold
 * 1x1/2x2 pivoting with delayed pivots inside fronts, Bunch-Kaufman at
 * roots. Replaces SparseLDL::factor (include/sparse_ldl.h:136-158) and, for
 * device-resident data, CSRMatFactorCuda::factor
 * (include/cuda/csr_factor_cuda.h:13-35). Synchronizes the handle's stream. */
int b200ldl_factor(b200ldl_t h, const double* vals, const double* diag);

/* Same with HOST vals/diag (copied in on the handle's stream). */
int b200ldl_factor_host(b200ldl_t h, const double* vals, const double* diag);

/* Solve K x = b in place for nrhs right-hand sides stored column-major with
 * leading dimension ldx >= n (DEVICE pointer). Replaces
 * SparseLDL::solve(int nrhs, T* x, int ldx) (include/sparse_ldl.h:191-197)
 * and CSRMatFactorCuda::solve. K is symmetric, so this is also the
 * transposed (adjoint) solve. */
int b200ldl_solve(b200ldl_t h, int nrhs, double* x, int ldx);

/* Same with a HOST array x (copied in and out). */
int b200ldl_solve_host(b200ldl_t h, int nrhs, double* x, int ldx);

/* Solve with FP64 iterative refinement against the matrix itself: x = K^-1 b
 * by the stored factor, then up to max_iter corrections x += K^-1 (b - K x)
 * with the residual from the CSR values `vals` and `diag` (DEVICE pointers,
 * the same matrix that was factored, or its exact FP64 version when the
 * factor is approximate) until every column's backward error
 * ||b - Kx||_inf / (||K||_inf ||x||_inf + ||b||_inf) is <= tol. b (ldb) is
 * left unchanged, x (ldx) receives the solution; both DEVICE. berr_out (HOST,
 * nrhs entries, may be NULL) receives the final backward errors and
 * iters_out (HOST, may be NULL) the most corrections any column used. The
 * reference has no refinement (amigo/algorithm/solvers/linear_solver.py:5-35
 * has no such method although newton_direction.py:6-8 asks for one). */
int b200ldl_solve_refine(b200ldl_t h, const double* vals, const double* diag,
                         int nrhs, const double* b, int ldb, double* x,
                         int ldx, int max_iter, double tol, double* berr_out,
                         int* iters_out);

/* Precision of the factorization (no counterpart in the reference, which
 * computes everything in FP64, include/sparse_ldl.h:1190-1215 and
 * 1316-1553). B200LDL_FP64 (the default): every update in FP64.
 * B200LDL_MIXED: in the blocked panels that fronts re-planned from a pivot
 * record use (b200ldl_set_pivot_record), the trailing-update tiles of the
 * contribution block (the rows the parent assembles, never pivoted in the
 * front) run on the tensor cores with about FP32 accuracy (see
 * b200ldl_schur_update_tc); the fully summed columns, every pivot decision
 * and all other fronts stay in FP64. Two checks keep the results those of
 * an FP64 factorization: a mixed factorization whose inertia differs from
 * the last FP64 factorization of the handle is redone in FP64 (FP32-level
 * rounding can flip the sign of a pivot that cancellation makes tiny; with
 * no FP64 factorization on the handle yet the factorization runs in FP64),
 * and b200ldl_solve / b200ldl_solve_host refine every solution in FP64
 * against the factored matrix (the vals and diag of the factor call, which
 * must stay valid until the solves) to the tolerance of
 * b200ldl_set_refinement, refactoring in FP64 and solving again if the
 * refinement stalls. Applies from the next factorization. */
#define B200LDL_FP64 0
#define B200LDL_MIXED 1
int b200ldl_set_precision(b200ldl_t h, int mode);

/* Refinement of the solves after a mixed-precision factorization: at most
 * max_iter corrections per solve, until every column's backward error is
 * <= tol (defaults 5 and 1e-12). */
int b200ldl_set_refinement(b200ldl_t h, int max_iter, double tol);

/* The last refinement: corrections used, the largest backward error,
 * whether the factor in use ran mixed tiles, and how many factorizations of
 * the handle the mixed-precision checks redid in FP64 (any pointer may be
 * NULL). */
int b200ldl_last_refinement(b200ldl_t h, int* iters, double* berr, int* mixed, int* fallbacks);

/* Inertia of the last factorization: numbers of positive and negative
 * pivots (zero pivots count as positive, as the reference does). Replaces
 * SparseLDL::get_inertia (include/sparse_ldl.h:205-213). */
int b200ldl_get_inertia(b200ldl_t h, int* npos, int* nneg);

/* Many independent systems in one handle, factored and solved together
 * (one level-scheduled forest). The reference factors them one at a time,
 * each with its own SparseLDL (include/sparse_ldl.h:65-118); each system
 * here gets the same symbolic phase as it would alone. sys_n[s], sys_nnz[s]:
 * size and nonzeros of system s; rowp_cat: the systems' CSR row pointers
 * one after another (n_s + 1 entries each, local offsets); cols_cat: their
 * column indices one after another (local indices). b200ldl_factor and
 * b200ldl_solve then take the systems' values, diagonals and right-hand
 * sides concatenated in the same order (total size sum n_s). */
int b200ldl_create_batch(b200ldl_t* out, int nsys, const int* sys_n, const int* sys_nnz,
                         const int* rowp_cat, const int* cols_cat, int solver_type,
                         double ustab, double pivot_tol, double delay_growth, int order);

/* Derivatives of a scalar loss through x = K^{-1} b (no counterpart in the
 * reference, which differentiates post-optimality with extra solves on the
 * host, amigo/algorithm/ipm_driver.py:297-353): given the solution x and the
 * adjoint lam = K^{-1} (dloss/dx) from b200ldl_solve on the same factor,
 * writes gvals[e] = -sum_r lam(i,r) x(j,r) for every stored entry e = (i,j)
 * of the CSR pattern and, if gdiag is not NULL, gdiag[i] = -sum_r lam(i,r)
 * x(i,r). dloss/db is lam itself. Device pointers, nrhs <= 8. For values
 * that are kept symmetric (K(i,j) and K(j,i) from the same parameter) the
 * entry-wise gradients sum to the exact derivative. */
int b200ldl_value_gradient(b200ldl_t h, int nrhs, const double* lam, int ldl, const double* x,
                           int ldx, double* gvals, double* gdiag);

/* Number of systems in the handle (1 for b200ldl_create). */
int b200ldl_num_systems(b200ldl_t h);

/* Inertia correction, one attempt per call (Algorithm IC of Waechter and
 * Biegler, as amigo/algorithm/solvers/inertia_correction.py:308-383 drives
 * it). b200ldl_set_perturbation_rows stores, once per pattern, the rows that
 * take +delta_x (primal, HOST array of nprimal distinct indices) and those
 * that take -delta_c (constraints, ndual distinct indices): the index sets
 * InertiaCorrector._compute_perturbation adds to (lines 280-293, which use
 * problem.get_primal_indices / get_constraint_indices). */
int b200ldl_set_perturbation_rows(b200ldl_t h, int nprimal, const int* primal, int ndual,
                                  const int* dual);

/* Factor K + diag(d) with d = diag (+ delta_x on the primal rows when
 * delta_x > 0) (- delta_c on the constraint rows when delta_c > 0), formed
 * on the device in that order (vals, diag DEVICE; diag may be NULL), and
 * return the inertia (npos, nneg: HOST, may be NULL). Replaces
 * InertiaCorrector._apply_and_factor (inertia_correction.py:308-316), whose
 * caller passes delta_x = numerical_eps + delta_w: the values and the
 * diagonal stay on the device across attempts and only the two counts come
 * back. delta_x and delta_c must be finite and >= 0. */
int b200ldl_factor_perturbed(b200ldl_t h, const double* vals, const double* diag,
                             double delta_x, double delta_c, int* npos, int* nneg);

/* The diagonal d of the last b200ldl_factor_perturbed into out [n] (DEVICE),
 * e.g. for b200ldl_solve_refine against the matrix that was factored. */
int b200ldl_copy_perturbed_diagonal(b200ldl_t h, double* out);

/* Inertia of every system of the last factorization (arrays of
 * b200ldl_num_systems entries), with get_inertia's counting rule. */
int b200ldl_system_inertia(b200ldl_t h, int* npos, int* nneg);

/* Message for the last non-zero status on this handle ("" if none). */
const char* b200ldl_last_error(b200ldl_t h);

/* Sizes of the symbolic structure: number of supernodes and total number
 * of contribution rows. */
int b200ldl_symbolic_sizes(b200ldl_t h, int* num_nodes, int* num_contrib);

/* Copy the supernodal structure the factorizations run on (the reference's
 * symbolic structure unless b200ldl_set_pivot_record replaced it) to host
 * arrays (any pointer may be NULL):
 * invperm [n], node_ptr [num_nodes+1], node_to_var [n], children_ptr
 * [num_nodes+2] (roots in slot num_nodes), children [num_nodes],
 * contrib_ptr [num_nodes+1], contrib_rows [num_contrib]. Same layout and
 * numbering as the reference's SparseLDL members (include/sparse_ldl.h:
 * 3269-3286). */
int b200ldl_get_symbolic(b200ldl_t h, int* invperm, int* node_ptr,
                         int* node_to_var, int* children_ptr, int* children,
                         int* contrib_ptr, int* contrib_rows);

/* Per-supernode pivot and delayed-pivot counts of the last factorization
 * (host arrays of length num_nodes). */
int b200ldl_node_pivots(b200ldl_t h, int* num_pivots, int* num_delayed);

/* Pivot-order reuse (no counterpart in the reference: every
 * SparseLDL::factor starts again from the symbolic supernodes,
 * include/sparse_ldl.h:136-158, and delays the same candidates through the
 * same fronts each time, factor_front_matrix_block, sparse_ldl.h:1316-1553).
 *
 * The pivot record of a factorization is, per supernode k, its front size
 * f[k], its pivots npiv[k], its delayed candidates ndel[k], and its front
 * variables after pivoting: npiv[k] pivots in elimination order (2x2 pairs
 * adjacent, each encoded -(v+1)), then the ndel[k] delayed candidates, then
 * the contribution rows; fv holds these lists one supernode after another
 * (sum of f[k] entries). b200ldl_get_pivot_record reads it from the last
 * factorization into host arrays (any may be NULL; *fv_len receives the
 * length of fv). */
int b200ldl_get_pivot_record(b200ldl_t h, int* f, int* npiv, int* ndel, int* fv,
                             long long* fv_len);

/* Re-plan the fronts from a pivot record (host arrays as above, num_nodes
 * entries each, from any factorization of this pattern): supernode k's
 * pivot columns become the variables it eliminated, in that order, and the
 * candidates it delayed become contribution rows, so each candidate is
 * tested in the front that accepted it instead of being delayed through the
 * fronts below it. The elimination tree is kept; the threshold tests and
 * delays still apply to every factorization, so a candidate that fails in
 * its new front is delayed as before. All four pointers NULL returns to the
 * reference's symbolic structure. The last factor is dropped; factor again
 * before solving. Status -4 if the record does not describe a valid
 * elimination of this pattern (the handle keeps its structure). */
int b200ldl_set_pivot_record(b200ldl_t h, const int* f, const int* npiv, const int* ndel,
                             const int* fv);

/* b200ldl_set_pivot_record with the last factorization's own record. */
int b200ldl_reuse_pivot_order(b200ldl_t h);

/* Statistics of the last factorization: stats[0] = factor flops actually
 * executed (dense partial factorizations of the fronts as sized at run
 * time), stats[1] = bytes of the factor L, stats[2] = bytes of the
 * contribution blocks, stats[3] = largest front, stats[4] = number of
 * delayed pivots summed over supernodes, stats[5] = number of levels. */
int b200ldl_stats(b200ldl_t h, double* stats, int nstats);

/* Profiling (no counterpart in the reference, which has no GPU timers):
 * when enabled, CUDA events on the handle's stream time each kernel class.
 * b200ldl_profile writes, for each class p in {fronts, big-front assembly,
 * big-front panels, big-front trailing updates, forward solve, backward
 * solve, fronts factored on chip in a thread-block cluster}, out[2p] =
 * accumulated milliseconds and out[2p+1] = kernel launches since the last
 * reset. */
int b200ldl_set_profiling(b200ldl_t h, int enable);
int b200ldl_reset_profile(b200ldl_t h);
int b200ldl_profile(b200ldl_t h, double* out, int n);

/* Kernels launched by this handle since creation. */
long long b200ldl_launch_count(b200ldl_t h);

/* Work of the last factorization: out[0] = flops executed in all fronts,
 * out[1] = of which in big-front panels, out[2] = in big-front trailing
 * updates, out[3] = bytes moved by the trailing updates, out[4] = flops in
 * fronts factored on chip in a thread-block cluster; after pivot-order
 * reuse, the blocked panels with a-posteriori tests: out[5] = panels,
 * out[6] = panels cut short because the a-posteriori test rejected a pivot,
 * out[7] = candidates delayed inside a panel's diagonal block. */
int b200ldl_work(b200ldl_t h, double* out, int n);

/* KKT assembly: element Hessian blocks into the values of the fixed CSR
 * pattern, on the device. Replaces the Hessian assembly of
 * OptimizationProblem::hessian (include/optimization_problem.h:1063-1088):
 * the matrix zeroed, then for each component group, element and column j of
 * the element's Hessian, the column added into CSR row conn[e][j] at
 * columns conn[e][i] with entries outside the pattern dropped
 * (ComponentGroup::add_hessian_kernel, include/component_group.h:144-162,
 * CSRMat::add_row, include/csr_matrix.h:554-567; the GPU backend's
 * atomicAdd scatter, include/cuda/component_group_backend.cuh:157-190).
 * The values are summed in exactly that order, so they are bit-identical to
 * the reference's CPU assembly. */
typedef struct b200ldl_assembly* b200ldl_assembly_t;

/* Plan the assembly on the host (no device work until the first
 * b200ldl_assembly_values). rowp/cols: the CSR pattern (n rows, sorted
 * columns), HOST. ngroups component groups; group g has nelems[g] elements
 * of ncomp[g] variables; conn: the groups' [nelems][ncomp] global variable
 * indices one after another (int32, HOST). On failure *out still holds a
 * handle whose b200ldl_assembly_last_error says why; destroy it. */
int b200ldl_assembly_create(b200ldl_assembly_t* out, int n, const int* rowp, const int* cols,
                            int ngroups, const int* nelems, const int* ncomp, const int* conn);

/* vals[nnz] = the assembled CSR values from blocks, the groups' element
 * blocks one after another, block[e][j][i] = column j, row i of element e's
 * Hessian, which must hold the number of block values b200ldl_assembly_info
 * reports in out[2] (DEVICE pointers; asynchronous on stream, a
 * cudaStream_t or NULL).
 * The output feeds b200ldl_factor directly. The plan is copied to the
 * current device at the first call and used there from then on. */
int b200ldl_assembly_values(b200ldl_assembly_t a, const double* blocks, double* vals,
                            void* stream);

/* out[0] = contributions kept, out[1] = contributions outside the pattern
 * (dropped, as add_row drops them), out[2] = block values expected,
 * out[3] = nnz; the first nout of them. */
int b200ldl_assembly_info(b200ldl_assembly_t a, long long* out, int nout);

/* The plan (HOST arrays, may be NULL): ptr [nnz + 1] and src [out[0] of
 * b200ldl_assembly_info]; CSR entry p sums blocks[src[ptr[p] .. ptr[p+1])]
 * in that order. */
int b200ldl_assembly_plan(b200ldl_assembly_t a, long long* ptr, long long* src);

const char* b200ldl_assembly_last_error(b200ldl_assembly_t a);
void b200ldl_assembly_destroy(b200ldl_assembly_t a);

/* Factor from element Hessian blocks without forming the CSR values: the
 * front assembly of b200ldl_factor reads each CSR entry as the sum of its
 * element contributions through the assembly plan a (built by
 * b200ldl_assembly_create for this handle's pattern), in the plan's order,
 * so every front receives the same bits as from b200ldl_assembly_values
 * followed by b200ldl_factor. blocks (the element blocks as
 * b200ldl_assembly_values takes them) and diag: DEVICE pointers. Replaces
 * the reference's assembly into a CSR matrix followed by the factorization:
 * ComponentGroup::add_hessian_kernel + CSRMat::add_row
 * (include/component_group.h:144-162, include/csr_matrix.h:554-567) or the
 * GPU hessian_kernel_atomic (include/cuda/component_group_backend.cuh:
 * 157-190), then SparseLDL::factor(diag) (include/sparse_ldl.h:136-158).
 * FP64 mode only (status -1 in the mixed mode, whose refinement needs the
 * CSR values); the solves work as after b200ldl_factor, b200ldl_solve_refine
 * excepted (it needs the values). */
int b200ldl_factor_elements(b200ldl_t h, b200ldl_assembly_t a, const double* blocks,
                            const double* diag);

/* Dense Schur-complement update on the Blackwell tensor cores (no
 * counterpart in the reference, whose frontal_trailing_update,
 * include/sparse_ldl.h:1190-1215, calls FP64 dgemm): C -= A B^T for A (m x
 * k, lda), B (n x k, ldb) and C (m x n, ldc), column-major FP64 DEVICE
 * arrays; with lower != 0 only entries with row >= column change. The
 * products run as 3xTF32 (each operand split into two TF32 parts) on
 * tcgen05.mma with FP32 accumulation in tensor memory, so the update has
 * about FP32 accuracy: the mixed-precision factorization applies it to the
 * contribution blocks of big fronts. Synchronizes the stream (cudaStream_t,
 * NULL = default). Status 1 if a tensor-core operation did not complete in
 * time. */
int b200ldl_schur_update_tc(int m, int n, int k, const double* a, int lda, const double* b,
                            int ldb, double* c, int ldc, int lower, void* stream);

/* Allocation-free dense solve (no counterpart in the reference; the
 * reference always allocates its factor storage). For callers that must not
 * allocate device memory while running, e.g. a real-time loop re-solving a
 * small KKT system, or a plugin in a process whose framework has reserved
 * the device memory. Factors the dense symmetric matrix a (n x n,
 * column-major, lower triangle read, leading dimension lda) with
 * Bunch-Kaufman LDL^T and overwrites b (n x nrhs, ldb) with the solution;
 * inertia (npos, nneg) goes to inertia[0..1] if not NULL. All pointers are
 * DEVICE pointers; stream is a cudaStream_t (NULL = default stream); the
 * call is asynchronous. Scratch is a fixed device array inside the library:
 * n must be <= 512 (status -6 otherwise), every GPU that loads the library
 * holds the array (2 MiB) until exit, all calls share it, and calls whose
 * kernels overlap on the GPU race on it (order them on one stream). The
 * first call on a device looks up the array's address; make it before any
 * stream capture. Calls no cudaMalloc/cudaFree or allocating routine.
 * A singular matrix is not an error: a zero pivot (a column that is zero at
 * its elimination) counts as positive in the inertia, as the reference
 * counts it, and the solution component it divides gets 0; the status is
 * still 0, so npos + nneg == n does not rule out singularity. */
int b200ldl_dense_solve_noalloc(int n, const double* a, int lda, double* b,
                                int ldb, int nrhs, int* inertia, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* B200LDL_H */
