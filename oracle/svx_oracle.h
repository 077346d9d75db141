/*
 * svx_oracle.h - CPU oracle for the Solvix linear-static path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a C++ restatement of the reference's
 * Rust arithmetic (crates/solvix-core/src/{element,assembly,solver,stress,
 * lib}.rs) used as the checker for the CUDA path and as the timed CPU
 * baseline.  Nothing in the product links it or calls it.
 *
 * Parity is pinned against the reference's published golden values for
 * examples/cantilever.inp, examples/cantilever3d.inp, examples/plate_hole.inp,
 * the bench patch deck and the cantilever refinement table (see the tests
 * under tests/ that load tests/golden/).
 */
#ifndef SVX_ORACLE_H
#define SVX_ORACLE_H

#include "solvix_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct svx_oracle_csr {
    int64_t n;
    int64_t nnz;
    int64_t* row_ptr; /* [n + 1] */
    int64_t* col_idx; /* [nnz] */
    double* vals;     /* [nnz] */
    double* f;        /* [n] assembled load vector (copy of the model's) */
} svx_oracle_csr_t;

/* Order in which csr_from_triplets sums duplicate (row, col) triplets:
 * 0 (default) = the reference's `sort_unstable_by_key` restated, so K is
 * bit-identical to the reference's; 1 = stable (triplet-stream order:
 * diagonal seed, then elements in enumeration order), the order the CUDA
 * assembly uses. */
void svx_oracle_set_sort_mode(int mode);

/* Element stiffness of one element (row-major N x N into ke); returns 0 or
 * the svx_elem_reason of the failure.  coords: [n_nodes][3]. */
int svx_oracle_element_stiffness(int kind, const double* coords, double E, double nu,
                                 double thickness, double* ke);

/* assembly::assemble_with restated (assembly.rs:291-386): triplets -> CSR,
 * duplicates summed in the order of the current sort mode. */
int svx_oracle_assemble(const svx_flat_model_t* m, int threads, svx_oracle_csr_t* out,
                        svx_error_t* err);
void svx_oracle_csr_free(svx_oracle_csr_t* csr);

/* Csr::mat_vec_with (assembly.rs:46-72). */
void svx_oracle_spmv(const svx_oracle_csr_t* k, const double* x, double* y, int threads);

/* solver::apply_dirichlet (solver.rs:45-62) in place on k and f. */
void svx_oracle_apply_dirichlet(svx_oracle_csr_t* k, double* f, const int64_t* rows,
                                int64_t n_rows);

/* solver::pcg_with_threads (solver.rs:82-149).  Returns SVX_OK or
 * SVX_NOT_CONVERGED (iterations / residual filled either way). */
int svx_oracle_pcg(const svx_oracle_csr_t* k, const double* f, double tol, int64_t max_iter,
                   int threads, double* u, int64_t* iterations, double* residual);

/* Full linear-static pipeline (lib.rs:593-716) with Method::Pcg.  Output
 * arrays of `sol` are caller-allocated. */
int svx_oracle_solve(const svx_flat_model_t* m, int threads, double tol, int64_t max_iter,
                     svx_solution_t* sol, svx_error_t* err);

/* lib.rs:525-535 Method. */
enum { SVX_ORACLE_METHOD_PCG = 0, SVX_ORACLE_METHOD_LDLT = 1, SVX_ORACLE_METHOD_AUTO = 2 };

/* The same pipeline with a Method (lib.rs:664-686): Ldlt factorizes directly,
 * Auto runs the PCG and factorizes when it returns NotConverged.  On the
 * direct path iterations is 0, final_residual ||f - K u|| / ||f|| and
 * cond_estimate max|D| / min|D|.  *method_used (may be NULL) receives the
 * method that produced u (PCG or LDLT). */
int svx_oracle_solve_method(const svx_flat_model_t* m, int threads, double tol,
                            int64_t max_iter, int method, svx_solution_t* sol,
                            int* method_used, svx_error_t* err);

/* Consistent mass of one element (modal.rs:82-146: CPS3 closed form, CPS4 /
 * CPE4 2x2 and C3D8 2x2x2 Gauss of rho [t] detJ N^T N), row-major N x N into
 * me; returns 0 or the svx_elem_reason of the failure. */
int svx_oracle_element_mass(int kind, const double* coords, double rho, double t, double* me);

/* assemble_mass (modal.rs:203-271): the consistent mass matrix on the
 * stiffness's pattern (diagonal seeds, then elements in order, summed in the
 * current sort mode); density rho is model-wide, thickness the model's. */
int svx_oracle_assemble_mass(const svx_flat_model_t* m, double rho, svx_oracle_csr_t* out,
                             svx_error_t* err);

/* Reverse Cuthill-McKee permutation of k's pattern, old -> new
 * (ldl.rs:27-60). */
void svx_oracle_rcm(const svx_oracle_csr_t* k, int64_t* perm);

/* Ldlt::factorize + Ldlt::solve (ldl.rs:144-251) of a Dirichlet-modified k,
 * then the residual and estimate of lib.rs:645-663.  d (optional, [n]) gets
 * D in the permuted order, nnz_l (optional) the entries of L.  Returns SVX_OK
 * or SVX_INVALID_MODEL with the reference's pivot message. */
int svx_oracle_ldlt(const svx_oracle_csr_t* k, const double* f, int threads, double* u,
                    double* residual, double* cond, double* d, int64_t* nnz_l,
                    svx_error_t* err);

/* Stress + reaction recovery for a given u (stress.rs:22-118); K_orig for
 * the reactions is assembled with the current sort mode.  Output arrays may
 * be NULL. */
int svx_oracle_stress(const svx_flat_model_t* m, const double* u, int threads, double* vm,
                      double* vm_node, double* reactions, svx_error_t* err);

/* Steady heat conduction: the public svx_thermal_model_t (solvix_gpu.h). */
typedef svx_thermal_model_t svx_oracle_thermal_t;

/* heat::solve_thermal restated (heat.rs:52-98) for CPS3, CPS4, CPE4 and
 * C3D8 elements: conduction matrices (heat.rs:149-296), flux loads
 * (heat.rs:298-358), nonhomogeneous Dirichlet rows (heat.rs:361-407) and
 * the Jacobi-PCG to tol with max(1000, 10 * nodes) iterations.  Returns
 * SVX_OK or the error code, with err's message in the reference's text. */
int svx_oracle_solve_thermal(const svx_oracle_thermal_t* m, int threads, double tol,
                             double* temperatures, int64_t* iterations, double* residual,
                             svx_error_t* err);

/* The conduction matrix (row-major N x N, N = nodes of the kind) and the
 * consistent heat-source load of one element; returns 0 or the
 * svx_elem_reason of the failure. */
int svx_oracle_conduction_element(int kind, const double* coords, double conductivity,
                                  double thickness, int has_source, double source, double* ke,
                                  double* fe);

#ifdef __cplusplus
}
#endif

#endif
