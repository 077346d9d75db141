/*
 * solvix_gpu.h - C ABI of the B200 linear-static path of Solvix.
 *
 * This header is the drop-in boundary for solvix-core's linear-static hot
 * path: Gauss-point element stiffness integration (CPS3 / CPS4 / C3D8),
 * global CSR assembly, symmetric Dirichlet elimination, Jacobi-PCG and
 * stress / reaction recovery.  In the reference these are the pub(crate)
 * functions called from `solve_with_thermal`
 * (crates/solvix-core/src/lib.rs:593-716, the steps at :614-703).
 *
 * Conventions
 *   - Every function returns an `int` status (SVX_OK on success) and, where
 *     a model can be rejected, fills a caller-owned `svx_error_t`.
 *   - The caller owns every host array.  The library copies inputs in and
 *     writes outputs into caller-allocated arrays.  Device memory is owned
 *     by the library behind opaque handles and released by the *_free /
 *     *_destroy functions.
 *   - Calls on different contexts are thread safe (one CUDA stream per
 *     context).  A single context or operator must not be used from two
 *     threads at once.  Calls block until their host outputs are written.
 *   - Indices are 0-based; node and element ids are the model's own ids and
 *     are only used for error messages and reaction records.
 *   - There is no CPU fallback: without a usable CUDA device every compute
 *     entry point returns SVX_CUDA_ERROR.
 */
#ifndef SOLVIX_GPU_H
#define SOLVIX_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Status codes.  1-4 are the reference's SolveError variants          */
/* (crates/solvix-core/src/lib.rs:515-521); the rest are device-side.  */
/* ------------------------------------------------------------------ */
enum svx_status {
    SVX_OK = 0,
    SVX_EMPTY_MESH = 1,      /* SolveError::EmptyMesh */
    SVX_NO_CONSTRAINTS = 2,  /* SolveError::NoConstraints */
    SVX_INVALID_MODEL = 3,   /* SolveError::InvalidModel(message) */
    SVX_NOT_CONVERGED = 4,   /* SolveError::NotConverged{iterations, residual} */
    SVX_OOM = 5,             /* device memory (or admission budget) exhausted */
    SVX_CUDA_ERROR = 6,      /* no device, launch failure, driver error */
    SVX_BAD_ARGUMENT = 7,    /* null pointer, inconsistent sizes */
    SVX_QUEUE_EMPTY = 8,     /* server poll: nothing completed yet */
    SVX_IO_ERROR = 9,        /* a file could not be written (std::io::Error) */
    SVX_PARSE_ERROR = 10,    /* a deck the reference's parser rejects (ParseError) */
    SVX_UNSUPPORTED = 11     /* a deck outside the linear-static reader's keywords */
};

/* Element kinds, in the order of the reference's ElemKind enum
 * (crates/solvix-core/src/lib.rs:54-73).  The GPU path integrates
 * CPS3, CPS4 and C3D8; the other kinds are rejected as InvalidModel. */
enum svx_elem_kind {
    SVX_CPS3 = 0,
    SVX_CPS4 = 1,
    SVX_CPS8 = 2,
    SVX_CPE4 = 3,
    SVX_CPE8 = 4,
    SVX_C3D8 = 5,
    SVX_C3D4 = 6,
    SVX_B31 = 7
};

/* Why an element was rejected (svx_error_t.reason). */
enum svx_elem_reason {
    SVX_REASON_NONE = 0,
    SVX_REASON_NO_MATERIAL = 1,      /* assembly.rs:144-146 */
    SVX_REASON_BAD_MATERIAL = 2,     /* assembly.rs:147-149 */
    SVX_REASON_SOLID_POISSON = 3,    /* assembly.rs:150-160 */
    SVX_REASON_DEGENERATE_TRI = 4,   /* assembly.rs:175 */
    SVX_REASON_BAD_JACOBIAN = 5,     /* assembly.rs:195, :259-261 */
    SVX_REASON_UNSUPPORTED_KIND = 6  /* kinds outside CPS3/CPS4/C3D8 */
};

/* Error record.  `message` holds the text the reference carries in the
 * SolveError payload (e.g. "element 7: non-positive Jacobian determinant
 * at a Gauss point" for InvalidModel), NUL terminated. */
typedef struct svx_error {
    int32_t code;        /* enum svx_status */
    int32_t reason;      /* enum svx_elem_reason for element failures */
    int64_t elem_index;  /* first failing element in enumeration order, or -1 */
    int64_t iterations;  /* NotConverged: iteration reached */
    double residual;     /* NotConverged: recursive ||r||/||f|| there */
    char message[512];
} svx_error_t;

/* ------------------------------------------------------------------ */
/* Reference-shaped model (solvix_core::Model after Model::load_state,  */
/* crates/solvix-core/src/lib.rs:250-307, :388-403).  Node and element  */
/* references are by id; materials are resolved through element sets.  */
/* ------------------------------------------------------------------ */
typedef struct svx_model_desc {
    int64_t n_nodes;
    const uint32_t* node_ids;     /* [n_nodes] */
    const double* node_coords;    /* [3 * n_nodes], x y z per node */

    int64_t n_elems;
    const uint32_t* elem_ids;     /* [n_elems] */
    const uint8_t* elem_kinds;    /* [n_elems] enum svx_elem_kind */
    const int64_t* elem_conn_ptr; /* [n_elems + 1] */
    const uint32_t* elem_conn;    /* node ids, [elem_conn_ptr[n_elems]] */

    int32_t n_materials;
    const char* const* material_names;
    const double* youngs_modulus;
    const double* poisson_ratio;

    int32_t n_elsets;
    const char* const* elset_names;
    const int64_t* elset_ptr;        /* [n_elsets + 1] */
    const uint32_t* elset_elem_ids;  /* element ids */

    int32_t n_assignments;           /* (elset, material) pairs, in order */
    const char* const* assign_elset;
    const char* const* assign_material;

    double thickness;

    int32_t n_bcs;                   /* BoundaryCondition{node_ids, dofs} */
    const int64_t* bc_node_ptr;      /* [n_bcs + 1] */
    const uint32_t* bc_node_ids;
    const int64_t* bc_dof_ptr;       /* [n_bcs + 1] */
    const int64_t* bc_dofs;          /* 1-based dofs */

    int64_t n_cloads;                /* ConcentratedLoad{node_id, dof, value} */
    const uint32_t* cload_node_ids;
    const int64_t* cload_dofs;       /* 1-based */
    const double* cload_values;

    /* Model::density (kg/m^3) for gravity loads; the reference's Model
     * default is 7850, so a caller building a model by hand sets it. */
    double density;
    int64_t n_dloads;                /* DistributedLoad{element_id, face, magnitude} */
    const uint32_t* dload_elem_ids;
    const int64_t* dload_faces;      /* 1-based plane edge (P1..P4) */
    const double* dload_values;      /* pressure, positive into the element */
    int32_t has_gravity;             /* the load state's gravity is Some((g, dir)) */
    double gravity_magnitude;        /* g */
    double gravity_dir[3];           /* dir (not normalised; plane models use x, y) */
} svx_model_desc_t;

/* ------------------------------------------------------------------ */
/* Flat, index-resolved model: what the device path consumes.          */
/* ------------------------------------------------------------------ */
typedef struct svx_flat_model {
    int64_t n_nodes;
    const double* xyz;            /* [3 * n_nodes] */
    const uint32_t* node_id;      /* [n_nodes] ids (NULL: index + 1) */

    int64_t n_elem;
    const uint8_t* kind;          /* [n_elem] enum svx_elem_kind */
    const int64_t* conn_ptr;      /* [n_elem + 1] */
    const int32_t* conn;          /* 0-based node indices */
    const double* youngs;         /* [n_elem] E per element */
    const double* poisson;        /* [n_elem] nu per element */
    const uint8_t* no_material;   /* [n_elem] 1 = no material (NULL: all 0) */
    const uint32_t* elem_id;      /* [n_elem] ids (NULL: index + 1) */

    double thickness;             /* model-wide, plane elements only */
    int32_t ndof;                 /* 2 (plane) or 3 (solid) */

    int64_t n_fixed;              /* constrained dof rows in BC order */
    const int64_t* fixed_row;     /* node_index * ndof + dof - 1 */
    const double* f;              /* [n_nodes * ndof] load vector */
} svx_flat_model_t;

/* Resolved model produced from a svx_model_desc_t (owned by the library). */
typedef struct svx_resolved svx_resolved_t;

/* Precision forms of the PCG solve. */
enum svx_precision {
    SVX_FP64 = 0,      /* FP64 K, FP64 PCG: the plain form */
    SVX_MIXED = 1,     /* one FP64 Jacobi-PCG (FP64 vectors, u and dots) whose operator
                          is relaxed as it converges: FP64 K until ||r||/||f|| <=
                          clamp(tol * 1e7, tol, 0.1), then the FP32-stored K on the same
                          search directions for at most as many iterations again, then
                          FP64 K; convergence is decided on the true FP64 residual, and
                          CG restarts on FP64 K if that is short of tol */
    SVX_MIXED_DEFECT = 2 /* single solves only: FP64 defect correction (u, r = f - K64 u
                          and the correction's update in FP64) around an inner Jacobi-PCG
                          whose K, vectors and preconditioner are FP32 and whose dots
                          accumulate in FP64, each inner solve to inner_tol; after two
                          corrections that cut ||r|| by less than 2x the inner solver is
                          the FP64 PCG */
};

/* Linear solver selection (Method, lib.rs:523-534; dispatch lib.rs:664-686). */
enum svx_method {
    SVX_METHOD_PCG = 0,   /* Jacobi-PCG; a budget overrun returns SVX_NOT_CONVERGED */
    SVX_METHOD_LDLT = 1,  /* the direct path: RCM-ordered band LDL^T factorized on the
                             device (replaces Ldlt::factorize / solve, ldl.rs:144-251) */
    SVX_METHOD_AUTO = 2   /* Jacobi-PCG, then the direct path when it returns
                             SVX_NOT_CONVERGED (Method::Auto, the reference's default) */
};

typedef struct svx_solve_opts {
    double tol;            /* relative residual tolerance (reference: 1e-10) */
    int64_t max_iter;      /* <= 0: max(1000, 10 * ndof_total) like lib.rs:632 */
    int32_t precision;     /* enum svx_precision */
    double inner_tol;      /* SVX_MIXED_DEFECT: relative residual of each inner FP32
                              solve; values outside (0, 1) select 1e-5.  Unused by the
                              other forms */
    int32_t check_every;   /* iterations per graph launch between host checks (0: auto) */
    int32_t want_stress;   /* 1: compute von Mises + reactions */
    int32_t method;        /* enum svx_method (svx_default_opts: SVX_METHOD_PCG) */
} svx_solve_opts_t;

/* Results of one static solve; arrays are caller-allocated (NULL skips). */
typedef struct svx_solution {
    double* u;                 /* [n_nodes * ndof] */
    double* displacements;     /* [3 * n_nodes] like Solution::displacements */
    double* von_mises;         /* [n_elem] centroid von Mises */
    double* nodal_von_mises;   /* [n_nodes] */
    double* reactions;         /* [n_fixed] K_orig u - f at constrained rows */
    int64_t iterations;        /* PCG iterations (outer+inner total for mixed) */
    int64_t outer_iterations;  /* mixed: defect-correction steps */
    double final_residual;     /* recursive ||r||/||f|| (mixed: true FP64 residual) */
    double cond_estimate;      /* max|diag| / min|diag| of the Dirichlet-modified K */
    double ms_assemble;        /* device time of element integration + assembly */
    double ms_solve;           /* device time of the PCG */
    double ms_stress;          /* device time of stress + reaction recovery */
    int64_t fp32_iterations;   /* mixed: iterations on the FP32 operator */
    int32_t solver_method;     /* SVX_METHOD_PCG or SVX_METHOD_LDLT: what produced u.  After
                                  the direct path iterations is 0, final_residual
                                  ||f - K u|| / ||f|| and cond_estimate max|D| / min|D|
                                  (lib.rs:645-663, ldl.rs:256-265) */
    int64_t factor_bandwidth;  /* direct path: half-bandwidth of K in the RCM order */
    double ms_factor;          /* direct path: device time of the factorization + solve */
} svx_solution_t;

typedef struct svx_ctx svx_ctx_t;
typedef struct svx_op svx_op_t;

/* Library version string. */
const char* svx_version(void);

/* Default options: tol 1e-10, max_iter auto, FP64, inner_tol 1e-5, method PCG. */
void svx_default_opts(svx_solve_opts_t* opts);

/* ---- context ----------------------------------------------------- */
int svx_ctx_create(int device, svx_ctx_t** out);
/* Free every operator of a context (svx_op_free) before destroying it. */
int svx_ctx_destroy(svx_ctx_t* ctx);
/* The context's CUDA stream (cudaStream_t), for callers that order their own
 * work or timing events with the library's. */
void* svx_ctx_stream(svx_ctx_t* ctx);
/* Copies the last error message of `ctx` (or of the calling thread when
 * ctx is NULL) into buf. */
int svx_last_error(const svx_ctx_t* ctx, char* buf, size_t len);

/* ---- a1: id / material / load resolution (host, O(N)) -------------- */
/* Replaces Mesh::node_index (lib.rs:106-108), Model::material_for_element
 * (lib.rs:357-367), validate (lib.rs:406-436), ndof_per_node
 * (lib.rs:725-752), the load vector of assemble_with: CLOADs
 * (assembly.rs:365-380), edge pressure (edge_pressure_forces,
 * assembly.rs:382, :393-452) and gravity (gravity_forces, assembly.rs:383,
 * :458-539), and constrained_dofs (solver.rs:15-41).  Errors the reference
 * raises before assembly are returned here; errors it raises after the
 * element loop (CLOAD, DLOAD, gravity, BC, in that order) are kept pending
 * inside the resolved model and reported by svx_solve_resolved only when no
 * element fails first. */
int svx_resolve(const svx_model_desc_t* desc, svx_resolved_t** out, svx_error_t* err);
/* Borrowed view of the resolved flat model (valid until svx_resolved_free). */
const svx_flat_model_t* svx_resolved_flat(const svx_resolved_t* res);
/* The CLOAD / BC error the reference raises after the element loop, if
 * any (SVX_OK when none): callers that solve the flat view themselves
 * (svx_serve_submit) report it when no element fails first. */
int svx_resolved_pending(const svx_resolved_t* res, svx_error_t* err);
int svx_resolved_free(svx_resolved_t* res);

/* ---- K1-K4: assembly on the device ------------------------------- */
/* Element integration + CSR pattern + fixed-order assembly + Dirichlet.
 * Replaces assembly::assemble (assembly.rs:281-386), constrained_dofs /
 * apply_dirichlet (solver.rs:15-62) and the K/f clones (lib.rs:623-628). */
enum svx_assemble_flags {
    SVX_KEEP_ORIGINAL = 1  /* keep a device copy of K before Dirichlet */
};
int svx_assemble(svx_ctx_t* ctx, const svx_flat_model_t* model, uint32_t flags,
                 svx_op_t** out, svx_error_t* err);
int svx_op_free(svx_op_t* op);
/* Re-runs element integration, assembly and Dirichlet from the operator's
 * device-resident model (the pattern is kept): the whole K1-K4 path with
 * no host traffic. */
int svx_op_reassemble(svx_op_t* op, svx_error_t* err);
/* CSR sizes of an assembled operator. */
int svx_op_dims(const svx_op_t* op, int64_t* n_rows, int64_t* nnz);
/* Copies the CSR to host arrays of n+1 / nnz / nnz entries (any may be
 * NULL).  which = 0: the PCG operator (K after Dirichlet); which = 1: the
 * assembled K before Dirichlet (needs SVX_KEEP_ORIGINAL). */
int svx_op_get_csr(const svx_op_t* op, int which, int64_t* row_ptr, int32_t* col_idx,
                   double* vals);
/* Copies the load vector (which = 0: after Dirichlet, 1: before) and the
 * Jacobi inverse diagonal (NULL skips) to host arrays of n_rows. */
int svx_op_get_vectors(const svx_op_t* op, int which, double* f, double* inv_diag);
/* y = K x with the PCG operator (x, y host arrays of n_rows). */
int svx_op_spmv(svx_op_t* op, const double* x, double* y);
/* Installs u (host, n_rows) as the operator's solution, e.g. to recover
 * stresses for a displacement field computed elsewhere. */
int svx_op_set_solution(svx_op_t* op, const double* u);

/* ---- consistent mass --------------------------------------------- */
/* The consistent mass matrix of a flat model of density `density` (kg/m^3;
 * plane elements take the model's thickness) assembled on the device: the
 * element mass matrices of CPS3 (closed form rho t A / 12 x [2 1 1; 1 2 1;
 * 1 1 2]), CPS4 / CPE4 (rho t det J N_i N_j under 2x2 Gauss) and C3D8
 * (rho det J N_i N_j under 2x2x2 Gauss) on every dof pair (d, d), summed by
 * the stiffness's fixed-order node-block assembly into the same CSR pattern
 * (zero entries and every diagonal included), with no Dirichlet rows.
 * Replaces assemble_mass (crates/solvix-core/src/modal.rs:203-271) with
 * cps3_mass / cps4_mass / c3d8_mass (modal.rs:82-146); the values are
 * bit-identical to summing the reference's triplets in element order.  The
 * operator answers svx_op_dims, svx_op_get_csr (which = 0), svx_op_spmv
 * (y = M x) and svx_op_reassemble; svx_op_solve, svx_op_stress and
 * svx_op_get_vectors return SVX_BAD_ARGUMENT for it.  Errors: the first
 * failing element in enumeration order with the reference's text
 * ("element 7: degenerate (zero-area) triangle", "... non-positive Jacobian
 * determinant at a Gauss point"); kinds outside the four are rejected as
 * InvalidModel like the stiffness; a negative or non-finite density is
 * SVX_BAD_ARGUMENT.  Material, load and constraint arrays are not read. */
int svx_assemble_mass(svx_ctx_t* ctx, const svx_flat_model_t* model, double density,
                      svx_op_t** out, svx_error_t* err);

/* ---- K5-K7: PCG --------------------------------------------------- */
/* Replaces solver::pcg (solver.rs:66-149) and jacobi_cond (lib.rs:634-644);
 * with opts->want_stress also K9-K10 (device-side, copied to the non-NULL
 * arrays of sol).  opts->method selects the Method dispatch of
 * lib.rs:664-686: SVX_METHOD_LDLT and the fallback of SVX_METHOD_AUTO run
 * the direct path on the device (Ldlt::factorize / solve, ldl.rs:144-265),
 * whose failed pivot returns SVX_INVALID_MODEL with the reference's text
 * ("stiffness matrix is not positive definite (pivot near-zero at equation
 * 12)") and whose band (half-bandwidth x rows doubles) must fit in the
 * device's free memory, else SVX_OOM. */
int svx_op_solve(svx_op_t* op, const svx_solve_opts_t* opts, svx_solution_t* sol,
                 svx_error_t* err);

/* The equation ordering of the direct path: the reverse Cuthill-McKee
 * permutation (old row -> new row) of a symmetric CSR pattern, as the
 * reference's rcm (ldl.rs:27-60) computes it, and the half-bandwidth
 * max |perm[r] - perm[c]| over the pattern's entries.  Host only. */
int svx_order_rcm(int64_t n, const int64_t* row_ptr, const int32_t* col_idx, int32_t* perm,
                  int64_t* bandwidth);

/* ---- K9-K10: stress + reactions ----------------------------------- */
/* svx_op_solve with opts->want_stress = 1 also recovers the stresses into
 * device buffers (copied out only where sol's arrays are non-NULL).
 * svx_op_stress uses the operator's last solution (svx_op_solve).  Replaces
 * stress::{von_mises_at_centroids, nodal_von_mises, reactions}
 * (stress.rs:22-118) and the displacement packaging of lib.rs:689-698. */
int svx_op_stress(svx_op_t* op, svx_solution_t* sol);

/* ---- steady heat conduction (one temperature dof per node) ----------- */
/* The model heat::solve_thermal reads (crates/solvix-core/src/heat.rs:52-98)
 * from a Model and its last Step, flattened like svx_flat_model_t (0-based
 * node indices).  Temperature constraints apply in array order, a later one
 * for the same node winning (heat.rs:367-375); heat fluxes act on the plane
 * edge `face` (1-based) of element flux_elem[i], positive into the element
 * (heat.rs:298-358). */
typedef struct svx_thermal_model {
    int64_t n_nodes;
    const double* xyz;          /* [3 * n_nodes] */
    int64_t n_elem;
    const uint8_t* kind;        /* [n_elem] enum svx_elem_kind */
    const int64_t* conn_ptr;    /* [n_elem + 1] */
    const int32_t* conn;        /* 0-based node indices */
    const uint32_t* elem_id;    /* [n_elem] ids for messages; NULL = e + 1 */
    double thickness;           /* model-wide (2D elements) */
    double conductivity;        /* model-wide */
    int32_t has_source;         /* the step's volumetric heat source is set */
    double source;
    int64_t n_temp;
    const int64_t* temp_node;   /* [n_temp] node indices */
    const double* temp_value;   /* [n_temp] */
    int64_t n_flux;
    const int64_t* flux_elem;   /* [n_flux] element indices */
    const int32_t* flux_face;   /* [n_flux] 1-based edge */
    const double* flux_value;   /* [n_flux] */
} svx_thermal_model_t;

/* Replaces heat::solve_thermal (heat.rs:52-98): conduction matrices of
 * CPS3, CPS4 / CPE4 and C3D8 elements (heat.rs:149-296) assembled on the
 * device in the mechanical path's fixed order, source and flux loads,
 * nonhomogeneous temperature rows (heat.rs:361-407) and the FP64 Jacobi-PCG
 * (opts: tol, max_iter <= 0 for max(1000, 10 * nodes), check_every; the
 * precision must be SVX_FP64).  temperatures: [n_nodes].  Errors and their
 * texts follow the reference (EmptyMesh, NoConstraints, InvalidModel,
 * NotConverged). */
int svx_solve_thermal_flat(svx_ctx_t* ctx, const svx_thermal_model_t* model,
                           const svx_solve_opts_t* opts, double* temperatures,
                           int64_t* iterations, double* residual, svx_error_t* err);

/* ---- .inp reader (linear-static decks) ------------------------------ */
/* The reference's parse_inp (crates/solvix-io/src/parser.rs:87-1370) for the
 * keywords of linear-static decks (*HEADING, *NODE, *ELEMENT, *NSET, *ELSET
 * [GENERATE], *MATERIAL, *ELASTIC, *DENSITY, *SOLID SECTION, *STEP,
 * *STATIC, *BOUNDARY, *CLOAD, *DLOAD [P1..P4, GRAV], *END STEP; unknown
 * keywords are warned and skipped like the reference does), producing the
 * model svx_resolve consumes with the BCs and loads of Model::load_state
 * (lib.rs:388-403).  Returns SVX_OK,
 * SVX_PARSE_ERROR (err->elem_index = the 1-based line, err->message the
 * reference's ParseError message) or SVX_UNSUPPORTED (a keyword the
 * reference reads with another meaning, or *STEP, NLGEOM=YES: parse that
 * deck with the reference's parser). */
typedef struct svx_inp svx_inp_t;
int svx_inp_parse(const char* text, int64_t len, svx_inp_t** out, svx_error_t* err);
/* The parsed model (valid until svx_inp_free). */
const svx_model_desc_t* svx_inp_model(const svx_inp_t* inp);
/* *STEP blocks read (the model's steps.len()). */
int32_t svx_inp_step_count(const svx_inp_t* inp);
/* ParseReport::warnings, in order. */
int32_t svx_inp_warning_count(const svx_inp_t* inp);
const char* svx_inp_warning(const svx_inp_t* inp, int32_t i);
void svx_inp_free(svx_inp_t* inp);

/* ---- VTU output ---------------------------------------------------- */
/* What the reference's writers read from a Model and a Solution
 * (crates/solvix-io/src/vtu.rs), with node ids already resolved to 0-based
 * indices.  Arrays shorter than the mesh print 0 beyond their length, as
 * the reference's `.get(i).unwrap_or(0)` does. */
typedef struct svx_vtu_data {
    int64_t n_nodes;
    const double* xyz;                  /* [3 * n_nodes] */
    int64_t n_elem;
    const uint8_t* kind;                /* [n_elem] enum svx_elem_kind */
    const int64_t* conn_ptr;            /* [n_elem + 1] */
    const int32_t* conn;                /* 0-based node indices */
    int64_t n_disp;                     /* displacement triplets available */
    const double* displacements;        /* [3 * n_disp] (Solution::displacements) */
    int64_t n_von_mises;                /* centroid values available */
    const double* von_mises;            /* [n_von_mises] */
    int32_t n_extra;                    /* extra scalar PointData arrays (ASCII only) */
    const char* const* extra_names;     /* [n_extra] */
    const double* const* extra_values;  /* [n_extra] */
    const int64_t* extra_len;           /* [n_extra] values available per array */
} svx_vtu_data_t;

/* Writes `path` byte for byte as the reference's ASCII writer
 * (vtu.rs:14-115, write_vtu / write_vtu_ex) when binary == 0, or as its
 * appended raw binary writer (vtu.rs:148-288, write_vtu_binary) when
 * binary == 1.  The ASCII lines are formatted on `threads` host threads
 * (<= 0: all cores); the bytes do not depend on the thread count.  Returns
 * SVX_OK, SVX_BAD_ARGUMENT, SVX_OOM or SVX_IO_ERROR (with the reference's
 * text when an appended block exceeds the Int32 byte-count header). */
int svx_write_vtu(const char* path, const svx_vtu_data_t* data, int32_t binary, int32_t threads,
                  svx_error_t* err);

/* ---- batched solves (many independent models in one launch) -------- */
typedef struct svx_batch_result {
    int64_t iterations;    /* PCG iterations of this model */
    double residual;       /* recursive ||r||/||f|| at exit */
    int32_t status;        /* SVX_OK, SVX_NOT_CONVERGED, or why the model was
                              rejected (SVX_EMPTY_MESH, SVX_NO_CONSTRAINTS,
                              SVX_INVALID_MODEL, SVX_BAD_ARGUMENT) */
    int32_t reason;        /* enum svx_elem_reason for SVX_INVALID_MODEL */
    double cond_estimate;  /* max|diag| / min|diag| of this model's modified K */
    int64_t nnz;           /* nonzeros of this model's K */
    int64_t elem_index;    /* failing element (index within the model) or -1 */
} svx_batch_result_t;

typedef struct svx_batch_stats {
    double ms_assemble;    /* device time: all models' K1-K4 */
    double ms_solve;       /* device time of the batched PCG launch */
    double ms_stress;      /* device time of the centroid von Mises */
    int32_t threads_per_cta;  /* autotuned CTA size of the batched PCG */
    int32_t lanes_per_node;   /* autotuned lanes per node of its SpMV */
    int64_t total_iterations; /* sum over models */
    int64_t total_dof;        /* sum over models */
    int32_t not_converged;    /* models that missed tol within their budget
                                 or were rejected */
    int32_t cluster_members;  /* models solved by a CTA cluster (3D >= 4096
                                 rows, 2D >= 16384 rows) */
    int64_t fp32_iterations;  /* mixed form: iterations on the FP32 operator */
} svx_batch_stats_t;

/* Solves `count` independent models of equal ndof.  They are
 * assembled as one block-diagonal operator; one launch per size class then
 * runs every model's Jacobi-PCG with its own scalars, convergence test and
 * iteration budget (max(1000, 10 n_model) unless opts->max_iter > 0): one
 * CTA per model for the small ones and one thread-block cluster per model
 * for the large ones, largest models first.  The CTA size and lanes
 * per node are autotuned once per context and ndof, and kept.  Per model
 * outputs: u[k] (n_nodes*ndof) and von_mises[k] (n_elem), host arrays, any
 * may be NULL.  Each model is checked on its own: one that is rejected
 * (empty mesh, no constraints, a bad element found on the host or by the
 * element kernel) gets that status in its result and the others are solved
 * as if it were absent.  Models of different ndof in one call are
 * SVX_BAD_ARGUMENT for the call.  opts->precision selects the FP64 or the
 * mixed form (FP32-stored K with FP64 residual replacement) per model. */
int svx_batch_solve(svx_ctx_t* ctx, int32_t count, const svx_flat_model_t* models,
                    const svx_solve_opts_t* opts, double* const* u, double* const* von_mises,
                    svx_batch_result_t* results, svx_batch_stats_t* stats, svx_error_t* err);

/* ---- served solves (continuous batching) ---------------------------- */
/* A request loop for `solvix serve --json`: decks are submitted as they
 * arrive and solved in batches on the device while later ones keep
 * arriving.  `lanes` dispatcher threads each own a CUDA stream; whenever a
 * lane is free it takes every waiting request (arrival order, equal ndof,
 * at most max_batch) whose device memory fits what is left of the budget,
 * solves them as one batch (svx_batch_solve's per-model isolation and
 * per-model convergence) and publishes each result as its batch completes.
 * Batches of different lanes run concurrently on the device.  A request is
 * admitted only while the estimated device bytes of all admitted, unfinished
 * requests stay within hbm_budget_bytes.  Each lane has its own device
 * memory pool (blocks are reused only on the stream that freed them) whose
 * arena, budget / lanes, is reserved at creation, so batches of any size
 * make no cudaMalloc / cudaFree calls in steady state; a lane's batch stays
 * within its arena (blocks that fragmentation leaves no room for fall back
 * to cudaMalloc). */
typedef struct svx_server svx_server_t;

typedef struct svx_serve_opts {
    int64_t hbm_budget_bytes;  /* admission budget; 0 = 40 GiB */
    int32_t lanes;             /* concurrent batches (streams); 0 = 2 */
    int32_t max_batch;         /* requests per batch at most; 0 = 4096 */
    svx_solve_opts_t solve;    /* tolerance, precision, max_iter, want_stress */
    int64_t max_batch_bytes;   /* estimated device bytes per batch at most;
                                  0 = 4/5 of a lane's arena (budget / lanes) */
} svx_serve_opts_t;

typedef struct svx_serve_result {
    uint64_t tag;              /* the caller's tag from svx_serve_submit */
    int32_t status;            /* as svx_batch_result_t.status */
    int32_t ndof;
    int64_t n_nodes;
    int64_t n_elem;
    int64_t iterations;
    double residual;
    double cond_estimate;
    double t_submit_ms;        /* server clock (ms since svx_serve_create) */
    double t_start_ms;         /* its batch was taken by a lane */
    double t_done_ms;          /* its batch's results were on the host */
    int32_t batch_size;        /* requests in its batch */
    int32_t lane;
    const double* u;           /* [n_nodes * ndof], owned by the result */
    const double* von_mises;   /* [n_elem] centroid von Mises (NULL if off) */
    svx_error_t error;         /* why a request failed (status != SVX_OK) */
    int64_t nnz;               /* stored nonzeros of its K (0 if it failed before assembly) */
} svx_serve_result_t;

typedef struct svx_serve_stats {
    int64_t submitted;
    int64_t rejected;          /* refused by svx_serve_submit */
    int64_t completed;         /* results published (any status) */
    int64_t batches;
    int64_t pending;           /* waiting for admission */
    int64_t in_flight;         /* admitted, not yet published */
    int64_t bytes_admitted;    /* estimated device bytes of in-flight work */
    int64_t peak_bytes_admitted;
    int64_t device_bytes;      /* device memory the lanes' pools hold: their
                                  arenas (budget / lanes each) or, if more,
                                  the blocks in use + cached */
    int64_t peak_device_bytes;
    /* summed over batches, ms of host wall clock per phase: member checks
     * and concatenation, upload + assembly, batched PCG, result copies;
     * and the device time of the batched PCG launches */
    double prep_ms, assemble_ms, solve_ms, output_ms, device_solve_ms;
    double pool_ms;            /* wall clock inside cudaMalloc / cudaFree */
    int64_t pool_mallocs;      /* cudaMalloc calls of the shared pool */
} svx_serve_stats_t;

void svx_serve_default_opts(svx_serve_opts_t* opts);
int svx_serve_create(int device, const svx_serve_opts_t* opts, svx_server_t** out,
                     svx_error_t* err);
/* Queues a copy of `model`.  Refused at once (not queued, no result) with
 * SVX_OOM when its estimated device bytes exceed the whole budget, and with
 * the reference's error for a deck the host can reject (bad sizes, empty
 * mesh, no constraints, a bad material); elements with a non-positive
 * Jacobian are found on the device and come back as a failed result. */
int svx_serve_submit(svx_server_t* srv, const svx_flat_model_t* model, uint64_t tag,
                     svx_error_t* err);
/* Estimated device bytes the server charges against the budget for a model. */
int64_t svx_serve_estimate_bytes(const svx_flat_model_t* model);
/* Next completed result (completion order), waiting up to wait_ms
 * (< 0: until one exists).  SVX_QUEUE_EMPTY when none arrived in time. */
int svx_serve_poll(svx_server_t* srv, int32_t wait_ms, svx_serve_result_t** out);
void svx_serve_result_free(svx_serve_result_t* res);
int svx_serve_stats(svx_server_t* srv, svx_serve_stats_t* stats);
/* Milliseconds on the server clock. */
double svx_serve_now_ms(const svx_server_t* srv);
/* Finishes every submitted request, then stops the lanes and frees the
 * server (results not yet polled are freed too). */
int svx_serve_destroy(svx_server_t* srv);

/* ---- measurement --------------------------------------------------- */
/* Kernels this process has launched through the library (graph nodes count
 * when their graph is launched). */
int64_t svx_launch_count(void);
/* Average device time in ms of the PCG iteration kernels of an operator,
 * each over `reps` back-to-back launches on the context stream: ms4[0] =
 * FP64 node-block SpMV + p.Kp, ms4[1] = u/r update + dots, ms4[2] = p
 * update, ms4[3] = the difference-form FP32 SpMV of the mixed form. */
int svx_op_time_kernels(svx_op_t* op, int reps, double* ms4);

/* ---- diagnostics ---------------------------------------------------- */
/* No counterpart in the reference.  Runs the persistent PCG kernels' grid
 * barrier with one block where it expects two, so that nothing ever
 * releases it, and a spin limit of `spins` polls (1..2^24).  Every wait in
 * the library's kernels is bounded this way; on a healthy device the wait
 * runs out, the kernel raises the barrier's error flag and returns, and the
 * context stays usable.  Fills *returned_ok (0 = the barrier reported the
 * time-out to its caller) and *error_flag (1 = the flag was raised). */
int svx_diag_barrier_timeout(int device, long long spins, int* returned_ok, int* error_flag);

/* ---- PCG without device allocation ---------------------------------- */
/* Largest system (rows) svx_pcg_solve_noalloc accepts. */
#define SVX_NOALLOC_MAX_DOF 262144

/* Jacobi-preconditioned CG on a CSR system that already lives on the
 * device, for callers that cannot let a library allocate device memory:
 * an application that manages all device memory through its own arena, or
 * a latency-bounded loop that cannot absorb the implicit synchronisation of
 * cudaMalloc / cudaFree.  This entry point has no counterpart in the
 * reference.  It runs the FP64 Jacobi-PCG recurrence and stopping rule of
 * svx_op_solve (||r|| / ||f|| <= tol checked after each r update, the same
 * iteration count semantics) on a row-CSR SpMV with its own launch
 * geometry, not on svx_op_solve's node-block kernels, so its reduction
 * order, and with it the last bits of u and the iteration count, can differ
 * from svx_op_solve's on the same system.
 *
 * Every pointer but `iterations` / `residual` (host) is a device pointer of
 * the current device: row_ptr [n + 1] and col_idx [nnz] (int32, sorted
 * columns, the diagonal present), vals [nnz], f [n], u [n] (output).  tol is
 * the relative residual tolerance (>= 0); max_iter <= 0 means
 * max(1000, 10 n).  stream is a cudaStream_t (NULL = the legacy default
 * stream); the call returns after the solve has finished on it.
 *
 * Nothing is allocated: the work vectors (4 x SVX_NOALLOC_MAX_DOF doubles,
 * about 8 MB) live in one static device array that every GPU loading this
 * library holds until the process exits.  All calls on a device share that
 * array and it keeps the previous call's contents (each call clears what
 * must start at zero), so calls whose work overlaps on the GPU (other
 * threads, other streams) race; serialise them.  The first call on each
 * device looks up the array's device address and keeps it.  A
 * cudaDeviceReset of that device afterwards leaves the kept address stale,
 * so do not call this entry point on a device again after resetting it in
 * the same process.
 *
 * Returns SVX_OK; SVX_NOT_CONVERGED when max_iter is reached or the
 * recurrence breaks down (p.Kp <= 0 or NaN), with iterations / residual
 * filled and u holding the last iterate; SVX_BAD_ARGUMENT (null pointer,
 * n <= 0, n > SVX_NOALLOC_MAX_DOF, tol negative or NaN) before any work; or
 * SVX_CUDA_ERROR. */
int svx_pcg_solve_noalloc(int64_t n, const int32_t* row_ptr, const int32_t* col_idx,
                          const double* vals, const double* f, double tol, int64_t max_iter,
                          double* u, int64_t* iterations, double* residual, void* stream);

/* ---- one-call pipelines -------------------------------------------- */
/* Whole linear-static path for a flat model: lib.rs:614-703. */
int svx_solve_flat(svx_ctx_t* ctx, const svx_flat_model_t* model,
                   const svx_solve_opts_t* opts, svx_solution_t* sol, svx_error_t* err);
/* Same, for a resolved reference-shaped model (reports pending CLOAD / BC
 * errors in the reference's order). */
int svx_solve_resolved(svx_ctx_t* ctx, const svx_resolved_t* res,
                       const svx_solve_opts_t* opts, svx_solution_t* sol, svx_error_t* err);

#ifdef __cplusplus
}
#endif

#endif /* SOLVIX_GPU_H */
