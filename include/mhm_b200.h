/*
 * mhm_b200.h - C ABI of the B200 Primal-MHM hot path (libmhm_b200.so).
 *
 * Plain pointers and sizes only.  Every pointer argument is a device pointer
 * unless its comment says "host"; every call is asynchronous on `stream`
 * (a cudaStream_t passed as void*, NULL = legacy default stream) and returns
 * an MHM_* status for argument/launch errors.  Per-cell numerical outcomes
 * are reported in caller-owned status arrays after the stream completes.
 * The library never allocates device memory: scratch space is passed in by
 * the caller and sized with the matching *_workspace_bytes query.
 *
 * Reference interfaces (PyMHM 1.3.2, paths relative to src/pymhm/):
 *   mhm_q1_condense        replaces _assemble_quad (_legacy/models/darcy/
 *                          cartesian.py:69-83) + condense_local
 *                          (core/condensation.py:21-122) + local_global_
 *                          contribution (core/contributions.py:14-74) for all
 *                          macrocells of a Cartesian Q1 problem at once.
 *                          With kappa_mode 3/4 its assembly follows the
 *                          cut-cell branch of quadrilateral_operators
 *                          (fem/scalar/quadrilateral.py:136-188, 215-234).
 *   mhm_skeleton_scatter   replaces assemble_hybrid_contributions
 *                          (core/contributions.py:77-195) and the Numba
 *                          leaves core/_assembly.py:10-42.
 *   mhm_skeleton_solve     replaces solve_hybrid_system's global solve
 *                          (core/system.py:355-528 -> linalg/linear.py:798)
 *                          for systems without gauges; with
 *   mhm_skeleton_fixed_rhs its elimination of fixed (Neumann) trace DOFs
 *                          (core/system.py:421-447).
 *   mhm_q1_reconstruct     replaces reconstruct_response (core/reconstruction.py:
 *                          130-141) and the flux samples of
 *                          QuadrilateralDarcySolution.evaluate
 *                          (postprocessing/solutions.py:278-324).
 *   mhm_batched_factor /   replace BatchedFactorization.__init__/solve
 *   mhm_batched_solve      (execution/cuda.py:165-288): equilibrated dense LU
 *                          with FP64 residual refinement.
 *   mhm_p1_batch_assemble  replaces assemble_p1_batch (execution/cuda.py:27-105):
 *                          dense P1 stiffness, mass and load of a batch of
 *                          triangle or tetrahedron meshes.
 *   mhm_q1_condense_offline / mhm_q1_source_response
 *                          replace OfflineLocalProblem's factor-once and
 *                          one-column response (core/offline.py:99-145) for
 *                          OfflineHybridSystem.solve (core/offline.py:234-307).
 *   mhm_q1_original_defect(_dd) / mhm_refine_norms / mhm_q1_correction_response /
 *   mhm_q1_flux / mhm_vector_accumulate(_dd)
 *                          replace the residual evaluation and the defect-source
 *                          correction of refine_hybrid (core/refinement.py:612-800)
 *                          for the Cartesian Q1 path.
 */
#ifndef MHM_B200_H
#define MHM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Call status (return value of every entry point). */
#define MHM_OK 0
#define MHM_ERR_ARGUMENT 1     /* invalid sizes, modes or null pointers        */
#define MHM_ERR_LAUNCH 2       /* a CUDA launch or attribute call failed        */
#define MHM_ERR_UNSUPPORTED 3  /* problem too large for the on-chip layout      */

/* Per-cell / per-matrix numerical status (written to status arrays). */
#define MHM_CELL_OK 0
#define MHM_CELL_KERNEL 1          /* declared constant kernel is not a nullspace  */
#define MHM_CELL_SINGULAR_PIVOT 2  /* zero or negative pivot                       */
#define MHM_CELL_RANK_DEFICIENT 3  /* pivot below eps * n * max pivot              */
#define MHM_CELL_RESIDUAL 4        /* refinement did not reach the tolerance       */
#define MHM_CELL_NONFINITE 5       /* non-finite input or result                   */
#define MHM_CELL_ZERO_ROW 6        /* equilibration met a zero row                  */
#define MHM_CELL_ZERO_COLUMN 7     /* equilibration met a zero column               */
#define MHM_CELL_SIZE 8            /* a ragged batch's matrix exceeds the launch maximum */
#define MHM_CELL_TIMEOUT 9         /* an on-chip copy did not complete within its wait limit */

/* Global solve status (mhm_skeleton_solve `info` array, entry 0). */
#define MHM_SOLVE_OK 0
#define MHM_SOLVE_NOT_CONVERGED 1
#define MHM_SOLVE_BREAKDOWN 2      /* non-positive curvature in projected CG        */
#define MHM_SOLVE_BARRIER_TIMEOUT 3 /* a grid barrier exceeded its spin limit        */
#define MHM_SOLVE_NONFINITE 4

/* Arithmetic of the local factorisations. */
#define MHM_PRECISION_FP64 0   /* factor + sweeps in binary64                    */
#define MHM_PRECISION_MIXED 1  /* factor + sweeps in binary32, FP64 refinement   */

/* ------------------------------------------------------------------------ */
/* Cartesian Q1 macrocells: assembly + constrained condensation + Schur block */
/* ------------------------------------------------------------------------ */
typedef struct mhm_q1_problem {
    int32_t macro_nx, macro_ny;   /* macro grid; cell = iy * macro_nx + ix       */
    int32_t rx, ry;               /* fine subdivisions per macrocell              */
    double hx, hy;                /* fine cell widths                             */
    double x0, y0;                /* lower-left corner of the domain              */
    int32_t tf_h, tf_v;           /* trace DOFs on horizontal / vertical faces    */
    /* coupling_table[kind][orient][k][j]: kind 0 = horizontal side (rx+1 nodes),
     * kind 1 = vertical side (ry+1 nodes); orient 0 = face parameter increases
     * with the coordinate, 1 = decreases; k = node along the side in increasing
     * coordinate order; j < tf (kind).  Physical face length is included, the
     * cell's orientation sign is not.  Shape [2][2][kmax][jmax],
     * kmax = max(rx,ry)+1, jmax = max(tf_h,tf_v).                              */
    const double* coupling_table;
    const int8_t* side_sign;      /* (cells, 4): +-1, sides bottom,right,top,left */
    const int8_t* side_orient;    /* (cells, 4): 0/1 as in coupling_table          */
    int32_t kappa_mode;           /* 0 constant, 1 isotropic per fine cell,
                                     2 (kxx,kxy,kyy) per fine cell,
                                     3 isotropic per pixel, 4 (kxx,kxy,kyy) per
                                     pixel: a pixel field whose lines may cut the
                                     fine cells, integrated exactly on each
                                     intersection (quadrilateral.py:136-188),
                                     5 isotropic / 6 (kxx,kxy,kyy) per Gauss point
                                     of every fine cell (quad_order points a side),
                                     integrated by that rule                       */
    const double* kappa;          /* modes 1/2: global fine grid [gx][gy][comp];
                                     modes 3/4: pixels [px][py][comp] (x-major);
                                     modes 5/6: [gx][gy][Q*Q + 1][comp], point
                                     qy*Q + qx, the last one the fine-cell centre
                                     (for the flux)                                */
    double kappa_const[3];        /* kxx, kxy, kyy for kappa_mode 0                */
    int32_t source_mode;          /* 0 constant, 1 per fine cell,
                                     2 per Gauss point of the fine cell,
                                     3 nodal load vector of each cell              */
    const double* source;         /* [gx][gy] or [gx][gy][q] (q = qy*order + qx);
                                     mode 3: [cell][node], node = iy*(rx+1)+ix     */
    double source_const;
    int32_t quad_order;           /* Gauss points per axis for source_mode 2      */
    double pixel_origin[2];       /* kappa_mode 3/4: lower-left corner of pixel 0  */
    double pixel_spacing[2];      /* kappa_mode 3/4: pixel widths                 */
    int32_t pixel_nx, pixel_ny;   /* kappa_mode 3/4: pixel counts; the field must
                                     cover the domain                              */
    double* cut_elements;         /* kappa_mode 3-6: device work buffer of
                                     10 x (global fine cells) doubles: the lower
                                     triangle of each fine cell's element stiffness,
                                     entry-major [entry][gx][gy]; every local entry
                                     point first writes it                         */
} mhm_q1_problem;

/* Width of the per-cell right-hand side block: 1 source + trace + 1 retained. */
int32_t mhm_q1_rhs_width(const mhm_q1_problem* p /* host */);

/* Shared-memory bytes one cell needs (0 if the size is unsupported). */
int64_t mhm_q1_condense_smem_bytes(const mhm_q1_problem* p /* host */, int32_t precision);

/*
 * Assemble, constrain, factor and solve every macrocell, then form its oriented
 * Schur block and reduced load.
 *   solution (cells, w, n+1): augmented responses, column-major per cell:
 *            column 0 = R f, columns 1..t = R B, column w-1 = R (A 1)
 *            (row n = constraint multiplier).
 *   blocks   (cells, t+1, t+1), loads (cells, t+1): local_global_contribution.
 *   corrected (cells): 1 when the assembled A 1 is not exactly zero.
 *   cell_status (cells): MHM_CELL_*; cell_iters (cells): refinement sweeps.
 * tol is the per-column relative residual of the augmented system
 * (||b - K x||_2 <= tol ||b||_2); max_refine bounds the correction sweeps.
 */
int mhm_q1_condense(const mhm_q1_problem* p /* host */, int32_t precision, int32_t max_refine,
                    double tol, double* solution, double* blocks, double* loads,
                    uint8_t* corrected, int32_t* cell_status, int32_t* cell_iters, void* stream);

/*
 * Offline / online reuse (replaces OfflineLocalProblem and the local part of
 * OfflineHybridSystem, core/offline.py:104-313): a condensation that keeps each
 * cell's factor, and later source responses that reuse it.
 *
 * Bytes of the stored factors: cells x (ry+1) x (rx+1)^2 values of the factor
 * type (binary64 for MHM_PRECISION_FP64, binary32 for MHM_PRECISION_MIXED);
 * -1 for invalid arguments.
 */
int64_t mhm_q1_factor_bytes(const mhm_q1_problem* p /* host */, int32_t precision);

/* mhm_q1_condense that also writes each cell's factor (the inverses of its line
 * Schur complements) to `factors` (mhm_q1_factor_bytes). */
int mhm_q1_condense_offline(const mhm_q1_problem* p /* host */, int32_t precision,
                            int32_t max_refine, double tol, double* solution, double* blocks,
                            double* loads, uint8_t* corrected, int32_t* cell_status,
                            int32_t* cell_iters, void* factors, void* stream);

/*
 * The local stage of up to 16 independent problems of one shape (macro grid, local
 * refinement, trace spaces, precision) in one launch: problem k's macrocells are the
 * CTAs (x, k), each reading problems[k] (host array) and writing problem k's own
 * outputs (host arrays of device pointers, as for mhm_q1_condense).  factors may be
 * NULL (a fresh condensation for every problem, mhm_q1_condense) or hold, per problem,
 * NULL or a factor store to keep that problem's cell factors in
 * (mhm_q1_condense_offline).  Permeability modes 0-2 only (no pre-pass); problems of
 * different shapes give MHM_ERR_ARGUMENT, modes 3-6 MHM_ERR_UNSUPPORTED.  Every
 * cell's arithmetic is that of the single-problem launch, so the outputs are
 * identical.  Serving requests that arrive together batch their local stages this way
 * (the per-request launches of a serving loop, core/offline.py:148-229, in one).
 */
int mhm_q1_condense_batch(int32_t count, const mhm_q1_problem* problems, int32_t precision,
                          int32_t max_refine, double tol, double* const* solution, double* const* blocks,
                          double* const* loads, uint8_t* const* corrected, int32_t* const* cell_status,
                          int32_t* const* cell_iters, void* const* factors, void* stream);

/*
 * Source response only (OfflineLocalProblem.response, core/offline.py:121-127):
 * re-assembles every cell with p's source and the offline permeability, reuses
 * `factors` instead of factoring, refines the source column and writes solution
 * column 0 (R f) and `loads`.  Solution columns 1..w-1, the Schur blocks and
 * `corrected` keep what mhm_q1_condense_offline wrote for the same operator; the
 * caller must not change the permeability in between.
 */
int mhm_q1_source_response(const mhm_q1_problem* p /* host */, int32_t precision,
                           int32_t max_refine, double tol, const void* factors, double* solution,
                           double* loads, uint8_t* corrected, int32_t* cell_status,
                           int32_t* cell_iters, void* stream);

/* ------------------------------------------------------------------------ */
/* Original-equation refinement (core/refinement.py:612-800)                 */
/* ------------------------------------------------------------------------ */
/*
 * Residual of the uncondensed equations at a hybrid solution (x: trace then
 * coarse unknowns; fields: (cells, n) nodal values), refinement.py:718-738:
 * defect[cell][i] = f - B lambda - A u (each row in double-double arithmetic),
 * slot_terms[cell][j] = (B^T u)_j, weak[g] = boundary[g] - the DOF's slot terms
 * (first cell, then second; boundary may be NULL = 0), and per cell
 * partial[cell] = {d.d, g.g, sum d} with g = f - B lambda_fixed, lambda_fixed
 * the trace values on the DOFs marked in `fixed` (T bytes; NULL = none, g = f),
 * refinement.py:704-709.  p's source and permeability are those of the original
 * problem.
 */
int mhm_q1_original_defect(const mhm_q1_problem* p /* host */, const int64_t* cell_dofs,
                           int64_t trace_size, const int32_t* dof_cells, const int32_t* dof_slot,
                           const uint8_t* fixed, const double* x, const double* fields,
                           const double* boundary, double* defect, double* slot_terms, double* weak,
                           double* partial, void* stream);

/*
 * The same for a double-double solution (x + x_lo, fields + fields_lo): the
 * extended correction storage of refine_hybrid(refinement_precision="extended")
 * (core/refinement.py:636-643, a wider NumPy type there).  Both low parts are
 * required.
 */
int mhm_q1_original_defect_dd(const mhm_q1_problem* p /* host */, const int64_t* cell_dofs,
                              int64_t trace_size, const int32_t* dof_cells, const int32_t* dof_slot,
                              const uint8_t* fixed, const double* x, const double* x_lo,
                              const double* fields, const double* fields_lo, const double* boundary,
                              double* defect, double* slot_terms, double* weak, double* partial,
                              void* stream);

/*
 * Norms of one refinement step, each summed in a fixed order:
 * out[0] = ||[defects; weak]||^2, out[1] = ||[loads; boundary]||^2,
 * out[2] = ||[weak; sum d per cell]||^2 and, if indptr is given, out[3] =
 * ||rhs||^2 and out[4] = || |K| |x| ||^2 of the assembled CSR system (size rows).
 * out holds 5 + 5 * 256 doubles: the block partials follow the five results.
 */
int mhm_refine_norms(int32_t cells, const double* partial, int64_t trace_size,
                     const uint8_t* fixed /* NULL: none; fixed DOFs and rows are left out */,
                     const double* weak, const double* boundary, int64_t size, const int64_t* indptr,
                     const int32_t* indices, const double* values, const double* x,
                     const double* rhs, double* out /* 5 + 1280 */, void* stream);

/*
 * Correction source responses (refinement.py:779-798): solution column 0 and
 * `loads` become the response to p's source and its reduced load, as in
 * mhm_q1_source_response; p carries the defects as nodal loads (source_mode 3).
 * factors from mhm_q1_condense_offline of the same operator, or NULL to factor
 * each cell again.  The corrected fields are the old ones plus the
 * reconstruction (mhm_q1_reconstruct) of this response with the correction's
 * trace and coarse values.
 */
int mhm_q1_correction_response(const mhm_q1_problem* p /* host */, int32_t precision,
                               int32_t max_refine, double tol, const void* factors,
                               double* solution, double* loads, uint8_t* corrected,
                               int32_t* cell_status, int32_t* cell_iters, void* stream);

/*
 * Mean-pressure gauge of a pure-Neumann solve (every boundary side fixed), the
 * reference's hybrid_mean_constraint with the cells' weights C = M 1
 * (core/system.py:531-566, _legacy/models/darcy/cartesian.py:136-142): with
 * s1 = sum_cells C . fields and s2 = sum_cells C . (1 - R A1) (solution column
 * w-1), adds alpha = (value - s1) / s2 to every coarse unknown x[T + cell].  The
 * caller reconstructs again.  partial: 2 cells + 1 doubles (the last = alpha).
 */
int mhm_q1_mean_gauge(const mhm_q1_problem* p /* host */, const double* solution,
                      const double* fields, double value, int64_t trace_size, double* x,
                      double* partial, void* stream);

/* Flux -K grad u at the fine-cell centres from given nodal fields (cells, n):
 * the flux part of mhm_q1_reconstruct (postprocessing/solutions.py:278-324). */
int mhm_q1_flux(const mhm_q1_problem* p /* host */, const double* fields, double* flux, void* stream);

/* dst[i] += src[i], i < n (the hybrid unknowns plus a correction). */
int mhm_vector_accumulate(int64_t n, double* dst, const double* src, void* stream);

/* (hi[i], lo[i]) += src[i] in double-double arithmetic, i < n (a correction added
 * to a double-double solution). */
int mhm_vector_accumulate_dd(int64_t n, double* hi, double* lo, const double* src, void* stream);

/* ------------------------------------------------------------------------ */
/* Ordered skeleton reduction                                                 */
/* ------------------------------------------------------------------------ */
/*
 * vals[s] = sum_{e in slot_ptr[s]..slot_ptr[s+1]} blocks_flat[contrib[e]] in
 * ascending cell order (precomputed by the host from the DOF maps); likewise
 * rhs[g] = sum loads_flat[load_contrib[.]] - boundary[g] (g < trace_size) and
 * load_scale[g] = sum |loads| + |boundary[g]|.  Deterministic, no atomics.
 */
int mhm_skeleton_scatter(int64_t nnz, const int64_t* slot_ptr, const int64_t* contrib,
                         const double* blocks, double* vals, int64_t size, int64_t trace_size,
                         const int64_t* load_ptr, const int64_t* load_contrib, const double* loads,
                         const double* boundary, double* rhs, double* load_scale, void* stream);

/*
 * The assembled matrix as the reference hands it on: CSC, entries whose sum is
 * exactly zero (either sign) dropped.  Replaces `coo_matrix(...).tocsc()` and
 * `matrix.eliminate_zeros()` (core/contributions.py:184-185).  Input: the
 * structural CSR (indptr size+1, indices sorted per row) with the values of
 * mhm_skeleton_scatter, and transpose[k] = the CSR slot of (i, j) for the CSR
 * slot k of (j, i) (the pattern is symmetric).  Output: csc_indptr (size+1),
 * csc_indices / csc_data (at least nnz entries; csc_indptr[size] are used).
 */
int mhm_skeleton_export_csc(int64_t size, const int64_t* indptr, const int32_t* indices,
                            const int64_t* transpose, const double* vals, int64_t* csc_indptr,
                            int32_t* csc_indices, double* csc_data, void* stream);

/* ------------------------------------------------------------------------ */
/* Global skeleton solve: projected PCG with an outer FP64 defect correction  */
/* ------------------------------------------------------------------------ */
typedef struct mhm_skeleton_system {
    int64_t size;                 /* N = trace_size + cells                        */
    int64_t trace_size;           /* T                                             */
    const int64_t* indptr;        /* CSR of the full matrix K (N+1)                */
    const int32_t* indices;       /* column indices, sorted per row                */
    const double* values;
    const int64_t* trace_end;     /* (T): first CSR slot of row r with col >= T    */
    int32_t faces;                /* number of skeleton faces                      */
    int32_t face_size;            /* DOFs per face (uniform skeleton)              */
    int32_t cells;
    int32_t cell_width;           /* t: trace DOFs per cell                        */
    const int64_t* cell_dofs;     /* (cells, t)                                    */
    const double* cell_g0;        /* (cells, t): geometric constraint column        */
    const int32_t* dof_cells;     /* (T, 2): cells sharing the DOF (-1 = none)      */
    const int32_t* dof_slot;      /* (T, 2): position of the DOF in each cell      */
    int32_t nx, ny;               /* macro grid of the coarse Poisson operator     */
    /* G0^T G0 = coarse_ay (T_y (x) I) + coarse_ax (I (x) T_x), T = tridiag(-1,2,-1) */
    double coarse_ax, coarse_ay;
    /* Optional (NULL allowed): the cells' own trace blocks, (cells, block_ld,
     * block_ld) row-major, top-left cell_width x cell_width used; S must equal
     * their sum scattered through cell_dofs (mhm_q1_condense's `blocks` with
     * block_ld = cell_width + 1).  With them the solve uses the cell-Dirichlet
     * preconditioner; without them it splits S from the CSR matrix and uses
     * additive Schwarz over the cells' 12 x 12 principal submatrices.          */
    const double* cell_blocks;
    int32_t block_ld;
    /* Optional (NULL allowed): fixed trace DOFs, T bytes (1 = fixed), the Neumann
     * faces' prescribed coefficients (core/system.py:421-447).  The solve then
     * works on the free DOFs: rhs must hold rhs - K x_fixed with zeros on the
     * fixed rows (mhm_skeleton_fixed_rhs), x is returned zero on them and the
     * caller adds x_fixed.  The fixed DOFs are all DOFs of their faces.  Whole
     * fixed sides are Neumann ends of T_y (coarse_neumann bit 0 = bottom y = y0,
     * bit 1 = top) and of T_x (bit 2 = left x = x0, bit 3 = right); faces on
     * parts of sides go through coarse_partial below.                           */
    const uint8_t* fixed;
    int32_t coarse_neumann;
    /* With coarse_neumann bit 2 (left side x = x0 fixed) or bit 3 (right side):
     * the eigenvectors and eigenvalues of T_x with those Neumann ends,
     * coarse_qx[cell][mode] (nx x nx, orthonormal columns) and coarse_lamx[mode]
     * (nx), which replace the sine basis.  Ignored otherwise (NULL allowed).  */
    const double* coarse_qx;
    const double* coarse_lamx;
    /* With all four sides fixed (coarse_neumann 15, pure Neumann): the ny x ny
     * pseudo-inverse of mode 0's T_y (row-major), the constant coarse mode being
     * the kernel of G0^T G0.  The solve then returns coarse unknowns without that
     * mode; mhm_q1_mean_gauge fixes it from the mean-pressure condition.        */
    const double* coarse_pinv0;
    /* Fixed DOFs on part of a side (Neumann faces that do not cover it): the
     * coarse operator above (those sides counted as Dirichlet) less a_y (a_x)
     * on the diagonal of each cell with such a horizontal (vertical) face.
     * coarse_partial = m cells (0: none; at most 2 (nx + ny)),
     * coarse_partial_cells[m] their indices, coarse_partial_R (cells x m,
     * row-major) = A_sep^-1 E (D^-1 - E^T A_sep^-1 E)^-1 (the Woodbury factor;
     * topology.coarse_partial_correction computes it).                        */
    int32_t coarse_partial;
    const int32_t* coarse_partial_cells;
    const double* coarse_partial_R;
} mhm_skeleton_system;

int64_t mhm_skeleton_workspace_bytes(const mhm_skeleton_system* s /* host */, int32_t grid);

/*
 * Elimination of prescribed trace DOFs before mhm_skeleton_solve:
 * reduced[i] = rhs[i] - sum_j K[i][j] xfixed[j] (double-double row sums) on the
 * free rows, 0 on the fixed ones (reduced may be rhs).  xfixed (N) holds the
 * prescribed values on the fixed trace DOFs and zeros elsewhere; fixed (T bytes)
 * marks them.  K is the CSR of mhm_skeleton_system.
 */
int mhm_skeleton_fixed_rhs(int64_t size, int64_t trace_size, const int64_t* indptr,
                           const int32_t* indices, const double* values, const uint8_t* fixed,
                           const double* xfixed, const double* rhs, double* reduced, void* stream);

/*
 * Solve K x = rhs.  x (N) is output.  info (device int32[4]): status, total
 * inner iterations, outer corrections, barrier error flag.  stats (device
 * double[4]): final relative residual ||rhs - K x|| / ||rhs||, the physical
 * certificate ||K x - rhs|| / max(||rhs||, ||load_scale||, || |K||x| ||),
 * relative residual after the first outer correction, unused.  rtol bounds the
 * outer FP64 residual; the first inner solve runs to inner_rtol, each later one
 * to rtol / (current outer residual), clipped to [1e-12, 0.1].  The solve runs as one persistent
 * cooperative kernel with one CTA per macro row (ny CTAs, all co-resident;
 * MHM_ERR_UNSUPPORTED when they do not fit or a row's tables exceed shared
 * memory); `grid` is accepted for ABI stability and ignored.  workspace is
 * sized by mhm_skeleton_workspace_bytes.
 */
int mhm_skeleton_solve(const mhm_skeleton_system* s /* host */, const double* rhs,
                       const double* load_scale, double* x, double rtol, double inner_rtol,
                       int32_t max_inner, int32_t max_outer, int32_t grid, void* workspace,
                       int64_t workspace_bytes, int32_t* info, double* stats, void* stream);

/*
 * Allocation-free form of mhm_skeleton_solve, for callers that cannot allocate
 * device memory (a C/Fortran/FFI host code without its own CUDA allocator, or a
 * serving process that reserves all device memory up front and must not call
 * cudaMalloc/cudaFree, which also synchronise the device).  It has no
 * counterpart in the reference, which solves the global system on the host.
 * The scratch is a fixed 4 MiB file-scope device array that every GPU loading
 * the library holds until exit; systems whose mhm_skeleton_workspace_bytes
 * exceeds 4 MiB are rejected with MHM_ERR_UNSUPPORTED (64x64 macrocells with
 * three DOFs per face need about 2.6 MiB).  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (other streams, other host threads) race
 * and must be serialised by the caller.  Arguments and results are those of
 * mhm_skeleton_solve.
 */
int mhm_skeleton_solve_static(const mhm_skeleton_system* s /* host */, const double* rhs,
                              const double* load_scale, double* x, double rtol, double inner_rtol,
                              int32_t max_inner, int32_t max_outer, int32_t grid, int32_t* info,
                              double* stats, void* stream);

/* ------------------------------------------------------------------------ */
/* Global skeleton solve on any macro mesh (tetrahedra, polygons, ...)        */
/* ------------------------------------------------------------------------ */
/*
 * Replaces solve_hybrid_system's global solve (core/system.py:355-528 ->
 * linalg/linear.py:798, SuperLU at rtol 1e-10) for macro meshes without the
 * Cartesian structure mhm_skeleton_solve relies on.  The caller describes the
 * assembled system K = [[S, -G], [-G^T, -C]] (the structural CSR of
 * mhm_skeleton_scatter) and the exact geometric constraint G0 = B^T 1 of every
 * cell, together with the dense inverse of the coarse operator G0^T G0, which
 * depends on the mesh only.  All pointers are device pointers; the struct itself
 * is read on the host.
 */
typedef struct mhm_general_system {
    int64_t size;                 /* N = trace_size + cells                         */
    int64_t trace_size;           /* T                                              */
    const int64_t* indptr;        /* CSR of K (N+1), columns sorted per row         */
    const int32_t* indices;
    const double* values;
    int32_t faces;                /* skeleton faces                                  */
    int32_t max_face_size;        /* largest DOF count of a face (1..8)             */
    const int64_t* face_ptr;      /* (faces+1): face f owns DOFs face_ptr[f]..[f+1]-1 */
    int32_t cells;
    const int64_t* cell_ptr;      /* (cells+1) into cell_dofs / cell_g0            */
    const int64_t* cell_dofs;     /* trace DOFs of every cell, in its local order   */
    const double* cell_g0;        /* G0 entry of each (cell, local DOF)              */
    const int32_t* dof_cells;     /* (T, 2): the cells holding each DOF (-1: none)  */
    const int64_t* dof_entry;     /* (T, 2): its index in cell_dofs / cell_g0       */
    const double* coarse_inverse; /* (cells, cells) row-major (G0^T G0)^-1           */
    int64_t cell_entries;         /* cell_ptr[cells]                                 */
    /* Optional (cell_blocks NULL: face block-Jacobi preconditioner).  The cells'
       condensed (t+1) x (t+1) blocks, row-major at block_off[c] (t = the cell's
       DOF count <= max_cell_dofs <= 32, local order of cell_dofs; the last row and
       column are the coarse unknown), select the cell-Dirichlet preconditioner.
       The workspace holds its buffers whenever block_off is set.               */
    const double* cell_blocks;
    const int64_t* block_off;     /* (cells)                                         */
    int64_t blocks_size;          /* doubles spanned by the blocks                   */
    int32_t max_cell_dofs;
    int32_t max_trace_row;        /* most trace columns (< T) in one row of the CSR  */
} mhm_general_system;

/* Workspace bytes of mhm_general_solve on the current device (-1: invalid). */
int64_t mhm_general_workspace_bytes(const mhm_general_system* s /* host */);

/*
 * x (N) = K^-1 rhs (N): flexible GMRES on K in FP64 (cycles of at most 8
 * steps, each restarted from the true residual) until ||rhs - K x|| <= rtol
 * ||rhs|| and every row's residual is within rtol of |rhs_i| + sum_j |K_ij|
 * |x_j| (or that componentwise error stopped improving).  Each step solves
 * with [[S, -G0], [-G0^T, 0]] by projected CG, preconditioned by face
 * block-Jacobi or, with cell_blocks, by the cells' D S_c^-1 D, until the
 * preconditioned residual norm fell by inner_rtol (at most max_inner CG
 * iterations in total and max_outer such solves).  Setup kernels, then one
 * persistent cooperative launch (one CTA per SM).
 * info (4 int32, device): status (MHM_SOLVE_*), inner iterations, inner
 * solves, barrier error flag; stats (3 doubles, device): final relative
 * residual, ||rhs||, componentwise backward error.  Every grid barrier is bounded.
 */
int mhm_general_solve(const mhm_general_system* s /* host */, const double* rhs, double* x,
                      void* workspace, int64_t workspace_bytes, double rtol, double inner_rtol,
                      int32_t max_inner, int32_t max_outer, int32_t* info, double* stats,
                      void* stream);

/* ------------------------------------------------------------------------ */
/* Dense local problems (tetrahedral macrocells)                             */
/* ------------------------------------------------------------------------ */
/*
 * Material pre-pass of tetra_operators (fem/scalar/tetrahedron.py:41-52,
 * 157-190) for a layered voxel permeability: for every macrocell (its refined
 * vertices points (cells, npoints, 3), as TetraMesh.submesh computes them) and
 * fine tetrahedron e (fine_cells (nfine, 4)), the quadrature average
 * sum_q w_q kappa(x_q) over quad_bary / quad_weights (nquad), kappa the voxel
 * value voxels[layer(z)][ix(x)][iy(y)] (layers x px x py over the unit cube).
 * Writes the isotropic tensors diffusion (cells, nfine, 3, 3).
 */
int mhm_tet_kappa(int64_t cells, const double* points, int32_t npoints, int32_t nfine,
                  const int32_t* fine_cells, int32_t nquad, const double* quad_bary,
                  const double* quad_weights, int32_t layers, int32_t px, int32_t py,
                  const double* voxels, double* diffusion, void* stream);

/*
 * Local contract and augmented systems of `count` dense local problems
 * (LocalProblem.__init__, core/contracts.py:92-211, with kernel 1 and
 * constraint M 1, divided by 1^T M 1 when `normalize` is set as the 2D primal
 * driver does, _legacy/models/darcy/primal.py:69-71; local_condensation_system,
 * core/condensation.py:125-174).  Cell k has n_of[k] unknowns and t_of[k] <= 28
 * trace columns; its stiffness and mass are rows of lds doubles at
 * k * lds * lds, its load at k * lds, its coupling (lds x tld) at k * lds * tld.
 * Writes aug (count, nb, nb), nb >= n + 1: [[A, c~], [c~^T, 0]] with
 * c~ = C min(1, max|A| / max|C|) and an identity block past n + 1; rhs
 * (count, nb, w), w >= t + 2: [f | B | A 1] (the A 1 column zero when the cell
 * is not corrected, zero rows past n); action (count, 3, nb) = A 1, A^T 1
 * (double-double sums) and M 1; corrected (count); status (count:
 * MHM_CELL_KERNEL when the constant is not a left and right kernel at 1e-10).
 */
int mhm_dense_systems(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w, int32_t normalize,
                      const int32_t* n_of, const int32_t* t_of, const double* stiffness, const double* mass,
                      const double* load, const double* coupling, double* aug, double* rhs,
                      double* action, uint8_t* corrected, int32_t* status, void* stream);

/*
 * Oriented Schur block ((t+1) x (t+1), at blocks + block_off[k]) and reduced
 * load (t+1, at loads + load_off[k]) of each cell from its solved augmented
 * system solution (count, nb, w) = [R f | R B | R A 1]
 * (local_global_contribution, core/contributions.py:14-74;
 * local_condensed_load, core/reconstruction.py:91-127).  The products run on
 * the tensor cores (FP64 mma.sync); max_t is the largest t_of (at most 28).
 */
int mhm_dense_contributions(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w, int32_t max_t,
                            const int32_t* n_of, const int32_t* t_of, const double* solution,
                            const double* coupling, const double* action, const double* load,
                            const int64_t* block_off, const int64_t* load_off, double* blocks,
                            double* loads, void* stream);

/*
 * P2 triangle operators of polygonal macrocells (scalar_operators,
 * fem/scalar/triangle.py:208-257, degree 2, a scalar permeability sampled at the
 * Duffy rule's points, constant source), dense per cell.  Every fine triangle of
 * every cell is one element: triangles (elements, 3) index points (x, y pairs).
 * The permeability is `inside` in the union of the discs (centres (D, 2), squared
 * radii radii2), else `outside`; grid > 0 gives a grid x grid cell list over the
 * unit square (grid_ptr (grid^2 + 1) into grid_discs, cell gx * grid + gy, every
 * disc meeting the cell listed); grid = 0 means a constant `outside`.
 * element_scratch: mhm_p2_element_bytes.  Node g of all cells is row node_row[g]
 * of cell node_cell[g]: its element incidences inc[inc_ptr[g] ..] (element * 6 +
 * local index, ascending), elem_dofs (elements, 6) the cell-local DOFs; the cell's
 * dense stiffness and mass start at dense_off[cell] with rows of ld_of[cell]
 * doubles and its load at load_off[cell].  Rows are summed in element order.
 */
int64_t mhm_p2_element_bytes(int64_t elements);
int mhm_p2_assemble(int64_t elements, const double* points, const int64_t* triangles, int32_t nquad,
                    const double* quad_bary, const double* quad_weights, int32_t grid,
                    const int32_t* grid_ptr, const int32_t* grid_discs, const double* centres,
                    const double* radii2, double inside, double outside, double source,
                    double* element_scratch, int64_t nodes, const int32_t* node_cell,
                    const int32_t* node_row, const int64_t* inc_ptr, const int64_t* inc,
                    const int32_t* elem_dofs, const int64_t* dense_off, const int32_t* ld_of,
                    const int64_t* load_off, double* stiffness, double* mass, double* load,
                    void* stream);

/*
 * The two passes of mhm_p2_assemble as separate calls (the same arithmetic), for
 * local matrices too large to hold at once: mhm_p2_elements fills element_scratch
 * for every fine triangle; mhm_p2_assemble_rows then builds the dense rows of any
 * contiguous range of nodes (node_cell, node_row and inc_ptr offset to its first
 * node; dense_off may address a workspace that holds only those cells).
 * Replaces, with mhm_p2_assemble, scalar_operators (fem/scalar/triangle.py:208-257)
 * for the cells of a polygon batch whose P2 spaces exceed 639 unknowns.
 */
int mhm_p2_elements(int64_t elements, const double* points, const int64_t* triangles, int32_t nquad,
                    const double* quad_bary, const double* quad_weights, int32_t grid,
                    const int32_t* grid_ptr, const int32_t* grid_discs, const double* centres,
                    const double* radii2, double inside, double outside, double source,
                    double* element_scratch, void* stream);
int mhm_p2_assemble_rows(int64_t nodes, const int32_t* node_cell, const int32_t* node_row,
                         const int64_t* inc_ptr, const int64_t* inc, const int32_t* elem_dofs,
                         const double* element_scratch, const int64_t* dense_off, const int32_t* ld_of,
                         const int64_t* load_off, double* stiffness, double* mass, double* load,
                         void* stream);

/* u_K = R f - (R B) lambda_K + (1 - R A 1) c_K for dense cells (core/reconstruction.py:
 * 130-141): cell k's n_of[k] values go to fields + field_off[k]; its trace DOFs
 * are cell_dofs[dof_off[k] ...], its coarse unknown x[trace_size + cell_id[k]]. */
int mhm_dense_reconstruct(int64_t count, int32_t nb, int32_t w, const int32_t* n_of, const int32_t* t_of,
                          const double* solution, const int64_t* cell_dofs, const int64_t* dof_off,
                          const int32_t* cell_id, int64_t trace_size, const double* x,
                          const int64_t* field_off, double* fields, void* stream);

/*
 * Mixed RT0 / P0 local problems of polygonal macrocells (the "mixed" branch of
 * _DarcyLocalFactory, _legacy/models/darcy/primal.py:80-103: rt0_operators,
 * fem/scalar/operators.py:324-364, and normal_flux_blocks, fem/hdiv/mixed.py:77-112).
 * Local unknowns: the fine faces' fluxes, the fine cells' pressures, the boundary
 * faces' multipliers.  mhm_rt0_elements writes every fine triangle's saddle block
 * [[M, -s, S], [-s^T, 0, 0], [S^T, 0, 0]] over the slots (face 0, face 1, face 2,
 * pressure, multiplier a, multiplier b) in the mhm_p2_elements layout (so that
 * mhm_p2_assemble_rows builds the dense rows): M_ab = sum_q w_q area
 * kappa(x_q)^-1 phi_a . phi_b with phi_s = sign_s (x - v_(s+2)%3) / (2 area) (the
 * triangle's vertices counter-clockwise), the pressure mass (the area) and the load
 * (-area sum_q w_q source) on the pressure slot.  info (elements, 5): the faces'
 * signs (+1 / -1) and the local faces (0..2, or -1) selected by the two multiplier
 * slots.  Permeability as mhm_p2_elements.
 */
int mhm_rt0_elements(int64_t elements, const double* points, const int64_t* triangles, const int32_t* info,
                     int32_t nquad, const double* quad_bary, const double* quad_weights, int32_t grid,
                     const int32_t* grid_ptr, const int32_t* grid_discs, const double* centres,
                     const double* radii2, double inside, double outside, double source,
                     double* element_scratch, void* stream);

/*
 * mhm_dense_systems, mhm_dense_contributions and mhm_dense_reconstruct for a
 * declared kernel Z other than the ones vector: kernel (0 / 1 per unknown, in the
 * load's layout; kernel_fields in the fields' layout).  The systems test A Z and
 * A^T Z at 1e-10 ||A||_F ||Z||, border with C = M Z / (Z^T M Z) (primal.py:99-100)
 * and put A Z in the corrected column; the contributions use E = Z - R A Z and
 * write the blocks and loads negated (the mixed blocks are negative semi-definite;
 * the negated system has the same solution); reconstruction adds E c_K.
 */
int mhm_mixed_systems(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w, const int32_t* n_of,
                      const int32_t* t_of, const double* matrix, const double* mass, const double* load,
                      const double* coupling, const double* kernel, double* aug, double* rhs, double* action,
                      uint8_t* corrected, int32_t* status, void* stream);
int mhm_mixed_contributions(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w, int32_t max_t,
                            const int32_t* n_of, const int32_t* t_of, const double* solution,
                            const double* coupling, const double* action, const double* load,
                            const double* kernel, const int64_t* block_off, const int64_t* load_off,
                            double* blocks, double* loads, void* stream);
int mhm_mixed_reconstruct(int64_t count, int32_t nb, int32_t w, const int32_t* n_of, const int32_t* t_of,
                          const double* solution, const int64_t* cell_dofs, const int64_t* dof_off,
                          const int32_t* cell_id, int64_t trace_size, const double* x,
                          const int64_t* field_off, const double* kernel_fields, double* fields,
                          void* stream);

/* ------------------------------------------------------------------------ */
/* Reconstruction u_K = R f - (R B) lambda_K + E c_K and flux -K grad u       */
/* ------------------------------------------------------------------------ */
int mhm_q1_reconstruct(const mhm_q1_problem* p /* host */, const double* solution,
                       const int64_t* cell_dofs, int64_t trace_size, const double* x,
                       double* fields, double* flux, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched dense equilibrated LU (BatchedFactorization contract)              */
/* ------------------------------------------------------------------------ */
/*
 * factors (count, n, n) receives the row/column-equilibrated LU of matrices
 * (count, n, n), row-major; pivots (count, n); row_scale/col_scale (count, n)
 * hold 1/max; status (count) receives MHM_CELL_*.
 */
int mhm_batched_factor(int64_t count, int32_t n, const double* matrices, double* factors,
                       int32_t* pivots, double* row_scale, double* col_scale, int32_t* status,
                       void* stream);

/*
 * Solve matrices @ x = rhs for rhs (count, n, nrhs) row-major using the factors,
 * with up to max_refine FP64 residual corrections; each column must satisfy
 * ||A x - b|| <= max(atol, rtol ||b||) with the reference's max-scaling, else
 * status = MHM_CELL_RESIDUAL.  x (count, n, nrhs); work (count, n, nrhs).
 */
int mhm_batched_solve(int64_t count, int32_t n, int32_t nrhs, const double* matrices,
                      const double* factors, const int32_t* pivots, const double* row_scale,
                      const double* col_scale, const double* rhs, double* x, double* work,
                      double rtol, double atol, int32_t max_refine, int32_t* status,
                      void* stream);

/*
 * Ragged batches: matrices of different orders in one launch (polygon cells binned
 * by padded size).  Matrix k has order n (its rows and columns, row-major, at
 * matrices / factors + mat_off), pivots and row / column scales at + vec_off,
 * nrhs right-hand sides and solutions (n, nrhs) row-major at rhs / x + rhs_off,
 * and its status word at status[slot].
 */
typedef struct mhm_ragged_matrix {
    int64_t mat_off;
    int64_t vec_off;
    int64_t rhs_off;
    int32_t n;
    int32_t nrhs;
    int32_t slot;
    int32_t reserved;
} mhm_ragged_matrix;

/*
 * mhm_batched_factor over count ragged matrices in one launch (descriptors on the
 * device; every n <= max_n <= 640, larger ones get MHM_CELL_SIZE).  CTAs start in
 * descriptor order, so listing the largest matrices first balances the SMs.
 */
int mhm_batched_factor_ragged(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                              const double* matrices, double* factors, int32_t* pivots,
                              double* row_scale, double* col_scale, int32_t* status, void* stream);

/*
 * mhm_batched_solve over count ragged systems (nrhs <= max_nrhs columns each), one
 * launch per group of 16 columns, with the same acceptance per column.
 */
int mhm_batched_solve_ragged(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                             int32_t max_nrhs, const double* matrices, const double* factors,
                             const int32_t* pivots, const double* row_scale, const double* col_scale,
                             const double* rhs, double* x, double rtol, double atol, int32_t max_refine,
                             int32_t* status, void* stream);

/*
 * mhm_dense_systems over ragged cells in one launch: cell k of the launch is described
 * by desc[k] (order nb = n with lds = nb, nrhs = w columns, its stiffness, mass and
 * augmented matrix at mat_off (the augmented matrix may overwrite the stiffness), its
 * load at vec_off, actions at 3 vec_off, right-hand sides at rhs_off, sizes, flag
 * and status at slot) and by cpl_off[k] / tld_of[k] (its coupling block and width).
 * Same arithmetic per cell as mhm_dense_systems.
 */
int mhm_dense_systems_ragged(int64_t count, const mhm_ragged_matrix* desc, const int64_t* cpl_off,
                             const int32_t* tld_of, int32_t normalize, const int32_t* n_of,
                             const int32_t* t_of, const double* stiffness, const double* mass,
                             const double* load, const double* coupling, double* aug, double* rhs,
                             double* action, uint8_t* corrected, int32_t* status, void* stream);

/*
 * Large orders (n <= 4096; larger get MHM_CELL_SIZE): ragged batches of the bordered
 * local systems [[A, c], [c^T, 0]] (A positive semi-definite with the constants as
 * its kernel, identity padding allowed).  The factorization is the blocked LU in
 * HBM with the row search of each column restricted to its 32-column panel's
 * diagonal window and the one row below it (the bordering row needs no more: the
 * node rows' leading blocks are positive definite); the factors, pivots (LAPACK
 * sequence), scales, rank test and status words are those of
 * mhm_batched_factor_ragged, so the solve contract is the same.  The solve handles
 * up to 32 right-hand sides per pass and keeps its solution and correction blocks in
 * `work`: 66 doubles per row of every system, system k's at work + 66 vec_off.  Replaces the reference's large-block route,
 * `_condense_device` (execution/cuda.py:314-343: sparse cuDSS through the checked
 * factorization for augmented sizes above dense_size_limit = 512, cuda.py:352), for
 * the polygon batch's local P2 systems of order 640 to 4096.
 */
int mhm_batched_factor_large(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                             const double* matrices, double* factors, int32_t* pivots,
                             double* row_scale, double* col_scale, int32_t* status, void* stream);
int mhm_batched_solve_large(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                            int32_t max_nrhs, const double* matrices, const double* factors,
                            const int32_t* pivots, const double* row_scale, const double* col_scale,
                            const double* rhs, double* x, double* work, double rtol, double atol,
                            int32_t max_refine, int32_t* status, void* stream);

/* Library version string (host). */
const char* mhm_version(void);

/* ------------------------------------------------------------------------ */
/* Batched dense P1 simplex assembly (execution/cuda.py:27-105)               */
/* ------------------------------------------------------------------------ */
/*
 * points (batch, npoints, dim), dim 2 or 3; every batch item shares
 * cells (ncells, dim+1), which the caller has checked (0 <= index < npoints).
 * diffusion holds dim x dim tensors: item b, cell e uses tensor
 * b * diffusion_batch_stride + e * diffusion_cell_stride (strides 0 broadcast);
 * source likewise holds one value per fine cell.  node_ptr (npoints+1) /
 * node_contrib list, per node, element * (dim+1) + local index in ascending
 * element order.  scratch: mhm_p1_batch_scratch_bytes.  Outputs: dense
 * stiffness and consistent mass (batch, npoints, npoints) and load
 * (batch, npoints); each entry sums its elements in ascending order.
 * status[0..3] is set to 1 for non-finite points, a degenerate simplex
 * (|det J| <= eps prod |J columns|), a diffusion tensor that is not finite,
 * symmetric (1e-12 relative) and positive definite, or a non-finite source.
 */
int mhm_p1_batch_assemble(int64_t batch, int32_t npoints, int32_t dim, const double* points,
                          int32_t ncells, const int32_t* cells, const double* diffusion,
                          int64_t diffusion_batch_stride, int64_t diffusion_cell_stride,
                          const double* source, int64_t source_batch_stride,
                          int64_t source_cell_stride, const int64_t* node_ptr,
                          const int32_t* node_contrib, double* scratch, double* stiffness,
                          double* mass, double* load, int32_t* status /* 4 */, void* stream);

int64_t mhm_p1_batch_scratch_bytes(int64_t batch, int32_t dim, int32_t ncells);

#ifdef __cplusplus
}
#endif

#endif /* MHM_B200_H */
