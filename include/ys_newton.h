/*
 * ys_newton.h -- C ABI of the yasps_b200 Newton inner-loop library.
 *
 * One shared library (libys_newton.so) built for sm_100a.  Every entry point
 * is `extern "C"`, takes plain device/host pointers and sizes, never throws,
 * and returns an int32 status (YS_OK == 0, negative on error; see below).
 * All device buffers are owned by the caller.  `stream` is a cudaStream_t
 * passed as `void*` (NULL = legacy default stream).  Calls on the same
 * stream are ordered; no call synchronises the device unless stated.
 *
 * Citations point at the reference (txstc55/yasps) interface each entry
 * replaces, relative to the reference project root, PKG = yasps/yasps.
 */
#ifndef YS_NEWTON_H
#define YS_NEWTON_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes (mirroring the reference's return codes) ------------- */
#define YS_OK 0
#define YS_ERR_CUDA (-1)              /* CUDA failure (hessianKernelHost.pyx:151-155)    */
#define YS_ERR_INVALID (-2)           /* invalid argument / unsupported shape           */
#define YS_ERR_CAPACITY (-3)          /* caller buffer or index range too small         */
#define YS_ERR_NOT_CONVERGED (-4)     /* PCG budget exhausted (solverKernel.pyx:686)     */
#define YS_ERR_INVALID_RESIDUAL (-5)  /* invalid initial residual (solverKernel.pyx:602) */
/* A non-positive curvature at PCG iteration `it` returns -(it + 4)
 * (solverKernel.pyx:670-673); MAS domain inversion failures return
 * YS_ERR_SINGULAR_DOMAIN with the failing domain count in the result.    */
#define YS_ERR_SINGULAR_DOMAIN (-6)

/* Last error message of the calling thread ("" if none). */
const char* ys_last_error(void);
/* Library ABI version (major * 100 + minor). */
int32_t ys_version(void);

/* ---- index slots (PKG/kernel/Coordinate/gradientIndicesKernel.pyx) ------ */

/* Slot codes of an energy whose argument list is a JOIN of dimension
 * `join_dim` through `connectivity` [n x join_dim] into a primitive union of
 * `num_children` children (num_children == 1: a plain primitive).  Child c
 * owns union indices [child_prefix[c], child_prefix[c+1]) and resolves to
 *   child_kind[c] == 2: target leaf, code = child_wrt_start[c] + i*size + 2
 *   child_kind[c] == 1: non-target DATA leaf, code 1
 *   child_kind[c] == 0: no differentiated leaf (CONSTANT / not a target of
 *                       a restricted energy): code 0, the space is padding.
 * With a union every argument takes two slots [child, pad] (the reference
 * reserves index_size+1 slots, gradientIndicesKernel.pyx:566-574); the pad
 * slot carries the size of an argument whose child has no leaf.
 * Output: codes [n x K], sizes [n x K], K = join_dim * (num_children > 1 ? 2 : 1).
 * `child_prefix`, `child_kind`, `child_wrt_start` are HOST arrays (<= 8 children).
 * Replaces the generated `int get_indices(...)`
 * (gradientIndicesKernel.pyx:869-946).                                      */
int32_t ys_join_union_indices(const uint32_t* connectivity, uint32_t n, uint32_t join_dim,
                              uint32_t num_children, const uint32_t* child_prefix,
                              const int32_t* child_kind, const uint32_t* child_wrt_start,
                              uint32_t leaf_size, uint32_t* codes, uint16_t* sizes, void* stream);

/* Local permutation + per-instance coordinate counts.  coord_outer has n+1
 * entries: coord_outer[0] = 0, coord_outer[i+1] = sum_{j<=i} u_j (u_j + 1)/2
 * with u_j the unique target slots of instance j.  total_sizes may be NULL.
 * Replaces `int compress_indices(...)` (gradientIndicesKernel.pyx:131-214);
 * the reference's grouping of instances by compressed size only selects its
 * per-size kernel templates and has no counterpart here.                   */
int32_t ys_compress_indices(const uint32_t* codes, const uint16_t* sizes, uint32_t n, uint32_t K,
                            int16_t* perm, uint16_t* total_sizes, uint32_t* coord_outer,
                            void* stream);

/* Same arguments and outputs as ys_compress_indices (bit-identical), but the
 * call allocates nothing: the count scan keeps its tile sums in a fixed
 * 128 KiB device array of the library instead of temporary storage from
 * cudaMallocAsync.  No counterpart in the reference.
 * Limit: n <= 67,108,864 instances; larger n returns YS_ERR_CAPACITY.
 * The first call on a device resolves the array's address (set-up), so make
 * it before any stream capture.  The address is kept for the life of the
 * process: after cudaDeviceReset (or any other teardown of the device's
 * primary context) it is stale, so do not call this entry point on that
 * device again in the same process.  All calls on a device share the array:
 * calls that overlap in time (other streams or threads) race on it.        */
int32_t ys_compress_indices_noalloc(const uint32_t* codes, const uint16_t* sizes, uint32_t n,
                                    uint32_t K, int16_t* perm, uint16_t* total_sizes,
                                    uint32_t* coord_outer, void* stream);

/* Upper-triangle block coordinates (scalar (row,col) pairs) and dims.
 * Replaces `int computeCoordinates(...)` (gradientIndicesKernel.pyx:276-318). */
int32_t ys_compute_coordinates(const uint32_t* codes, const int16_t* perm, const uint16_t* sizes,
                               const uint32_t* coord_outer, uint32_t n, uint32_t K,
                               uint32_t* coords, uint16_t* dims, void* stream);

/* ---- sparsity pattern (PKG/kernel/Coordinate/coordinateCompressionKernel.pyx) */

/* Device workspace for ys_pattern_build with `n_coords` occurrences. */
int32_t ys_pattern_workspace_bytes(uint32_t n_coords, uint64_t* bytes);

typedef struct ys_pattern_out {
  /* device outputs, capacity n_coords (n_coords + 1 for value_offset) */
  uint32_t* positions;     /* [2*nu] unique scalar (row, col), order (h, w, row, col) */
  uint16_t* block_dims;    /* [2*nu] (h, w)                                       */
  uint32_t* value_offset;  /* [nu+1] exclusive scan of h*w                         */
  uint32_t* lookup;        /* [n_coords] value offset of each occurrence           */
  uint32_t* record;        /* [n_coords] record offset of each occurrence          */
  uint32_t* record_begin;  /* [nu] record offset of each unique block's first record */
  uint32_t* record_count;  /* [nu] occurrences of each unique block                */
  /* host outputs */
  uint32_t num_unique;
  uint32_t num_categories;     /* <= 16 */
  uint16_t category_dims[32];  /* (h, w) per category                              */
  uint32_t category_counts[16];
  uint32_t category_starts[17];/* value offsets; [num_categories] = total values  */
  uint64_t total_records;      /* sum of h*w over occurrences                      */
} ys_pattern_out;

/* Global unique sort of all occurrences by (h, w, row, col), stable in the
 * occurrence index.  Besides the reference outputs (unique coordinates,
 * category metadata, lookup) it returns the deterministic assembly plan:
 * the records of one unique block are contiguous, in occurrence order.
 * Synchronises `stream` once to read the category metadata.
 * Replaces `get_unique_coords` + `compress_unique_coords`
 * (coordinateCompressionKernel.pyx:92-144, 350-419).                       */
int32_t ys_pattern_build(const uint32_t* coords, const uint16_t* dims, uint32_t n_coords,
                         void* workspace, uint64_t workspace_bytes, ys_pattern_out* out,
                         void* stream);

/* ---- element evaluation (PKG/kernel/Hessian) ------------------------------ */

#define YS_MAX_UNION 8

/* A gathered 3-vector attribute: a union of up to 8 children (AoS xyz FP64). */
typedef struct ys_union3 {
  const double* child[YS_MAX_UNION];
  uint32_t prefix[YS_MAX_UNION + 1];
  uint32_t num_children;
} ys_union3;

/* Per-term DoF plan produced from the slot codes and the pattern. */
typedef struct ys_term_plan {
  const uint32_t* codes;        /* [n x K] slot codes                              */
  uint32_t K;                   /* slots per instance                              */
  uint32_t slot_stride;         /* slots per argument (1 plain, 2 union)           */
  const uint32_t* coord_outer;  /* [n+1] first occurrence of each instance          */
  const uint32_t* record;       /* pattern record offset of each occurrence (term slice) */
  const uint32_t* grad_outer;   /* [n+1] first target-argument occurrence           */
  const uint32_t* grad_record;  /* gradient record offset of each target argument    */
} ys_term_plan;

typedef struct ys_snh_args {
  ys_union3 position;           /* current positions (DATA)                         */
  ys_union3 rest;               /* rest positions (CONSTANT)                        */
  const uint32_t* tets;         /* [n x 4] union indices                            */
  uint32_t num_elements;
  const double* mu;             /* per element, or NULL to use mu_value             */
  const double* lam;            /* per element, or NULL to use lam_value            */
  double mu_value, lam_value, dt;
  int32_t projection_method;    /* -1/0 none, 1 |lambda|, 2 max(lambda, 0)          */
  ys_term_plan plan;
  double* block_records;        /* pattern records (FP64)                           */
  double* grad_records;         /* gradient records (FP64)                          */
  double* energy;               /* [n] per-element energy, or NULL                  */
  uint32_t* work_list;          /* [n] scratch: elements needing the eigen-projection */
  uint32_t* work_count;         /* [1] scratch counter                               */
} ys_snh_args;

/* Stable Neo-Hookean tetrahedra (examples/dropping_in_container_mixed/helpers.py:102-127):
 * gradient, Hessian, SPD projection of the full 12x12 local Hessian (the
 * inner projection of differentiator.pyx:794-799), merge of repeated
 * vertices and the scatter into pattern/gradient records
 * (hessianKernelNoProject.pyx:63-264).  Replaces the generated
 * `compute_hessian_and_gradient_with_compression` for this energy
 * (hessianKernelHost.pyx:27-161).                                          */
int32_t ys_snh_eval(const ys_snh_args* args, void* stream);
/* With block_records and grad_records NULL, ys_snh_eval, ys_inertia_eval and
 * ys_energy_eval write only the per-element energies to `energy` (the
 * reference's per-instance energy kernel, PKG/kernel/globalKernel.pyx:35-434,
 * used by minimizer.computeTotalEnergy, minimizer.pyx:396-407).           */

typedef struct ys_inertia_args {
  const double* position;       /* [n x 3] (DATA target primitive)                  */
  const double* x_before;       /* [n x 3] positions at the start of the step       */
  const double* velocity;       /* [n x 3] or NULL (zero)                           */
  const double* mass;           /* [n]                                              */
  double dt;
  double gravity[3];            /* x~ = x_before + v dt + gravity dt^2              */
  uint32_t num_vertices;
  ys_term_plan plan;
  double* block_records;
  double* grad_records;
  double* energy;               /* [n] or NULL                                      */
} ys_inertia_args;

/* Implicit-Euler inertia 1/2 (x - x~)^T m (x - x~) per vertex
 * (examples/dropping_in_container_mixed/helpers.py:138-141).               */
int32_t ys_inertia_eval(const ys_inertia_args* args, void* stream);

/* ---- vertex-tuple energies (cloth, contact, friction) --------------------
 * Energies over a JOIN of `arity` 3-DoF vertices (examples/
 * dropping_in_container_mixed/helpers.py, friction_helpers.py): gradient and
 * Hessian by second-order forward-mode differentiation of the formula, the
 * local Hessian projected like SNH (LDL^T PSD test, then |lambda| or
 * max(lambda, 0) of the negative modes), merged and scattered into records.
 * values[] by kind:
 *   barriers (PP/PE/PT/EE, helpers.py:143-199): dHat, kappa; d is the
 *     squared distance, E = kappa (d - dHat)^2 log^2(d / dHat);
 *   BENDING (helpers.py:213-234): bendStiff, dt; rest = x_init;
 *   BARAFF_WITKIN (helpers.py:272-292): stretchS, shearS, thickness, dt;
 *     rest = x_init;
 *   STVK_MEMBRANE: mu, lam, thickness, dt; rest = x_init, the Baraff-Witkin
 *     rest frame (no counterpart in the reference);
 *   FRICTION_PT / _PE / _EE / _PP (friction_helpers.py:12-66; :73-182,
 *     :188-276, :283-405, :411-500): fDhat, dt, frictionRate; rest =
 *     positions at the start of the step; params per element (stride >= 9):
 *     the lagged closest-point coordinates (beta1, beta2 / eta, 0 /
 *     gamma1, gamma2 / 0, 0), tangent0[3], tangent1[3], lambda_last_h.    */
#define YS_ENERGY_POINT_POINT 1
#define YS_ENERGY_POINT_EDGE 2
#define YS_ENERGY_POINT_TRIANGLE 3
#define YS_ENERGY_EDGE_EDGE 4
#define YS_ENERGY_BENDING 5
#define YS_ENERGY_BARAFF_WITKIN 6
#define YS_ENERGY_STVK_MEMBRANE 7
#define YS_ENERGY_FRICTION_PT 8
#define YS_ENERGY_FRICTION_PE 9
#define YS_ENERGY_FRICTION_EE 10
#define YS_ENERGY_FRICTION_PP 11

typedef struct ys_energy_args {
  int32_t kind;                 /* YS_ENERGY_*                                      */
  ys_union3 position;           /* current positions (DATA)                         */
  ys_union3 rest;               /* rest / initial / previous positions by kind      */
  const uint32_t* conn;         /* [n x arity] union indices                        */
  uint32_t arity;               /* 2 (PP), 3 (PE, membranes), 4 (PT, EE, bending) */
  uint32_t num_elements;
  const double* params;         /* [n x param_stride] per-element parameters or NULL */
  uint32_t param_stride;
  double values[8];             /* scalar parameters by kind (above)                */
  int32_t projection_method;    /* -1/0 none, 1 |lambda|, 2 max(lambda, 0)          */
  ys_term_plan plan;
  double* block_records;
  double* grad_records;
  double* energy;               /* [n] or NULL                                      */
} ys_energy_args;

/* Replaces the generated `compute_hessian_and_gradient_with_compression` of
 * these energies (hessianKernelHost.pyx:27-161).                           */
int32_t ys_energy_eval(const ys_energy_args* args, void* stream);

/* ---- rectangular second-order Jacobians (PKG/matrixAndVector/matrix/
 * secondOrderJacobian.pyx, PKG/kernel/Jacobian/secondOrderJacobianKernel*.pyx,
 * PKG/kernel/Coordinate/secondOrderJacobianIndicesKernel.pyx) -------------
 * d2E / (d rows d cols) of a scalar energy, rows and columns two target
 * lists.  The values of an instance come from its unprojected local Hessian
 * over the energy's arguments (the reference's no-project Jacobian kernel);
 * every argument carries a row code and a column code (ys_join_union_indices
 * run once with the row targets and once with the column targets).        */

/* Unprojected local Hessians, packed upper (3A(3A+1)/2 doubles an element,
 * row-major upper triangle), of the vertex-tuple energies (args->kind, the
 * position arguments; rest, lagged data and parameters as for
 * ys_energy_eval, the plan and record fields unused).                      */
int32_t ys_local_hessians(const ys_energy_args* args, double* out, void* stream);

/* Unprojected local Hessians over the positions and the rest positions of
 * the cloth energies (YS_ENERGY_BENDING, _BARAFF_WITKIN, _STVK_MEMBRANE):
 * arguments [x0 .. x(A-1), X0 .. X(A-1)], packed upper (6A)x(6A), the rest
 * quantities (rest frame, rest dihedral, rest edge length and area)
 * differentiated with the positions.  One hyper-dual evaluation of the
 * energy a vertex pair (3x3 block).  No counterpart kernel in the reference
 * (its differentiator forms these derivatives symbolically).              */
int32_t ys_rest_local_hessians(const ys_energy_args* args, double* out, void* stream);
/* Same for the SNH tetrahedra (12x12, 78 doubles an element).              */
int32_t ys_snh_local_hessians(const ys_snh_args* args, double* out, void* stream);
/* SNH over the positions and the rest positions of the tet, arguments
 * [x0..x3, X0..X3] (24x24 packed upper, 300 doubles an element): the x-x
 * block as ys_snh_local_hessians, the x-X block the derivative of the
 * position gradient in the rest positions (first-order dual numbers over
 * one rest vertex at a time), the X-X block the energy's second derivatives
 * in the rest positions (hyper-dual numbers over two rest vertices at a
 * time, 10 pairs a tet).                                                  */
int32_t ys_snh_rest_local_hessians(const ys_snh_args* args, double* out, void* stream);
/* Same for the inertia 1/2 m |x - x_before - dt v - dt^2 g|^2 per vertex
 * over its arguments (x, x_before) (args = 2) or (x, x_before, v) (args = 3):
 * m [[I, -I, -dt I], [-I, I, dt I], [-dt I, dt I, dt^2 I]] (helpers.py:
 * 138-141).  `mass` may be NULL (then mass_value for every vertex).        */
int32_t ys_inertia_local_hessians(const double* mass, double mass_value, double dt, uint32_t n,
                                  uint32_t args, double* out, void* stream);

/* Coordinates of the (row target, column target) pairs of every instance:
 * the distinct row codes >= 2 (first occurrence order) times the distinct
 * column codes >= 2, row-major, as scalar (row, col) pairs with dims (3, 3).
 * With coords NULL: coord_outer (n+1) = exclusive counts.  Otherwise
 * coords [2 m], dims [2 m] at the offsets of coord_outer.  Codes are
 * [n x K] with the argument a at column a * slot_stride, args <= 8.
 * Replaces count/generate_rectangular_coordinates
 * (secondOrderJacobianIndicesKernel.pyx:16-84).                            */
int32_t ys_rect_coordinates(const uint32_t* row_codes, const uint32_t* col_codes, uint32_t n, uint32_t K,
                            uint32_t slot_stride, uint32_t args, uint32_t* coord_outer, uint32_t* coords,
                            uint16_t* dims, void* stream);

/* Records (9 doubles, row-major) of every pair, in the order of
 * ys_rect_coordinates, at record[coord_outer[t] + k] (the assembly plan of
 * ys_pattern_build over those coordinates): the sum of the local Hessian's
 * argument blocks of the pair's row group and column group.  Sum them with
 * ys_assemble3.  difference_args = D > 0 (args = 2 D): the local Hessians
 * cover the first D arguments of an energy of x - x_old only (the lagged
 * friction kinds), arguments D .. 2D-1 are the step-start positions, and
 * their blocks are the first ones negated once per step-start side.
 * Replaces compute_second_order_jacobian_no_project
 * (secondOrderJacobianKernel.pyx:86-140).                                  */
int32_t ys_rect_records(const double* local_hessians, uint32_t args, uint32_t difference_args,
                        const uint32_t* row_codes, const uint32_t* col_codes, uint32_t n, uint32_t K,
                        uint32_t slot_stride, const uint32_t* coord_outer, const uint32_t* record, double* records,
                        void* stream);

/* Material-parameter columns (the reference's diff2(E, [position], [young])
 * of its material-optimization examples): the derivative of an element's
 * position gradient in one of its own scalar parameters, per argument,
 * [n x 3 args] doubles.  SNH: which 0 mu, 1 lambda (the per-tet Lame
 * arrays of ys_snh_args); inertia: the vertex mass over its 2 or 3
 * arguments (x, x_before[, v]).                                            */
int32_t ys_snh_param_jacobian(const ys_snh_args* args, uint32_t which, double* out, void* stream);
int32_t ys_inertia_mass_jacobian(const ys_inertia_args* args, uint32_t arguments, double* out, void* stream);
/* Coordinates and records of the parameter columns: one (3 x 1) pair per
 * distinct row code of element t and column param_start + t (coord_outer
 * alone when coords is NULL, as ys_rect_coordinates); records are the sums
 * of the pair's argument derivatives, 3 doubles at record[coord_outer[t] + k]. */
int32_t ys_rect_param_coordinates(const uint32_t* row_codes, uint32_t n, uint32_t K, uint32_t slot_stride,
                                  uint32_t args, uint32_t param_start, uint32_t* coord_outer, uint32_t* coords,
                                  uint16_t* dims, void* stream);
int32_t ys_rect_param_records(const double* derivatives, uint32_t args, const uint32_t* row_codes, uint32_t n,
                              uint32_t K, uint32_t slot_stride, const uint32_t* coord_outer, const uint32_t* record,
                              double* records, void* stream);

/* First-order Jacobian of the affine-body vertex positions x_i = A_b xbar_i
 * + t_b (firstOrderJacobian.pyx of the reference's diff1 on a vector
 * source): rows 3 i, a (3 x 9) block in the columns of A (row r holds xbar_i
 * at 3 r .. 3 r + 2) and a (3 x 3) identity in those of t, per vertex in
 * that order (a column start < 0 leaves that target out).  With record NULL
 * it writes the coordinates and dims of the n (or 2 n) occurrences; with
 * the assembly plan of ys_pattern_build over them, the records.           */
int32_t ys_affine_position_jacobian(const uint32_t* vertex_body, const double* xbar, uint32_t n,
                                    int64_t a_column_start, int64_t t_column_start, uint32_t* coords,
                                    uint16_t* dims, const uint32_t* record, double* records, void* stream);

/* Products with one category of the assembled rectangular matrix (unique
 * blocks of 3 rows and col_width = 1, 3 or 9 columns, sorted by (row, col),
 * scalar positions, 3 col_width values a block).  ys_rect_plan builds
 * row_ptr [block_rows + 1], col_ptr [block_cols + 1] (block_cols column
 * units of col_width) and col_order [num_blocks] (blocks by column, stable);
 * ys_rect_spmv computes y = J x (transpose 0, 3 block_rows outputs) or
 * y = J^T x (transpose 1, col_width block_cols outputs), each output summed
 * in block order, written (accumulate 0) or added (1).  Replaces matrix.spmv
 * of secondOrderJacobian (PKG/matrixAndVector/matrix/matrix.pyx).         */
int32_t ys_rect_plan_workspace_bytes(uint32_t num_blocks, uint64_t* bytes);
int32_t ys_rect_plan(const uint32_t* positions, uint32_t num_blocks, uint32_t block_rows, uint32_t block_cols,
                     uint32_t col_width, uint32_t* row_ptr, uint32_t* col_ptr, uint32_t* col_order, void* workspace,
                     uint64_t workspace_bytes, void* stream);
int32_t ys_rect_spmv(const double* values, const uint32_t* positions, const uint32_t* row_ptr,
                     const uint32_t* col_ptr, const uint32_t* col_order, uint32_t block_rows, uint32_t block_cols,
                     uint32_t col_width, const double* x, double* y, uint32_t transpose, uint32_t accumulate,
                     void* stream);

/* ---- affine (ABD) bodies ------------------------------------------------
 * A body carries a 3x3 affine matrix A (9 DoF, row-major, the reference's
 * `affine_matrices` attribute, examples/dropping_in_container_mixed/
 * dropping_in_container.py:241-245) and a translation t (3 DoF); its
 * vertices sit at x = A xbar + t (:261-270, xbar the body-frame rest
 * position).  The 9 DoF of A are stored as three 3-DoF rows, so every block
 * of the assembled matrix stays 3x3: an element's arguments are the rows
 * a0, a1, a2 of its body's A and t (K = 3 or 4 arguments of size 3, codes
 * from ys_join_union_indices over the rows-view [A rows (3 per body), t]).
 * Kinds:
 *   ORTHOGONALITY (helpers.py:201-211): stiffness * 1/2 |A^T A - I|_F^2 per
 *     body, 3 arguments;
 *   INERTIA (helpers.py:138-141 with x = A xbar + t, dropping_in_container.py:
 *     378): 1/2 m |x - x~|^2 per vertex, x~ = x_before + v dt +
 *     gravity dt^2, 4 arguments;
 *   SNH (helpers.py:129-136 on the tet positions xbar A^T + t,
 *     dropping_in_container.py:280-320, 370): Stable Neo-Hookean of one
 *     single-body tetrahedron, 4 arguments.
 * Gradients and Hessians by second-order forward-mode differentiation in
 * the (A, t) coordinates, local Hessian projected (PSD test, then the
 * negative modes) over the full 9x9 / 12x12, merged and scattered like
 * ys_energy_eval.  No counterpart of the split rows in the reference, whose
 * pattern keeps 9x9 / 9x3 blocks: the assembled matrix is the same.       */
#define YS_AFFINE_ORTHOGONALITY 1
#define YS_AFFINE_INERTIA 2
#define YS_AFFINE_SNH 3

typedef struct ys_affine_args {
  int32_t kind;                 /* YS_AFFINE_*                                      */
  const double* affine;         /* [num_bodies x 9] A per body, row-major           */
  const double* translation;    /* [num_bodies x 3] t per body (INERTIA, SNH)       */
  uint32_t num_bodies;
  uint32_t num_elements;
  const uint32_t* body;         /* [n] body of each element; NULL: element i is body i */
  const double* rest;           /* INERTIA: [n x 3] xbar per vertex;                */
                                /* SNH: [num_rest x 3] body-frame rest positions    */
  const uint32_t* tets;         /* SNH: [n x 4] indices into rest                   */
  uint32_t num_rest;
  const double* x_before;       /* INERTIA: [n x 3]                                 */
  const double* velocity;       /* INERTIA: [n x 3] or NULL (zero)                  */
  const double* mass;           /* INERTIA: [n]                                     */
  const double* mu;             /* SNH: per element, or NULL to use mu_value        */
  const double* lam;            /* SNH: per element, or NULL to use lam_value       */
  double mu_value, lam_value;
  double dt;                    /* INERTIA, SNH                                     */
  double gravity[3];            /* INERTIA                                          */
  double stiffness;             /* ORTHOGONALITY                                    */
  int32_t projection_method;    /* -1/0 none, 1 |lambda|, 2 max(lambda, 0)          */
  ys_term_plan plan;
  double* block_records;
  double* grad_records;
  double* energy;               /* [n] or NULL; records NULL: energies only         */
} ys_affine_args;

int32_t ys_affine_eval(const ys_affine_args* args, void* stream);

/* ---- contact through affine-body vertices --------------------------------
 * The PP / PE / PT / EE barriers and the four lagged friction kinds of
 * ys_energy_eval over a position union one child of which is the vertices of
 * affine bodies, whose position is the computed x = A_b xbar + t_b (the
 * collision union [soft, abd, container] of
 * examples/dropping_in_container_mixed/dropping_in_container.py:344, and
 * :270 for the position).  The map from the leaves (a free position, or the
 * A and t of a vertex's body) to the pair's vertex positions is linear, so
 * the reference projects the Hessian with respect to the vertex positions
 * (3V x 3V) and maps it to the leaves, J^T proj(H) J, merging repeated
 * leaves (one body's A and t seen from several vertices)
 * (PKG/differentiator/differentiator.pyx:795-799; the reference's test
 * expectation tests/differentiator/test_hessian_sparsity_permutation_gpu.py:269).
 *
 * Codes (ys_coupled_indices): K = 4 slots per vertex, slot stride 1; a plain
 * vertex fills its first slot (target position code, 1 for a non-target
 * leaf, 0 for a CONSTANT one) and pads the other three with code 0, size 0;
 * an affine vertex fills the four with the codes of its body's A rows
 * (wrt_start_A + 3 (3b + r) + 2) and t (wrt_start_t + 3b + 2).  Compression,
 * coordinates and the pattern then work unchanged (A as three 3-DoF rows).
 *
 * Evaluation (ys_coupled_energy_eval): the energy's value, gradient and
 * Hessian in the 3V vertex coordinates, the PSD test and negative-mode
 * projection of that Hessian, then the chain rule through the linear map
 * Jhat (vertex coordinates <- compressed leaves), written merged per leaf.
 * Friction kinds read base.rest (the old positions of the union's vertices,
 * same child layout) and base.params (9 lagged values per element).  An
 * element naming a vertex outside the union or a body beyond num_bodies sets
 * *status to its index + 1 (first one wins) and is skipped.              */
typedef struct ys_coupled_args {
  ys_energy_args base;          /* barrier or friction kind; base.position child `affine_child` unused */
  uint32_t affine_child;        /* union child of the affine-body vertices                   */
  const uint32_t* vertex_body;  /* [affine vertices] body of each                            */
  const double* rest;           /* [affine vertices x 3] body-frame rest position xbar      */
  const double* affine;         /* [num_bodies x 9] A per body, row-major                    */
  const double* translation;    /* [num_bodies x 3] t per body                               */
  uint32_t num_bodies;
  int32_t* status;              /* [1] or NULL: first element (+1) with an invalid vertex    */
} ys_coupled_args;

int32_t ys_coupled_indices(const uint32_t* connectivity, uint32_t n, uint32_t arity, uint32_t num_children,
                           const uint32_t* child_prefix, const int32_t* child_kind,
                           const uint32_t* child_wrt_start, uint32_t affine_child,
                           const uint32_t* vertex_body, uint32_t num_bodies, int32_t affine_kind,
                           uint32_t affine_wrt_start, int32_t translation_kind,
                           uint32_t translation_wrt_start, uint32_t* codes, uint16_t* sizes,
                           void* stream);

int32_t ys_coupled_energy_eval(const ys_coupled_args* args, void* stream);

/* Deterministic sum of n doubles into out[0] (device), fixed reduction order
 * for a given n; workspace: ys_sum_workspace_doubles() doubles.            */
uint64_t ys_sum_workspace_doubles(void);
int32_t ys_sum(const double* values, uint32_t n, double* out, double* workspace, void* stream);

/* ---- deterministic assembly --------------------------------------------- */

/* out[offset[u] + e] = sum_{c < count[u]} records[begin[u] + c*hw_u + e] for
 * e < hw_u, summed in occurrence order (no float atomics).  When out32 is
 * not NULL an FP32 copy of the sums is written as well.  `dims` gives (h, w)
 * per unique entry (the gradient uses (size, 1)).                          */
int32_t ys_assemble(const double* records, const uint32_t* begin, const uint32_t* count,
                    const uint32_t* offset, const uint16_t* dims, uint32_t nu,
                    double* out, float* out32, void* stream);

/* Per-variable diagonal blocks and scalar diagonal from assembled block sets.
 * Variable v of attribute a (count_a instances of size s_a) has scalar
 * offset seg_start[a] + i*s_a and diagonal block at diag_start[a] + i*s_a^2.
 * Stored blocks smaller than s_a inside one variable (the 3x3 row blocks of
 * an affine matrix) are placed at their offsets, off-diagonal ones mirrored.
 * Adds (accumulate != 0) or writes.  Replaces the diagonal / diagonal-block
 * accumulation of hessianKernelFullProject.pyx:186-212.                    */
int32_t ys_extract_diagonal(const double* values, const uint32_t* positions,
                            const uint16_t* block_dims, const uint32_t* value_offset, uint32_t nu,
                            uint32_t num_attributes, const uint32_t* seg_start /*host*/,
                            const uint32_t* attr_size /*host*/, const uint32_t* diag_start /*host*/,
                            double* diag_blocks, double* diagonal, int32_t accumulate, void* stream);

/* Block pseudo-inverse of the diagonal blocks, |lambda| -> |1/lambda|
 * (|lambda| < 1e-6 -> |lambda|).  Replaces `invert_diagonal_blocks`
 * (PKG/kernel/Solver/diagonalBlockInverseKernel.pyx:123-176).              */
int32_t ys_invert_diagonal_blocks(const double* diag_blocks, double* inverse, uint32_t num_attributes,
                                  const uint32_t* diag_start /*host*/, const uint32_t* count /*host*/,
                                  const uint32_t* attr_size /*host*/, void* stream);

/* ---- symmetric block SpMV ------------------------------------------------ */

/* Row plan of symmetric upper block storage over 3-DoF variables: for
 * variable i, the stored blocks with row i (direct) and col i (transposed).
 * entries: [2*nu] capacity; row_ptr: [num_vars+1].  Requires all blocks 3x3
 * and positions on 3-aligned scalar offsets.                               */
int32_t ys_spmv_plan_build(const uint32_t* positions, uint32_t nu, uint32_t num_vars,
                           void* workspace, uint64_t workspace_bytes, uint32_t* row_ptr,
                           uint32_t* entry_block, uint32_t* entry_col, void* stream);
int32_t ys_spmv_plan_workspace_bytes(uint32_t nu, uint32_t num_vars, uint64_t* bytes);

/* y = H x (beta == 0) or y += H x (beta == 1) for a 3x3 symmetric upper
 * block set with FP64 (values, 9 doubles a block) or FP32 (values32, 12-float
 * 16-byte aligned slots, see ys_assemble3) blocks, one of which is NULL.  Deterministic (row-gather, fixed order).  Replaces `spmv_blocks`
 * (PKG/matrixAndVector/matrix/matrix.pyx:21-86) and `spmvOffDiagonalBlocks`
 * (PKG/kernel/Solver/solverKernel.pyx:156-215).                            */
int32_t ys_spmv3(const double* values, const float* values32, const uint32_t* row_ptr,
                 const uint32_t* entry_block, const uint32_t* entry_col, uint32_t num_vars,
                 const double* x, double* y, int32_t beta, void* stream);

/* FP32 copy of a 3-vector per variable in 16-byte slots (x, y, z, 0):
 * x32[4 i + k] = (float)x[3 i + k].  x32 16-byte aligned.  The FP32 PCG keeps
 * its search direction in this form next to the FP64 one.               */
int32_t ys_pack_x32(const double* x, uint32_t num_vars, float* x32, void* stream);

/* ys_spmv3 with FP32 blocks reading x from its ys_pack_x32 copy (one 16-byte
 * load per neighbour instead of three 8-byte ones); the same products as
 * ys_spmv3 with values32 and the FP64 x.  The SpMV of the FP32 PCG loop. */
int32_t ys_spmv3_x32(const float* values32, const uint32_t* row_ptr, const uint32_t* entry_block,
                     const uint32_t* entry_col, uint32_t num_vars, const float* x32, double* y,
                     int32_t beta, void* stream);

/* Tile plan of a 3x3 block set for the tiled SpMV: rows in tiles of
 * YS_SPMV_TILE_ROWS, row_block[i] = first stored block of row i (the blocks
 * are (row, col)-sorted, so a tile's blocks are one contiguous range),
 * *tile_cap_host = the most blocks in one tile and *entry_cap_host = the
 * most row-plan entries in one tile's 16-byte aligned entry range (a
 * multiple of 4).  row_block has num_vars + 4 entries (the last three are
 * scratch here).  Synchronises `stream` (set-up, once per pattern).
 * YS_ERR_INVALID when the blocks are not (row, col)-sorted or do not match
 * the row plan.  No counterpart in the reference.                         */
#define YS_SPMV_TILE_ROWS 64
int32_t ys_spmv_tile_plan(const uint32_t* positions, uint32_t nu, const uint32_t* row_ptr,
                          const uint32_t* entry_block, uint32_t num_vars, uint32_t* row_block,
                          uint32_t* tile_cap_host, uint32_t* entry_cap_host, void* stream);

/* ys_spmv3_x32 by tiles: persistent CTAs stage each tile's contiguous run of
 * FP32 block slots, its row-plan entries and its row pointers into shared
 * memory with bulk copies (cp.async.bulk, mbarrier completion, a ring of
 * `stages` buffers, 2..4, 0 = as many as let two CTAs share an SM), so
 * every stored block crosses HBM once per product;
 * direct blocks and the transposed blocks of rows in the tile are read from
 * shared memory, the transposed blocks of earlier tiles from global memory.
 * Bit-identical to ys_spmv3_x32.  Padding: row_ptr and row_block hold
 * num_vars + 4 entries, entry_block and entry_col (row_ptr[num_vars] + 3)
 * & ~3 (the copies move whole 16-byte words).  `stage_status` (device word
 * or NULL) is OR-ed with 1 when a CTA's wait for a copy ran out (it then
 * reads global memory: the result is the same).  Replaces the reference's
 * `yasps_mas_specialized_fine_block_spmv`
 * (PKG/solver/mas/cuda/block_spmv.cu:279-398).                            */
int32_t ys_spmv3_x32_tiled(const float* values32, const uint32_t* row_ptr,
                           const uint32_t* entry_block, const uint32_t* entry_col,
                           const uint32_t* row_block, uint32_t tile_cap, uint32_t entry_cap,
                           uint32_t stages, uint32_t num_vars, const float* x32, double* y,
                           int32_t beta, uint32_t* stage_status, void* stream);

/* Streamed-tile plan of a 3x3 block set (ys_spmv_stream_plan): tiles of
 * YS_SPMV_TILE_ROWS rows, each with one contiguous run of packed FP32
 * blocks (its own stored blocks, then the blocks of earlier tiles that its
 * rows use transposed), one run of entry words and its distinct neighbour
 * variables.  block_cap == 0: no plan.  No counterpart in the reference.  */
typedef struct ys_spmv_stream {
  const float* blocks32;         /* 9 floats a slot, ys_spmv_stream_words slots (ys_spmv_stream_fill) */
  const uint32_t* desc;          /* 4 words a tile (+ 4 scratch): base, blocks, entries, columns      */
  const uint32_t* rows;          /* 68 words a tile: row offsets into the entry words, column count  */
  const uint32_t* words;         /* entry words: column index | block slot << 16 | transposed << 31  */
  const uint32_t* halo;          /* distinct neighbour variables of each tile, ascending             */
  uint32_t block_cap;            /* most blocks, entries, distinct columns of a tile (multiples of 4) */
  uint32_t entry_cap;
  uint32_t halo_cap;
} ys_spmv_stream;

/* Slots (and words) each array of a streamed-tile plan needs: num_entries
 * = row_ptr[num_vars] of the row plan.  No counterpart in the reference.  */
int32_t ys_spmv_stream_words(uint32_t num_entries, uint32_t num_vars, uint64_t* words);

/* Builds the streamed-tile plan of a 3x3 block set from its row plan and
 * ys_spmv_tile_plan's row_block: desc [4 * (tiles + 1)] words, rows
 * [68 * tiles], words / halo / src [capacity_words] (>= ys_spmv_stream_words),
 * all 16-byte aligned; src[s] = the stored block of stream slot s (or
 * 0xffffffff); slot_of [2 * num_blocks] (8-byte aligned) = each stored
 * block's slot in its row's tile and its cross slot in a later tile (or
 * 0xffffffff).  caps_host[3] = block_cap, entry_cap, halo_cap.  Synchronises
 * `stream` (set-up, once per pattern).  YS_ERR_CAPACITY when a tile has more
 * than 4096 entries, 512 distinct columns or 32768 stream slots (the tiled
 * SpMV then stays the product of the FP32 loop); YS_ERR_INVALID when the
 * blocks are not (row, col)-sorted along the row plan.  No counterpart in
 * the reference.                                                          */
int32_t ys_spmv_stream_plan(const uint32_t* row_ptr, const uint32_t* entry_block,
                            const uint32_t* entry_col, const uint32_t* row_block, uint32_t num_vars,
                            uint64_t capacity_words, uint32_t* desc, uint32_t* rows, uint32_t* words,
                            uint32_t* halo, uint32_t* src, uint32_t num_blocks, uint32_t* slot_of,
                            uint32_t* caps_host, void* stream);

/* ys_assemble3 that also writes every block's FP32 values into the streamed
 * plan's packed blocks (blocks32 of ys_spmv_stream_fill) at its own slot
 * slot_of[2 b] and, when a later tile uses it transposed, at slot_of[2 b + 1]:
 * the fill after the assembly is then not needed.  No counterpart in the
 * reference.                                                              */
int32_t ys_assemble3_streamed(const double* records, const uint32_t* begin, const uint32_t* count,
                              const uint32_t* offset, uint32_t nu, double* out, float* out32,
                              const uint32_t* slot_of, float* blocks32, void* stream);

/* blocks32[9 s + k] = values32[12 src[s] + k] for every slot s < slots with
 * a block (zeros elsewhere): the streamed plan's packed FP32 blocks, current
 * after each update of values32.  slots = ys_spmv_stream_words (a multiple
 * of 4); src and blocks32 16-byte aligned.  No counterpart in the
 * reference.                                                              */
int32_t ys_spmv_stream_fill(const float* values32, const uint32_t* src, uint64_t slots, float* blocks32,
                            void* stream);

/* ys_spmv3_x32 over a streamed-tile plan: persistent CTAs stage each tile's
 * packed blocks, entry words, distinct columns and row offsets into shared
 * memory with bulk copies (cp.async.bulk, mbarrier completion, a ring of
 * `stages` buffers: 2 or 3, 0 = three when three CTAs still share an SM,
 * else two) and gather the tile's distinct neighbour vectors once
 * (cp.async), so every block read is a streamed HBM read and no neighbour is
 * fetched twice by a tile.  Bit-identical to ys_spmv3_x32.  The row plan
 * (values32, row_ptr, entry_block, entry_col) is read instead by a CTA whose
 * copy wait ran out (`stage_status` OR-ed with 1; the result is the same).
 * max_ctas > 0 caps the grid (tests: several tiles a CTA).  Replaces the
 * reference's `yasps_mas_specialized_fine_block_spmv`
 * (PKG/solver/mas/cuda/block_spmv.cu:279-398).                            */
int32_t ys_spmv3_x32_streamed(const ys_spmv_stream* plan, const float* values32, const uint32_t* row_ptr,
                              const uint32_t* entry_block, const uint32_t* entry_col, uint32_t num_vars,
                              const float* x32, double* y, int32_t beta, uint32_t stages,
                              uint32_t max_ctas, uint32_t* stage_status, void* stream);

/* ---- preconditioned CG ----------------------------------------------------- */

#define YS_PREC_BLOCK_JACOBI 0
#define YS_PREC_MAS 1

#define YS_STOP_PRECONDITIONED 0   /* r^T M^-1 r <= tol * r0^T M^-1 r0 (reference rule) */
#define YS_STOP_RESIDUAL 1         /* ||r||_2 <= tol * ||rhs||_2                        */

typedef struct ys_matrix3 {
  /* up to two 3x3 block sets (static + dynamic), each with an SpMV row plan */
  uint32_t num_sets;
  const double* values[2];
  const float* values32[2];      /* 12-float block slots (ys_assemble3)           */
  const uint32_t* row_ptr[2];
  const uint32_t* entry_block[2];
  const uint32_t* entry_col[2];
  uint32_t num_vars;             /* 3-DoF variables; n = 3 * num_vars             */
  /* optional tile plan of each set (ys_spmv_tile_plan); tile_cap 0: none.
   * With one set, FP32 blocks and a tile plan the PCG loop runs the tiled
   * SpMV (ys_spmv3_x32_tiled; its padding rules apply).                   */
  const uint32_t* row_block[2];
  uint32_t tile_cap[2];
  uint32_t entry_cap[2];
  /* optional streamed-tile plan of each set (ys_spmv_stream_plan, blocks
   * current with values32); with one set and FP32 blocks the PCG loop runs
   * ys_spmv3_x32_streamed in preference to the tiled SpMV.               */
  ys_spmv_stream stream[2];
} ys_matrix3;

typedef struct ys_pcg_args {
  ys_matrix3 matrix;
  int32_t precision;            /* 0: FP64 blocks, 1: FP32 blocks (values32)      */
  int32_t preconditioner;       /* YS_PREC_*                                      */
  const double* jacobi_inverse; /* [num_vars * 9] block-Jacobi inverse            */
  void* mas;                    /* ys_mas handle for YS_PREC_MAS                  */
  int32_t stop_rule;            /* YS_STOP_*                                      */
  double tolerance;
  uint32_t max_iterations;
  const double* rhs;            /* [n]                                            */
  double* solution;             /* [n] in: initial guess unless zero_initial_guess */
  int32_t zero_initial_guess;
  double* workspace;            /* ys_pcg_workspace_doubles(n) doubles             */
  /* Block-Jacobi with targets wider than 3 (a 9-DoF affine matrix is three
   * 3-DoF variables whose 9x9 diagonal block is inverted whole,
   * diagonalBlockInverseKernel.pyx:40-215): jacobi_group[i] = first variable
   * of i's group | (group size << 30), group size 1 or 3, and
   * jacobi_inverse holds per variable the 3 x 9 row strip of its group's
   * inverse (27 doubles, row-major, columns of the group's variables in
   * order).  NULL: every group is one variable and jacobi_inverse holds 3x3
   * blocks (9 doubles a variable).                                         */
  const uint32_t* jacobi_group;
} ys_pcg_args;

/* With YS_PREC_MAS a finite non-positive curvature p^T H p (rounding on an
 * ill-conditioned SPD system) takes a zero step and restarts the direction
 * from M^-1 r, as the reference's MAS PCG does (mas/cuda/pcg.cu:183-189);
 * block-Jacobi ends the solve with -(it+4) as solverKernel.pyx:388-404. */
typedef struct ys_pcg_result {
  int32_t status;        /* reference convention: >=0 iterations (0: converged at start), <0 error */
  uint32_t iterations;
  double delta0, delta;  /* preconditioned r^T z at start / end                   */
  double residual0, residual;  /* recursive ||r||_2 at start / end                  */
} ys_pcg_result;

uint64_t ys_pcg_workspace_doubles(uint32_t n);

/* ---- multilevel additive Schwarz (PKG/solver/mas) -------------------------- */

/* Static description of a MAS hierarchy over 3-DoF variables, produced on
 * the host once per static structure (mas/hierarchy.py:150-271).  Packed
 * node space: level l owns nodes [level_node_offset[l], level_node_offset[l+1]),
 * level 0 being the fine variables.  All pointers are device arrays unless
 * marked host; the handle keeps the pointers (the caller keeps them alive). */
typedef struct ys_mas_desc {
  uint32_t num_fine_vars;
  uint32_t num_levels;                 /* 1..8                                        */
  const uint32_t* level_node_offset;   /* host [num_levels+1]                         */
  const double* level_weights;         /* host [num_levels] (mas/preconditioner.py:32-36) */
  const uint32_t* cmap;                /* [num_levels * num_fine_vars] packed node of each fine var */
  const uint32_t* child_ptr;           /* [coarse nodes + 1] children of every coarse node:  */
  const uint32_t* child_fine;          /* packed ids of its nodes on the level below          */
  uint32_t num_domains;
  const uint32_t* dom_node_ptr;        /* [num_domains+1]                             */
  const uint32_t* dom_nodes;           /* packed node ids, local order                 */
  const uint64_t* inv_offset;          /* [num_domains] float offset of each inverse,  */
                                       /* a multiple of 4; ys_mas_inverse_floats(3 * */
                                       /* domain nodes) floats each                    */
  const uint32_t* dom_entry_ptr;       /* [num_domains+1]                             */
  const uint32_t* dom_entry;           /* [3 * entries] (local i, local j, level block) */
  uint32_t fine_blocks;                /* level-0 blocks = the static 3x3 upper blocks */
  uint32_t coarse_blocks;
  const uint32_t* cb_src_ptr;          /* [coarse_blocks+1]                           */
  const uint32_t* cb_src;              /* block index | mode << 30 (0 B, 1 B^T, 2 B+B^T) */
  const uint32_t* cb_level_begin;      /* host [num_levels+1] coarse block ranges       */
  uint32_t max_domain_dofs;            /* <= 128                                      */
  double* coarse_values;               /* [coarse_blocks * 9] scratch                  */
  float* inverse;                      /* FP32 domain inverses (4x4 tile layout below) */
  float* level_residual;               /* [3 * packed nodes] scratch                   */
  float* level_correction;             /* [3 * packed nodes] scratch                   */
  int32_t* status;                     /* [1] scratch                                  */
  double* level_residual64;            /* [3 * packed nodes] scratch (FP64 restriction) */
} ys_mas_desc;

/* Floats of one domain's FP32 inverse: the n x n inverse padded to 4T rows
 * (T = ceil(n/4) rounded up to even; zero padding) stored as its upper 4x4
 * tiles (A <= B, diagonal tiles in full), 16 floats a tile, row-major in the
 * tile; tile (A, B) at slot A (T+1) + B - A for A < T/2, else at
 * q (T+1) + T - q + B - A with q = T-1-A (the triangle folded into a
 * T/2 x (T+1) rectangle).  Equals 8 T (T+1).  Host function.             */
uint64_t ys_mas_inverse_floats(uint32_t dofs);

int32_t ys_mas_create(const ys_mas_desc* desc, void** handle);
/* Level Galerkin sums and FP64 Gauss-Jordan inverses of every domain from
 * the assembled FP64 fine blocks (mas/numeric_assembly.py:64-83,
 * mas/cuda/local_inverse.cu:190-545).  When failed_domains is not NULL the
 * call synchronises and reports singular domains (YS_ERR_SINGULAR_DOMAIN). */
int32_t ys_mas_numeric_update(void* handle, const double* fine_values, void* stream, int32_t* failed_domains);
/* FP64 values of the union of two 3x3 block sets on their union pattern
 * (the MAS fine level of a Hessian with a dynamic contact set): block u is
 * a[9 a_index[u] ..] + b[9 b_index[u] ..], a negative index meaning no block
 * of that set; pass the result to ys_mas_numeric_update of a handle whose
 * fine blocks are the union pattern.  The reference adds the dynamic blocks
 * into the domain matrices of every level
 * (PKG/solver/mas/cuda/dynamic_assembly_specialized.cu:81-112,
 * mas/numeric_assembly.py:64-83 over "both" block sets).                    */
int32_t ys_mas_union_values(const double* a, const int32_t* a_index, const double* b, const int32_t* b_index,
                            uint32_t num_blocks, double* out, void* stream);
/* Singular domains of the last ys_mas_numeric_update on `stream` (which may
 * have been called without failed_domains, so the check can wait for a
 * later synchronisation); synchronises the stream; YS_ERR_SINGULAR_DOMAIN
 * when any.                                                              */
int32_t ys_mas_failed_domains(void* handle, void* stream, int32_t* failed_domains);
/* z = M^-1 r (mas/preconditioner.py:128-154). */
int32_t ys_mas_apply(void* handle, const double* r, double* z, void* stream);
int32_t ys_mas_destroy(void* handle);
/* The domain-GEMV stage of ys_mas_apply alone, on the level residuals of the
 * last apply (used to time the preconditioner's dominant kernel).  When
 * algorithmic_bytes is not NULL it receives the bytes one launch must move
 * (the n(n+1)/2 distinct FP32 entries of every inverse + gathered residuals,
 * node ids and corrections); that query synchronises.                     */
int32_t ys_mas_gemv(void* handle, void* stream, uint64_t* algorithmic_bytes);

/* ---- extras -------------------------------------------------------------- */

/* Gradient occurrences: one (dof, dof) coordinate with dims (size, 1) per
 * target slot (repeated slots included); grad_outer[n+1] prefix counts. */
int32_t ys_gradient_coordinates(const uint32_t* codes, const uint16_t* sizes, uint32_t n, uint32_t K,
                                uint32_t* grad_outer, uint32_t* coords, uint16_t* dims, void* stream);
/* ys_assemble specialised for 3x3 blocks.  out32 (when not NULL) receives
 * the FP32 copy in 16-byte aligned slots of 12 floats per block (block u at
 * out32 + 12 u, the last 3 floats unused): the layout ys_spmv3, the tiled
 * SpMV and the PCG read FP32 blocks in.                                   */
int32_t ys_assemble3(const double* records, const uint32_t* begin, const uint32_t* count, const uint32_t* offset,
                     uint32_t nu, double* out, float* out32, void* stream);
/* ys_assemble with out offset offset[u * offset_stride] (the gradient passes
 * the pattern positions with stride 2). */
int32_t ys_assemble_strided(const double* records, const uint32_t* begin, const uint32_t* count,
                            const uint32_t* offset, uint32_t offset_stride, const uint16_t* dims, uint32_t nu,
                            double* out, void* stream);
/* FP64 iterative-refinement residual: x += delta (when delta is not NULL),
 * r = rhs - H x with the FP64 blocks of `m`, and ||r||^2, ||rhs||^2 (host
 * norms_host[0..1] when not NULL, synchronising `stream`).  x NULL stands
 * for the zero vector (r = rhs, no product; delta must then be NULL).  workspace holds
 * ys_refine_workspace_doubles(num_vars) doubles.  The FP64 audit of the
 * reference's mixed_spmv mode (PKG/solver/mas/solver.py:643-688).           */
uint64_t ys_refine_workspace_doubles(uint32_t num_vars);
int32_t ys_refine_residual(const ys_matrix3* m, const double* rhs, double* x, const double* delta, double* r,
                           double* workspace, double* norms_host, void* stream);
/* Change the tolerance / iteration budget of an existing solver (the graph
 * reads them from device memory, so no rebuild). */
int32_t ys_pcg_set_params(void* handle, double tolerance, uint32_t max_iterations);
/* Polls a block of the MAS loop makes at its grid barrier (the cooperative
 * collect + direction kernel) before it gives up; default 2^24.  A block that
 * gives up marks the solve void and ys_pcg_status returns YS_ERR_CUDA; the
 * loop then ends at its iteration budget.  The waiting grid is co-resident,
 * so the default bound is never reached in a healthy run; a small bound
 * exercises the failure path without hanging the device.  Applies from the
 * next launch.  No counterpart in the reference (its loop has no grid-wide
 * wait).                                                                    */
int32_t ys_pcg_set_barrier_poll_limit(void* handle, uint32_t polls);
/* Asynchronous halves of ys_pcg_run. */
int32_t ys_pcg_launch(void* handle, void* stream);
int32_t ys_pcg_status(void* handle, void* stream, ys_pcg_result* result);

/* Opaque solver: owns the CUDA graph of one PCG configuration (the loop runs
 * on the device behind a conditional while node; one device->host read of
 * the status per solve).  Replaces `computeSolution`
 * (PKG/kernel/Solver/solverKernel.pyx:547-687, block-Jacobi) and the MAS
 * PCG runtime (PKG/solver/mas/cuda_runtime.py:3549-3751, mas/cuda/pcg.cu). */
int32_t ys_pcg_create(const ys_pcg_args* args, void** handle);
int32_t ys_pcg_run(void* handle, void* stream, ys_pcg_result* result);
int32_t ys_pcg_destroy(void* handle);

/* ---- serving form: batched MAS-PCG over resident solves ------------------
 * Many Newton-step solves ("slots") advance together: one launch runs
 * `passes_per_launch` pipeline passes over every attached slot, each pass a
 * PCG iteration of every live slot (FP32 blocks and MAS inside, FP64
 * vectors, dots and refinement residuals; the precision form of masSolver
 * with mixed_spmv).  Converged slots retire on the device; the host attaches
 * new slots between launches.  A slot's arithmetic does not depend on the
 * other slots in the launch, so its result is bit-identical alone and in a
 * mix.  The reference has no serving form (its MAS PCG solves one system,
 * PKG/solver/mas/cuda_runtime.py:3549-3751).                              */
#define YS_SERVE_EMPTY 0   /* no solve attached                               */
#define YS_SERVE_INIT 1    /* attached, not started                           */
#define YS_SERVE_REFINE 2  /* FP64 residual of x in the next pass             */
#define YS_SERVE_START 3   /* inner PCG restart in this pass                  */
#define YS_SERVE_ITER 4    /* inner PCG iterating                             */
#define YS_SERVE_DONE 5    /* ||g - H x|| <= tolerance ||g|| (FP64 blocks)     */
#define YS_SERVE_FAILED 6  /* non-SPD curvature / preconditioner, or budget   */

typedef struct ys_serve_slot_desc {
  void* mas;                   /* ys_mas handle of this solve, numeric update done */
  ys_matrix3 matrix;           /* one 3x3 block set: values (FP64) + values32 (FP32) */
  const double* rhs;           /* g [3 * num_vars]                                   */
  double* solution;            /* x [3 * num_vars] (written)                         */
  double* workspace;           /* ys_serve_workspace_doubles(num_vars), 16-B aligned */
  double tolerance;            /* target true relative residual                      */
  double refinement_tolerance; /* lower bound of every inner relative tolerance      */
  uint32_t max_iterations;     /* inner iterations over all refinements              */
} ys_serve_slot_desc;

typedef struct ys_serve_slot_status {
  int32_t phase;               /* YS_SERVE_*                                         */
  uint32_t iterations;         /* inner PCG iterations so far                        */
  uint32_t refinements;        /* FP64 residual evaluations after the first          */
  double relative_residual;    /* ||g - H x|| / ||g|| at the last FP64 evaluation     */
} ys_serve_slot_status;

uint64_t ys_serve_workspace_doubles(uint32_t num_vars);
/* max_slots <= 256; passes_per_launch <= 64. */
int32_t ys_serve_create(uint32_t max_slots, uint32_t passes_per_launch, void** handle);
/* Attach a solve to a free slot (takes effect at the next launch). */
int32_t ys_serve_attach(void* handle, uint32_t slot, const ys_serve_slot_desc* desc);
/* Detach a slot (its buffers are no longer read after the next launch). */
int32_t ys_serve_detach(void* handle, uint32_t slot);
/* Run passes_per_launch passes over the attached slots on `stream`
 * (asynchronous; one CUDA graph per size bucket of the CTA tables). */
int32_t ys_serve_launch(void* handle, void* stream);
/* Synchronise `stream` and report every slot: out[max_slots]. */
int32_t ys_serve_status(void* handle, void* stream, ys_serve_slot_status* out);
int32_t ys_serve_destroy(void* handle);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* YS_NEWTON_H */
