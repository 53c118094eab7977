/*
 * rbffd_sm100.h -- C ABI of librbffd_sm100.so, the B200 (sm_100a) RBF-FD hot path.
 *
 * The path: per-stencil RBF-FD weights (batched FP64 solves of the
 * RBF + polynomial saddle-point systems), ELL application of derivative and
 * hyperviscosity operators (applyWeightsForDeriv), and the classical RK4
 * update with the PDE right-hand side fused into each stage.
 *
 * Every entry point returns an int status (RBFFD_OK = 0, negative on error),
 * never exits and never traps; the message of the last failure on a context
 * is available from rbffd_ctx_last_error().  Host pointers are plain C arrays;
 * device pointers appear only in the *_dev variants and are typed void*.
 * Handles are not reentrant: one host thread per handle at a time.
 *
 * Layout conventions: node coordinates xyz are [N][3] doubles (unit sphere);
 * stencils are [N][n_pad] int32 row-major, row i listing the st_len[i] node
 * indices of stencil i with the centre i first (the reference's StencilType,
 * src/common_typedefs.h:16; centre check rbffd.cpp:916-928); weights on the
 * host are [N][n_pad] doubles in the same order; solution vectors with T
 * tracers are [N][T] (tracer fastest).
 */
#ifndef RBFFD_SM100_H
#define RBFFD_SM100_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum rbffd_status {
    RBFFD_OK = 0,
    RBFFD_ERR_INVALID = -1,     /* bad argument, size or handle */
    RBFFD_ERR_OOM = -2,         /* device or host allocation failed */
    RBFFD_ERR_CUDA = -3,        /* CUDA runtime error (message in last_error) */
    RBFFD_ERR_TIMEOUT = -4,     /* a bounded wait expired */
    RBFFD_ERR_UNSUPPORTED = -5, /* combination not implemented */
    RBFFD_ERR_STATE = -6,       /* call out of order (e.g. weights missing) */
    RBFFD_ERR_SINGULAR = -7,    /* a stencil system had an exactly zero pivot */
    RBFFD_ERR_BUDGET = -8,      /* admission refused: over the HBM budget */
    RBFFD_ERR_NO_DEVICE = -9,   /* no CUDA device / driver */
    RBFFD_ERR_CANCELLED = -10   /* serving: the request was cancelled */
};

/* Arithmetic type of a kernel path. */
enum rbffd_dtype { RBFFD_F32 = 0, RBFFD_F64 = 1 };

/* Derivative operator flags; identical values to RBFFD::DerType
 * (src/rbffd/rbffd.h:43-60). */
enum rbffd_der_type {
    RBFFD_X = 0x1, RBFFD_Y = 0x2, RBFFD_Z = 0x4, RBFFD_LAPL = 0x8, RBFFD_R = 0x10, RBFFD_HV = 0x20,
    RBFFD_LAMBDA = 0x40, RBFFD_THETA = 0x80, RBFFD_LSFC = 0x100, RBFFD_XSFC = 0x200, RBFFD_YSFC = 0x400,
    RBFFD_ZSFC = 0x800, RBFFD_ALT_XSFC = 0x1000, RBFFD_ALT_YSFC = 0x2000, RBFFD_ALT_ZSFC = 0x4000,
    RBFFD_INTERP = 0x8000
};

typedef struct rbffd_ctx rbffd_ctx;
typedef struct rbffd_grid rbffd_grid;
typedef struct rbffd_pde rbffd_pde;

/* ---- library / context ------------------------------------------------ */
const char* rbffd_version(void);
const char* rbffd_status_string(int status);
int rbffd_device_count(int* count);

/* One context per device; owns a CUDA stream and all device memory of the
 * grids and PDEs created from it.  Replaces the OpenCL context/queue the
 * reference GPU classes set up (src/utils/opencl/cl_base_class.cpp:16-66). */
int rbffd_ctx_create(int device, rbffd_ctx** out);
int rbffd_ctx_destroy(rbffd_ctx* ctx);
const char* rbffd_ctx_last_error(const rbffd_ctx* ctx);
int rbffd_ctx_synchronize(rbffd_ctx* ctx);
/* Bytes this context holds on the device, and the device's free/total bytes. */
int rbffd_ctx_mem_info(rbffd_ctx* ctx, size_t* held, size_t* free_bytes, size_t* total_bytes);
/* The context's CUDA stream (cudaStream_t), for callers that order their own work after ours. */
int rbffd_ctx_stream(rbffd_ctx* ctx, void** stream);
/* FP64 arithmetic of the derivative application and time stepping.
 *   RBFFD_ARITH_FUSED (default): every multiply-add of the SpMV, the
 *     right-hand side and the RK4 update is one fused multiply-add;
 *   RBFFD_ARITH_UNFUSED: every such multiply-add is a rounded product, then a
 *     rounded sum, in the reference's source order -- the arithmetic of the
 *     reference's RBFFD::applyWeightsForDeriv (rbffd.cpp:669-688),
 *     CosineBell::solve (cosine_bell.cpp:47-57), VortexRollup::solve and
 *     TimeDependentPDE::advanceRungeKutta4 (time_dependent_pde.cpp:172-304) as
 *     the reference's own build compiles them (g++ -O3 for x86-64, which has no
 *     FMA instruction): with it the device's FP64 results equal that build's
 *     bit for bit.  One lane per stencil row, gathers from global memory.
 * The context's setting applies to FP64 rbffd_apply / rbffd_apply_dev calls
 * and to FP64 one-tracer PDEs created after it; rbffd_pde_set_arithmetic sets
 * one PDE's (FP64, one tracer).  FP32 paths are unaffected. */
enum { RBFFD_ARITH_FUSED = 0, RBFFD_ARITH_UNFUSED = 1 };
int rbffd_ctx_set_arithmetic(rbffd_ctx* ctx, int arith);
int rbffd_ctx_get_arithmetic(rbffd_ctx* ctx, int* arith);

/* ---- host-side inputs (no GPU) ----------------------------------------- */
/* N Fibonacci-spiral points on the unit sphere under a seeded uniform random
 * rotation; xyz[N][3].  Stands in for the reference's node files. */
int rbffd_nodes_fibonacci(int N, uint64_t seed, double* xyz);
/* n nearest neighbours of every node, closest first, centre at [0]:
 * Grid::generateStencilsKDTree (src/grids/grid_interface.cpp:688-725) with the
 * k-d tree of external/kdtree/KDTree.h:407-433.  st[N][n].  *ties (optional)
 * receives the number of stencils whose distance list had an exact tie. */
int rbffd_stencils_knn(const double* xyz, int N, int n, int* st, int* ties, int nthreads);
/* Grid::generateStencils(st_generator_t) (src/grids/grid_interface.cpp:514-536)
 * for the reference's default generator and its k-d tree, in the caller's
 * numbering, with the grid's max_st_radius:
 *   RBFFD_ST_BRUTE_FORCE: Grid::generateStencilsBruteForce
 *     (grid_interface.cpp:637-686): nodes by squared distance, equal
 *     distances in decreasing node number (its std::set with a `<=`
 *     comparator, grid_interface.h:442-461) -- a duplicate point with a
 *     higher number then comes before the centre, as in the reference;
 *   RBFFD_ST_KDTREE: the lists of rbffd_stencils_knn.
 * Each list stops at the first node whose distance is not below max_radius
 * (DBL_MAX: the reference's default, no trimming); st_len[N] receives the
 * lengths and the rest of each row is the centre (padding).  Searched over a
 * cell grid, not O(N^2).  RBFFD_ERR_INVALID for max_radius <= 0 (the
 * reference's stencils would all be empty). */
enum { RBFFD_ST_BRUTE_FORCE = 0, RBFFD_ST_KDTREE = 1 };
/* RBFFD::setVariableEpsilon (src/rbffd/rbffd.cpp:1378-1420, Sarler 2006
 * form): eps[st[i][0]] = 1 / (alpha * r_max(i)), r_max the distance from the
 * centre to the stencil's last node.  st_len NULL: every stencil n_pad long.
 * eps[N] entries of nodes that are no stencil's centre are left as given.
 * Host only. */
int rbffd_variable_epsilon(int N, const double* xyz, int n_pad, const int* st, const int* st_len, double alpha,
                           double* eps);
int rbffd_stencils_generate(const double* xyz, int N, int n, int method, double max_radius, int* st, int* st_len,
                            int* ties, int nthreads);
/* The same stencils (identical lists and tie count) computed on ctx's device:
 * the host bins the points into a uniform cell grid, one warp per node
 * searches the surrounding cells.  Replaces the same reference call
 * (grid_interface.cpp:688-725, KDTree.h:407-433); n <= 255. */
int rbffd_stencils_knn_gpu(rbffd_ctx* ctx, const double* xyz, int N, int n, int* st, int* ties);
/* rbffd_stencils_generate on ctx's device (both generators, max_radius, the
 * same lists and lengths); n <= 255. */
int rbffd_stencils_generate_gpu(rbffd_ctx* ctx, const double* xyz, int N, int n, int method, double max_radius,
                                int* st, int* st_len, int* ties);
/* Hash-grid stencils as the reference's cosine-bell experiment generates
 * them: Grid::generateStencilsHash (src/grids/grid_interface.cpp:733-966,
 * called at tests/experiments/cosine_bell_on_sphere/main.cpp:197-200).  Not
 * an exact kNN: candidates come from the nbx x nby x nbz overlay cells around
 * a node's cell (levels until they hold n nodes, at least one ring).  The
 * reference renumbers the grid by cell; order[k] is the node placed at k and
 * st[N][n] (centre first, closest first, ties in decreasing number) and
 * st_len[N] use the new numbering; stencils are trimmed to the nodes closer
 * than max_radius (DBL_MAX: no trimming), padding is the centre.  extents
 * [xmin, xmax, ymin, ymax, zmin, zmax], or NULL for the reference grid's
 * defaults widened by the nodes (Grid::refreshExtents).  RBFFD_ERR_INVALID
 * where the reference would not terminate or index out of range (fewer
 * reachable nodes than n, nodes outside the extents, a flat extent).  As in
 * the reference, the z cell index is bounded by nby: with nbz > nby some
 * cells are never searched and some stencils miss their own centre (such
 * stencils are refused by rbffd_grid_create). */
int rbffd_stencils_hash(const double* xyz, int N, int n, int nbx, int nby, int nbz, const double* extents,
                        double max_radius, int* order, int* st, int* st_len);
/* Cosine bell ExactAdvection::operator() (tests/experiments/cosine_bell_on_sphere/exact_advection.h:37-53). */
int rbffd_exact_cosine_bell(int N, const double* xyz, double sphere_radius, double* h);
/* Vortex roll-up (VortexRollup::solve, src/pdes/hyperbolic/vortex_rollup.cpp:27-57):
 * w(theta) = Vt / rho per node, rho = 3 cos(theta), Vt = (3 sqrt(3) / 2)
 * sech(rho)^2 tanh(rho), 0 where |rho| < 4 eps; theta the latitude of
 * cart2sph.  f = -w D_lambda h is RBFFD_RHS_ADVECTION with cu = w, cv = NULL. */
int rbffd_vortex_rollup_coefficients(int N, const double* xyz, double* w);
/* ExactRollup::operator() (tests/experiments/vortex_rollup_on_sphere/exact_rollup.h:25-35):
 * h = 1 - tanh((rho / 5) sin(lambda - w t)). */
int rbffd_exact_vortex_rollup(int N, const double* xyz, double t, double* h);
/* PDE::calcSolNorms (src/pdes/pde.cpp:467-510; src/utils/norms.cpp): out[0..5]
 * = l1 absolute, l1 relative, l2 absolute, l2 relative, linf absolute, linf
 * relative of sol against exact over n values, sums in index order; a
 * relative norm whose exact norm is at most 1e-10 is (abs + 1) / (exact + 1),
 * as in the reference.  Host only. */
int rbffd_sol_norms(const double* sol, const double* exact, int n, double* out);
/* Heat on the unit sphere: u = sum_{l<=lmax,m} c_lm exp(-kappa l(l+1) t) Y_lm (real orthonormal Y_lm). */
int rbffd_exact_sph_heat(int N, const double* xyz, int lmax, const double* coeffs, double kappa, double t, double* u);

/* ---- node orders -------------------------------------------------------- */
/* The order in which a grid stores its rows and nodes (the reordering step
 * before the SpMV: tests/util/cuthill_mckee/{main.cpp,reorder.h}).  order[k]
 * is the node placed at position k, as the reference's `order` vector
 * (reorder.h: inv_order[order[i]] = i).  MORTON: along a 3-D Morton curve of
 * the coordinates (xyz needed), the order grids use by default.  RCM: reverse
 * Cuthill-McKee on the stencil graph (stencils needed), the order the
 * reference's utility computes with Boost's cuthill_mckee_ordering
 * (reorder.h:50-60); ties may break differently from Boost's, whose
 * neighbour lists keep insertion order.  GIVEN: the caller's order.  Host
 * only, no GPU. */
enum rbffd_order_method { RBFFD_ORDER_MORTON = 0, RBFFD_ORDER_RCM = 1, RBFFD_ORDER_GIVEN = 2 };
int rbffd_node_order(int N, const double* xyz, int n_pad, const int* stencils, const int* st_len, int method,
                     int* order);

/* ---- grid (nodes + stencils resident on the device) -------------------- */
/* Uploads nodes and stencils; replaces RBFFD_CL::updateStencilsOnGPU /
 * updateNodesOnGPU (src/rbffd/rbffd_cl.cpp:186-257).  st_len may be NULL
 * (every stencil has n_pad nodes).  Padding slots hold the centre index and
 * weight 0, as the reference's ELL packing does (rbffd_cl.cpp:238-242). */
int rbffd_grid_create(rbffd_ctx* ctx, int N, const double* xyz, int n_pad, const int* stencils, const int* st_len,
                      rbffd_grid** out);
/* The same with the grid's internal order chosen (rbffd_order_method);
 * rbffd_grid_create uses RBFFD_ORDER_MORTON.  The order changes where rows
 * and nodes sit in device memory, never a row's arithmetic: results are the
 * same bits in every order. */
int rbffd_grid_create_ordered(rbffd_ctx* ctx, int N, const double* xyz, int n_pad, const int* stencils,
                              const int* st_len, int order_method, rbffd_grid** out);
int rbffd_grid_destroy(rbffd_grid* grid);
/* Device bytes held by the grid (nodes, stencils, all weights). */
int rbffd_grid_nbytes(const rbffd_grid* grid, size_t* bytes);

/* ---- weights ------------------------------------------------------------ */
typedef struct rbffd_weight_params {
    unsigned der_types; /* OR of rbffd_der_type */
    int dim;            /* RBF dimension used by LAPL and HV (RBFFD ctor dim_num, rbffd.h:192) */
    int poly_deg;       /* -1 none; 0 constant (the reference build, rbffd.cpp:1,230-234);
                           1 {1,x,y,z} (rbffd.cpp:150-172); 2..4 tangent-plane polynomials
                           of total degree <= d, (d+1)(d+2)/2 terms (beyond the reference) */
    int hv_k;           /* hyperviscosity power (RBFFD::setHVScalars, rbffd.h:241-245) */
    double hv_gamma;    /* HV scale = -hv_gamma * hv_nodes^-hv_k (RBFFD::getHVScalar, rbffd.h:227-238) */
    double hv_nodes;    /* global node count for the HV scale; <= 0 means the grid's N */
} rbffd_weight_params;

/* Batched FP64 weight computation on the device, all stencils, all selected
 * operators: replaces RBFFD::computeAllWeightsForAllStencils
 * (src/rbffd/rbffd.cpp:90-103) and computeAllWeightsForStencil_Direct
 * (rbffd.cpp:225-352).  eps is per node (var_epsilon, the stencil uses
 * eps[centre], rbffd.cpp:395-400) or NULL to use eps_uniform (setEpsilon,
 * rbffd.h:352-362).  deg_per_row (optional) overrides poly_deg per stencil
 * for mixed-size batches.  Returns RBFFD_ERR_SINGULAR if any system had a
 * zero pivot (first failing row in last_error). */
int rbffd_weights_compute(rbffd_grid* grid, const rbffd_weight_params* params, const double* eps, double eps_uniform,
                          const int* deg_per_row);
/* Elimination used by rbffd_weights_compute on this context (no reference
 * counterpart: the reference calls LAPACK through arma::solve).  Every
 * method performs dgetf2's arithmetic (first-maximum partial pivoting,
 * multipliers by division, fused updates in step order) and gives the same
 * weights bit for bit; they differ in where the system lives:
 *   RBFFD_ELIM_AUTO       the autotuner picks per system size (default);
 *   RBFFD_ELIM_UNBLOCKED  shared memory, one pass over the trailing rows per step;
 *   RBFFD_ELIM_BLOCKED    shared memory, panels of 8 steps with register-tiled updates;
 *   RBFFD_ELIM_ROW_MAP    shared memory, rows never swapped (a row map), one barrier per step;
 *   RBFFD_ELIM_REGISTERS  the rows in registers of one CTA (m <= 128 and m + K <= 128).
 * A method that does not apply to a system size leaves that size to the
 * autotuner. */
enum { RBFFD_ELIM_AUTO = 0, RBFFD_ELIM_UNBLOCKED = 1, RBFFD_ELIM_BLOCKED = 2, RBFFD_ELIM_ROW_MAP = 3,
       RBFFD_ELIM_REGISTERS = 4 };
int rbffd_weights_set_elimination(rbffd_ctx* ctx, int method);
int rbffd_weights_get_elimination(rbffd_ctx* ctx, int* method);
/* The assembled augmented systems [A | B] (m x (m+K), row-major, K = number
 * of selected operators) of the listed stencils, as the weight solver builds
 * them before elimination: RBFFD::getStencilLHS + getStencilMultiRHS
 * (rbffd.cpp:106-191), for inspection and parity checks.  All listed rows
 * must have the same system size m.  out: host [count][m][m+K]. */
int rbffd_weights_assemble(rbffd_grid* grid, const rbffd_weight_params* params, const double* eps, double eps_uniform,
                           const int* deg_per_row, const int* rows, int count, double* out);
/* Install host FP64 weights of one operator, [N][n_pad] (e.g. computed by the
 * reference CPU path): RBFFD_CL::updateWeightsDouble (rbffd_cl.cpp:306-385). */
int rbffd_weights_set(rbffd_grid* grid, unsigned der_type, const double* w);
/* Read one operator's FP64 weights back, [N][n_pad]; padding slots are 0.
 * RBFFD::getStencilWeights (rbffd.h:395). */
int rbffd_weights_get(rbffd_grid* grid, unsigned der_type, double* w);
/* Weight files in the reference's Matrix Market forms, host only (no GPU):
 * RBFFD::writeToAsciiFile / writeToBinaryFile (src/rbffd/rbffd.cpp:1265-1375)
 * and loadFromAsciiFile / loadFromBinaryFile (rbffd.cpp:983-1210).  binary = 0
 * writes "row col %24.16le" text entries, 1 raw int/int/double records after
 * the same text header; rows are the stencils' centres, columns their nodes,
 * 1-based, in stencil order.  stencils [N][n_pad] with lengths st_len (NULL:
 * all n_pad); w [N][n_pad] (read: padding set to 0).  Reading refuses
 * (RBFFD_ERR_INVALID) a file whose sizes, order or stencil nodes differ from
 * the given stencils; unreadable / unwritable files also give RBFFD_ERR_INVALID. */
int rbffd_weights_file_write(const char* filename, int binary, int N, int n_pad, const int* stencils,
                             const int* st_len, const double* w);
int rbffd_weights_file_read(const char* filename, int binary, int N, int n_pad, const int* stencils,
                            const int* st_len, double* w);

/* ---- eigenvalue stability check ---------------------------------------- */
/* RBFFD::EigenvalueOutput (src/rbffd/rbffd.h:91-100). */
typedef struct rbffd_eig_output {
    double max_pos_eig, min_pos_eig, max_neg_eig, min_neg_eig;
    int nb_positive, nb_negative, nb_zero;
} rbffd_eig_output;
/* The classification of RBFFD::computeEigenvalues (src/rbffd/rbffd.cpp:781-858)
 * over real parts re[0..n): counts of real parts > zero_tol, < -zero_tol and
 * in between (the reference's tolerance is 1e-8), with the largest and
 * smallest magnitude among the positive and among the negative ones, all four
 * starting from |re[0]| as in the reference.  *max_neg_eig (optional) gets the
 * reference's return value.  Host only, no GPU. */
int rbffd_eig_classify(const double* re, int n, double zero_tol, rbffd_eig_output* out, double* max_neg_eig);
/* RBFFD::computeEigenvalues (rbffd.cpp:703-873): every eigenvalue of the
 * grid's N x N operator der_type, plus the HV operator when use_hv (the
 * reference adds its hyperviscosity weights, rbffd.cpp:737-749), from the
 * dense nonsymmetric eigenproblem the reference solves with eig_gen: the
 * matrix is assembled on the device from the FP64 weights and solved with
 * cuSOLVER's geev (loaded at first use; RBFFD_ERR_UNSUPPORTED if absent).
 * Sphere grids have no boundary nodes, so the reference's identity rows for
 * them do not occur.  eig_re / eig_im (optional, host, N each) receive the
 * eigenvalues in the solver's order; out and max_neg_eig as
 * rbffd_eig_classify with tolerance 1e-8.  N <= RBFFD_EIG_MAX_N. */
#define RBFFD_EIG_MAX_N 16384
int rbffd_eigenvalues(rbffd_grid* grid, unsigned der_type, int use_hv, double* eig_re, double* eig_im,
                      rbffd_eig_output* out, double* max_neg_eig);
/* The rightmost eigenvalues (largest real part) of the operator der_type
 * (+ RBFFD_HV when use_hv) on grids too large for the dense check: the
 * stability question of RBFFD::computeEigenvalues (rbffd.cpp:703-873) -- any
 * eigenvalue with positive real part? -- answered by implicitly restarted
 * Arnoldi on the device's FP64 sliced-ELL operator (basis of ncv vectors,
 * classical Gram-Schmidt with reorthogonalisation, exact shifts, a seeded
 * start vector).  Writes the nev rightmost Ritz values (re, im; rightmost
 * first) and their residual estimates; *nconv of them met
 * |h_{m+1,m}| |e_m^T y| <= tol * max(|theta|, 1e-3 |theta_max|).  nev >= 1,
 * nev + 2 <= ncv <= 256, ncv < N. */
int rbffd_eigen_rightmost(rbffd_grid* grid, unsigned der_type, int use_hv, int nev, int ncv, double tol,
                          int max_restarts, unsigned long long seed, double* re, double* im, double* ritz_resid,
                          int* nconv, int* restarts, int* matvecs);
/* Eigenvalues of a real upper Hessenberg n x n matrix (row-major), by the
 * shifted QR algorithm in complex arithmetic (the projected problem of
 * rbffd_eigen_rightmost); host only.  RBFFD_ERR_UNSUPPORTED if it does not
 * converge. */
int rbffd_hessenberg_eigenvalues(int n, const double* H, double* re, double* im);

/* ---- apply (derivative evaluation) ------------------------------------- */
/* deriv[i] = sum_s w[i][s] * u[st_i[s]] for i in [start, start+count):
 * RBFFD::applyWeightsForDeriv(which, start_indx, nb_stencils, u, deriv)
 * (src/rbffd/rbffd.cpp:669-688; GPU form RBFFD_CL::applyWeightsForDerivDouble/
 * Single, rbffd_cl.cpp:526-694).  u has all N values; deriv is written only on
 * [start, start+count).  Host buffers; dtype selects the FP64 or FP32 kernel
 * (FP32 casts u to float and returns doubles, as rbffd_cl.cpp:669-682). */
int rbffd_apply(rbffd_grid* grid, unsigned der_type, int dtype, unsigned start, unsigned count, const double* u,
                double* deriv);
/* Device-pointer form on the context stream: u_dev and deriv_dev hold N*ntracers
 * values of the dtype ([N][ntracers]). */
int rbffd_apply_dev(rbffd_grid* grid, unsigned der_type, int dtype, int ntracers, const void* u_dev, void* deriv_dev);

/* ---- batched dense FP64 solves (the weight solver's core) ------------- */
/* Solves batch independent systems A_b X_b = B_b in place, A_b m x m and B_b
 * m x nrhs, both row-major and contiguous per system on the device
 * (A_dev[batch][m][m], B_dev[batch][m][nrhs]); X overwrites B; A is destroyed.
 * Gaussian elimination with partial pivoting (first maximal |pivot|), the
 * arithmetic of LAPACK dgesv that arma::solve calls (rbffd.cpp:259).
 * info_dev[b] = 0 or k+1 for an exactly zero pivot at step k.  m <= 160. */
int rbffd_batched_gesv_dev(rbffd_ctx* ctx, int m, int nrhs, int batch, void* A_dev, void* B_dev, void* info_dev);

/* ---- time-dependent PDE (RK4 with fused right-hand side) --------------- */
enum rbffd_rhs_kind {
    /* CosineBell::solve (src/pdes/hyperbolic/cosine_bell.cpp:23-70):
     * f = -(vel_u/a * D_lambda h + vel_v/a * D_theta h) [+ D_hv h]  */
    RBFFD_RHS_COSINE_BELL = 1,
    /* heat on the sphere: f = kappa * D_lsfc u (one Laplace-Beltrami operator, rbffd.cpp:458-464) */
    RBFFD_RHS_HEAT = 2,
    /* advection with caller-given per-node coefficients cu, cv:
     * f = -(cu * D_lambda h + cv * D_theta h) [+ D_hv h]; with cv = NULL,
     * f = -cu * D_lambda h [+ D_hv h] (no D_theta weights needed), the form of
     * VortexRollup::solve (src/pdes/hyperbolic/vortex_rollup.cpp:27-57) with
     * cu = rbffd_vortex_rollup_coefficients */
    RBFFD_RHS_ADVECTION = 3
};

typedef struct rbffd_pde_params {
    int rhs_kind;         /* rbffd_rhs_kind */
    int ntracers;         /* T >= 1 right-hand sides sharing the operators */
    int dtype;            /* RBFFD_F32 or RBFFD_F64 state, weights and accumulation */
    int use_hv;           /* add the HV operator's output to f (advection kinds) */
    double sphere_radius; /* a (cosine bell) */
    double alpha;         /* advection angle (cosine bell) */
    double u0;            /* cosine bell speed 2*pi*a / (one revolution) */
    double kappa;         /* heat diffusivity */
    const double* cu;     /* RBFFD_RHS_ADVECTION: host [N] coefficients */
    const double* cv;     /* (NULL: no D_theta term) */
} rbffd_pde_params;

/* Creates the device-resident state of a TimeDependentPDE
 * (src/pdes/time_dependent_pde.h:9-126) on a grid whose weights are ready:
 * replaces TimeDependentPDE_CL's buffers (time_dependent_pde_cl.cpp:677-708). */
int rbffd_pde_create(rbffd_grid* grid, const rbffd_pde_params* params, rbffd_pde** out);
int rbffd_pde_destroy(rbffd_pde* pde);
/* Copy the solution [N][T] host <-> device (PDE::syncCPUtoGPU, pde.h:166). */
int rbffd_pde_set_state(rbffd_pde* pde, const double* u);
int rbffd_pde_get_state(rbffd_pde* pde, double* u);
int rbffd_pde_set_time(rbffd_pde* pde, double t);
int rbffd_pde_get_time(rbffd_pde* pde, double* t);

enum rbffd_advance_flags {
    RBFFD_ADVANCE_GRAPH = 0x1,   /* capture the steps in a CUDA graph and replay it */
    RBFFD_ADVANCE_UNFUSED = 0x2, /* plain path: one SpMV launch per operator, separate RHS/axpy
                                    launches and a host synchronisation after every step,
                                    the structure of TimeDependentPDE_CL::advanceRK4
                                    (time_dependent_pde_cl.cpp:496-537) */
    RBFFD_ADVANCE_ASYNC = 0x4,   /* return without waiting for the device */
    RBFFD_ADVANCE_RESIDENT = 0x8 /* one tracer, small grids: all steps in one launch of a 16-CTA
                                    thread-block cluster that keeps the weights, stencils and
                                    state in its shared memory (each CTA copies its halo of
                                    the stage input from the other CTAs through distributed
                                    shared memory, then gathers locally; a cluster barrier
                                    per stage);
                                    the one-lane-per-row kernels' arithmetic, fused or unfused
                                    per the PDE's arithmetic.  RBFFD_ERR_UNSUPPORTED when the
                                    grid's weights do not fit 16 CTAs' shared memory (about
                                    N x n x operators x 8 bytes <= 3.3 MB in FP64) */
};
/* nsteps classical RK4 steps of size dt: TimeDependentPDE::advance(RK4, dt)
 * (src/pdes/time_dependent_pde.cpp:53-73,172-304), nsteps times.
 * scheme must be 2 (TimeDependentPDE::RK4); EULER (0) and MIDPOINT (1) return
 * RBFFD_ERR_UNSUPPORTED, as the reference's GPU class compiles them out and
 * exits on them (TimeDependentPDE_CL::advance, time_dependent_pde_cl.cpp:350-375). */
int rbffd_pde_advance(rbffd_pde* pde, int scheme, double dt, int nsteps, int flags);
/* Heat-equation RK4 that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that cannot let a library allocate on the
 * GPU -- applications that reserve the device's memory for their own pool, or
 * latency-critical loops where cudaMalloc/cudaFree would synchronise the
 * device.  The caller passes the state u_dev, N values of dtype in its own
 * device memory, advanced in place by nsteps RK4 steps of
 * u_t = kappa * LSFC u on the grid's Laplace-Beltrami weights (computed or
 * set beforehand).  A copy of the state in the grid's internal node order and
 * the three RK4 stage buffers live in one fixed 8 MiB array inside the
 * library.  rbffd_ctx_create loads this path's device code on its GPU, which
 * reserves the array there (held until the process exits); so a host that
 * reserves nearly all GPU memory for its own pool creates its context first,
 * and no call of this entry point then takes device memory, the first one
 * included.  Grids above 262144 nodes (FP64) or 524288 nodes (FP32) are
 * rejected with RBFFD_ERR_INVALID.  Every call looks up the array's device
 * address (cudaGetSymbolAddress, no allocation).  All calls on a device share the array and
 * leave their stage values in it: calls that overlap on the GPU race and
 * must be serialised by the caller.  Runs on the context stream and returns
 * after the steps complete. */
int rbffd_heat_rk4_noalloc(rbffd_grid* grid, int dtype, double kappa, double dt, int nsteps, void* u_dev);
/* The FP64 arithmetic of this PDE (RBFFD_ARITH_*, see rbffd_ctx_set_arithmetic);
 * RBFFD_ARITH_UNFUSED needs an FP64 one-tracer PDE (else RBFFD_ERR_UNSUPPORTED)
 * and fixes the stage kernel to one lane per row (set_shape may still pick the
 * block size; tiled shapes are refused).  Setting RBFFD_ARITH_FUSED returns the
 * PDE to the autotuned shape. */
int rbffd_pde_set_arithmetic(rbffd_pde* pde, int arith);
int rbffd_pde_get_arithmetic(rbffd_pde* pde, int* arith);
/* Kernel-shape choice for this PDE's stage kernel (lanes per stencil row and
 * threads per block); 0 = autotuned. */
int rbffd_pde_set_shape(rbffd_pde* pde, int lanes_per_row, int block_threads);
int rbffd_pde_get_shape(rbffd_pde* pde, int* lanes_per_row, int* block_threads);
/* Tiled stage kernel: each thread block takes rows_per_block consecutive rows
 * (a multiple of 32) and stages the node values their stencils gather in
 * shared memory; lanes (1, 2 or 4) split each row's slots.  flags (one lane
 * per row):
 *   RBFFD_TILE_STREAM_WEIGHTS: the block's weights and indices are also
 *     streamed into shared memory by asynchronous bulk copies (TMA), several
 *     stages ahead; its waits are bounded and a timeout is reported by
 *     rbffd_pde_advance as RBFFD_ERR_TIMEOUT;
 *   RBFFD_TILE_SLOT_SCHEDULE: FP32 PDEs with 4, 8 or 16 tracers (heat, a
 *     fused advection operator, or the two or three advection operators,
 *     each kept in the same order): each row reads its slots in an order
 *     chosen so that the rows sharing a shared-memory wavefront read
 *     different bank groups (fewer bank conflicts).  Changes each row's FP32
 *     summation order;
 *   RBFFD_TILE_PREFETCH: the block's lanes ask L2 for the weights and indices
 *     of chunks a few steps ahead (pays where the weight stream comes from
 *     HBM); the arithmetic is unchanged;
 *   RBFFD_TILE_PIPELINE: PDEs that stream one operator (heat, or a fused
 *     advection operator) with 1, 4, 8, 16 or 32 (FP32) / 1, 2, 4, 8 or 16
 *     (FP64) values per node: each lane keeps the local indices and weights of
 *     its row's next four chunks in flight in registers; the arithmetic is
 *     unchanged;
 *   RBFFD_TILE_DOUBLE_BUFFER: the same PDEs: a persistent grid (as many
 *     blocks as fit on the device) whose blocks walk the tiles and copy the
 *     next tile's node values into a second shared-memory buffer (cp.async)
 *     while they compute the current one; the arithmetic is unchanged.
 *     Refused where a block's halo exceeds 8 nodes per row.
 * At most one of the first three; RBFFD_TILE_PIPELINE combines with
 * RBFFD_TILE_SLOT_SCHEDULE only, RBFFD_TILE_DOUBLE_BUFFER with none.
 * (flags = 1, the former stream_weights argument, keeps its meaning.)
 * Returns RBFFD_ERR_UNSUPPORTED if the staged data do not fit shared memory
 * or the flags do not apply to the PDE.
 * get_tiling reports 0 when the stage kernel gathers from global memory;
 * get_tile_flags the flags of the shape in use (set or autotuned). */
enum {
    RBFFD_TILE_STREAM_WEIGHTS = 1,
    RBFFD_TILE_SLOT_SCHEDULE = 2,
    RBFFD_TILE_PREFETCH = 4,
    RBFFD_TILE_PIPELINE = 8,
    RBFFD_TILE_DOUBLE_BUFFER = 16
};
int rbffd_pde_set_tiled_shape(rbffd_pde* pde, int rows_per_block, int lanes, int flags);
int rbffd_pde_get_tiling(rbffd_pde* pde, int* rows_per_block);
int rbffd_pde_get_tile_flags(rbffd_pde* pde, int* flags);
/* Advection with time-independent coefficients: replace the three
 * operators of each stage (CosineBell::solve's Dlambda, Dtheta and HV,
 * cosine_bell.cpp:47-57) by one fused operator
 * Wf = -(cu W_lambda + cv W_theta) + W_hv, formed once in FP64 from the FP64
 * weights and rounded to the PDE's dtype, so a stage streams one weight array
 * instead of three (beyond the reference; results within the dtype's rounding
 * of the three-operator path, not bit-identical: FP64 PDEs that must keep the
 * reference's operation order stay on three operators).  on = 0 returns to
 * three operators.  RBFFD_ERR_UNSUPPORTED for heat PDEs and for PDEs in the
 * unfused (reference) arithmetic. */
int rbffd_pde_set_fused_operator(rbffd_pde* pde, int on);
/* FP32 PDEs: keep the state with a compensated update (beyond the reference,
 * which steps in FP64 only).  An RK4 step moves u by a small fraction of
 * itself, and rounding u + increment to FP32 every step drops most of the
 * increment's bits: over thousands of small steps the FP32 state drifts from
 * the FP64 one by far more than one rounding.  With on = 1 stage 3 adds the
 * increment with an exact two-sum and keeps minus the lost part in an extra
 * N x ntracers FP32 array, added back by the next step; rbffd_pde_get_state
 * returns u - that correction (computed in FP64); set_state clears it.  Costs
 * one more FP32 read and write per value and step.  The weights, gathers,
 * sums and stages 0-2 stay FP32 as before.  on = 0 frees the array.
 * RBFFD_ERR_UNSUPPORTED for FP64 PDEs; every stepping path applies it except
 * RBFFD_ADVANCE_RESIDENT, which refuses a PDE that has it on. */
int rbffd_pde_set_compensated_state(rbffd_pde* pde, int on);

/* ---- serving: persistent request loop with continuous batching --------- *
 * No counterpart in the reference, whose drivers run one PDE per process
 * (tests/experiments/cosine_bell_on_sphere/main.cpp:280-515).  A server owns
 * two host threads: one admits requests in arrival order while the
 * context's device memory plus the request's stays within hbm_fraction of
 * the device's memory and fewer than max_active requests run (allocation and
 * upload overlap the running steps); the other advances every admitted
 * request by batches of RK4 steps.  Each stage of a step is one launch per
 * dtype and group size over the rows of all active requests, so requests of
 * different grids, stencil sizes and right-hand sides share the device, and
 * requests on the same grid share one read of its weights and indices.
 * Requests admitted while others run join at the next step boundary.  Each
 * request's sums run over its own stencil with the arithmetic of
 * rbffd_pde_advance with one lane per row, so its result does not depend on
 * what else is in the batch.  FP64 requests sum in stencil order and equal
 * the one-lane rbffd_pde_advance result bit for bit; FP32 requests sum in a
 * fixed per-grid slot order chosen against shared-memory bank conflicts (and
 * FP32 advection uses one fused operator), and FP32 requests add each step's
 * increment to the state with a compensated sum (the rounding lost in u +
 * increment carried into the next step, the result read out as u minus that
 * compensation), so long runs of small steps stay close to the FP64 result:
 * closer than the one-lane FP32 result, from which they differ within FP32
 * rounding.  The server's threads build per-grid tables on
 * demand: while it holds requests on a grid, the caller uses that grid from
 * no other thread. */
typedef struct rbffd_server rbffd_server;

typedef struct rbffd_request {
    rbffd_grid* grid;     /* grid with the operators' weights on the device (kept by the caller) */
    rbffd_pde_params pde; /* right-hand side and dtype; ntracers must be 1 */
    const double* u0;     /* [N] initial state in the caller's node order, copied at submission */
    double dt;            /* RK4 step */
    int nsteps;           /* RK4 steps, >= 0 */
    double* out;          /* [N] result, written before the request reports done; the caller
                             keeps it valid until then (or until rbffd_server_cancel returns) */
} rbffd_request;

typedef struct rbffd_server_stats {
    long long submitted, completed, failed, cancelled; /* completed: results written */
    long long pending, active, max_active_seen;
    long long ticks;        /* batches of steps issued */
    long long launches;     /* stage-kernel launches */
    long long slots_reused; /* admissions that reused a finished request's device buffers */
    double node_updates;    /* sum over executed request steps of the request's N */
    double gpu_busy_s;      /* device time of the issued batches (CUDA events) */
    double stage_bytes;     /* algorithmic bytes of the issued stage launches: per group and
                               row the stencil's indices and each operator's weights once, per
                               request and row four state values (+ two coefficients) */
    double budget_bytes, held_bytes;
} rbffd_server_stats;

/* Start the loop on ctx's device.  hbm_fraction in (0, 1]; max_active <= 0
 * means no slot limit. */
int rbffd_server_start(rbffd_ctx* ctx, double hbm_fraction, int max_active, rbffd_server** out);
/* Which waiting request the admission thread takes next when a slot or
 * memory frees up (beyond the reference, which has no server):
 *   RBFFD_ADMIT_ARRIVAL (default): arrival order;
 *   RBFFD_ADMIT_SHORTEST: the request with the least work left to do (grid
 *     nodes x padded stencil size x steps), ties in arrival order.  With a
 *     max_active limit on an overloaded stream, short requests overtake long
 *     ones, which lowers the median latency; a long request waits while
 *     shorter ones keep arriving.
 * Takes effect for the next admission; results are the same either way. */
enum { RBFFD_ADMIT_ARRIVAL = 0, RBFFD_ADMIT_SHORTEST = 1 };
int rbffd_server_set_admission_order(rbffd_server* srv, int order);
/* Queue a request; *id identifies it.  Returns RBFFD_ERR_BUDGET when the
 * request alone could never fit the budget, RBFFD_ERR_INVALID /
 * RBFFD_ERR_STATE / RBFFD_ERR_UNSUPPORTED for a malformed request. */
int rbffd_server_submit(rbffd_server* srv, const rbffd_request* req, uint64_t* id);
/* done = 1 once the request has finished, failed or been cancelled; status is
 * then its outcome (RBFFD_OK: out holds the result).  latency_s: submission to
 * completion; queue_s: submission to admission (-1 while unknown). */
int rbffd_server_poll(rbffd_server* srv, uint64_t id, int* done, int* status, double* latency_s, double* queue_s);
/* Block until the request is done (returns its status) or timeout_s passes
 * (RBFFD_ERR_TIMEOUT). */
int rbffd_server_wait(rbffd_server* srv, uint64_t id, double timeout_s);
/* Block until nothing is pending or active, or timeout_s passes. */
int rbffd_server_wait_idle(rbffd_server* srv, double timeout_s);
/* Cancel a pending or active request (an active one leaves at the next step
 * boundary; out is not written afterwards).  Returns after it has left. */
int rbffd_server_cancel(rbffd_server* srv, uint64_t id);
int rbffd_server_get_stats(rbffd_server* srv, rbffd_server_stats* stats);
/* paused != 0: issue no further batches of steps (requests are still
 * admitted, and a batch already issued completes); 0 resumes.  Stopping a
 * paused server resumes it to finish the admitted requests. */
int rbffd_server_pause(rbffd_server* srv, int paused);
/* Fault injection on the host: the next count admissions fail as if the
 * device allocation had failed (status RBFFD_ERR_OOM). */
int rbffd_server_inject_admission_failures(rbffd_server* srv, int count);
/* Stop the loop: pending requests end with RBFFD_ERR_CANCELLED, active ones
 * run to completion first; all device memory of the server is released. */
int rbffd_server_stop(rbffd_server* srv);

#ifdef __cplusplus
}
#endif
#endif /* RBFFD_SM100_H */
