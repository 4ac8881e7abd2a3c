/*
 * pmg_b200.h -- C ABI of the B200 implementation of ParMooN's 3D scalar
 * convection-diffusion hot path: finite-element assembly (Galerkin / SUPG /
 * mass forms) into a host-defined CSR pattern, and the geometric-multigrid
 * preconditioned flexible GMRES solve.
 *
 * The entry points take plain pointers and sizes only.  Every call returns 0
 * (PMG_OK) or a negative PMG_ERR_* code; nothing calls exit().  A handle owns
 * one CUDA stream and the device mirrors of everything it was given; the
 * caller keeps ownership of its host arrays.  Calls on one handle are not
 * thread-safe (the reference is single-threaded and non-reentrant too).
 *
 * Which reference interface each entry point stands in for is given beside
 * it (paths relative to the ParMooN source tree).
 */
#ifndef PMG_B200_H
#define PMG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- codes */
#define PMG_OK                   0
#define PMG_ERR_ARG             -1  /* bad argument / size / ordering */
#define PMG_ERR_CUDA            -2  /* CUDA runtime error (message via pmg_last_error) */
#define PMG_ERR_STATE           -3  /* call out of order (e.g. solve before assemble) */
#define PMG_ERR_NOT_CONVERGED   -4  /* iteration limit reached before the tolerance */
#define PMG_ERR_DIVERGED        -5  /* residual grew beyond SC_DIV_FACTOR * r0 */
#define PMG_ERR_SLOT            -6  /* element coupling missing from the CSR pattern */
#define PMG_ERR_NONFINITE       -7  /* NaN/Inf detected in assembled data or residual */
#define PMG_ERR_SINGULAR        -8  /* zero pivot in the coarsest-level factorisation */
#define PMG_ERR_UNSUPPORTED     -9  /* element/form/coefficient combination not built */

/* ------------------------------------------------------------ elements */
/* Element families (reference: include/FE3D/BF_C_H_Q1_3D.h, BF_C_H_Q2_3D.h,
 * BF_C_T_P1_3D.h, BF_C_T_P2_3D.h).  Local basis ordering follows the
 * reference tables: hexahedra are tensor-ordered (x fastest) on the nodes of
 * [-1,1]^3, tetrahedra follow the reference vertex/edge numbering. */
#define PMG_ELEM_Q1_HEX   1   /*  8 local dofs */
#define PMG_ELEM_Q2_HEX   2   /* 27 local dofs */
#define PMG_ELEM_NQ1_HEX  3   /*  6 local dofs: the non-conforming rotated trilinear element N_Q1
                                 (include/FE3D/BF_N_H_Q1_3D.h, point-value nodal functionals at the
                                 face midpoints, NF_N_H_Q1_3D.h) of the non-conforming levels of
                                 SC_MG_TYPE_SCALAR = 1 */
#define PMG_ELEM_P1_TET  11   /*  4 local dofs */
#define PMG_ELEM_P2_TET  12   /* 10 local dofs */

/* Local forms (reference: src/FE/ConvDiff3D.C:87-214, src/FE/TCD3D.C:37-421). */
#define PMG_FORM_GALERKIN     1  /* BilinearAssemble:   A = eps grad.grad + (b.grad u) v + c u v ; f v */
#define PMG_FORM_SUPG         2  /* BilinearAssemble_SD: Galerkin + delta (b.grad u + c u)(b.grad v) */
#define PMG_FORM_MASS         3  /* MatrixMRhsAssemble: M = u v ; f v */
#define PMG_FORM_MASS_SUPG    4  /* MatrixMRhsAssemble_SUPG: M = u (v + delta b.grad v) ; f (v + delta b.grad v) */
#define PMG_FORM_STIFF_SUPG   5  /* MatricesAKRhsAssemble_SUPG (A part): SUPG stiffness, rhs f (v + delta b.grad v) */

/* Coefficient descriptors: the device-evaluable stand-in for the host
 * CoeffFct3D callback (include/General/Constants.h:148-149).  Coefficient
 * order follows the reference: c0=eps, c1..c3=b, c4=c (reaction), c5=f. */
#define PMG_COEF_CONST        0  /* eps, b, c, f constant */
#define PMG_COEF_SINE_RHS     1  /* Laplace.h: f = 3 pi^2 eps sin(pi x) sin(pi y) sin(pi z) */
#define PMG_COEF_LOGNORMAL    2  /* eps(x) = exp(sum_k a_k cos(2 pi k.x + phi_k)) ; b, c, f constant */
#define PMG_COEF_CURL_FOURIER 3  /* b = curl psi, psi = sum of Fourier modes (scaled) ; eps, c, f constant */
#define PMG_COEF_ROTATING     4  /* b = (-(y-.5), x-.5, 0.2 sin(2 pi t)) ; eps, c, f constant */
#define PMG_COEF_AMC          5  /* amc.h: eps=1, f=(3 pi^2 - 0.1) e^{-0.1 t} sin(pi x) cos(pi y) cos(pi z) */
#define PMG_COEF_TABLE        6  /* values per cell and quadrature point from pmg_set_coefficient_table */

typedef struct pmg_coeff_desc {
    int    kind;          /* PMG_COEF_* */
    double eps;           /* c0 */
    double b[3];          /* c1..c3 (constant kinds) / scale (curl kind: b[0]) */
    double c;             /* c4 */
    double f;             /* c5 (constant kinds) */
    double t;             /* current time for time-dependent kinds */
    int    n_modes;       /* Fourier modes for LOGNORMAL / CURL_FOURIER */
    const double *modes;  /* n_modes x 8 doubles: kx ky kz amp phase ax ay az (host pointer, copied) */
} pmg_coeff_desc;

/* ------------------------------------------------------------ solver knobs */
/* POD mirror of the TDatabase::ParamDB fields the reference reads on this
 * path (src/General/Database.C:660-780).  pmg_default_params fills the
 * reference defaults. */
#define PMG_SMOOTHER_JACOBI   1  /* TMGLevel3D::Jacobi (src/FE/MGLevel3D.C:469-560) */
#define PMG_SMOOTHER_SOR      2  /* TMGLevel3D::SOR (src/FE/MGLevel3D.C:280-361), rows in colour order */
#define PMG_SMOOTHER_SSOR     3  /* TMGLevel3D::SSOR (src/FE/MGLevel3D.C:363-467), rows in colour order */
#define PMG_SMOOTHER_LEARNED 30  /* stencil-network smoother with SSOR fallback */
#define PMG_COARSE_JACOBI     1
#define PMG_COARSE_SOR        2
#define PMG_COARSE_SSOR       3
#define PMG_COARSE_DIRECT    17  /* dense LU of the coarsest level (reference: SolveExact) */
#define PMG_PREC_FP64         0  /* V-cycle stores level matrices and vectors in FP64 */
#define PMG_PREC_FP32         1  /* V-cycle in FP32, outer FGMRES / true residual in FP64 */

/* quadrature rules selectable through pmg_params.quad_rule (Gauss: hexahedra,
 * Keast: tetrahedra; src/QuadFormulas/QuadFormulaHexa.C, QuadFormulaTetra.C;
 * the 5-point degree-3 tetrahedral rule has no reference counterpart) */
#define PMG_QUAD_AUTO     0
#define PMG_QUAD_GAUSS2   2
#define PMG_QUAD_GAUSS3   3
#define PMG_QUAD_GAUSS4   4
#define PMG_QUAD_KEAST4   104
#define PMG_QUAD_KEAST5   105
#define PMG_QUAD_KEAST11  111

typedef struct pmg_params {
    int    smoother;           /* SC_SMOOTHER_SCALAR */
    int    pre_smooth;         /* SC_PRE_SMOOTH_SCALAR */
    int    post_smooth;        /* SC_POST_SMOOTH_SCALAR */
    int    coarse_smoother;    /* SC_COARSE_SMOOTHER_SCALAR */
    int    coarse_maxit;       /* SC_COARSE_MAXIT_SCALAR */
    double coarse_red;         /* SC_COARSE_RED_FACTOR_SCALAR */
    double smooth_omega;       /* SC_SMOOTH_DAMP_FACTOR_SCALAR (Parameters[0]) */
    double gmg_damp;           /* SC_GMG_DAMP_FACTOR_SCALAR */
    double lin_red;            /* SC_LIN_RED_FACTOR_SCALAR  (stop when |r| < lin_red |r0|) */
    double lin_res_min;        /* SC_LIN_RES_NORM_MIN_SCALAR (stop when |r| < lin_res_min) */
    int    lin_maxit;          /* SC_LIN_MAXIT_SCALAR */
    int    restart;            /* SC_GMRES_RESTART */
    double div_factor;         /* SC_DIV_FACTOR */
    int    precision;          /* PMG_PREC_* (V-cycle storage/compute precision) */
    int    sdfem_type;         /* SDFEM_TYPE (2 supported) */
    int    poly_degree;        /* INTERNAL_POLYNOMIAL_DEGREE used in the SUPG delta */
    double delta0;             /* DELTA0 */
    int    reference_restart_rule; /* 1: FGMRES restart resets r0 like FgmresIte.C:546-566; 0: always relative to the first r0 */
    int    problem_linear;     /* INTERNAL_PROBLEM_LINEAR: 1 -> Q1 Gauss2 / Q2 Gauss3 / P1 Keast4 / P2 Keast11,
                                  0 -> Q1 Gauss3 / Q2 Gauss4 / P1 Keast11 (FEDatabase3D.C:1203-1309) */
    int    learned_steps;      /* learned-smoother steps per pre/post phase (0: pre_smooth / post_smooth) */
    int    assembly_kernel;    /* 0: automatic -- space-constant eps, b, c, and pure diffusion with a varying
                                  eps on Q1 / P1 / P2, contract reference tables on the FP64 tensor cores;
                                  the rest runs per quadrature point; 1: per-quadrature-point kernel for
                                  every coefficient kind; 2: reference-matrix kernel on the FP64 CUDA cores
                                  for space-constant coefficients (per point otherwise) */
    int    slc_all;            /* SC_STEP_LENGTH_CONTROL_ALL_SCALAR: step-length control on every level >= 1 */
    int    slc_fine;           /* SC_STEP_LENGTH_CONTROL_FINE_SCALAR: step-length control on the finest level
                                  (TMultiGrid3D::Cycle, src/FE/MultiGrid3D.C:517-523, 655-663;
                                  TMGLevel3D::StepLengthControl, src/FE/MGLevel3D.C:908-961) */
    int    quad_rule;          /* 0 (default): the reference's rule for the element (problem_linear above);
                                  else one of PMG_QUAD_* for the element's shape (PMG_ERR_UNSUPPORTED at
                                  assembly otherwise) */
    int    learned_guard_off;  /* 0 (default): with PMG_SMOOTHER_LEARNED the solve measures the plain SSOR
                                  V-cycle's contraction over the first 2 cycles, then runs the learned
                                  smoother and hands back to SSOR as soon as its measured per-cycle
                                  contraction exceeds the plain one; 1: the learned smoother runs in every
                                  cycle (for measuring it alone) */
    int    assembly_scatter;   /* how local matrices reach the CSR matrix (same sums, same order, bitwise
                                  equal results): 0 (default) automatic -- the row gather for Q1, N_Q1,
                                  P1 and P2, the colour scatter for Q2; 1: colour by colour, each colour's
                                  cells adding into the matrix (TAssembleMat3D::Assemble order); 2: row
                                  gather -- local matrices of all cells in one pass, then each CSR row
                                  summed from its cells' rows in colour order and written once (rows up to
                                  768 / (32 / n_loc) entries; colour scatter otherwise) */
} pmg_params;

typedef struct pmg_solve_stats {
    int    iterations;         /* FGMRES iterations (= V-cycles applied) */
    double res0;               /* |b - A x0| (FP64, all rows) */
    double res_final;          /* true |b - A x| recomputed in FP64 after the solve */
    double rel_res;            /* res_final / res0 */
    double mean_contraction;   /* (res_final/res0)^(1/iterations) */
    int    smoother_used;      /* PMG_SMOOTHER_* actually used (learned may fall back) */
    double seconds;            /* device time of the solve (CUDA events) */
    double setup_seconds;      /* of which per-solve set-up: SELL values, coarsest factorisation, graph capture */
    double vcycle_seconds;     /* device time of the first preconditioner application (one V-cycle) */
    double rho_plain;          /* learned smoother: the plain SSOR cycles' measured contraction per cycle (0 if
                                  not measured) */
    double rho_learned;        /* learned smoother: its measured contraction per cycle over the cycles it ran
                                  (0 if it ran fewer than 2) */
    int    learned_cycles;     /* V-cycles that used the learned smoother */
} pmg_solve_stats;

typedef struct pmg_handle_s *pmg_handle;

/* ------------------------------------------------------------ lifecycle */
void        pmg_default_params(pmg_params *p);
/* sizeof(pmg_params) of this build of the library: pmg_default_params writes
 * that many bytes, so a program compiled against another revision of this
 * header (sizeof differs) must check it before the first call */
int         pmg_params_size(void);
const char *pmg_last_error(void);
int         pmg_device_count(int *n);

/* TSystemCD3D ctor (src/System/SystemCD3D.C:62-227): creates the per-level
 * containers; levels are numbered 0 (coarsest) .. n_levels-1 (finest).
 * pmg_create and pmg_set_params reject parameter sets this library does not
 * build (unknown smoother codes, out-of-range counts) with PMG_ERR_ARG. */
int pmg_create(pmg_handle *h, int n_levels, const pmg_params *p);
int pmg_destroy(pmg_handle h);
int pmg_set_params(pmg_handle h, const pmg_params *p);

/* ------------------------------------------------------------ mesh / space */
/* TFESpace3D (src/FE/FESpace3D.C:81-239): element->dof map of one level in the
 * reference's GlobalNumbers + BeginIndex form flattened to n_cells x n_loc,
 * plus each cell's vertex coordinates in the cell's own vertex order
 * in 8 vertex slots per cell (tetrahedra use the first 4; n_cells x 8 x 3).
 * Affine maps only (HexaAffin, TetraAffin): parallelepipeds / tetrahedra.
 * brick != 0 declares every hexahedron axis-aligned (needed for SUPG on hexes,
 * whose convection-direction mesh size uses the physical trilinear interpolant). */
int pmg_set_level_mesh(pmg_handle h, int level, int elem_type, int n_cells,
                       const int *elem_dof, const double *cell_vert, int brick);

/* TSquareStructure3D + Sort (src/FE/SquareStructure3D.C:58-527,
 * src/FE/SquareStructure.C:91-110): the CSR pattern of one level, columns
 * sorted ascending in each row, rows [active_bound, n_rows) Dirichlet (one
 * diagonal entry each).  The device keeps a mirror; the host keeps ownership. */
int pmg_set_level_csr(pmg_handle h, int level, int n_rows, int active_bound,
                      const int *row_ptr, const int *kcol);

/* The same pattern built on the device from the element -> dof map
 * (GlobalNumbers + BeginIndex flattened, n_cells x nloc): every dof of every
 * cell holding an active row, sorted; a Dirichlet row (>= active_bound) its
 * diagonal alone -- what TSquareStructure3D + Sort produce for conforming
 * spaces.  Installed as the level's pattern as pmg_set_level_csr would;
 * nnz_out (may be NULL) receives its size.  Rows may gather at most 1024
 * candidate columns (incident cells x nloc), else PMG_ERR_UNSUPPORTED. */
int pmg_build_level_csr(pmg_handle h, int level, int n_rows, int active_bound, int n_cells, int nloc,
                        const int *elem_dof, int *nnz_out);
/* Wall times of the last pmg_build_level_csr: the pattern built on the device
 * (element map upload included) and its installation (pattern checks, greedy
 * row colouring, host mirror). */
int pmg_setup_timings(pmg_handle h, double *csr_device_s, double *csr_install_s);
/* Copy a level's pattern out (TSquareStructure3D::GetRowPtr / GetKCol
 * consumers): row_ptr n_rows + 1 entries, kcol (may be NULL) nnz entries. */
int pmg_get_level_csr(pmg_handle h, int level, int *row_ptr, int *kcol);

/* Optional multicolour ordering of the rows of one level for the parallel
 * SSOR (n_rows colour ids in [0, n_colors)).  Rows sharing a matrix entry
 * must have different colours.  Without it a greedy colouring is built. */
int pmg_set_level_row_colors(pmg_handle h, int level, int n_colors, const int *colors);

/* Prolongation from level-1 to level (GetProlongationMatrix3D,
 * src/FE/FEDatabase3D.C:1656-1815, averaged by dof multiplicity as in
 * Prolongate, src/FE/MGComponents3D.C:208-488).  n_fine rows, CSR.
 * Restriction is its transpose (DefectRestriction, :732-1014). */
int pmg_set_transfer(pmg_handle h, int level, int n_fine, int n_coarse,
                     const int *p_row_ptr, const int *p_col, const double *p_val);

/* The prolongation from level-1 to level built on the device for conforming
 * nested spaces (what pmg_nested_prolongation in pmg_mesh.h builds on the
 * host): fine dof r (position f_dof_xyz[3r..3r+2]) lies in coarse cell
 * f_dof_cell[r] (the caller's cell index of level-1, whose mesh must be set);
 * its row holds that cell's coarse basis at the dof, entries below 1e-12
 * dropped.  R = P^T is formed on the device.  pmg_get_transfer copies P out
 * (p_row_ptr n_fine + 1 entries; p_col / p_val may be NULL). */
int pmg_build_transfer(pmg_handle h, int level, int n_fine, const double *f_dof_xyz, const int *f_dof_cell);
int pmg_get_transfer(pmg_handle h, int level, int *p_row_ptr, int *p_col, double *p_val);

/* Dirichlet values of one level (the BoundValueFunct3D callback evaluated at
 * the dof nodes, AssembleMat3D.C:1031-1081): n_rows - active_bound values. */
int pmg_set_dirichlet_values(pmg_handle h, int level, const double *values);

/* CoeffFct3D stand-in (include/General/Constants.h:148-149). */
int pmg_set_coefficients(pmg_handle h, const pmg_coeff_desc *c);

/* Tabulated coefficients, for a host CoeffFct3D callback the device cannot
 * call (TDiscreteForm3D::GetLocalForms calls it at the cell's quadrature points,
 * src/FE/DiscreteForm3D.C:264, after GetOrig maps them, AssembleMat3D.C:461-466).
 * pmg_quad_points returns, for the rule pmg_assemble uses with the current
 * params (INTERNAL_PROBLEM_LINEAR), the number of points per cell and, when
 * xyz is non-NULL, their physical coordinates: n_cells x nq x 3 in the
 * caller's cell order of pmg_set_level_mesh, mapped as the reference maps them
 * (HexaAffin / TetraAffin).  The caller evaluates its callback there and
 * passes n_cells x nq x 6 values c0..c5 (eps, b1, b2, b3, c, f) to
 * pmg_set_coefficient_table; the level's assembly reads them when the
 * coefficient kind is PMG_COEF_TABLE (|b| is formed on the device). */
int pmg_quad_points(pmg_handle h, int level, int *nq, double *xyz);
int pmg_set_coefficient_table(pmg_handle h, int level, const double *values);

/* ------------------------------------------------------------ assembly */
/* TAssembleMat3D::Reset + Assemble3D (src/System/AssembleMat3D.C:261-535,
 * 751-857, 913-1200) for one level with one local form; the matrix and rhs
 * stay on the device.  entries_out / rhs_out, when non-NULL, receive host
 * copies (TSquareMatrix3D::GetEntries() consumers).  level = -1: all levels
 * (TSystemCD3D::Assemble, src/System/SystemCD3D.C:340-365). */
int pmg_assemble(pmg_handle h, int level, int form, double *entries_out, double *rhs_out);

/* Copy a level's matrix (or rhs) between host and device. */
int pmg_get_matrix(pmg_handle h, int level, int which, double *entries_out);
int pmg_set_matrix(pmg_handle h, int level, int which, const double *entries);
int pmg_get_rhs(pmg_handle h, int level, double *rhs_out);
/* which: 0 = system matrix A, 1 = mass matrix M (time-dependent problems) */

/* TSystemTCD3D::AssembleSystMat (src/System/SystemTCD3D.C:260-326), after
 * pmg_assemble of the mass form (AssembleMRhs) and of the stiffness form at
 * the new time (AssembleARhs):
 *   B := tau*theta3*f_old + tau*theta4*f_new + (M - tau*theta2*A) u_old   (active rows)
 *   B := f_new, start vector := f_new                                  (Dirichlet rows)
 *   A := M + tau*theta1*A on every level (active rows; A is kept for
 *   pmg_tcd_restore).  B becomes the finest level's rhs for pmg_solve, whose
 *   start vector (sol == NULL) is u_old.  f_old / u_old: host arrays of the
 *   finest level, or NULL for the device copies (f_old = the rhs of the
 *   previous pmg_tcd_system call or of the mass assembly, u_old = the last
 *   solution).  rhs_out (optional) receives B. */
int pmg_tcd_system(pmg_handle h, double tau, const double theta[4],
                   const double *f_old, const double *u_old, double *rhs_out);

/* TSystemTCD3D::RestoreMassMat (src/System/SystemTCD3D.C:328-347): the
 * stiffness matrices saved by pmg_tcd_system are put back on every level. */
int pmg_tcd_restore(pmg_handle h);

/* ------------------------------------------------------------ kernels */
/* MatVect_Scalar / Defect_Scalar plug-ins (src/FE/Blas2.C:86-126) on the
 * finest level's FP64 matrix: y = A x, r = b - A x.  Host arrays. */
int pmg_matvec(pmg_handle h, int level, const double *x, double *y);
int pmg_defect(pmg_handle h, int level, const double *x, const double *b, double *r, double *norm);

/* Allocation-free variant of pmg_defect (no counterpart in the reference).
 * For callers that must not have the library allocate device memory during a
 * call: hosts whose GPU memory is owned by their own pool or framework
 * allocator, and latency-critical loops that cannot absorb cudaFree's
 * device-wide wait.  x, b, r and norm are DEVICE pointers (N, N, N and 1
 * doubles) the caller owns; the call computes r = b - A x and norm = |r|_2 on
 * the level's FP64 matrix and returns after the handle's stream is done.
 * The kernels run on the handle's own stream, which is not ordered after the
 * caller's streams: x and b must be completely written on the device before
 * the call (synchronize the stream that produced them, or the device), and r
 * and norm may be read on any stream once the call has returned.  The level
 * must hold an assembled (or pmg_set_matrix) matrix, else PMG_ERR_STATE.
 * Its only scratch is a fixed array inside the library (512 KiB per GPU,
 * kept until the process exits), shared by all calls: calls that overlap on
 * the GPU race on it.  The first call on a device looks up the array's
 * address (once per device).  Levels with more than PMG_NOALLOC_MAX_ROWS
 * rows are rejected with PMG_ERR_ARG; it calls no allocating routine. */
#define PMG_NOALLOC_MAX_ROWS 16777216
int pmg_defect_noalloc(pmg_handle h, int level, const double *x, const double *b, double *r, double *norm);

/* One multicolour SSOR sweep pair (forward+backward) on a level, FP64
 * (TMGLevel3D::SSOR, src/FE/MGLevel3D.C:363-467, in colour order). */
int pmg_ssor(pmg_handle h, int level, const double *rhs, double *sol, int n_sweeps);

/* Prolongate (P c) and restrict (P^T d) between level-1 and level. */
int pmg_prolongate(pmg_handle h, int level, const double *coarse, double *fine);
int pmg_restrict(pmg_handle h, int level, const double *fine, double *coarse);

/* ------------------------------------------------------------ solve */
/* TFgmresIte::Iterate with TMultiGridScaIte (src/FE/FgmresIte.C:245-624,
 * src/FE/MultiGridScaIte.C:89-130) on the finest level.  sol is the start
 * vector on input (its Dirichlet part is overwritten by the rhs like
 * SetDirichletNodes) and the solution on output; rhs == NULL uses the
 * device-resident assembled rhs; sol == NULL keeps the solution on the
 * device (start vector = assembled Dirichlet values, zero elsewhere). */
int pmg_solve(pmg_handle h, double *sol, const double *rhs, pmg_solve_stats *stats);

/* ------------------------------------------------------------ domain decomposition */
/* The parallel path of the reference (TParFECommunicator3D::CommUpdate /
 * CommUpdateReduce and the all-reduced inner products, src/Parallel/
 * ParFECommunicator3D.C:218-346, src/FE/MGLevel3D.C:220-272) with the transport
 * left to the caller.  Each rank's handle holds one subdomain: its levels are
 * the cells of the subdomain plus a layer of neighbouring cells, numbered with
 * the rank's active owned dofs first; its own Dirichlet dofs and the ghost
 * dofs (dofs of the neighbouring layer owned by other ranks) are rows past
 * active_bound.  pmg_set_halo names, on the finest level, the owned dofs the
 * neighbours need (send_idx, packed in the order the transport delivers them)
 * and the ghost rows (recv_idx) filled from the neighbours, with two device
 * buffers of n_send / n_recv doubles the transport reads and writes. */
typedef struct pmg_comm {
    void *ctx;
    /* sum v[0..n) over all ranks in place (host memory); 0 on success */
    int (*allreduce_sum)(void *ctx, double *v, int n);
    /* send_dev (n_send doubles, packed by the library) to the neighbours and
     * fill recv_dev (n_recv doubles) with theirs; called after the library's
     * stream is idle, must return with recv_dev written; 0 on success */
    int (*exchange)(void *ctx, const double *send_dev, int n_send, double *recv_dev, int n_recv);
} pmg_comm;
int pmg_set_halo(pmg_handle h, int n_send, const int *send_idx, int n_recv, const int *recv_idx,
                 double *send_buf_dev, double *recv_buf_dev);
/* FGMRES over the ranks' subdomains (every rank calls it with its own handle
 * and the same parameters): products with the neighbours' ghost values, every
 * inner product summed over the ranks, each rank's V-cycle on its subdomain
 * with the ghost rows held at zero as the preconditioner (overlapping additive
 * Schwarz with multigrid inside each subdomain).  sol / rhs / stats as
 * pmg_solve (local arrays; only the owned entries of sol are the solution). */
int pmg_solve_dd(pmg_handle h, const pmg_comm *comm, double *sol, const double *rhs, pmg_solve_stats *stats);

/* Copy the device-resident finest-level solution out. */
int pmg_get_solution(pmg_handle h, double *sol_out);

/* ------------------------------------------------------------ output */
/* TOutput3D::WriteVtk (src/FE/Output3D.C:1773-2292) for one scalar function:
 * legacy ASCII VTK unstructured grid of the level's cells (VTK_HEXAHEDRON /
 * VTK_TETRA, corners in the cell's own vertex order, the caller's cell order)
 * with the function's vertex values as POINT_DATA `name` and the cells'
 * region ids (region_ids, n_cells values, or NULL for 0) as CELL_DATA
 * RegionID.  values: host array of the level's N coefficients, or NULL for
 * the device-resident solution of the finest level (the last pmg_solve); the
 * vertex values are gathered on the device.  Vertices are numbered in dof
 * order (the reference numbers them by memory address, so files agree up to
 * that numbering). */
int pmg_write_vtk(pmg_handle h, int level, const double *values, const int *region_ids, const char *path,
                  const char *name);

/* ------------------------------------------------------------ learned smoother */
/* No counterpart in the reference.  A stencil network maps each node's
 * normalised matrix stencil to a 27-point correction stencil W; with
 * params.smoother = PMG_SMOOTHER_LEARNED every pre/post smoothing step is
 * x += omega W (f - A x).  The solve measures the per-cycle contraction of
 * the first cycles with SSOR and with the learned step and keeps SSOR when
 * the learned one contracts worse (stats.smoother_used tells which ran).
 * Levels need one dof per node of a cubic n1^3 lattice (Q1 hexahedra):
 * dof_lat[d] = i + n1 (j + n1 k) for dof d. */
int pmg_set_level_lattice(pmg_handle h, int level, int nx, int ny, int nz, const int *dof_lat);
/* Network parameters: conv 27->32, 32->32, 32->27 (3x3x3 each) with biases,
 * flat FP32 array [W1 b1 W2 b2 W3 b3], W laid out [c_out][c_in][27]. */
int pmg_learned_num_params(int *n);
int pmg_set_learned_weights(pmg_handle h, const float *weights);
int pmg_get_learned_weights(pmg_handle h, float *weights);
/* Stencil W of a level, 27 x N floats (lattice order, channel-major). */
int pmg_learned_stencil(pmg_handle h, int level, float *W_out);
/* One training step on a level from n_samples (error, residual = A error)
 * pairs in device memory (n_samples x N doubles each): loss = mean |A (e -
 * W r)|^2 / |r|^2; lr > 0 applies an Adam step on the device. */
int pmg_learned_train_step(pmg_handle h, int level, int n_samples, const double *e_dev, const double *r_dev, float lr,
                           double *loss_out, float *grad_out);
/* One Adam step from a host gradient (e.g. the mean of the ranks' gradients
 * of pmg_learned_train_step with lr = 0, for data-parallel training). */
int pmg_learned_apply_gradient(pmg_handle h, const float *grad, float lr);
/* One V-cycle z = MG(v) (the preconditioner) on device vectors of the
 * finest level (TMultiGridScaIte::Iterate with zero start). */
int pmg_vcycle(pmg_handle h, const double *v_dev, double *z_dev);

/* ------------------------------------------------------------ timing */
/* Device time in seconds of the last pmg_assemble / pmg_solve call, and the
 * device time of the dominant kernel of the last assembly (CUDA events). */
int pmg_last_timings(pmg_handle h, double *assemble_s, double *solve_s, double *assemble_kernel_s);

/* Time one device kernel family on `level` with CUDA events on the handle's
 * stream (reps launches after one warm-up) and report its algorithmic bytes
 * and flops per launch:
 *   PMG_KERNEL_SPMV64 / SPMV32     y = A x on the solve's SELL-32 copy (FP64 / FP32 values)
 *   PMG_KERNEL_SSOR64 / SSOR32     one SSOR step = forward + backward colour sweeps (SELL-32)
 *   PMG_KERNEL_CSR_SPMV64          y = A x on the CSR pattern (the pmg_matvec plug-in)
 *   PMG_KERNEL_ASSEMBLE            the level's assembly kernel launches (form = current SUPG/Galerkin choice in arg)
 * The matrix must be assembled. */
#define PMG_KERNEL_SPMV64    0
#define PMG_KERNEL_SPMV32    1
#define PMG_KERNEL_SSOR64    2
#define PMG_KERNEL_SSOR32    3
#define PMG_KERNEL_ASSEMBLE  4
#define PMG_KERNEL_CSR_SPMV64 5
#define PMG_KERNEL_COARSE_FACTOR 6  /* LU + inverse of the coarsest level (level must be 0) */
#define PMG_KERNEL_LEARNED_FWD 7    /* the stencil network's forward on the level's lattice (features, three
                                       tensor-core convolutions, stencil); flops = 2 x 27 x (27*32 + 32*32 +
                                       32*27) per lattice node; needs weights and a lattice */
int pmg_time_kernel(pmg_handle h, int kernel, int level, int form, int reps,
                    double *seconds_per_launch, double *bytes_per_launch, double *flops_per_launch);

/* Number of kernel launches this library has issued in the process (graph
 * replays count every kernel node of the graph). */
int pmg_launch_count(unsigned long long *n);

/* Throughput of the arithmetic paths the kernels use, measured on the current
 * device by register-only probe kernels (8 blocks of 256 threads per SM, one
 * timed launch after a warm-up): FP64 FMA on the CUDA cores, FP64
 * mma.sync.m8n8k4 (DMMA) and BF16 mma.sync.m16n8k16 with FP32 accumulation,
 * in TFLOP/s.  Diagnostic only; no handle needed. */
int pmg_measure_peaks(double *fp64_fma_tflops, double *fp64_dmma_tflops, double *bf16_mma_sync_tflops);

#ifdef __cplusplus
}
#endif
#endif /* PMG_B200_H */
