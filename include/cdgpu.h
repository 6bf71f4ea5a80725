/*
 * cdgpu.h -- C ABI of libcdgpu, the B200 (sm_100a) implementation of ParMooN's
 * scalar convection-diffusion hot path: Galerkin/SUPG assembly of Q1/Q2
 * quadrilaterals and hexahedra into the CSR TSquareMatrix, and the
 * geometric-multigrid-preconditioned FGMRES / fixed-point solve.
 *
 * Plain C types only.  Every call returns a status code (CDGPU_OK = 0); the
 * reference instead prints a message and calls exit(4711), which a host shim
 * maps back to (see cdgpu_status_string).  Pointers named h_* are host memory,
 * d_* device memory of the context's device.  Calls on one context are
 * serialised on the context's CUDA stream; a context must not be used by two
 * host threads at once.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the ParMooN_CMG tree).
 */
#ifndef CDGPU_H
#define CDGPU_H

#ifdef __cplusplus
extern "C" {
#endif

enum cdgpu_status
{
  CDGPU_OK = 0,
  CDGPU_ERR_INVALID = 1,       /* bad argument or id */
  CDGPU_ERR_OOM = 2,           /* device allocation failed */
  CDGPU_ERR_CUDA = 3,          /* a CUDA call failed (see cdgpu_last_error) */
  CDGPU_ERR_NOT_CONVERGED = 4, /* maximal iterations reached (reference: "not converged" message) */
  CDGPU_ERR_DIVERGED = 5,      /* residual > SC_DIV_FACTOR * initial (reference: exit(4711)) */
  CDGPU_ERR_UNSUPPORTED = 6,   /* input outside the implemented scope (hanging nodes, ...) */
  CDGPU_ERR_PATTERN = 7,       /* a cell coupling is missing from the given CSR pattern */
  CDGPU_ERR_NO_DEVICE = 8      /* no CUDA device */
};

/* discretisation types, include/General/Constants.h:188-190 */
#define CDGPU_GALERKIN 1
#define CDGPU_SUPG 2
/* the mass-matrix form of the time-dependent system (MatrixMRhsAssemble,
 * src/FE/ConvDiff2D.C:411, src/FE/TCD3D.C:11): M_ij = (phi_j, phi_i), rhs_i = (f, phi_i) */
#define CDGPU_MASS 10

/* coefficient kinds: how BilinearCoeffs (Examples/CD_2D, CD_3D) is evaluated */
#define CDGPU_COEFF_CONSTANT 0 /* eps, b, c, f constant in space */
#define CDGPU_COEFF_SINE 1     /* Examples/CD_2D/SineLaplace.h: f = 2 pi^2 eps sin(pi x) sin(pi y) */
#define CDGPU_COEFF_ROTATING 2 /* b = (0.5 - y, x - 0.5), eps, c, f constant (TCD2D config) */
#define CDGPU_COEFF_TABLE 3    /* host-evaluated record per cell and quadrature point */

typedef struct cdgpu_coeffs
{
  int kind;        /* CDGPU_COEFF_* */
  int poly_degree; /* INTERNAL_POLYNOMIAL_DEGREE used by the SUPG parameter (reference default 1) */
  double eps;      /* diffusion, coeff[0] */
  double b1, b2, b3; /* convection, coeff[1..2] (2D) / [1..3] (3D) */
  double c;        /* reaction */
  double f;        /* source */
  double delta0;   /* DELTA0 (src/General/Database.C:456, default 1) */
} cdgpu_coeffs;

/* multigrid / Krylov parameters, named after the reference's ParamDB keys
 * (defaults src/General/Database.C:639-760) */
typedef struct cdgpu_solver_params
{
  int solver;          /* SC_SOLVER_SCALAR: 16 FGMRES (flexible), 11 fixed point */
  int restart;         /* SC_GMRES_RESTART */
  int maxit;           /* SC_LIN_MAXIT_SCALAR */
  int minit;           /* SC_MINIT */
  int smoother;        /* SC_SMOOTHER_SCALAR: 1 damped Jacobi (only value implemented on the GPU) */
  int coarse_smoother; /* SC_COARSE_SMOOTHER_SCALAR: 1 Jacobi, 3 SSOR, 17 exact (dense FP64) */
  int pre, post;       /* SC_PRE_SMOOTH_SCALAR, SC_POST_SMOOTH_SCALAR */
  int coarse_maxit;    /* SC_COARSE_MAXIT_SCALAR */
  int cycle;           /* SC_MG_CYCLE_SCALAR: 1 V, 2 W, 0 F */
  int slc;             /* SC_STEP_LENGTH_CONTROL_ALL_SCALAR (must be 0 on the GPU) */
  int precision;       /* 0: FP64 multigrid (drop-in); 1: FP32 multigrid inside FP64 FGMRES */
  int stop_rule;       /* 0: the reference's rule, red_factor relative to the residual at the last
                          restart (FgmresIte.C:430-431, 557); 1: red_factor relative to the initial
                          residual of the solve (no counterpart in the reference) */
  int pad_;
  double red_factor;   /* SC_LIN_RED_FACTOR_SCALAR */
  double res_norm_min; /* SC_LIN_RES_NORM_MIN_SCALAR */
  double div_factor;   /* SC_DIV_FACTOR */
  double omega;        /* SC_SMOOTH_DAMP_FACTOR_SCALAR */
  double coarse_red;   /* SC_COARSE_RED_FACTOR_SCALAR */
  double gmg_damp;     /* SC_GMG_DAMP_FACTOR_SCALAR */
} cdgpu_solver_params;

typedef struct cdgpu_solve_info
{
  int iterations;        /* the value TFgmresIte::Iterate / TFixedPointIte::Iterate returns */
  int status;            /* CDGPU_OK, CDGPU_ERR_NOT_CONVERGED or CDGPU_ERR_DIVERGED */
  double initial_residual;
  double final_residual; /* |s_{i+1}| (FGMRES) or ||f - A x|| (fixed point) at exit */
} cdgpu_solve_info;

typedef struct cdgpu_ctx cdgpu_ctx;

/* --- context ------------------------------------------------------------- */
/* No reference counterpart (the reference is a process-wide CPU library).   */
int cdgpu_create(cdgpu_ctx **ctx, int device);
void cdgpu_destroy(cdgpu_ctx *ctx);
const char *cdgpu_status_string(int status);
const char *cdgpu_last_error(const cdgpu_ctx *ctx);
/* the cudaStream_t all work of this context is issued on, as an integer handle */
unsigned long long cdgpu_stream(const cdgpu_ctx *ctx);
/* number of kernels this context has launched so far */
long long cdgpu_kernel_launches(const cdgpu_ctx *ctx);

/* --- finite element space -------------------------------------------------
 * Replaces the data TFESpace2D/TFESpace3D hands to the assembler
 * (include/FE/FESpace.h:135-197: GetGlobalNumbers, GetBeginIndex,
 * GetActiveBound, GetHangingBound, GetN_Dirichlet) plus the cell vertices
 * (TBaseCell::GetVertex, include/Geometry/BaseCell.h:165).
 * h_vert: n_cells x (4|8) x dim doubles, cell vertices in the reference's
 * counter-clockwise order; h_global_numbers / h_begin_index as in TFESpace;
 * DOFs ordered [active | Dirichlet].  Hanging nodes are not supported
 * (hanging_bound must equal n_active). */
int cdgpu_upload_space(cdgpu_ctx *ctx, int dim, int order, int n_cells, const double *h_vert,
                       const int *h_global_numbers, const int *h_begin_index, int n_dof,
                       int n_active, int hanging_bound, int *space_id);

/* --- matrix structure ------------------------------------------------------
 * Replaces TSquareStructure2D/3D(TFESpace*) + TSquareStructure::Sort()
 * (src/FE/SquareStructure3D.C:32, SquareStructure2D.C:46, SquareStructure.C:65):
 * builds the CSR pattern from the space's DOF map (bit-identical to the
 * reference's), or takes the host's own RowPtr/KCol.  *nnz receives the count. */
int cdgpu_build_pattern(cdgpu_ctx *ctx, int space_id, int *nnz);
int cdgpu_upload_pattern(cdgpu_ctx *ctx, int space_id, const int *h_row_ptr, const int *h_kcol,
                         int nnz);
/* The same pattern as cdgpu_build_pattern, built on the device (one warp per row sorts the
 * DOFs of the row's cells; row lengths, a scan, then the columns), for callers that set up
 * many meshes (a request loop's new mesh sizes).  Bit-identical to the host build, which it
 * falls back to for rows with more than 512 candidate columns. */
int cdgpu_build_pattern_device(cdgpu_ctx *ctx, int space_id, int *nnz);
int cdgpu_get_pattern(cdgpu_ctx *ctx, int space_id, int *h_row_ptr, int *h_kcol);

/* --- coefficients ----------------------------------------------------------
 * Replaces the CoeffFct2D/CoeffFct3D callback (include/General/Constants.h:120-125)
 * bound by TDiscreteForm2D/3D.  h_table (kind CDGPU_COEFF_TABLE only):
 * n_cells x n_quad x 6 doubles (eps, b1, b2, b3, c, f) at the assembly's
 * quadrature points, see cdgpu_quadrature_points. */
int cdgpu_set_coeffs(cdgpu_ctx *ctx, int space_id, const cdgpu_coeffs *coeffs,
                     const double *h_table);
/* quadrature points (physical coordinates, n_cells x n_quad x dim) at which a
 * CDGPU_COEFF_TABLE must be evaluated; *n_quad receives the points per cell. */
int cdgpu_quadrature_points(cdgpu_ctx *ctx, int space_id, double *h_xyz, int *n_quad);

/* --- error evaluation ---------------------------------------------------------
 * Replaces TFEFunction2D::GetErrors (src/FE/FEFunction2D.C:73) for the exact solution of
 * the SineLaplace example, u = sin(pi x) sin(pi y) (Examples/CD_2D/SineLaplace.h:27-30):
 * *l2 = ||u_h - u||_L2, *h1semi = |u_h - u|_H1 with the assembly's Gauss rule on every cell,
 * computed on the device.  h_sol: the full solution vector (n_dof values).  Only 2D spaces
 * whose coefficients are of kind CDGPU_COEFF_SINE have this exact solution; others return
 * CDGPU_ERR_UNSUPPORTED. */
int cdgpu_errors(cdgpu_ctx *ctx, int space_id, const double *h_sol, double *l2, double *h1semi);
/* The same errors against any exact solution, for the MEASURE_ERRORS branch of the mains
 * (TFEFunction3D::GetErrors with L2H1Errors, src/FE/FEFunction3D.C:57; 2D FEFunction2D.C:73):
 * the host tabulates the example's Exact() at the points of cdgpu_quadrature_points,
 * h_exact = n_cells x n_quad x (1 + dim) doubles (u, du/dx, du/dy[, du/dz]); the device
 * evaluates u_h and grad u_h there and sums w |det J| (u_h - u)^2 and |grad(u_h - u)|^2.
 * h_sol: the full solution (n_dof values).  2D and 3D, Q1 and Q2. */
int cdgpu_errors_table(cdgpu_ctx *ctx, int space_id, const double *h_sol, const double *h_exact, double *l2,
                       double *h1semi);

/* --- output ------------------------------------------------------------------
 * Replaces TOutput3D::WriteVtk / TOutput2D::WriteVtk (src/FE/Output3D.C:1747) for one scalar
 * function: legacy ASCII VTK with the mesh vertices, the cells and the function's vertex
 * values (name: the SCALARS name, NULL = "u").  sol: n_dof values on the device
 * (sol_on_device = 1, e.g. a batch or device solve's result) or on the host.  The vertices are
 * numbered in ascending order of their DOFs (the reference numbers them by vertex address, so
 * the files list the same points and values in another order). */
int cdgpu_write_vtk(cdgpu_ctx *ctx, int space_id, const double *sol, int sol_on_device, const char *path,
                    const char *name);

/* --- assembly ---------------------------------------------------------------
 * Replaces TSystemCD3D::Assemble / TAssembleMat3D::Reset + Assemble3D
 * (src/System/SystemCD3D.C:314-339, src/System/AssembleMat3D.C:230-505) and
 * TSystemCD2D::Assemble / Assemble2D (src/System/SystemCD2D.C:125-179,
 * src/FE/Assemble2D.C:33-1206): local Galerkin (ConvDiff2D.C:32, ConvDiff3D.C:61)
 * or SUPG (ConvDiff2D.C:96, ConvDiff3D.C:124) forms, scattered into the CSR
 * entries; Dirichlet rows become identity rows whose right-hand side is the
 * boundary value.  The matrix and right-hand side stay on the device;
 * h_entries / h_rhs (nullable) receive copies like TSquareMatrix::GetEntries().
 * h_dirichlet: values of DOFs [n_active, n_dof) (BoundValue at the nodes), NULL = 0. */
int cdgpu_assemble(cdgpu_ctx *ctx, int space_id, int disctype, const double *h_dirichlet,
                   double *h_entries, double *h_rhs);
/* Neumann boundary data: adds sum_q |J_q| w_q g_q phi_k(x_q) to active rows, like the
 * NEUMANN branch of Assemble2D (src/FE/Assemble2D.C:797-827) and the NEUMANN / ROBIN branch of
 * TAssembleMat3D::Assemble3D (src/System/AssembleMat3D.C:1068-1170).  2D: per edge its cell,
 * local edge m (vertices m, m+1) and g at the (order+1) Gauss points from vertex m; 3D: per face
 * its cell, local face m (THexahedron's face-vertex table) and g at the (order+1)^2 Gauss points
 * of the face, in the order cdgpu_boundary_points lists them.  h_rhs (nullable) receives the
 * updated right-hand side. */
int cdgpu_add_neumann(cdgpu_ctx *ctx, int space_id, int n_edges, const int *h_cell,
                      const int *h_local_edge, const double *h_g, double *h_rhs);
/* physical coordinates (n x points x dim) of the Gauss points of boundary edges (2D) or faces
 * (3D) at which cdgpu_add_neumann expects g (the points where the reference calls BoundValue) */
int cdgpu_boundary_points(cdgpu_ctx *ctx, int space_id, int n, const int *h_cell, const int *h_local, double *h_xyz);

/* --- matrix-vector products -------------------------------------------------
 * Replace MatVect / MatVect_Scalar and ScalarDefect / Defect_Scalar
 * (src/FE/Blas2.C:11-99) on the assembled matrix of a space. */
int cdgpu_spmv(cdgpu_ctx *ctx, int space_id, const double *h_x, double *h_y);
int cdgpu_defect(cdgpu_ctx *ctx, int space_id, const double *h_x, const double *h_f, double *h_d,
                 double *res);
int cdgpu_spmv_device(cdgpu_ctx *ctx, int space_id, const double *d_x, double *d_y);
/* The FP64 product, defect and Jacobi sweep of a matrix larger than L2 stream its tiles into
 * shared memory with bulk copies; the tile shape (nonzeros per tile, pipeline stages, CTAs
 * per SM) is chosen by timing every variant on the matrix at the first solve that uses it.
 * This copies a one-line report of that choice (or "not tuned yet") into buf.  No reference
 * counterpart (MatVect / Defect, src/FE/Blas2.C:11-99, are the operations). */
int cdgpu_product_tuning(cdgpu_ctx *ctx, int space_id, char *buf, int len);
/* y = A x with an FP32 form of the assembled operator, the forms the mixed multigrid cycle
 * applies (TMGLevel3D's MatVect/Defect on the FP32 levels, src/FE/MGLevel3D.C:194-252):
 * form 0 the FP32 copy of the CSR entries; 1 the matrix-free per-cell products
 * A_c x_c = sum_t coef_{c,t} R_t x_c on CUDA cores; 2 the same products on the tensor cores
 * (tcgen05, TF32 inputs, FP32 accumulation).  Dirichlet rows are identity rows.  Forms 1 and 2
 * need Q2 hexahedra assembled from affine cells with constant coefficients
 * (CDGPU_ERR_UNSUPPORTED otherwise).  h_x, h_y: host arrays of n_dof floats. */
int cdgpu_apply_fp32(cdgpu_ctx *ctx, int space_id, int form, const float *h_x, float *h_y);
/* y = A x with an FP64 form of the assembled operator (MatVect, src/FE/Blas2.C:11-99):
 * form 0 the CSR entries (what cdgpu_spmv applies); 1 the matrix-free sum-factorised per-cell
 * products A_c x_c = sum_t coef_{c,t} R_t x_c, values and gradients at the 3 x 3 x 3 Gauss
 * points by one-dimensional passes, the form the mixed solve (precision 1) applies in its
 * FGMRES iteration on a finest level of at least 16,384 such cells.  Equal to form 0 up to
 * rounding; Dirichlet rows are identity rows.  Form 1 needs Q2 hexahedra assembled from affine
 * cells with constant coefficients (CDGPU_ERR_UNSUPPORTED otherwise).  h_x, h_y: host arrays
 * of n_dof doubles. */
int cdgpu_apply_fp64(cdgpu_ctx *ctx, int space_id, int form, const double *h_x, double *h_y);
/* The same on device vectors of n_dof doubles, enqueued on the context's stream (no
 * synchronisation; like cdgpu_spmv_device). */
int cdgpu_apply_fp64_device(cdgpu_ctx *ctx, int space_id, int form, const double *d_x, double *d_y);
/* The defect d = f - A x and *h_res = ||d||, like cdgpu_defect, for callers that cannot
 * allocate device memory (for example while another allocator holds the whole device, or
 * where the device synchronisation of cudaFree is not acceptable).  No counterpart in the
 * reference.  d_x, d_f, d_d: device vectors of the space's length; h_res: host (nullable).
 * Allocates nothing: the partial sums live in a fixed 32 KB array of the library, so at most
 * 8,388,608 rows (CDGPU_ERR_UNSUPPORTED beyond).  cdgpu_create looks up that array's address
 * on its device (which, under lazy module loading, also loads it), so create the context
 * before another allocator takes the device; if that lookup failed, the first call repeats it
 * and should then come before any stream capture.  Calls that overlap on the GPU share the
 * array and race. */
int cdgpu_defect_noalloc(cdgpu_ctx *ctx, int space_id, const double *d_x, const double *d_f,
                         double *d_d, double *h_res);

/* --- multigrid hierarchy ------------------------------------------------------
 * Replaces TMultiGrid3D/TMultiGrid2D + AddLevel(TMGLevel) (src/System/SystemCD3D.C:
 * 147-151, 295-308) and the cell-wise transfer operators Prolongate /
 * DefectRestriction (src/FE/MGComponents3D.C:182-988, MGComponents2D.C:118-1022),
 * which are built here once as sparse matrices.  space_ids: coarsest first;
 * h_parent[l] (l >= 1): for each cell of level l, its parent cell on level l-1
 * (TBaseCell::GetParent); h_parent[0] is ignored. */
int cdgpu_hierarchy(cdgpu_ctx *ctx, int n_levels, const int *space_ids, const int *const *h_parent,
                    int *mg_id);

/* --- solve -----------------------------------------------------------------
 * Replaces TSystemCD3D::Solve (GMG branch, src/System/SystemCD3D.C:342-368):
 * TFgmresIte (src/FE/FgmresIte.C:219-582) or TFixedPointIte (FixedPointIte.C:150)
 * preconditioned by one TMultiGridScaIte cycle (MultiGridScaIte.C:63-104) of
 * TMultiGrid3D::Cycle (src/FE/MultiGrid3D.C:423-669).  Uses the finest level's
 * assembled matrix.  h_sol: initial guess in, solution out. */
int cdgpu_solve(cdgpu_ctx *ctx, int mg_id, const cdgpu_solver_params *params, const double *h_rhs,
                double *h_sol, cdgpu_solve_info *info);
/* same with device vectors (length n_dof of the finest level) */
int cdgpu_solve_device(cdgpu_ctx *ctx, int mg_id, const cdgpu_solver_params *params,
                       const double *d_rhs, double *d_sol, cdgpu_solve_info *info);
/* assemble every level of a hierarchy, as TSystemCD3D::Assemble loops over all levels
 * (src/System/SystemCD3D.C:314-339).  disctype is used on the finest level,
 * coarse_disctype on the others (the reference uses one DISCTYPE for all levels; a SUPG
 * coarse-grid operator under a Galerkin fine level only changes the preconditioner).
 * The device-side checks of an assembly (every cell coupling present in the pattern, rows
 * within the kernel's length) depend on the pattern only, so the call waits for the device
 * and reports them on the first assembly of each level's pattern; later calls return as
 * soon as the work is enqueued on the library's stream. */
int cdgpu_assemble_hierarchy(cdgpu_ctx *ctx, int mg_id, int disctype, int coarse_disctype);
/* copy of a space's assembled right-hand side (n_dof values), the rhs array that
 * TSystemCD3D::Assemble leaves on the host (src/System/SystemCD3D.C:314-339); waits for the
 * device */
int cdgpu_get_rhs(cdgpu_ctx *ctx, int space_id, double *h_rhs);
/* device pointer of the assembled right-hand side of a space */
int cdgpu_rhs_device(cdgpu_ctx *ctx, int space_id, double **d_rhs);

/* --- time-dependent problems (theta schemes) --------------------------------
 * Replace TSystemTCD2D (src/System/SystemTCD2D.C): the constructor (mass and stiffness
 * matrices on the hierarchy's levels), AssembleMRhs (94-123), AssembleARhs (124-153) and
 * one step of AssembleSystMat + Solve + RestoreMassMat (154-235) as called by the time
 * loop of 2DPrograms/TCD2D_ParMooN.C:241-290.  The mass matrix is updated in place like
 * the reference's, so every step rounds like the reference.  The solve is the multigrid
 * FGMRES of cdgpu_solve on the system matrices M + tau*theta1*A of every level.
 * cdgpu_tcd_assemble_stiffness first saves the current right-hand side as the old one
 * (the time loop's memcpy(oldrhs, rhs)).  Galerkin forms only.  On a 3D hierarchy the
 * steps follow TSystemTCD3D (src/System/SystemTCD3D.C:228-305, 3DPrograms/TCD3D_ParMooN.C):
 * M - tau*theta2*A is formed on the finest level only and the coarser levels' system
 * matrices are M + tau*theta1*A. */
int cdgpu_tcd_create(cdgpu_ctx *ctx, int mg_id, int disctype, int *tcd_id);
int cdgpu_tcd_assemble_mass(cdgpu_ctx *ctx, int tcd_id);
int cdgpu_tcd_assemble_stiffness(cdgpu_ctx *ctx, int tcd_id);
int cdgpu_tcd_step(cdgpu_ctx *ctx, int tcd_id, const cdgpu_solver_params *params, double tau,
                   double theta1, double theta2, double theta3, double theta4, double *h_sol,
                   cdgpu_solve_info *info);
int cdgpu_tcd_step_device(cdgpu_ctx *ctx, int tcd_id, const cdgpu_solver_params *params, double tau,
                          double theta1, double theta2, double theta3, double theta4, double *d_sol,
                          cdgpu_solve_info *info);
int cdgpu_tcd_rhs(cdgpu_ctx *ctx, int tcd_id, double *h_rhs);
/* Dirichlet values (n_dof - n_active values of the finest level, BoundValue at the DOFs at
 * the current time) that the following cdgpu_tcd_assemble_mass / _stiffness calls put into
 * the right-hand side, as the reference's assembly evaluates BoundValue at CURRENTTIME
 * (src/System/SystemTCD3D.C:176-226 through Assemble3D); NULL = zero values (the default).
 * The values are copied. */
int cdgpu_tcd_set_dirichlet(cdgpu_ctx *ctx, int tcd_id, const double *h_dirichlet);
/* copies (nnz values of level `level`, 0 = coarsest; each pointer nullable) of the mass matrix
 * M as updated in place by the steps, the stiffness matrix A, and the system matrix the last
 * step solved with: the sqmatrixM / sqmatrixA members of TSystemTCD2D / TSystemTCD3D
 * (include/System/SystemTCD2D.h, SystemTCD3D.h) after RestoreMassMat. */
int cdgpu_tcd_matrices(cdgpu_ctx *ctx, int tcd_id, int level, double *h_M, double *h_A, double *h_S);

/* --- batched solves and serving ---------------------------------------------
 * No single reference function: the reference solves one system per process
 * (TSystemCD2D/3D::Solve).  A batch runs many independent solves of the GMG-FGMRES kind of
 * cdgpu_solve at once: every kernel launch of an FGMRES iteration serves all running
 * instances (grouped launches, one thread block range per instance), and the FGMRES
 * control (Givens rotations, stopping tests, restarts) runs on the device per instance, so
 * instances at different iterations, of different sizes, orders and dimensions share the
 * launches.  Instances can be submitted while others run (they start at the next
 * iteration) and released when done, which is how a request loop admits new solves as
 * memory frees up.
 *
 * The mesh structure (pattern, transfer operators, colour classes) comes from a hierarchy
 * built with cdgpu_hierarchy and is shared by every instance that names it; each instance
 * owns its coefficients, matrices on every level (FP64 and FP32), multigrid vectors and
 * Krylov workspace.  The multigrid cycle runs in FP32 inside FP64 FGMRES (the mixed form of
 * cdgpu_solve) with the exact FP64 coarse solve.  params->smoother: 1 damped Jacobi
 * (MGLevel3D.C:443), 2 multicolour SOR, 3 multicolour SSOR (the colouring is a greedy
 * colouring of the matrix graph, so SOR/SSOR sweep the rows colour by colour rather than in
 * the reference's lexicographic order).  params->coarse_smoother must be 17 (exact).
 * stop_rule, red_factor, res_norm_min, maxit, restart (<= 32) as for cdgpu_solve. */
int cdgpu_batch_create(cdgpu_ctx *ctx, const cdgpu_solver_params *params, int *batch_id);
/* add one instance: coefficients co on every level of hierarchy mg_id, assembled with
 * disctype on the finest level and coarse_disctype on the others (Dirichlet values 0),
 * initial guess 0; the instance joins at the next cdgpu_batch_advance.  *slot identifies
 * it until cdgpu_batch_release. */
int cdgpu_batch_submit(cdgpu_ctx *ctx, int batch_id, int mg_id, const cdgpu_coeffs *co, int disctype,
                       int coarse_disctype, int *slot);
/* run up to `iterations` FGMRES iterations of every running instance; *running (nullable)
 * = instances still running afterwards.  The iterations run in a device-side loop: one CUDA
 * graph per running set whose WHILE node repeats an iteration of every running solve until
 * all have finished or `iterations` are done, so one call is one graph launch and one wait. */
int cdgpu_batch_advance(cdgpu_ctx *ctx, int batch_id, int iterations, int *running);
/* how cdgpu_batch_advance ran: *mode (nullable) 1 = device-side loop, 2 = device-side loop
 * without programmatic dependent launch inside the loop body (a driver that refused it),
 * 0 = host loop (a driver without conditional graph nodes), -1 = not yet run;
 * *graph_launches, *host_iterations (nullable) = advance calls run as one graph launch,
 * iterations launched from the host loop. */
int cdgpu_batch_loop_info(cdgpu_ctx *ctx, int batch_id, int *mode, long long *graph_launches,
                          long long *host_iterations);
/* a time-dependent instance (theta scheme, as cdgpu_tcd_* per instance, SystemTCD2D.C:
 * 154-235): mass matrix M and stiffness matrix A (disctype, every level) with coefficients
 * co, system matrices M + tau*theta1*A on every level and K = M - tau*theta2*A on the finest,
 * formed in the reference's order of in-place updates; h_u0 = initial solution (n_dof
 * values; its Dirichlet entries are replaced by the boundary values).  The coefficients are
 * constant in time, so f_old = f.  The instance idles until cdgpu_batch_tcd_step. */
int cdgpu_batch_submit_tcd(cdgpu_ctx *ctx, int batch_id, int mg_id, const cdgpu_coeffs *co, int disctype,
                           double tau, double theta1, double theta2, double theta3, double theta4,
                           const double *h_u0, int *slot);
/* one time step of every time-dependent instance of the batch: right-hand side
 * tau*theta3*f_old + tau*theta4*f + K u_old, then FGMRES from u_old to the batch's stopping
 * rule.  The step is one CUDA graph (captured on the first step, replayed while the batch's
 * instances are unchanged): the right-hand sides, then the device-side iteration loop of
 * cdgpu_batch_advance until every solve has finished (at most maxit + 1 iterations).  A
 * driver without conditional graph nodes gets a graph of the right-hand sides and `iterations`
 * FGMRES iterations, and solves that need more continue in rounds of `iterations`.
 * *max_iterations (nullable) = the iterations the slowest instance was given. */
int cdgpu_batch_tcd_step(cdgpu_ctx *ctx, int batch_id, int iterations, int *max_iterations);
/* current solution of a time-dependent instance (same as cdgpu_batch_fetch) */
int cdgpu_batch_tcd_solution(cdgpu_ctx *ctx, int batch_id, int slot, double *h_sol, cdgpu_solve_info *info);
/* slots that finished since the last poll (at most max_slots; *count = how many) */
int cdgpu_batch_poll(cdgpu_ctx *ctx, int batch_id, int *slots, int max_slots, int *count);
/* solution (finest level, n_dof values) and statistics of a finished instance */
int cdgpu_batch_fetch(cdgpu_ctx *ctx, int batch_id, int slot, double *h_sol, cdgpu_solve_info *info);
/* free an instance's device memory (finished or not); the slot number may be reused */
int cdgpu_batch_release(cdgpu_ctx *ctx, int batch_id, int slot);
/* device bytes held by the batch's instances (for admission under a memory budget) */
int cdgpu_batch_memory(cdgpu_ctx *ctx, int batch_id, unsigned long long *bytes);
/* device bytes one instance on hierarchy mg_id would take */
int cdgpu_batch_instance_bytes(cdgpu_ctx *ctx, int batch_id, int mg_id, unsigned long long *bytes);

#ifdef __cplusplus
}
#endif

#endif /* CDGPU_H */
