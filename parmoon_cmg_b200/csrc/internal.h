// Internal declarations of libcdgpu (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cdgpu.h"

#define CD_MAXBF 27   // Q2 hexahedron
#define CD_MAXQ 64    // Gauss4 on hexahedra
#define CD_MAXT 14    // reference tensors of the affine fast path
#define CD_MAXROW 128 // longest CSR row of a conforming Q2 hexahedral mesh is 125

// ---------------------------------------------------------------------------
// reference element: tensor-product Lagrange basis, Gauss rules, reference tensors
// ---------------------------------------------------------------------------
struct RefElement
{
  int dim = 0, order = 0, nbf = 0, nq = 0, nv = 0;
  std::vector<double> qx, qw;          // nq x dim, nq
  std::vector<double> phi, dphi, hphi; // nq x nbf, nq x nbf x dim, nq x nbf x dim x dim
};
void make_ref_element(int dim, int order, RefElement &re);
void basis_eval(int dim, int order, const double *xi, double *val, double *grad);
int n_tensors(int dim, int disctype);
int n_rhs_tensors(int dim, int disctype);
// R[(i*nbf + j)*T + t] and r[i*Tr + t]
void reference_tensors(const RefElement &re, int disctype, std::vector<double> &R,
                       std::vector<double> &r);

// ---------------------------------------------------------------------------
// launch shape of the CSR kernels of a matrix (csr.cuh): gs threads per row, each issuing
// up to 8 (16 when gs = 8) loads of the row at once; set from the longest row
// ---------------------------------------------------------------------------
struct CsrShape
{
  int gs = 8;
};
CsrShape csr_shape(const int *row_ptr, int n_rows);

// ---------------------------------------------------------------------------
// finite element space with its matrix
// ---------------------------------------------------------------------------
struct Space
{
  int dim = 0, order = 0, nbf = 0, nv = 0, n_cells = 0, n_dof = 0, n_active = 0;
  std::vector<double> h_coords;
  std::vector<int> h_gn;
  bool all_affine = true;
  double *d_coords = nullptr;
  int *d_gn = nullptr;
  // CSR pattern (bit-identical to TSquareStructure + Sort)
  long nnz = -1;
  std::vector<int> h_row_ptr, h_kcol;
  int *d_row_ptr = nullptr, *d_kcol = nullptr;
  int *d_dir_start = nullptr; // first slot of each row whose column is a Dirichlet DOF
  int *d_dir_rows = nullptr;  // the active rows that have Dirichlet columns
  int n_dir_rows = 0;
  CsrShape shape;
  // tiles of the bulk-copy (TMA) FP64 product (csr.cuh, csr_tma_kernel): tile t covers rows
  // [d_tiles[t].x, d_tiles[t+1].x) and nonzeros from d_tiles[t].y; n_tiles = 0 when the matrix
  // keeps the plain CSR kernels (small, or a row longer than a tile)
  int2 *d_tiles = nullptr;
  int n_tiles = 0;
  // the variant of the TMA product chosen by the autotuner on the first assembly of this
  // pattern (index into the variant table of solve.cu; -1 = not tuned yet) and its report
  int tma_var = -1;
  int tma_ctas = 0; // resident CTAs per SM of the chosen variant
  // assembly_version at the last bulk-copy launch that waited for its predecessor before
  // streaming the matrix: later launches of the same assembly may stream it before their wait
  mutable long tma_safe_version = -1;
  std::string tma_report;
  // DOF -> (cell, local index) incidence, ascending cell per DOF
  int *d_inc_ptr = nullptr, *d_inc = nullptr;
  // slot map of the row gather: for incidence t of an active row and local column j, the
  // position of column gn[cell][j] within the row (rows are at most CD_MAXROW long); built
  // from the pattern on the first assembly
  unsigned char *d_slot = nullptr;
  long slot_pattern = -1; // nnz of the pattern the slot map was built for
  bool pattern_checked = false; // an assembly with this pattern passed the device-side checks
  // values
  double *d_a = nullptr, *d_rhs = nullptr, *d_diag = nullptr;
  float *d_a32 = nullptr, *d_diag32 = nullptr;
  bool assembled = false;
  long assembly_version = 0;
  // coefficients
  cdgpu_coeffs co{};
  bool co_set = false;
  double *d_tab = nullptr;
  // assembly scratch
  double *d_cellcoef = nullptr; // affine path: n_cells x (T + Tr)
  // matrix-free FP32 operator for the FP32 multigrid cycle (mf.cuh), available after an
  // affine constant-coefficient assembly: mf_T = its number of reference tensors (0: none)
  int mf_T = 0;
  long mf_version = -1;         // assembly the FP32 copies were made from
  float *d_cf32 = nullptr;      // n_cells x T cell coefficients
  float *d_R32 = nullptr;       // T x nbf x nbf reference tensors, [t][i][j]
  float *d_R32img = nullptr;    // the tensor-core kernel's B operand as its shared-memory image
  float *d_ybuf = nullptr;      // nbf x n_cells per-cell products
  // matrix-free FP64 operator (mf64.cuh) of the mixed form's FGMRES products: nbf x n_cells
  // per-cell products, and the assembly at the last launch that waited for its predecessor
  // before reading the cell data (later launches of that assembly may read it before the wait)
  double *d_ybuf64 = nullptr;
  mutable long mf64_safe_version = -1;
  // the active rows' incidences as 8-wide records of per-cell-buffer indices (mf.cuh,
  // mf_inc8_kernel); null when not built or when a row has more than 8 cells
  int *d_inc8 = nullptr;
  bool inc8_tried = false;
  double *d_local = nullptr;    // quadrature path: n_cells x (nbf*nbf + nbf)
  double *d_dir = nullptr;      // Dirichlet values
  double *d_ref = nullptr;      // reference tensors (affine path)
  double *d_quadtab = nullptr;  // reference-element tables (quadrature path)
  int ref_disctype = -1;
  int n_tab = 0;
  RefElement re;                // reference element of (dim, order), built on first use
  bool re_ready = false;
};

// ---------------------------------------------------------------------------
// multigrid hierarchy
// ---------------------------------------------------------------------------
template <typename T> struct LevelVec
{
  T *sol = nullptr, *alt = nullptr, *rhs = nullptr, *def = nullptr;
};

struct Level
{
  Space *sp = nullptr;
  // prolongation from the next coarser level (rows = this level's DOFs) and its transpose
  int *d_p_row = nullptr, *d_p_col = nullptr, *d_r_row = nullptr, *d_r_col = nullptr;
  double *d_p_val = nullptr, *d_r_val = nullptr;
  float *d_p_val32 = nullptr, *d_r_val32 = nullptr;
  long p_nnz = 0;
  CsrShape p_shape, r_shape;
  // colour classes of the active rows (greedy distance-1 colouring of the matrix graph) for
  // the multicolour SOR/SSOR smoothers of the batched solver: rows of colour c are
  // d_color_rows[h_color_ptr[c] .. h_color_ptr[c+1])
  int n_colors = -1;
  std::vector<int> h_color_ptr;
  int *d_color_rows = nullptr;
  LevelVec<double> v64, c64; // working pointers (ping-pong swapped) and their initial assignment
  LevelVec<float> v32, c32;
};

struct Hierarchy
{
  std::vector<Level> lev;
  double *d_cinv = nullptr; // explicit inverse of the coarsest matrix (exact coarse solve)
  int *d_cpiv = nullptr;    // pivots of its Gauss-Jordan inversion + error flag
  long cinv_version = -1;
  // FGMRES workspace
  int m = 0;
  double *d_V = nullptr, *d_Z = nullptr, *d_w = nullptr, *d_ctl = nullptr, *d_partial = nullptr;
  double *h_ctl = nullptr; // pinned mirror of the control block
  int partial_blocks = 0;
  double *d_x = nullptr, *d_b = nullptr; // host-API staging vectors
  // captured multigrid cycle per precision (0 FP64, 1 FP32) and its in/out pointer slot
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  unsigned mf_mask = 0; // levels whose FP32 cycle in gexec[1] uses the matrix-free operator
  // the running solve applies the finest operator matrix-free in FP64 (mixed form, Q2
  // hexahedra from the affine constant-coefficient assembly), not from the CSR entries
  bool mf64 = false;
  cdgpu_solver_params gparams[2] = {};
  long long graph_nodes[2] = {0, 0};
  double **d_io = nullptr;
  double **h_io = nullptr; // pinned ring of 64 (in, out) pairs
  unsigned io_slot = 0;
  double *h_slot = nullptr;            // pinned: two slots of an FGMRES iteration's control block
  cudaEvent_t ev_slot[2] = {nullptr, nullptr}; // recorded behind each slot's copy
  // the slots' copies run on their own stream, after the iteration's Gram-Schmidt passes
  // (ev_ready) and beside the rest of the iteration; ev_beta: the initial residual's copy
  cudaStream_t cstream = nullptr;
  cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_beta = nullptr;
  // side stream of the hierarchy's assembly: the coarse levels (and the exact coarse inverse,
  // once a solve has used it) are assembled there beside the finest level
  cudaStream_t astream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int *h_cflag = nullptr;     // pinned copy of the coarse inversion's zero-pivot flag
  bool cflag_pending = false; // copy enqueued, not yet checked
  unsigned *d_gs_count = nullptr; // arrival counter of the Gram-Schmidt passes' last-block reduction
};

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct Tcd; // time-dependent system (tcd.cu)
void free_tcd(Tcd *t);
struct Batch; // batched solves (batch.cu)
void free_batch(Batch *b);

struct cdgpu_ctx
{
  std::vector<Tcd *> tcds;
  std::vector<Batch *> batches;
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  std::string err;
  long long launches = 0;
  std::vector<Space *> spaces;
  std::vector<Hierarchy *> mgs;
  // resident CTAs per SM of kernels launched with a dynamic shared-memory attribute, found
  // once per context (the attribute is set at the same time)
  std::vector<std::pair<const void *, int>> occupancy;
  // set while the multigrid cycle is recorded into its graph: its kernels load the data that
  // no kernel of the cycle writes before waiting for their predecessor
  bool pdl_pre = false;
  bool mf_attr_set = false; // the tensor-core kernel's shared-memory attribute is set
  int *d_err = nullptr; // assembly error flag (device) and its pinned host mirror
  int *h_err = nullptr;
};

// the device error flag (ctx->d_err) and its pinned host mirror, allocated on first use
int ensure_err_flag(cdgpu_ctx *ctx);
// CSR arrays are allocated this many elements longer than the pattern, so that the bulk
// copies of the TMA product may round their end up to a 16-byte boundary
constexpr int kCsrPad = 8;

// error helpers: set ctx->err and return a status
int fail(cdgpu_ctx *ctx, int status, const std::string &msg);
int cuda_fail(cdgpu_ctx *ctx, cudaError_t e, const char *what);
#define CD_CUDA(ctx, call)                                   \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)
#define CD_LAUNCHED(ctx)                                                  \
  do {                                                                    \
    (ctx)->launches++;                                                    \
    cudaError_t e_ = cudaGetLastError();                                  \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, "kernel launch");   \
  } while (0)

// Programmatic dependent launch (sm_90+): a kernel started with cd_launch may be scheduled
// while the previous kernel of the stream (or captured graph) still runs.  Every kernel
// launched that way waits until its predecessor has completed and its memory is visible
// (griddepcontrol.wait) before it reads or writes anything the predecessor may touch, and
// only then lets its own successor be scheduled (griddepcontrol.launch_dependents).  So at
// most two kernels of a chain are resident at once, and the later one runs only the part
// before its wait: the launch, the CTA scheduling and, in kernels of the captured multigrid
// cycle, loads of data that no kernel of the cycle writes (matrices, transfer operators,
// incidence lists, reference tensors).  Without the launch attribute both instructions
// return at once.
#define CD_PDL_WAIT() asm volatile("griddepcontrol.wait;" ::: "memory")
#define CD_PDL_TRIGGER() asm volatile("griddepcontrol.launch_dependents;" ::: "memory")
#define CD_PDL_ENTRY() \
  do {                 \
    CD_PDL_WAIT();     \
    CD_PDL_TRIGGER();  \
  } while (0)

// false while this thread captures a graph whose kernels must not carry programmatic
// dependencies (a conditional node's body, where a driver may refuse them)
inline bool &cd_pdl_enabled()
{
  static thread_local bool on = true;
  return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t cd_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                             Args &&...args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = cd_pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <typename T> int dev_alloc(cdgpu_ctx *ctx, T **p, size_t n)
{
  if (*p) { cudaFree(*p); *p = nullptr; }
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) { *p = nullptr; cudaGetLastError(); return fail(ctx, CDGPU_ERR_OOM, "cudaMalloc failed"); }
  return CDGPU_OK;
}

// host-side setup algorithms (setup.cpp)
void build_pattern(const Space &s, std::vector<int> &row_ptr, std::vector<int> &kcol);
void build_incidence(const Space &s, std::vector<int> &ptr, std::vector<int> &inc);
bool cell_is_affine(int dim, const double *V);
void ref_map(int dim, bool affine, const double *V, const double *xi, double *x, double *J);
double invert(int dim, const double *J, double *Ji);
double cell_diameter(int dim, const double *V);
void build_prolongation(const Space &coarse, const Space &fine, const int *parent,
                        std::vector<int> &row, std::vector<int> &col, std::vector<double> &val);
bool dense_inverse(int n, std::vector<double> &a); // in place, row-major; false if singular

// device entry points (assemble.cu / solve.cu)
// assemble one space; with check = false the error flag is left for assemble_check
int assemble_space(cdgpu_ctx *ctx, Space &s, int disctype, const double *h_dir, bool check = true);
// L2 and H1-semi errors against the SineLaplace solution (2D, coefficient kind SINE)
int space_errors_sine(cdgpu_ctx *ctx, Space &s, const double *d_u, double *l2, double *h1semi);
// the same against an exact solution tabulated at the quadrature points (u and its gradient)
int space_errors_table(cdgpu_ctx *ctx, Space &s, const double *d_u, const double *d_ex, double *l2, double *h1semi);
int assemble_check(cdgpu_ctx *ctx);
int err_flag_status(cdgpu_ctx *ctx);
int add_neumann(cdgpu_ctx *ctx, Space &s, int n_edges, const int *cell, const int *edge,
                const double *g);
void boundary_points(const Space &s, int n, const int *cell, const int *local, double *xyz);
int spmv64(cdgpu_ctx *ctx, const Space &s, const double *x, double *y);
int defect64(cdgpu_ctx *ctx, const Space &s, const double *x, const double *f, double *d,
             double *res);
int setup_hierarchy_buffers(cdgpu_ctx *ctx, Hierarchy &h, int m);
int run_solve(cdgpu_ctx *ctx, Hierarchy &h, const cdgpu_solver_params &p, const double *d_rhs,
              double *d_sol, cdgpu_solve_info *info);
int apply_fp32_form(cdgpu_ctx *ctx, Space &s, int form, const float *d_x, float *d_y);
int apply_fp64_form(cdgpu_ctx *ctx, Space &s, int form, const double *d_x, double *d_y, bool check);
// the explicit inverse of the coarsest level's matrix for the exact coarse solve, when its
// assembly changed since the last inversion (enqueued on ctx->stream)
int refresh_coarse_inverse(cdgpu_ctx *ctx, Hierarchy &h);
// the CSR pattern built on the device (pattern.cu)
int build_pattern_device(cdgpu_ctx *ctx, Space &s, int **d_kcol_out, bool *fallback);
// tiles of the TMA product for a freshly installed pattern (solve.cu)
int build_csr_tiles(cdgpu_ctx *ctx, Space &s);
// the TMA product's variant choice for a space, as text
int csr_tuning_report(cdgpu_ctx *ctx, Space &s, std::string &out);
// looks up the allocation-free defect's scratch array on a device (noalloc.cu)
void noalloc_prepare(int device);
