// C ABI of libcdgpu (declared in include/cdgpu.h).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

int fail(cdgpu_ctx *ctx, int status, const std::string &msg)
{
  if (ctx) ctx->err = msg;
  return status;
}

int cuda_fail(cdgpu_ctx *ctx, cudaError_t e, const char *what)
{
  if (ctx) ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? CDGPU_ERR_OOM : CDGPU_ERR_CUDA;
}

int ensure_err_flag(cdgpu_ctx *ctx)
{
  if (ctx->d_err) return CDGPU_OK;
  int rc = dev_alloc(ctx, &ctx->d_err, 1);
  if (rc) return rc;
  CD_CUDA(ctx, cudaMallocHost((void **)&ctx->h_err, sizeof(int)));
  *ctx->h_err = 0;
  CD_CUDA(ctx, cudaMemset(ctx->d_err, 0, sizeof(int)));
  return CDGPU_OK;
}

static Space *get_space(cdgpu_ctx *ctx, int id)
{
  if (!ctx || id < 0 || id >= (int)ctx->spaces.size()) return nullptr;
  return ctx->spaces[id];
}

static Hierarchy *get_mg(cdgpu_ctx *ctx, int id)
{
  if (!ctx || id < 0 || id >= (int)ctx->mgs.size()) return nullptr;
  return ctx->mgs[id];
}

static void free_space(Space *s)
{
  if (!s) return;
  void *ptrs[] = {s->d_coords, s->d_gn,  s->d_row_ptr, s->d_kcol,     s->d_dir_start, s->d_dir_rows, s->d_slot, s->d_inc_ptr, s->d_tiles,
                  s->d_inc,    s->d_a,   s->d_rhs,     s->d_diag,     s->d_a32,       s->d_diag32,
                  s->d_tab,    s->d_cellcoef, s->d_local, s->d_dir, s->d_ref, s->d_quadtab,
                  s->d_cf32,   s->d_R32, s->d_R32img, s->d_ybuf, s->d_ybuf64, s->d_inc8};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete s;
}

static void free_mg(Hierarchy *h)
{
  if (!h) return;
  for (auto &L : h->lev)
  {
    void *ptrs[] = {L.d_p_row, L.d_p_col, L.d_r_row, L.d_r_col, L.d_p_val, L.d_r_val, L.d_p_val32,
                    L.d_r_val32, L.d_color_rows, L.c64.sol, L.c64.alt, L.c64.rhs, L.c64.def, L.c32.sol, L.c32.alt,
                    L.c32.rhs, L.c32.def};
    for (void *p : ptrs)
      if (p) cudaFree(p);
  }
  for (auto &g : h->gexec)
    if (g) cudaGraphExecDestroy(g);
  void *ptrs[] = {h->d_cinv, h->d_cpiv, h->d_V, h->d_Z, h->d_w, h->d_ctl, h->d_partial, h->d_x, h->d_b,
                  h->d_io, h->d_gs_count};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  if (h->h_io) cudaFreeHost(h->h_io);
  if (h->h_cflag) cudaFreeHost(h->h_cflag);
  if (h->h_slot) cudaFreeHost(h->h_slot);
  for (auto &e : h->ev_slot)
    if (e) cudaEventDestroy(e);
  for (auto &e : h->ev_ready)
    if (e) cudaEventDestroy(e);
  if (h->ev_beta) cudaEventDestroy(h->ev_beta);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->astream) cudaStreamDestroy(h->astream);
  if (h->cstream) cudaStreamDestroy(h->cstream);
  delete h;
}

extern "C" {

int cdgpu_create(cdgpu_ctx **out, int device)
{
  if (!out) return CDGPU_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
  {
    cudaGetLastError();
    return CDGPU_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return CDGPU_ERR_INVALID;
  cdgpu_ctx *ctx = new cdgpu_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return CDGPU_ERR_CUDA; }
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
  {
    delete ctx;
    return CDGPU_ERR_CUDA;
  }
  noalloc_prepare(device);
  *out = ctx;
  return CDGPU_OK;
}

void cdgpu_destroy(cdgpu_ctx *ctx)
{
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto *t : ctx->tcds) free_tcd(t);
  for (auto *b : ctx->batches) free_batch(b);
  for (auto *h : ctx->mgs) free_mg(h);
  for (auto *s : ctx->spaces) free_space(s);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->h_err) cudaFreeHost(ctx->h_err);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char *cdgpu_status_string(int status)
{
  switch (status)
  {
    case CDGPU_OK: return "ok";
    case CDGPU_ERR_INVALID: return "invalid argument";
    case CDGPU_ERR_OOM: return "out of device memory";
    case CDGPU_ERR_CUDA: return "CUDA error";
    case CDGPU_ERR_NOT_CONVERGED: return "solver not converged";
    case CDGPU_ERR_DIVERGED: return "solver diverged";
    case CDGPU_ERR_UNSUPPORTED: return "unsupported input";
    case CDGPU_ERR_PATTERN: return "matrix pattern does not contain a cell coupling";
    case CDGPU_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char *cdgpu_last_error(const cdgpu_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

unsigned long long cdgpu_stream(const cdgpu_ctx *ctx)
{
  return ctx ? (unsigned long long)(uintptr_t)ctx->stream : 0ull;
}

long long cdgpu_kernel_launches(const cdgpu_ctx *ctx) { return ctx ? ctx->launches : 0; }

int cdgpu_upload_space(cdgpu_ctx *ctx, int dim, int order, int n_cells, const double *h_vert,
                       const int *h_gn, const int *h_bi, int n_dof, int n_active, int hanging_bound,
                       int *space_id)
{
  if (!ctx || !space_id || !h_vert || !h_gn || !h_bi) return fail(ctx, CDGPU_ERR_INVALID, "upload_space: null argument");
  if ((dim != 2 && dim != 3) || (order != 1 && order != 2))
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "upload_space: only Q1/Q2 on quadrilaterals and hexahedra");
  if (n_cells <= 0 || n_dof <= 0 || n_active < 0 || n_active > n_dof)
    return fail(ctx, CDGPU_ERR_INVALID, "upload_space: bad sizes");
  if (hanging_bound != n_active) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "upload_space: hanging nodes are not supported");
  cudaSetDevice(ctx->device);
  Space *s = new Space();
  s->dim = dim;
  s->order = order;
  s->nbf = dim == 2 ? (order + 1) * (order + 1) : (order + 1) * (order + 1) * (order + 1);
  s->nv = dim == 2 ? 4 : 8;
  s->n_cells = n_cells;
  s->n_dof = n_dof;
  s->n_active = n_active;
  for (int c = 0; c <= n_cells; c++)
    if (h_bi[c] != c * s->nbf)
    {
      delete s;
      return fail(ctx, CDGPU_ERR_INVALID, "upload_space: BeginIndex must step by the number of basis functions");
    }
  s->h_coords.assign(h_vert, h_vert + (size_t)n_cells * s->nv * dim);
  s->h_gn.assign(h_gn, h_gn + (size_t)n_cells * s->nbf);
  for (int v : s->h_gn)
    if (v < 0 || v >= n_dof)
    {
      delete s;
      return fail(ctx, CDGPU_ERR_INVALID, "upload_space: global number out of range");
    }
  for (int c = 0; c < n_cells && s->all_affine; c++)
    s->all_affine = cell_is_affine(dim, &s->h_coords[(size_t)c * s->nv * dim]);
  int rc;
  // GlobalNumbers get 4 spare ints: bulk copies of a tile's numbers round their size up to 16 bytes
  if ((rc = dev_alloc(ctx, &s->d_coords, s->h_coords.size())) || (rc = dev_alloc(ctx, &s->d_gn, s->h_gn.size() + 4)))
  {
    free_space(s);
    return rc;
  }
  cudaError_t e = cudaMemcpy(s->d_coords, s->h_coords.data(), s->h_coords.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->d_gn, s->h_gn.data(), s->h_gn.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { free_space(s); return cuda_fail(ctx, e, "upload_space"); }
  // DOF -> cell incidence for the row-gather assembly
  std::vector<int> ptr, inc;
  build_incidence(*s, ptr, inc);
  if ((rc = dev_alloc(ctx, &s->d_inc_ptr, ptr.size())) || (rc = dev_alloc(ctx, &s->d_inc, inc.size())))
  {
    free_space(s);
    return rc;
  }
  e = cudaMemcpy(s->d_inc_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->d_inc, inc.data(), inc.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { free_space(s); return cuda_fail(ctx, e, "upload_space"); }
  ctx->spaces.push_back(s);
  *space_id = (int)ctx->spaces.size() - 1;
  return CDGPU_OK;
}

// d_kcol_built: the columns already on the device (built there, nnz + kCsrPad entries; the
// space takes ownership), else they are uploaded from s.h_kcol
static int install_pattern(cdgpu_ctx *ctx, Space &s, int *d_kcol_built = nullptr)
{
  int rc;
  s.nnz = s.h_row_ptr[s.n_dof];
  std::vector<int> dir_start(s.n_dof), dir_rows;
  for (int r = 0; r < s.n_dof; r++)
  {
    int j = s.h_row_ptr[r + 1];
    while (j > s.h_row_ptr[r] && s.h_kcol[j - 1] >= s.n_active) j--;
    dir_start[r] = j;
    if (r < s.n_active && j < s.h_row_ptr[r + 1]) dir_rows.push_back(r);
  }
  if (s.d_dir_rows) { cudaFree(s.d_dir_rows); s.d_dir_rows = nullptr; }
  s.n_dir_rows = (int)dir_rows.size();
  if (d_kcol_built)
  {
    if (s.d_kcol) cudaFree(s.d_kcol);
    s.d_kcol = d_kcol_built;
  }
  if ((rc = dev_alloc(ctx, &s.d_row_ptr, s.n_dof + 1 + kCsrPad)) ||
      (!d_kcol_built && (rc = dev_alloc(ctx, &s.d_kcol, s.nnz + kCsrPad))) ||
      (rc = dev_alloc(ctx, &s.d_dir_start, s.n_dof)) ||
      (rc = dev_alloc(ctx, &s.d_dir_rows, std::max<size_t>(1, dir_rows.size()))))
    return rc;
  CD_CUDA(ctx, cudaMemcpy(s.d_row_ptr, s.h_row_ptr.data(), sizeof(int) * (s.n_dof + 1), cudaMemcpyHostToDevice));
  if (!d_kcol_built)
    CD_CUDA(ctx, cudaMemcpy(s.d_kcol, s.h_kcol.data(), sizeof(int) * s.nnz, cudaMemcpyHostToDevice));
  CD_CUDA(ctx, cudaMemcpy(s.d_dir_start, dir_start.data(), sizeof(int) * s.n_dof, cudaMemcpyHostToDevice));
  if (!dir_rows.empty())
    CD_CUDA(ctx, cudaMemcpy(s.d_dir_rows, dir_rows.data(), sizeof(int) * dir_rows.size(), cudaMemcpyHostToDevice));
  CD_CUDA(ctx, cudaMemset(s.d_row_ptr + s.n_dof + 1, 0, sizeof(int) * kCsrPad));
  CD_CUDA(ctx, cudaMemset(s.d_kcol + s.nnz, 0, sizeof(int) * kCsrPad));
  s.shape = csr_shape(s.h_row_ptr.data(), s.n_dof);
  if ((rc = build_csr_tiles(ctx, s))) return rc;
  // a new pattern invalidates values sized for the old one and the slot map
  s.slot_pattern = -1;
  s.pattern_checked = false;
  void **vals[] = {(void **)&s.d_a, (void **)&s.d_a32};
  for (void **p : vals)
    if (*p) { cudaFree(*p); *p = nullptr; }
  s.assembled = false;
  return CDGPU_OK;
}

int cdgpu_build_pattern(cdgpu_ctx *ctx, int space_id, int *nnz)
{
  Space *s = get_space(ctx, space_id);
  if (!s) return fail(ctx, CDGPU_ERR_INVALID, "build_pattern: bad space id");
  cudaSetDevice(ctx->device);
  build_pattern(*s, s->h_row_ptr, s->h_kcol);
  int rc = install_pattern(ctx, *s);
  if (rc) return rc;
  if (nnz) *nnz = (int)s->nnz;
  return CDGPU_OK;
}

int cdgpu_build_pattern_device(cdgpu_ctx *ctx, int space_id, int *nnz)
{
  Space *s = get_space(ctx, space_id);
  if (!s) return fail(ctx, CDGPU_ERR_INVALID, "build_pattern_device: bad space id");
  cudaSetDevice(ctx->device);
  int *d_kcol = nullptr;
  bool fallback = false;
  int rc = build_pattern_device(ctx, *s, &d_kcol, &fallback);
  if (rc) return rc;
  if (fallback) build_pattern(*s, s->h_row_ptr, s->h_kcol); // a row beyond the kernel's buffer
  if ((rc = install_pattern(ctx, *s, d_kcol))) return rc;
  if (nnz) *nnz = (int)s->nnz;
  return CDGPU_OK;
}

int cdgpu_upload_pattern(cdgpu_ctx *ctx, int space_id, const int *h_row_ptr, const int *h_kcol, int nnz)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !h_row_ptr || !h_kcol) return fail(ctx, CDGPU_ERR_INVALID, "upload_pattern: bad argument");
  if (h_row_ptr[0] != 0 || h_row_ptr[s->n_dof] != nnz) return fail(ctx, CDGPU_ERR_INVALID, "upload_pattern: row_ptr does not match nnz");
  for (int r = 0; r < s->n_dof; r++)
  {
    if (h_row_ptr[r + 1] < h_row_ptr[r]) return fail(ctx, CDGPU_ERR_INVALID, "upload_pattern: row_ptr not monotone");
    for (int j = h_row_ptr[r]; j < h_row_ptr[r + 1]; j++)
    {
      if (h_kcol[j] < 0 || h_kcol[j] >= s->n_dof) return fail(ctx, CDGPU_ERR_INVALID, "upload_pattern: column out of range");
      if (j > h_row_ptr[r] && h_kcol[j] <= h_kcol[j - 1])
        return fail(ctx, CDGPU_ERR_INVALID, "upload_pattern: columns must be sorted ascending (TSquareStructure::Sort)");
    }
  }
  cudaSetDevice(ctx->device);
  s->h_row_ptr.assign(h_row_ptr, h_row_ptr + s->n_dof + 1);
  s->h_kcol.assign(h_kcol, h_kcol + nnz);
  return install_pattern(ctx, *s);
}

int cdgpu_get_pattern(cdgpu_ctx *ctx, int space_id, int *h_row_ptr, int *h_kcol)
{
  Space *s = get_space(ctx, space_id);
  if (!s || s->nnz < 0) return fail(ctx, CDGPU_ERR_INVALID, "get_pattern: no pattern");
  if (h_row_ptr) std::copy(s->h_row_ptr.begin(), s->h_row_ptr.end(), h_row_ptr);
  if (h_kcol) std::copy(s->h_kcol.begin(), s->h_kcol.end(), h_kcol);
  return CDGPU_OK;
}

int cdgpu_quadrature_points(cdgpu_ctx *ctx, int space_id, double *h_xyz, int *n_quad)
{
  Space *s = get_space(ctx, space_id);
  if (!s) return fail(ctx, CDGPU_ERR_INVALID, "quadrature_points: bad space id");
  RefElement re;
  make_ref_element(s->dim, s->order, re);
  if (n_quad) *n_quad = re.nq;
  if (!h_xyz) return CDGPU_OK;
  for (int c = 0; c < s->n_cells; c++)
  {
    const double *V = &s->h_coords[(size_t)c * s->nv * s->dim];
    bool aff = cell_is_affine(s->dim, V);
    for (int q = 0; q < re.nq; q++)
    {
      double J[9];
      ref_map(s->dim, aff, V, &re.qx[q * s->dim], h_xyz + ((size_t)c * re.nq + q) * s->dim, J);
    }
  }
  return CDGPU_OK;
}

int cdgpu_set_coeffs(cdgpu_ctx *ctx, int space_id, const cdgpu_coeffs *co, const double *h_table)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !co) return fail(ctx, CDGPU_ERR_INVALID, "set_coeffs: bad argument");
  if (co->kind < 0 || co->kind > 3) return fail(ctx, CDGPU_ERR_INVALID, "set_coeffs: unknown coefficient kind");
  if ((co->kind == CDGPU_COEFF_SINE || co->kind == CDGPU_COEFF_ROTATING) && s->dim != 2)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "set_coeffs: sine and rotating coefficients are 2D examples");
  if (!std::isfinite(co->eps) || !std::isfinite(co->b1) || !std::isfinite(co->b2) || !std::isfinite(co->b3) ||
      !std::isfinite(co->c) || !std::isfinite(co->f) || !std::isfinite(co->delta0))
    return fail(ctx, CDGPU_ERR_INVALID, "set_coeffs: non-finite coefficient");
  cudaSetDevice(ctx->device);
  s->co = *co;
  if (co->kind == CDGPU_COEFF_TABLE)
  {
    if (!h_table) return fail(ctx, CDGPU_ERR_INVALID, "set_coeffs: table kind needs a table");
    RefElement re;
    make_ref_element(s->dim, s->order, re);
    size_t n = (size_t)s->n_cells * re.nq * 6;
    for (size_t i = 0; i < n; i++)
      if (!std::isfinite(h_table[i])) return fail(ctx, CDGPU_ERR_INVALID, "set_coeffs: non-finite table entry");
    int rc = dev_alloc(ctx, &s->d_tab, n);
    if (rc) return rc;
    CD_CUDA(ctx, cudaMemcpy(s->d_tab, h_table, n * sizeof(double), cudaMemcpyHostToDevice));
  }
  s->co_set = true;
  return CDGPU_OK;
}

int cdgpu_assemble(cdgpu_ctx *ctx, int space_id, int disctype, const double *h_dirichlet, double *h_entries,
                   double *h_rhs)
{
  Space *s = get_space(ctx, space_id);
  if (!s) return fail(ctx, CDGPU_ERR_INVALID, "assemble: bad space id");
  cudaSetDevice(ctx->device);
  int rc = assemble_space(ctx, *s, disctype, h_dirichlet);
  if (rc) return rc;
  if (h_entries)
    CD_CUDA(ctx, cudaMemcpyAsync(h_entries, s->d_a, sizeof(double) * s->nnz, cudaMemcpyDeviceToHost, ctx->stream));
  if (h_rhs)
    CD_CUDA(ctx, cudaMemcpyAsync(h_rhs, s->d_rhs, sizeof(double) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CDGPU_OK;
}

int cdgpu_add_neumann(cdgpu_ctx *ctx, int space_id, int n_edges, const int *h_cell, const int *h_edge,
                      const double *h_g, double *h_rhs)
{
  Space *s = get_space(ctx, space_id);
  if (!s || (n_edges > 0 && (!h_cell || !h_edge || !h_g))) return fail(ctx, CDGPU_ERR_INVALID, "add_neumann: bad argument");
  cudaSetDevice(ctx->device);
  int rc = add_neumann(ctx, *s, n_edges, h_cell, h_edge, h_g);
  if (rc) return rc;
  if (h_rhs)
  {
    CD_CUDA(ctx, cudaMemcpyAsync(h_rhs, s->d_rhs, sizeof(double) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return CDGPU_OK;
}

int cdgpu_boundary_points(cdgpu_ctx *ctx, int space_id, int n, const int *h_cell, const int *h_local, double *h_xyz)
{
  Space *s = get_space(ctx, space_id);
  if (!s || n < 0 || (n > 0 && (!h_cell || !h_local || !h_xyz))) return fail(ctx, CDGPU_ERR_INVALID, "boundary_points: bad argument");
  for (int e = 0; e < n; e++)
    if (h_cell[e] < 0 || h_cell[e] >= s->n_cells || h_local[e] < 0 || h_local[e] > (s->dim == 2 ? 3 : 5))
      return fail(ctx, CDGPU_ERR_INVALID, "boundary_points: bad cell or edge/face index");
  boundary_points(*s, n, h_cell, h_local, h_xyz);
  return CDGPU_OK;
}

int cdgpu_rhs_device(cdgpu_ctx *ctx, int space_id, double **d_rhs)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !d_rhs || !s->assembled) return fail(ctx, CDGPU_ERR_INVALID, "rhs_device: not assembled");
  *d_rhs = s->d_rhs;
  return CDGPU_OK;
}

int cdgpu_get_rhs(cdgpu_ctx *ctx, int space_id, double *h_rhs)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !h_rhs || !s->assembled) return fail(ctx, CDGPU_ERR_INVALID, "get_rhs: not assembled");
  cudaSetDevice(ctx->device);
  CD_CUDA(ctx, cudaMemcpyAsync(h_rhs, s->d_rhs, sizeof(double) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CDGPU_OK;
}

int cdgpu_spmv_device(cdgpu_ctx *ctx, int space_id, const double *d_x, double *d_y)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !s->assembled) return fail(ctx, CDGPU_ERR_INVALID, "spmv: matrix not assembled");
  cudaSetDevice(ctx->device);
  return spmv64(ctx, *s, d_x, d_y);
}

int cdgpu_spmv(cdgpu_ctx *ctx, int space_id, const double *h_x, double *h_y)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !s->assembled || !h_x || !h_y) return fail(ctx, CDGPU_ERR_INVALID, "spmv: bad argument");
  cudaSetDevice(ctx->device);
  double *dx = nullptr, *dy = nullptr;
  int rc;
  if ((rc = dev_alloc(ctx, &dx, s->n_dof)) || (rc = dev_alloc(ctx, &dy, s->n_dof))) return rc;
  CD_CUDA(ctx, cudaMemcpyAsync(dx, h_x, sizeof(double) * s->n_dof, cudaMemcpyHostToDevice, ctx->stream));
  rc = spmv64(ctx, *s, dx, dy);
  if (!rc)
  {
    CD_CUDA(ctx, cudaMemcpyAsync(h_y, dy, sizeof(double) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->d_err) rc = assemble_check(ctx); // wait flag of the bulk-copy product
  }
  cudaFree(dx);
  cudaFree(dy);
  return rc;
}

int cdgpu_apply_fp64_device(cdgpu_ctx *ctx, int space_id, int form, const double *d_x, double *d_y)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !s->assembled || !d_x || !d_y || form < 0 || form > 1)
    return fail(ctx, CDGPU_ERR_INVALID, "apply_fp64: bad argument");
  cudaSetDevice(ctx->device);
  return apply_fp64_form(ctx, *s, form, d_x, d_y, false);
}

int cdgpu_apply_fp64(cdgpu_ctx *ctx, int space_id, int form, const double *h_x, double *h_y)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !s->assembled || !h_x || !h_y || form < 0 || form > 1)
    return fail(ctx, CDGPU_ERR_INVALID, "apply_fp64: bad argument");
  cudaSetDevice(ctx->device);
  double *dx = nullptr, *dy = nullptr;
  int rc;
  if ((rc = dev_alloc(ctx, &dx, s->n_dof)) || (rc = dev_alloc(ctx, &dy, s->n_dof)))
  {
    if (dx) cudaFree(dx);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(dx, h_x, sizeof(double) * s->n_dof, cudaMemcpyHostToDevice, ctx->stream);
  rc = e == cudaSuccess ? apply_fp64_form(ctx, *s, form, dx, dy, true) : cuda_fail(ctx, e, "apply_fp64: copy");
  if (!rc)
  {
    e = cudaMemcpyAsync(h_y, dy, sizeof(double) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "apply_fp64: copy back");
  }
  cudaStreamSynchronize(ctx->stream);
  cudaFree(dx);
  cudaFree(dy);
  return rc;
}

int cdgpu_apply_fp32(cdgpu_ctx *ctx, int space_id, int form, const float *h_x, float *h_y)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !s->assembled || !h_x || !h_y || form < 0 || form > 2)
    return fail(ctx, CDGPU_ERR_INVALID, "apply_fp32: bad argument");
  cudaSetDevice(ctx->device);
  float *dx = nullptr, *dy = nullptr;
  int rc;
  if ((rc = dev_alloc(ctx, &dx, s->n_dof)) || (rc = dev_alloc(ctx, &dy, s->n_dof)))
  {
    if (dx) cudaFree(dx);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(dx, h_x, sizeof(float) * s->n_dof, cudaMemcpyHostToDevice, ctx->stream);
  rc = e == cudaSuccess ? apply_fp32_form(ctx, *s, form, dx, dy) : cuda_fail(ctx, e, "apply_fp32: copy");
  if (!rc)
  {
    e = cudaMemcpyAsync(h_y, dy, sizeof(float) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "apply_fp32: copy back");
  }
  cudaStreamSynchronize(ctx->stream);
  cudaFree(dx);
  cudaFree(dy);
  return rc;
}

int cdgpu_errors(cdgpu_ctx *ctx, int space_id, const double *h_sol, double *l2, double *h1semi)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !h_sol || !l2 || !h1semi) return fail(ctx, CDGPU_ERR_INVALID, "errors: bad argument");
  cudaSetDevice(ctx->device);
  double *du = nullptr;
  int rc;
  if ((rc = dev_alloc(ctx, &du, s->n_dof))) return rc;
  cudaError_t e = cudaMemcpyAsync(du, h_sol, sizeof(double) * s->n_dof, cudaMemcpyHostToDevice, ctx->stream);
  rc = e == cudaSuccess ? space_errors_sine(ctx, *s, du, l2, h1semi) : cuda_fail(ctx, e, "errors: copy");
  cudaStreamSynchronize(ctx->stream);
  cudaFree(du);
  return rc;
}

int cdgpu_product_tuning(cdgpu_ctx *ctx, int space_id, char *buf, int len)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !buf || len <= 0) return fail(ctx, CDGPU_ERR_INVALID, "product_tuning: bad argument");
  std::string r;
  csr_tuning_report(ctx, *s, r);
  snprintf(buf, len, "%s", r.c_str());
  return CDGPU_OK;
}

// Legacy-VTK output of a solution, in the form TOutput3D::WriteVtk / TOutput2D::WriteVtk write
// it (src/FE/Output3D.C:1747-2010): ASCII UNSTRUCTURED_GRID, the mesh vertices as POINTS, one
// hexahedron (type 12) or quadrilateral (type 9) per cell, the function's values at the vertices
// as POINT_DATA, 6 significant digits in scientific notation.  The vertices are the vertex DOFs
// of the Q1/Q2 space (a conforming function's value there is its DOF value), numbered in
// ascending DOF order; the reference numbers them by sorting vertex addresses.  sol may be on
// the device (sol_on_device != 0: it is copied back first) or on the host.
int cdgpu_write_vtk(cdgpu_ctx *ctx, int space_id, const double *sol, int sol_on_device, const char *path,
                    const char *name)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !sol || !path) return fail(ctx, CDGPU_ERR_INVALID, "write_vtk: bad argument");
  std::vector<double> u(s->n_dof);
  if (sol_on_device)
  {
    cudaSetDevice(ctx->device);
    CD_CUDA(ctx, cudaMemcpyAsync(u.data(), sol, sizeof(double) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  else
    std::copy(sol, sol + s->n_dof, u.begin());
  // local index of every cell vertex among the cell's DOFs (tensor order, x fastest)
  const int p1 = s->order + 1;
  int vdof[8];
  for (int v = 0; v < s->nv; v++)
  {
    const int ix = (v == 1 || v == 2 || v == 5 || v == 6) ? s->order : 0;
    const int iy = (v == 2 || v == 3 || v == 6 || v == 7) ? s->order : 0;
    const int iz = v >= 4 ? s->order : 0;
    vdof[v] = ix + p1 * iy + (s->dim == 3 ? p1 * p1 * iz : 0);
  }
  std::vector<int> point(s->n_dof, -1);
  std::vector<double> xyz((size_t)s->n_dof * 3, 0.0);
  for (int c = 0; c < s->n_cells; c++)
    for (int v = 0; v < s->nv; v++)
    {
      const int d = s->h_gn[(size_t)c * s->nbf + vdof[v]];
      point[d] = 0;
      for (int a = 0; a < s->dim; a++) xyz[(size_t)d * 3 + a] = s->h_coords[((size_t)c * s->nv + v) * s->dim + a];
    }
  int np = 0;
  for (int d = 0; d < s->n_dof; d++)
    if (point[d] >= 0) point[d] = np++;
  FILE *f = fopen(path, "w");
  if (!f) return fail(ctx, CDGPU_ERR_INVALID, std::string("write_vtk: cannot open ") + path);
  fprintf(f, "# vtk DataFile Version 4.2\nfile created by libcdgpu\nASCII\nDATASET UNSTRUCTURED_GRID\n\n");
  fprintf(f, "POINTS %d double\n", np);
  for (int d = 0; d < s->n_dof; d++)
    if (point[d] >= 0) fprintf(f, "%.6e %.6e %.6e\n", xyz[(size_t)d * 3], xyz[(size_t)d * 3 + 1], xyz[(size_t)d * 3 + 2]);
  fprintf(f, "\nCELLS %d %d\n", s->n_cells, s->n_cells * (s->nv + 1));
  for (int c = 0; c < s->n_cells; c++)
  {
    fprintf(f, "%d ", s->nv);
    for (int v = 0; v < s->nv; v++) fprintf(f, "%d ", point[s->h_gn[(size_t)c * s->nbf + vdof[v]]]);
    fprintf(f, "\n");
  }
  fprintf(f, "\nCELL_TYPES %d\n", s->n_cells);
  for (int c = 0; c < s->n_cells; c++) fprintf(f, "%d ", s->dim == 3 ? 12 : 9);
  fprintf(f, "\n\nPOINT_DATA %d\nSCALARS %s double\nLOOKUP_TABLE default\n", np, name && name[0] ? name : "u");
  for (int d = 0; d < s->n_dof; d++)
    if (point[d] >= 0) fprintf(f, "%.6e\n", u[d]);
  const bool ok = fclose(f) == 0;
  return ok ? CDGPU_OK : fail(ctx, CDGPU_ERR_INVALID, "write_vtk: write failed");
}

int cdgpu_errors_table(cdgpu_ctx *ctx, int space_id, const double *h_sol, const double *h_exact, double *l2,
                       double *h1semi)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !h_sol || !h_exact || !l2 || !h1semi) return fail(ctx, CDGPU_ERR_INVALID, "errors_table: bad argument");
  cudaSetDevice(ctx->device);
  if (!s->re_ready)
  {
    make_ref_element(s->dim, s->order, s->re);
    s->re_ready = true;
  }
  const size_t ne = (size_t)s->n_cells * s->re.nq * (1 + s->dim);
  double *du = nullptr, *dex = nullptr;
  int rc;
  if ((rc = dev_alloc(ctx, &du, s->n_dof)) || (rc = dev_alloc(ctx, &dex, ne)))
  {
    if (du) cudaFree(du);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(du, h_sol, sizeof(double) * s->n_dof, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dex, h_exact, sizeof(double) * ne, cudaMemcpyHostToDevice, ctx->stream);
  rc = e == cudaSuccess ? space_errors_table(ctx, *s, du, dex, l2, h1semi) : cuda_fail(ctx, e, "errors_table: copy");
  cudaStreamSynchronize(ctx->stream);
  cudaFree(du);
  cudaFree(dex);
  return rc;
}

int cdgpu_defect(cdgpu_ctx *ctx, int space_id, const double *h_x, const double *h_f, double *h_d, double *res)
{
  Space *s = get_space(ctx, space_id);
  if (!s || !s->assembled || !h_x || !h_f) return fail(ctx, CDGPU_ERR_INVALID, "defect: bad argument");
  cudaSetDevice(ctx->device);
  double *dx = nullptr, *df = nullptr, *dd = nullptr;
  int rc;
  if ((rc = dev_alloc(ctx, &dx, s->n_dof)) || (rc = dev_alloc(ctx, &df, s->n_dof)) || (rc = dev_alloc(ctx, &dd, s->n_dof)))
    return rc;
  CD_CUDA(ctx, cudaMemcpyAsync(dx, h_x, sizeof(double) * s->n_dof, cudaMemcpyHostToDevice, ctx->stream));
  CD_CUDA(ctx, cudaMemcpyAsync(df, h_f, sizeof(double) * s->n_dof, cudaMemcpyHostToDevice, ctx->stream));
  rc = defect64(ctx, *s, dx, df, dd, res);
  if (!rc && h_d)
  {
    CD_CUDA(ctx, cudaMemcpyAsync(h_d, dd, sizeof(double) * s->n_dof, cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (!rc && ctx->d_err) rc = assemble_check(ctx); // wait flag of the bulk-copy product
  cudaFree(dx);
  cudaFree(df);
  cudaFree(dd);
  return rc;
}

int cdgpu_hierarchy(cdgpu_ctx *ctx, int n_levels, const int *space_ids, const int *const *h_parent, int *mg_id)
{
  if (!ctx || n_levels < 1 || n_levels > 60 || !space_ids || !mg_id) return fail(ctx, CDGPU_ERR_INVALID, "hierarchy: bad argument");
  cudaSetDevice(ctx->device);
  Hierarchy *h = new Hierarchy();
  for (int l = 0; l < n_levels; l++)
  {
    Space *s = get_space(ctx, space_ids[l]);
    if (!s || s->nnz < 0) { free_mg(h); return fail(ctx, CDGPU_ERR_INVALID, "hierarchy: every level needs a space with a pattern"); }
    if (l > 0 && (s->dim != h->lev[0].sp->dim || s->order != h->lev[0].sp->order))
    {
      free_mg(h);
      return fail(ctx, CDGPU_ERR_UNSUPPORTED, "hierarchy: all levels must use the same element");
    }
    Level L;
    L.sp = s;
    h->lev.push_back(L);
  }
  for (int l = 1; l < n_levels; l++)
  {
    if (!h_parent || !h_parent[l]) { free_mg(h); return fail(ctx, CDGPU_ERR_INVALID, "hierarchy: missing parent map"); }
    Space &c = *h->lev[l - 1].sp, &f = *h->lev[l].sp;
    for (int i = 0; i < f.n_cells; i++)
      if (h_parent[l][i] < 0 || h_parent[l][i] >= c.n_cells)
      {
        free_mg(h);
        return fail(ctx, CDGPU_ERR_INVALID, "hierarchy: parent index out of range");
      }
    std::vector<int> row, col;
    std::vector<double> val;
    build_prolongation(c, f, h_parent[l], row, col, val);
    // transpose = restriction
    std::vector<int> rrow(c.n_dof + 1, 0), rcol(col.size());
    std::vector<double> rval(col.size());
    for (int v : col) rrow[v + 1]++;
    for (int i = 0; i < c.n_dof; i++) rrow[i + 1] += rrow[i];
    std::vector<int> fill(c.n_dof, 0);
    for (int i = 0; i < f.n_dof; i++)
      for (int j = row[i]; j < row[i + 1]; j++)
      {
        int p = rrow[col[j]] + fill[col[j]]++;
        rcol[p] = i;
        rval[p] = val[j];
      }
    std::vector<float> val32(val.begin(), val.end()), rval32(rval.begin(), rval.end());
    Level &L = h->lev[l];
    L.p_nnz = (long)col.size();
    int rc;
    if ((rc = dev_alloc(ctx, &L.d_p_row, row.size())) || (rc = dev_alloc(ctx, &L.d_p_col, col.size())) ||
        (rc = dev_alloc(ctx, &L.d_p_val, val.size())) || (rc = dev_alloc(ctx, &L.d_p_val32, val.size())) ||
        (rc = dev_alloc(ctx, &L.d_r_row, rrow.size())) || (rc = dev_alloc(ctx, &L.d_r_col, rcol.size())) ||
        (rc = dev_alloc(ctx, &L.d_r_val, rval.size())) || (rc = dev_alloc(ctx, &L.d_r_val32, rval.size())))
    {
      free_mg(h);
      return rc;
    }
    cudaMemcpy(L.d_p_row, row.data(), row.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(L.d_p_col, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(L.d_p_val, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(L.d_p_val32, val32.data(), val32.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(L.d_r_row, rrow.data(), rrow.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(L.d_r_col, rcol.data(), rcol.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(L.d_r_val, rval.data(), rval.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaError_t e = cudaMemcpy(L.d_r_val32, rval32.data(), rval32.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { free_mg(h); return cuda_fail(ctx, e, "hierarchy"); }
    L.p_shape = csr_shape(row.data(), f.n_dof);
    L.r_shape = csr_shape(rrow.data(), c.n_dof);
  }
  int rc = setup_hierarchy_buffers(ctx, *h, 30);
  if (rc) { free_mg(h); return rc; }
  ctx->mgs.push_back(h);
  *mg_id = (int)ctx->mgs.size() - 1;
  return CDGPU_OK;
}

int cdgpu_assemble_hierarchy(cdgpu_ctx *ctx, int mg_id, int disctype, int coarse_disctype)
{
  Hierarchy *h = get_mg(ctx, mg_id);
  if (!h) return fail(ctx, CDGPU_ERR_INVALID, "assemble_hierarchy: bad id");
  cudaSetDevice(ctx->device);
  bool need_check = false;
  for (auto &L : h->lev) need_check = need_check || !L.sp->pattern_checked;
  const size_t nl = h->lev.size();
  int rc = CDGPU_OK;
  // The levels are independent: the coarse ones are assembled on the hierarchy's side stream
  // beside the finest one, and so is the exact coarse inverse once a solve has used it (it
  // depends on the coarsest level only); the stream of the context waits for both at the end.
  if (nl > 1)
  {
    if (!h->astream)
    {
      CD_CUDA(ctx, cudaStreamCreateWithFlags(&h->astream, cudaStreamNonBlocking));
      CD_CUDA(ctx, cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
      CD_CUDA(ctx, cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    }
    CD_CUDA(ctx, cudaEventRecord(h->ev_fork, ctx->stream));
    CD_CUDA(ctx, cudaStreamWaitEvent(h->astream, h->ev_fork, 0));
    cudaStream_t main_stream = ctx->stream;
    ctx->stream = h->astream;
    for (size_t l = 0; l + 1 < nl && !rc; l++) rc = assemble_space(ctx, *h->lev[l].sp, coarse_disctype, nullptr, false);
    if (!rc && h->d_cinv) rc = refresh_coarse_inverse(ctx, *h);
    ctx->stream = main_stream;
    if (rc) return rc;
    CD_CUDA(ctx, cudaEventRecord(h->ev_join, h->astream));
  }
  rc = assemble_space(ctx, *h->lev[nl - 1].sp, disctype, nullptr, false);
  if (nl > 1) CD_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, h->ev_join, 0));
  if (rc) return rc;
  if (!need_check) return CDGPU_OK; // the checks depend on the patterns only
  rc = assemble_check(ctx);
  if (!rc)
    for (auto &L : h->lev) L.sp->pattern_checked = true;
  return rc;
}

int cdgpu_solve_device(cdgpu_ctx *ctx, int mg_id, const cdgpu_solver_params *p, const double *d_rhs, double *d_sol,
                       cdgpu_solve_info *info)
{
  Hierarchy *h = get_mg(ctx, mg_id);
  if (!h || !p || !d_rhs || !d_sol) return fail(ctx, CDGPU_ERR_INVALID, "solve: bad argument");
  cudaSetDevice(ctx->device);
  return run_solve(ctx, *h, *p, d_rhs, d_sol, info);
}

int cdgpu_solve(cdgpu_ctx *ctx, int mg_id, const cdgpu_solver_params *p, const double *h_rhs, double *h_sol,
                cdgpu_solve_info *info)
{
  Hierarchy *h = get_mg(ctx, mg_id);
  if (!h || !p || !h_rhs || !h_sol) return fail(ctx, CDGPU_ERR_INVALID, "solve: bad argument");
  cudaSetDevice(ctx->device);
  int n = h->lev.back().sp->n_dof;
  CD_CUDA(ctx, cudaMemcpyAsync(h->d_b, h_rhs, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  CD_CUDA(ctx, cudaMemcpyAsync(h->d_x, h_sol, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  int rc = run_solve(ctx, *h, *p, h->d_b, h->d_x, info);
  if (rc) return rc;
  CD_CUDA(ctx, cudaMemcpyAsync(h_sol, h->d_x, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CDGPU_OK;
}

} // extern "C"
