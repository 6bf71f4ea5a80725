// Time-dependent convection-diffusion (theta schemes) on top of a multigrid hierarchy:
// the GPU counterpart of TSystemTCD2D (src/System/SystemTCD2D.C) -- AssembleMRhs,
// AssembleARhs, AssembleSystMat, Solve, RestoreMassMat -- with the multigrid-preconditioned
// FGMRES of libcdgpu as the solver on every level.
//
// The mass matrix is kept and updated in place exactly like the reference's sqmatrixM:
//   M <- M - tau*theta2*A                    (MatAdd, Blas2.C:132, active rows only)
//   B  = tau*theta3*f_old + tau*theta4*f + M_active u_old;  B, u on Dirichlet rows <- f
//   M <- M + (tau*theta2 + tau*theta1)*A     (the system matrix)
//   solve M u = B
//   M <- M - tau*theta1*A                    (RestoreMassMat)
// so the rounding of every step is the reference's.
#include <cmath>

#include "internal.h"

struct Tcd
{
  Hierarchy *h = nullptr;
  int disctype = CDGPU_GALERKIN;
  std::vector<double *> M, A; // per level, same CSR pattern as the level's space
  double *d_f_old = nullptr, *d_f = nullptr, *d_B = nullptr, *d_x = nullptr;
  bool have_mass = false, have_stiff = false;
  // BoundValue at the finest level's Dirichlet DOFs for the next assemblies (empty = 0)
  std::vector<double> h_dir;
};

static std::vector<Tcd *> &tcds(cdgpu_ctx *ctx) { return ctx->tcds; }

void free_tcd(Tcd *t)
{
  if (!t) return;
  for (double *p : t->M) cudaFree(p);
  for (double *p : t->A) cudaFree(p);
  double *v[] = {t->d_f_old, t->d_f, t->d_B, t->d_x};
  for (double *p : v)
    if (p) cudaFree(p);
  delete t;
}

// y += alpha * x over the entries of the active rows [0, n_active_entries)
__global__ void matadd_kernel(long n, double alpha, const double *__restrict__ x, double *__restrict__ y)
{
  CD_PDL_ENTRY();
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += alpha * x[i];
}

// B = tau*th3*f_old + tau*th4*f + (M x) on active rows; B = f and x = f on Dirichlet rows
__global__ void tcd_rhs_kernel(int n, int n_active, const int *__restrict__ rp, const int *__restrict__ kc,
                               const double *__restrict__ M, const double *__restrict__ f_old,
                               const double *__restrict__ f, double c3, double c4, double *__restrict__ x,
                               double *__restrict__ B)
{
  CD_PDL_ENTRY();
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  if (r >= n_active)
  {
    B[r] = f[r];
    return;
  }
  double s = 0;
  for (int j = rp[r]; j < rp[r + 1]; j++) s += M[j] * x[kc[j]];
  double b = 0.0;
  b += c3 * f_old[r];
  b += c4 * f[r];
  B[r] = b + s;
}

__global__ void dirichlet_copy_kernel(int n, int n_active, const double *__restrict__ f, double *__restrict__ x)
{
  CD_PDL_ENTRY();
  int r = n_active + blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) x[r] = f[r];
}

// system matrix of a level into the space's value arrays (f64, f32 copy, diagonals)
__global__ void install_system_kernel(int n, const int *__restrict__ rp, const int *__restrict__ kc,
                                      const double *__restrict__ M, double *__restrict__ a, float *__restrict__ a32,
                                      double *__restrict__ diag, float *__restrict__ diag32)
{
  CD_PDL_ENTRY();
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  for (int j = rp[r]; j < rp[r + 1]; j++)
  {
    double v = M[j];
    a[j] = v;
    a32[j] = (float)v;
    if (kc[j] == r) { diag[r] = v; diag32[r] = (float)v; }
  }
}

static int matadd(cdgpu_ctx *ctx, const Space &s, double alpha, const double *x, double *y)
{
  long n = s.h_row_ptr[s.n_active];
  if (n == 0) return CDGPU_OK;
  (void)cd_launch(matadd_kernel, (unsigned)((n + 255) / 256), 256, 0, ctx->stream, n, alpha, x, y);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

static Tcd *get_tcd(cdgpu_ctx *ctx, int id)
{
  auto &v = tcds(ctx);
  return id >= 0 && id < (int)v.size() ? v[id] : nullptr;
}

// assemble one form on every level and keep the values in dst[l]; the finest right-hand
// side goes to rhs_dst
static int assemble_into(cdgpu_ctx *ctx, Tcd &t, int disctype, std::vector<double *> &dst, double *rhs_dst)
{
  for (size_t l = 0; l < t.h->lev.size(); l++)
  {
    Space &s = *t.h->lev[l].sp;
    const bool fine = l + 1 == t.h->lev.size();
    const double *dir = fine && !t.h_dir.empty() ? t.h_dir.data() : nullptr;
    int rc = assemble_space(ctx, s, disctype, dir, false);
    if (rc) return rc;
    CD_CUDA(ctx, cudaMemcpyAsync(dst[l], s.d_a, sizeof(double) * s.nnz, cudaMemcpyDeviceToDevice, ctx->stream));
    if (l + 1 == t.h->lev.size() && rhs_dst)
      CD_CUDA(ctx, cudaMemcpyAsync(rhs_dst, s.d_rhs, sizeof(double) * s.n_dof, cudaMemcpyDeviceToDevice,
                                   ctx->stream));
  }
  return assemble_check(ctx);
}

extern "C" {

int cdgpu_tcd_create(cdgpu_ctx *ctx, int mg_id, int disctype, int *tcd_id)
{
  if (!ctx || mg_id < 0 || mg_id >= (int)ctx->mgs.size() || !tcd_id)
    return fail(ctx, CDGPU_ERR_INVALID, "tcd_create: bad argument");
  if (disctype != CDGPU_GALERKIN)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "tcd_create: only the Galerkin time-dependent forms are implemented");
  cudaSetDevice(ctx->device);
  Tcd *t = new Tcd();
  t->h = ctx->mgs[mg_id];
  t->disctype = disctype;
  int rc;
  for (auto &L : t->h->lev)
  {
    double *m = nullptr, *a = nullptr;
    if ((rc = dev_alloc(ctx, &m, L.sp->nnz)) || (rc = dev_alloc(ctx, &a, L.sp->nnz))) return rc;
    t->M.push_back(m);
    t->A.push_back(a);
  }
  int n = t->h->lev.back().sp->n_dof;
  if ((rc = dev_alloc(ctx, &t->d_f_old, n)) || (rc = dev_alloc(ctx, &t->d_f, n)) || (rc = dev_alloc(ctx, &t->d_B, n)) ||
      (rc = dev_alloc(ctx, &t->d_x, n)))
    return rc;
  tcds(ctx).push_back(t);
  *tcd_id = (int)tcds(ctx).size() - 1;
  return CDGPU_OK;
}

// the boundary values that the reference's assembly takes from BoundValue at the current
// time (Assemble3D / Assemble2D set the Dirichlet entries of rhs), for the finest level's
// Dirichlet DOFs [n_active, n_dof); NULL returns to zero values
int cdgpu_tcd_set_dirichlet(cdgpu_ctx *ctx, int tcd_id, const double *h_dirichlet)
{
  Tcd *t = get_tcd(ctx, tcd_id);
  if (!t) return fail(ctx, CDGPU_ERR_INVALID, "tcd_set_dirichlet: bad id");
  const Space &f = *t->h->lev.back().sp;
  if (!h_dirichlet)
    t->h_dir.clear();
  else
    t->h_dir.assign(h_dirichlet, h_dirichlet + (f.n_dof - f.n_active));
  return CDGPU_OK;
}

// TSystemTCD2D::AssembleMRhs (SystemTCD2D.C:94-123): mass matrices of every level; the
// finest (f, phi) becomes the current right-hand side
int cdgpu_tcd_assemble_mass(cdgpu_ctx *ctx, int tcd_id)
{
  Tcd *t = get_tcd(ctx, tcd_id);
  if (!t) return fail(ctx, CDGPU_ERR_INVALID, "tcd_assemble_mass: bad id");
  cudaSetDevice(ctx->device);
  int rc = assemble_into(ctx, *t, CDGPU_MASS, t->M, t->d_f);
  if (rc) return rc;
  t->have_mass = true;
  return CDGPU_OK;
}

// TSystemTCD2D::AssembleARhs (SystemTCD2D.C:124-153) after the time loop's
// memcpy(oldrhs, rhs) (2DPrograms/TCD2D_ParMooN.C:265)
int cdgpu_tcd_assemble_stiffness(cdgpu_ctx *ctx, int tcd_id)
{
  Tcd *t = get_tcd(ctx, tcd_id);
  if (!t) return fail(ctx, CDGPU_ERR_INVALID, "tcd_assemble_stiffness: bad id");
  cudaSetDevice(ctx->device);
  int n = t->h->lev.back().sp->n_dof;
  CD_CUDA(ctx, cudaMemcpyAsync(t->d_f_old, t->d_f, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  int rc = assemble_into(ctx, *t, t->disctype, t->A, t->d_f);
  if (rc) return rc;
  t->have_stiff = true;
  return CDGPU_OK;
}

// AssembleSystMat (SystemTCD2D.C:154-186) + Solve + RestoreMassMat (187-210) for one step
int cdgpu_tcd_step_device(cdgpu_ctx *ctx, int tcd_id, const cdgpu_solver_params *p, double tau,
                          double theta1, double theta2, double theta3, double theta4, double *d_sol,
                          cdgpu_solve_info *info)
{
  Tcd *t = get_tcd(ctx, tcd_id);
  if (!t || !p || !d_sol) return fail(ctx, CDGPU_ERR_INVALID, "tcd_step: bad argument");
  if (!t->have_mass || !t->have_stiff) return fail(ctx, CDGPU_ERR_INVALID, "tcd_step: assemble mass and stiffness first");
  cudaSetDevice(ctx->device);
  Hierarchy &h = *t->h;
  const int L = (int)h.lev.size();
  int rc;
  const Space &f = *h.lev[L - 1].sp;
  // 2D (SystemTCD2D.C): M <- M - tau theta2 A on every level, so that the coarse levels get
  // the finest level's sequence of updates; 3D (SystemTCD3D.C:257-278): on the finest level
  // only, the coarser levels' system matrices are M + tau theta1 A
  const bool fine_only = f.dim == 3;
  for (int l = 0; l < L; l++)
    if (!(fine_only && l < L - 1) && (rc = matadd(ctx, *h.lev[l].sp, -tau * theta2, t->A[l], t->M[l]))) return rc;
  (void)cd_launch(tcd_rhs_kernel, (f.n_dof + 255) / 256, 256, 0, ctx->stream, f.n_dof, f.n_active, f.d_row_ptr, f.d_kcol,
                                                                t->M[L - 1], t->d_f_old, t->d_f, tau * theta3,
                                                                tau * theta4, d_sol, t->d_B);
  CD_LAUNCHED(ctx);
  if (f.n_dof > f.n_active)
  {
    (void)cd_launch(dirichlet_copy_kernel, (f.n_dof - f.n_active + 255) / 256, 256, 0, ctx->stream, f.n_dof, f.n_active, t->d_f,
                                                                                     d_sol);
    CD_LAUNCHED(ctx);
  }
  const double gamma = -tau * theta2;
  for (int l = 0; l < L; l++)
  {
    Space &s = *h.lev[l].sp;
    const double c = fine_only && l < L - 1 ? tau * theta1 : -gamma + tau * theta1;
    if ((rc = matadd(ctx, s, c, t->A[l], t->M[l]))) return rc;
    s.mf_T = 0; // the system matrix is a combination, not one affine assembly
    (void)cd_launch(install_system_kernel, (s.n_dof + 255) / 256, 256, 0, ctx->stream, s.n_dof, s.d_row_ptr, s.d_kcol, t->M[l],
                                                                        s.d_a, s.d_a32, s.d_diag, s.d_diag32);
    CD_LAUNCHED(ctx);
    s.assembly_version++;
  }
  cdgpu_solve_info local{};
  rc = run_solve(ctx, h, *p, t->d_B, d_sol, info ? info : &local);
  // RestoreMassMat: M <- M - tau theta1 A, whatever the solve returned
  for (int l = 0; l < L; l++)
  {
    int r2 = matadd(ctx, *h.lev[l].sp, -tau * theta1, t->A[l], t->M[l]);
    if (!rc) rc = r2;
  }
  return rc;
}

int cdgpu_tcd_step(cdgpu_ctx *ctx, int tcd_id, const cdgpu_solver_params *p, double tau, double theta1,
                   double theta2, double theta3, double theta4, double *h_sol, cdgpu_solve_info *info)
{
  Tcd *t = get_tcd(ctx, tcd_id);
  if (!t || !h_sol) return fail(ctx, CDGPU_ERR_INVALID, "tcd_step: bad argument");
  cudaSetDevice(ctx->device);
  int n = t->h->lev.back().sp->n_dof;
  CD_CUDA(ctx, cudaMemcpyAsync(t->d_x, h_sol, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  int rc = cdgpu_tcd_step_device(ctx, tcd_id, p, tau, theta1, theta2, theta3, theta4, t->d_x, info);
  if (rc) return rc;
  CD_CUDA(ctx, cudaMemcpyAsync(h_sol, t->d_x, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CDGPU_OK;
}

// copies of one level's mass matrix M (as updated in place), stiffness matrix A and the system
// matrix the last step's solve used (the level's installed entries), each nullable; like
// TSystemTCD2D's sqmatrixM / sqmatrixA members (include/System/SystemTCD2D.h)
int cdgpu_tcd_matrices(cdgpu_ctx *ctx, int tcd_id, int level, double *h_M, double *h_A, double *h_S)
{
  Tcd *t = get_tcd(ctx, tcd_id);
  if (!t || level < 0 || level >= (int)t->h->lev.size()) return fail(ctx, CDGPU_ERR_INVALID, "tcd_matrices: bad argument");
  if ((h_M && !t->have_mass) || (h_A && !t->have_stiff)) return fail(ctx, CDGPU_ERR_INVALID, "tcd_matrices: not assembled");
  const Space &s = *t->h->lev[level].sp;
  if (h_S && !s.assembled) return fail(ctx, CDGPU_ERR_INVALID, "tcd_matrices: no system matrix yet");
  cudaSetDevice(ctx->device);
  const size_t bytes = sizeof(double) * s.nnz;
  if (h_M) CD_CUDA(ctx, cudaMemcpyAsync(h_M, t->M[level], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (h_A) CD_CUDA(ctx, cudaMemcpyAsync(h_A, t->A[level], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (h_S) CD_CUDA(ctx, cudaMemcpyAsync(h_S, s.d_a, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CDGPU_OK;
}

// the current finest right-hand side (f, phi) of the last assembly, to the host
int cdgpu_tcd_rhs(cdgpu_ctx *ctx, int tcd_id, double *h_rhs)
{
  Tcd *t = get_tcd(ctx, tcd_id);
  if (!t || !h_rhs) return fail(ctx, CDGPU_ERR_INVALID, "tcd_rhs: bad argument");
  int n = t->h->lev.back().sp->n_dof;
  CD_CUDA(ctx, cudaMemcpyAsync(h_rhs, t->d_f, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CDGPU_OK;
}

} // extern "C"
