// Solver kernels and drivers of libcdgpu (sm_100a): CSR SpMV / defect, damped
// Jacobi, transfer operators, coarse solves, and the multigrid-preconditioned
// FGMRES and fixed-point iterations.
//
// The V-cycle follows TMultiGrid3D::Cycle (src/FE/MultiGrid3D.C:423-669) state for
// state: pre-smoothing, defect, restriction with CorrectDefect and Reset of the
// coarse solution, recursion, prolongation with CorrectNodes, Update with
// SC_GMG_DAMP_FACTOR_SCALAR, post-smoothing.  The three defects the reference
// computes only to print residuals (before pre-smoothing, after the update, after
// post-smoothing) change no state and are not computed.  Jacobi sweeps write into a
// second buffer and swap pointers instead of copying sol into aux first
// (MGLevel3D.C:455), which gives the same values.  A level whose solution is known
// to be zero (after Reset) starts with a sweep that reads no matrix row.
//
// FGMRES follows TFgmresIte::Iterate (src/FE/FgmresIte.C:236-582): same restart,
// stopping and divergence rules, the same Givens rotations computed on the host in
// FP64; the Arnoldi orthogonalisation is classical Gram-Schmidt applied twice
// (two fused passes over the basis) instead of modified Gram-Schmidt (one kernel
// launch per basis vector).  Both are accurate to working precision; iterates
// differ from the reference's by rounding only.
#include <climits>
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include <type_traits>

#include "internal.h"
#include "csr.cuh"
#include "mf.cuh"
#include "mf64.cuh"

namespace cg = cooperative_groups;

static const int kBlock = 256;

// ---------------------------------------------------------------------------
// The CSR operations (product, defect, Jacobi sweep, restriction, prolongation) are the
// kernels of csr.cuh.  group_sum: sum over aligned groups of GS lanes; every
// lane of the warp must call it.
// ---------------------------------------------------------------------------
template <int GS, typename T> __device__ __forceinline__ T group_sum(T v)
{
#pragma unroll
  for (int o = GS / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, GS);
  return v;
}

// first sweep when the active part of x is zero: only Dirichlet columns (numbered last,
// so at the end of every sorted row, from dir_start[r]) can contribute
template <typename T>
__global__ void jacobi_first_kernel(int n, int n_active, const int *__restrict__ rp,
                                    const int *__restrict__ kc, const int *__restrict__ dir_start,
                                    const T *__restrict__ a, const T *__restrict__ diag,
                                    const T *__restrict__ x, const T *__restrict__ f,
                                    T *__restrict__ xo, T omega, int x_all_zero)
{
  CD_PDL_ENTRY();
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  if (r >= n_active) { xo[r] = f[r]; return; }
  T s = f[r];
  if (!x_all_zero)
    for (int j = dir_start[r]; j < rp[r + 1]; j++) s -= a[j] * x[kc[j]];
  xo[r] = omega * s / diag[r];
}

// start of a cycle on the finest level fused with its first damped-Jacobi sweep: the
// right-hand side is the (FP64) input vector read through the pointer slot io[0]; the start
// vector is zero on active rows and the right-hand side on Dirichlet rows
// (MultiGridScaIte.C:79-85), so the sweep gives y = omega (f - A_D f_D) / a_rr on active rows
// (A_D: the Dirichlet columns, from dir_start[r]) and y = f on Dirichlet rows.
// Blocks [0, nb1): one thread per row, every row's rhs, y on the rows without Dirichlet
// columns; the remaining blocks: 8 threads per row of the list dir_rows (the active rows
// with Dirichlet columns), each thread issuing its first 4 column/value loads at once.
// Every lane of a warp of the second part reaches the shuffle.
template <typename T>
__global__ void __launch_bounds__(256) mg_start_first_kernel(int n, int n_active, int nb1, int n_dir_rows,
                                                             const int *__restrict__ dir_rows,
                                                             const int *__restrict__ rp,
                                                             const int *__restrict__ kc,
                                                             const int *__restrict__ dir_start,
                                                             const T *__restrict__ a, const T *__restrict__ diag,
                                                             double *const *__restrict__ io, T *__restrict__ rhs,
                                                             T *__restrict__ y, T omega)
{
  CD_PDL_ENTRY();
  const double *in = io[0];
  if ((int)blockIdx.x < nb1)
  {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const T f = (T)in[r];
    rhs[r] = f;
    if (r >= n_active)
      y[r] = f;
    else if (dir_start[r] == rp[r + 1])
      y[r] = omega * (f - T(0)) / diag[r];
    return;
  }
  constexpr int U = 4;
  const int lane = threadIdx.x % 8;
  const int q = (int)(((long)(blockIdx.x - nb1) * blockDim.x + threadIdx.x) / 8);
  const int r = q < n_dir_rows ? dir_rows[q] : -1;
  T t = 0;
  if (r >= 0)
  {
    const int b = dir_start[r], e = rp[r + 1];
    int c[U];
    T v[U];
#pragma unroll
    for (int u = 0; u < U; u++)
    {
      const int j = b + lane + u * 8;
      c[u] = j < e ? kc[j] : -1;
      v[u] = j < e ? a[j] : T(0);
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (c[u] >= 0) t += v[u] * (T)in[c[u]];
    for (int j = b + lane + U * 8; j < e; j += 8) t += a[j] * (T)in[kc[j]];
  }
  t = group_sum<8>(t);
  if (r >= 0 && lane == 0) y[r] = omega * ((T)in[r] - t) / diag[r];
}

// exact coarse solve (SolveExact, MGLevel3D.C:839) with the explicit FP64 inverse of the
// active block: Dirichlet rows are identity rows, so sol_D = rhs_D and
// sol_A = inv(A_AA) (rhs_A - A_AD rhs_D); A_AD is read from the CSR values of each active
// row from its first Dirichlet column (dir_start) on.
template <typename T>
__global__ void coarse_exact_kernel(int n, int na, const int *__restrict__ rp, const int *__restrict__ kc,
                                    const int *__restrict__ dir_start, const double *__restrict__ a,
                                    const double *__restrict__ cinv, const T *__restrict__ rhs,
                                    T *__restrict__ sol)
{
  CD_PDL_ENTRY();
  extern __shared__ double b[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) b[i] = (double)rhs[i];
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nw = blockDim.x / 32;
  // one warp per active row for the Dirichlet columns (a row of the coarsest level can have
  // ~100 of them)
  for (int i = warp; i < na; i += nw)
  {
    double v = 0.0;
    for (int j = dir_start[i] + lane; j < rp[i + 1]; j += 32) v += a[j] * b[kc[j]];
    v = group_sum<32>(v);
    if (lane == 0) b[n + i] = b[i] - v;
  }
  for (int i = na + threadIdx.x; i < n; i += blockDim.x) sol[i] = (T)b[i];
  __syncthreads();
  for (int r = warp; r < na; r += nw)
  {
    double s = 0;
    for (int j = lane; j < na; j += 32) s += cinv[(size_t)r * na + j] * b[n + j];
    s = group_sum<32>(s);
    if (lane == 0) sol[r] = (T)s;
  }
}

// coarse smoother loop (MultiGrid3D.C:199-311): iterate the coarse smoother until the
// defect norm drops by SC_COARSE_RED_FACTOR_SCALAR or SC_COARSE_MAXIT_SCALAR sweeps,
// in one CTA; mode 1 Jacobi, 2 SOR, 3 SSOR (MGLevel3D.C:254-537)
template <typename T>
__global__ void coarse_smooth_kernel(int n, int n_active, const int *__restrict__ rp,
                                     const int *__restrict__ kc, const T *__restrict__ a,
                                     const T *__restrict__ f, T *__restrict__ sol, double omega,
                                     int mode, int maxit, double red_factor)
{
  CD_PDL_ENTRY();
  extern __shared__ double sh[];
  double *x = sh, *aux = sh + n;
  __shared__ double red[32];
  __shared__ double res_s;
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (double)sol[i];
  __syncthreads();
  auto defect_norm = [&]() {
    double acc = 0;
    for (int r = threadIdx.x; r < n; r += blockDim.x)
    {
      double s = (double)f[r];
      for (int j = rp[r]; j < rp[r + 1]; j++) s -= (double)a[j] * x[kc[j]];
      acc += s * s;
    }
    acc = group_sum<32>(acc);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
    __syncthreads();
    if (threadIdx.x == 0)
    {
      double t = 0;
      for (int w = 0; w < (int)blockDim.x / 32; w++) t += red[w];
      res_s = sqrt(t);
    }
    __syncthreads();
    return res_s;
  };
  double res = defect_norm();
  double target = red_factor * res;
  int it = 0;
  while (res > target && it < maxit)
  {
    // Dirichlet rows take the right-hand side
    for (int i = n_active + threadIdx.x; i < n; i += blockDim.x) x[i] = (double)f[i];
    __syncthreads();
    if (mode == 1)
    {
      for (int i = threadIdx.x; i < n; i += blockDim.x) aux[i] = x[i];
      __syncthreads();
      for (int r = threadIdx.x; r < n_active; r += blockDim.x)
      {
        double s = (double)f[r], dg = 1;
        for (int j = rp[r]; j < rp[r + 1]; j++)
        {
          int c = kc[j];
          if (c == r) dg = (double)a[j]; else s -= (double)a[j] * aux[c];
        }
        x[r] = (1 - omega) * aux[r] + omega * s / dg;
      }
      __syncthreads();
    }
    else
    {
      if (threadIdx.x < 32)
      {
        const int lane = threadIdx.x;
        for (int pass = 0; pass < (mode == 3 ? 2 : 1); pass++)
          for (int ii = 0; ii < n_active; ii++)
          {
            int r = pass == 0 ? ii : n_active - 1 - ii;
            double s = 0, dg = 0;
            for (int j = rp[r] + lane; j < rp[r + 1]; j += 32)
            {
              int c = kc[j];
              if (c == r) dg = (double)a[j]; else s += (double)a[j] * x[c];
            }
            s = group_sum<32>(s);
            dg = group_sum<32>(dg);
            if (lane == 0)
            {
              double t = x[r];
              x[r] = omega * (((double)f[r] - s) / dg - t) + t;
            }
            __syncwarp();
          }
      }
      __syncthreads();
    }
    res = defect_norm();
    it++;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) sol[i] = (T)x[i];
}

// ---------------------------------------------------------------------------
// dense vector kernels for FGMRES (FP64)
// ---------------------------------------------------------------------------
// One fused pass of classical Gram-Schmidt over K basis vectors Y[0..K) (row stride n):
//   GS_DOTS            partial dots  w . Y_j
//   GS_AXPY_DOTS_NORM  w -= sum_j coef_j Y_j, then partial dots d_j of the new w with every
//                      Y_j and ||w||^2; the last block then leaves ||w - sum_j d_j Y_j||^2 =
//                      ||w||^2 - sum_j d_j^2 (Y orthonormal, d = Y^T w) in *norm_out, so the
//                      second classical Gram-Schmidt pass needs no third pass: the next basis
//                      vector (w - Y d) / norm is formed by axpy_scale_kernel
// Every thread keeps the K basis values of its row in registers; per-block partials go to
// partial[block * 33 + slot] and are summed in block order by the pass's last block.
enum { GS_DOTS = 0, GS_AXPY_DOTS_NORM = 1 };

// Block partials of NS sums and their reduction by the last block to arrive (an arrival
// counter, reset by that block): partial[block * 33 + slot], then out[slot] summed in block
// order (lanes over blocks, then a fixed warp tree).  Every thread of the block calls it.
// With norm_out, out[0..NS-1) are dot products d_j of a vector with orthonormal vectors and
// out[NS-1] the vector's squared norm; the last block also stores max(0, out[NS-1] - sum d_j^2).
template <int NS>
__device__ __forceinline__ void gs_reduce(const double (&acc)[NS], double *__restrict__ partial,
                                          double *__restrict__ out, unsigned *__restrict__ counter,
                                          double *__restrict__ norm_out = nullptr)
{
  __shared__ double red[kBlock / 32][NS];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
#pragma unroll
  for (int j = 0; j < NS; j++)
  {
    double v = group_sum<32>(acc[j]);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < NS)
  {
    double t = 0;
    for (int g = 0; g < kBlock / 32; g++) t += red[g][threadIdx.x];
    partial[(size_t)blockIdx.x * 33 + threadIdx.x] = t;
    __threadfence();
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the other blocks' partials are read from L2 (ld.global.cg), eight at a time in flight, and
  // added in block order
  for (int j = warp; j < NS; j += kBlock / 32)
  {
    double t = 0;
    for (int b0 = lane; b0 < (int)gridDim.x; b0 += 32 * 8)
    {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; u++)
      {
        const int b = b0 + 32 * u;
        v[u] = b < (int)gridDim.x ? __ldcg(partial + (size_t)b * 33 + j) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) t += v[u];
    }
    t = group_sum<32>(t);
    if (lane == 0) out[j] = t;
  }
  if (norm_out)
  {
    __syncthreads();
    if (threadIdx.x == 0)
    {
      double r = out[NS - 1];
      for (int j = 0; j < NS - 1; j++) r -= out[j] * out[j];
      norm_out[0] = r > 0.0 ? r : 0.0;
    }
  }
  if (threadIdx.x == 0) *counter = 0u;
}

template <int K, int MODE>
__global__ void __launch_bounds__(kBlock) gs_pass_kernel(int n, const double *__restrict__ Y,
                                                         double *__restrict__ w,
                                                         const double *__restrict__ coef,
                                                         double *__restrict__ partial,
                                                         double *__restrict__ out, unsigned *__restrict__ counter,
                                                         double *__restrict__ norm_out)
{
  CD_PDL_ENTRY();
  constexpr int NS = MODE == GS_AXPY_DOTS_NORM ? K + 1 : K;
  double acc[NS];
#pragma unroll
  for (int j = 0; j < NS; j++) acc[j] = 0;
  double cf[K];
#pragma unroll
  for (int j = 0; j < K; j++) cf[j] = MODE == GS_DOTS ? 0.0 : coef[j];
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
  {
    double y[K];
#pragma unroll
    for (int j = 0; j < K; j++) y[j] = __ldg(Y + (size_t)j * n + i);
    double wi = w[i];
    if (MODE != GS_DOTS)
    {
#pragma unroll
      for (int j = 0; j < K; j++) wi -= cf[j] * y[j];
      w[i] = wi;
    }
#pragma unroll
    for (int j = 0; j < K; j++) acc[j] += wi * y[j];
    if constexpr (MODE == GS_AXPY_DOTS_NORM) acc[NS - 1] += wi * wi;
  }
  gs_reduce<NS>(acc, partial, out, counter, MODE == GS_AXPY_DOTS_NORM ? norm_out : nullptr);
}

template <int MODE>
static void launch_gs(int k, int grid, cudaStream_t st, int n, const double *Y, double *w, const double *coef,
                      double *partial, double *out, unsigned *counter, double *norm_out = nullptr)
{
  switch (k)
  {
#define CD_GS_CASE(K) case K: (void)cd_launch(gs_pass_kernel<K, MODE>, grid, kBlock, 0, st, n, Y, w, coef, partial, out, counter, norm_out); break;
    CD_GS_CASE(1) CD_GS_CASE(2) CD_GS_CASE(3) CD_GS_CASE(4) CD_GS_CASE(5) CD_GS_CASE(6) CD_GS_CASE(7)
    CD_GS_CASE(8) CD_GS_CASE(9) CD_GS_CASE(10) CD_GS_CASE(11) CD_GS_CASE(12) CD_GS_CASE(13) CD_GS_CASE(14)
    CD_GS_CASE(15) CD_GS_CASE(16) CD_GS_CASE(17) CD_GS_CASE(18) CD_GS_CASE(19) CD_GS_CASE(20) CD_GS_CASE(21)
    CD_GS_CASE(22) CD_GS_CASE(23) CD_GS_CASE(24) CD_GS_CASE(25) CD_GS_CASE(26) CD_GS_CASE(27) CD_GS_CASE(28)
    CD_GS_CASE(29) CD_GS_CASE(30) CD_GS_CASE(31) CD_GS_CASE(32)
#undef CD_GS_CASE
    default: break;
  }
}

// Phase 2 of the matrix-free FP64 product fused with the first Gram-Schmidt pass: w = A x from
// the per-cell products (8-wide incidence records, ascending cell order; Dirichlet rows w = x)
// and the partial dots w . Y_j of the K basis vectors, reduced like a GS_DOTS pass.
template <int K>
__global__ void __launch_bounds__(kBlock) mf64_row_dots_kernel(int n, int na, const int *__restrict__ inc8,
                                                               const double *__restrict__ ybuf,
                                                               const double *__restrict__ x, double *__restrict__ w,
                                                               const double *__restrict__ Y, double *__restrict__ partial,
                                                               double *__restrict__ out, unsigned *__restrict__ counter)
{
  CD_PDL_ENTRY();
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; j++) acc[j] = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
  {
    double y[K];
#pragma unroll
    for (int j = 0; j < K; j++) y[j] = __ldg(Y + (size_t)j * n + r);
    double s;
    if (r >= na)
      s = x[r];
    else
    {
      const int4 i0 = __ldg((const int4 *)(inc8 + (size_t)r * 8)), i1 = __ldg((const int4 *)(inc8 + (size_t)r * 8) + 1);
      const int ix[8] = {i0.x, i0.y, i0.z, i0.w, i1.x, i1.y, i1.z, i1.w};
      double yv[8];
#pragma unroll
      for (int j = 0; j < 8; j++) yv[j] = ix[j] >= 0 ? ybuf[ix[j]] : 0.0;
      s = 0;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (ix[j] >= 0) s += yv[j];
    }
    w[r] = s;
#pragma unroll
    for (int j = 0; j < K; j++) acc[j] += s * y[j];
  }
  gs_reduce<K>(acc, partial, out, counter);
}

static void launch_row_dots(int k, int grid, cudaStream_t st, int n, int na, const int *inc8, const double *ybuf,
                            const double *x, double *w, const double *Y, double *partial, double *out,
                            unsigned *counter)
{
  switch (k)
  {
#define CD_RD_CASE(K) case K: (void)cd_launch(mf64_row_dots_kernel<K>, grid, kBlock, 0, st, n, na, inc8, ybuf, x, w, Y, partial, out, counter); break;
    CD_RD_CASE(1) CD_RD_CASE(2) CD_RD_CASE(3) CD_RD_CASE(4) CD_RD_CASE(5) CD_RD_CASE(6) CD_RD_CASE(7)
    CD_RD_CASE(8) CD_RD_CASE(9) CD_RD_CASE(10) CD_RD_CASE(11) CD_RD_CASE(12) CD_RD_CASE(13) CD_RD_CASE(14)
    CD_RD_CASE(15) CD_RD_CASE(16) CD_RD_CASE(17) CD_RD_CASE(18) CD_RD_CASE(19) CD_RD_CASE(20) CD_RD_CASE(21)
    CD_RD_CASE(22) CD_RD_CASE(23) CD_RD_CASE(24) CD_RD_CASE(25) CD_RD_CASE(26) CD_RD_CASE(27) CD_RD_CASE(28)
    CD_RD_CASE(29) CD_RD_CASE(30) CD_RD_CASE(31) CD_RD_CASE(32)
#undef CD_RD_CASE
    default: break;
  }
}

__global__ void sum_blocks_kernel(int nblocks, const double *__restrict__ partial, double *out)
{
  CD_PDL_ENTRY();
  __shared__ double red[32];
  double t = 0;
  // fixed per-thread order, then fixed tree
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) t += partial[b];
  t = group_sum<32>(t);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = t;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double s = 0;
    for (int w = 0; w < (int)blockDim.x / 32; w++) s += red[w];
    out[0] = s;
  }
}

// y = x / sqrt(*nrm2) unless *nrm2 == 0 (the next Arnoldi vector, scaled on the device so that
// the host need not have read the norm yet)
// With io, the first thread also sets the multigrid cycle graph's (in, out) slot to (y, z_next):
// y is the next preconditioner input, so the cycle needs no pointer kernel of its own.
__global__ void scale_norm_kernel(int n, const double *__restrict__ nrm2, const double *__restrict__ x,
                                  double *__restrict__ y, double **io, double *z_next)
{
  CD_PDL_ENTRY();
  const double hn = sqrt(*nrm2);
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (io && i == 0)
  {
    io[0] = y;
    io[1] = z_next;
  }
  if (hn != 0 && i < n) y[i] = (1.0 / hn) * x[i];
}

// y = (w - sum_j coef_j Y_j) / sqrt(*nrm2) unless *nrm2 == 0: the second Gram-Schmidt pass's
// update of w (in the order of the GS passes) and the next basis vector in one pass
template <int K>
__global__ void __launch_bounds__(256) axpy_scale_kernel(int n, const double *__restrict__ Y,
                                                         const double *__restrict__ w, const double *__restrict__ coef,
                                                         const double *__restrict__ nrm2, double *__restrict__ y,
                                                         double **io, double *z_next)
{
  CD_PDL_ENTRY();
  const double hn = sqrt(*nrm2);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (io && i == 0)
  {
    // the cycle graph's (in, out) slot for the next preconditioner application
    io[0] = y;
    io[1] = z_next;
  }
  if (hn == 0 || i >= n) return;
  double v[K];
#pragma unroll
  for (int j = 0; j < K; j++) v[j] = __ldg(Y + (size_t)j * n + i);
  double wi = w[i];
#pragma unroll
  for (int j = 0; j < K; j++) wi -= coef[j] * v[j];
  y[i] = (1.0 / hn) * wi;
}

static void launch_axpy_scale(int k, int grid, cudaStream_t st, int n, const double *Y, const double *w,
                              const double *coef, const double *nrm2, double *y, double **io, double *z_next)
{
  switch (k)
  {
#define CD_AS_CASE(K) case K: (void)cd_launch(axpy_scale_kernel<K>, grid, 256, 0, st, n, Y, w, coef, nrm2, y, io, z_next); break;
    CD_AS_CASE(1) CD_AS_CASE(2) CD_AS_CASE(3) CD_AS_CASE(4) CD_AS_CASE(5) CD_AS_CASE(6) CD_AS_CASE(7)
    CD_AS_CASE(8) CD_AS_CASE(9) CD_AS_CASE(10) CD_AS_CASE(11) CD_AS_CASE(12) CD_AS_CASE(13) CD_AS_CASE(14)
    CD_AS_CASE(15) CD_AS_CASE(16) CD_AS_CASE(17) CD_AS_CASE(18) CD_AS_CASE(19) CD_AS_CASE(20) CD_AS_CASE(21)
    CD_AS_CASE(22) CD_AS_CASE(23) CD_AS_CASE(24) CD_AS_CASE(25) CD_AS_CASE(26) CD_AS_CASE(27) CD_AS_CASE(28)
    CD_AS_CASE(29) CD_AS_CASE(30) CD_AS_CASE(31) CD_AS_CASE(32)
#undef CD_AS_CASE
    default: break;
  }
}

__global__ void set_io_kernel(double **io, const double *r, double *z)
{
  CD_PDL_ENTRY();
  io[0] = const_cast<double *>(r);
  io[1] = z;
}

__global__ void scale_kernel(int n, double alpha, const double *__restrict__ x, double *__restrict__ y)
{
  CD_PDL_ENTRY();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = alpha * x[i];
}

// x += sum_j c[j] Z[j]
__global__ void update_kernel(int n, int k, const double *__restrict__ c, const double *__restrict__ Z,
                              double *__restrict__ x)
{
  CD_PDL_ENTRY();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0;
  for (int j = 0; j < k; j++) s += c[j] * Z[(size_t)j * n + i];
  x[i] += s;
}

__global__ void axpy_kernel(int n, double alpha, const double *__restrict__ x, double *__restrict__ y)
{
  CD_PDL_ENTRY();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += alpha * x[i];
}

template <typename A, typename B> __global__ void convert_kernel(int n, const A *__restrict__ x, B *__restrict__ y)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (B)x[i];
}

// zero a vector and copy the Dirichlet part of rhs into it (MultiGridScaIte.C:79-85:
// zero start + SetDirichletNodes, MultiGrid3D.C:671)
// The input vector is read through a device-side pointer slot so that one captured
// CUDA graph serves every FGMRES basis vector.
template <typename T>
__global__ void mg_start_kernel(int n, int n_active, double *const *__restrict__ io, T *__restrict__ rhs,
                                T *__restrict__ sol)
{
  CD_PDL_ENTRY();
  const double *rhs_in = io[0];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T v = (T)rhs_in[i];
  rhs[i] = v;
  sol[i] = i < n_active ? T(0) : v;
}

template <typename T>
__global__ void mg_finish_kernel(int n, const T *__restrict__ sol, double *const *__restrict__ io)
{
  CD_PDL_ENTRY();
  double *out = io[1];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)sol[i];
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
template <typename T> static const T *mat(const Space &s);
template <> const double *mat<double>(const Space &s) { return s.d_a; }
template <> const float *mat<float>(const Space &s) { return s.d_a32; }
template <typename T> static const T *dg(const Space &s);
template <> const double *dg<double>(const Space &s) { return s.d_diag; }
template <> const float *dg<float>(const Space &s) { return s.d_diag32; }
template <typename T> static const T *pval(const Level &l);
template <> const double *pval<double>(const Level &l) { return l.d_p_val; }
template <> const float *pval<float>(const Level &l) { return l.d_p_val32; }
template <typename T> static const T *rval(const Level &l);
template <> const double *rval<double>(const Level &l) { return l.d_r_val; }
template <> const float *rval<float>(const Level &l) { return l.d_r_val32; }
template <typename T> static LevelVec<T> &vecs(Level &l);
template <> LevelVec<double> &vecs<double>(Level &l) { return l.v64; }
template <> LevelVec<float> &vecs<float>(Level &l) { return l.v32; }
template <typename T> static LevelVec<T> &canon(Level &l);
template <> LevelVec<double> &canon<double>(Level &l) { return l.c64; }
template <> LevelVec<float> &canon<float>(Level &l) { return l.c32; }

// the CSR operations of the solver (csr.cuh)
template <typename T> static CsrArgs<T> csr_args(const Space &s, const T *x)
{
  CsrArgs<T> p;
  p.n = s.n_dof;
  p.n_active = s.n_active;
  p.rp = s.d_row_ptr;
  p.kc = s.d_kcol;
  p.a = mat<T>(s);
  p.x = x;
  return p;
}
// FP64 operations on a matrix with TMA tiles go through csr_tma_kernel in the variant (tile
// capacity, stages) the autotuner chose for the matrix (variant 0 until it has run):
// persistent CTAs, as many per SM as the variant's shared memory allows, never more than
// there are tiles
struct TmaVariant
{
  int cap, stages, tpr; // nonzeros per tile, shared-memory stages, threads per row
};
// (variants with 8 threads per row and 32-row tiles measured 43.4-47.1 us against 41.4 us for
// the best 64-row one on the 32^3 Q2 matrix, and are not tried)
static const TmaVariant kTmaVariants[] = {{2048, 4, 4}, {2048, 2, 4}, {3072, 3, 4}, {3072, 2, 4},
                                          {4096, 2, 4}, {2048, 3, 4}, {1536, 2, 4}};
constexpr int kNumTmaVariants = sizeof(kTmaVariants) / sizeof(kTmaVariants[0]);

template <int MODE> static void (*tma_kernel(int v))(CsrArgs<double>, const int2 *, int, int *)
{
  switch (v)
  {
    case 1: return csr_tma_kernel<MODE, 2048, 2>;
    case 2: return csr_tma_kernel<MODE, 3072, 3>;
    case 3: return csr_tma_kernel<MODE, 3072, 2>;
    case 4: return csr_tma_kernel<MODE, 4096, 2>;
    case 5: return csr_tma_kernel<MODE, 2048, 3>;
    case 6: return csr_tma_kernel<MODE, 1536, 2>;
    default: return csr_tma_kernel<MODE, 2048, 4>;
  }
}
// rows per tile of a variant: the consumer warps' rows (8 warps x 32 / threads per row)
static int tma_rows(int v) { return kTmaWarps * 32 / kTmaVariants[v].tpr; }
static int tma_smem(int v) { return tma_smem_bytes(kTmaVariants[v].cap, kTmaVariants[v].stages); }
static int tma_var(const Space &s) { return s.tma_var < 0 ? 0 : s.tma_var; }

// resident CTAs per SM of a variant (its shared-memory attribute set on the way)
static int tma_ctas_per_sm(int v)
{
  const int sm = tma_smem(v);
  int nb = 0;
  for (auto k : {tma_kernel<CM_SPMV>(v), tma_kernel<CM_DEFECT>(v), tma_kernel<CM_JACOBI>(v)})
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, tma_kernel<CM_SPMV>(v), (kTmaWarps + 1) * 32, sm) != cudaSuccess)
  {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

static int tma_grid(const cdgpu_ctx *ctx, const Space &s)
{
  const int per_sm = s.tma_var < 0 ? 2 : std::max(1, s.tma_ctas);
  return std::max(1, std::min(s.n_tiles, ctx->sm_count * per_sm));
}

template <typename T, int MODE> static bool launch_tma(cdgpu_ctx *ctx, const Space &s, const CsrArgs<T> &pa, int grid)
{
  if constexpr (std::is_same<T, double>::value)
  {
    if (s.n_tiles > 0 && ctx->d_err)
    {
      CsrArgs<double> p = pa;
      // the producer streams the matrix before waiting for the predecessor when no kernel
      // that writes the matrix can still be running: inside the captured cycle, or once a
      // launch of the same assembly has waited (every later kernel starts after that one's
      // wait, hence after the assembly)
      p.pre = ctx->pdl_pre || s.tma_safe_version == s.assembly_version ? 1 : 0;
      if (!p.pre) s.tma_safe_version = s.assembly_version;
      const int v = tma_var(s);
      (void)cd_launch(tma_kernel<MODE>(v), grid, (kTmaWarps + 1) * 32, tma_smem(v), ctx->stream, p,
                      (const int2 *)s.d_tiles, s.n_tiles, ctx->d_err);
      return true;
    }
  }
  return false;
}
template <typename T> static void csr_jacobi(cdgpu_ctx *ctx, const Space &s, const T *x, const T *f, T *xo, T omega)
{
  CsrArgs<T> p = csr_args<T>(s, x);
  p.f = f;
  p.diag = dg<T>(s);
  p.y = xo;
  p.omega = omega;
  if (launch_tma<T, CM_JACOBI>(ctx, s, p, tma_grid(ctx, s))) return;
  launch_csr<T, CM_JACOBI>(ctx, s.shape, p, csr_grid(ctx, s.shape, s.n_dof));
}
// grid: the launch's number of blocks (and of partial sums), from defect_grid
template <typename T>
static void csr_defect(cdgpu_ctx *ctx, const Space &s, const T *x, const T *f, T *d, double *partial, int grid)
{
  CsrArgs<T> p = csr_args<T>(s, x);
  p.f = f;
  p.y = d;
  p.partial = partial;
  if (launch_tma<T, CM_DEFECT>(ctx, s, p, grid)) return;
  launch_csr<T, CM_DEFECT>(ctx, s.shape, p, grid);
}
template <typename T> static int defect_grid(const cdgpu_ctx *ctx, const Space &s)
{
  if (std::is_same<T, double>::value && s.n_tiles > 0 && ctx->d_err) return tma_grid(ctx, s);
  return csr_grid(ctx, s.shape, s.n_dof);
}
template <typename T> static void csr_spmv(cdgpu_ctx *ctx, const Space &s, const T *x, T *y)
{
  CsrArgs<T> p = csr_args<T>(s, x);
  p.y = y;
  if (launch_tma<T, CM_SPMV>(ctx, s, p, tma_grid(ctx, s))) return;
  launch_csr<T, CM_SPMV>(ctx, s.shape, p, csr_grid(ctx, s.shape, s.n_dof));
}
// coarse rhs = R d (zero on non-active coarse rows), coarse solution reset
template <typename T>
static void csr_restrict(cdgpu_ctx *ctx, const Level &L, const Space &sc, const T *d, T *crhs, T *csol)
{
  CsrArgs<T> p;
  p.n = sc.n_dof;
  p.n_active = sc.n_active;
  p.rp = L.d_r_row;
  p.kc = L.d_r_col;
  p.a = rval<T>(L);
  p.x = d;
  p.y = crhs;
  p.y2 = csol;
  launch_csr<T, CM_RESTRICT>(ctx, L.r_shape, p, csr_grid(ctx, L.r_shape, p.n));
}
// sol += damp * P xc on active fine rows
template <typename T>
static void csr_prolong(cdgpu_ctx *ctx, const Level &L, const Space &s, const T *xc, T *sol, T damp)
{
  CsrArgs<T> p;
  p.n = s.n_dof;
  p.n_active = s.n_active;
  p.rp = L.d_p_row;
  p.kc = L.d_p_col;
  p.a = pval<T>(L);
  p.x = xc;
  p.y = sol;
  p.omega = damp;
  launch_csr<T, CM_PROLONG>(ctx, L.p_shape, p, csr_grid(ctx, L.p_shape, p.n_active));
}

template <typename T> static int jacobi_sweep(cdgpu_ctx *ctx, Level &L, T omega)
{
  LevelVec<T> &v = vecs<T>(L);
  const Space &s = *L.sp;
  if constexpr (std::is_same<T, float>::value)
  {
    if (use_mf(s))
    {
      mf_apply_cells(ctx, s, v.sol);
      CD_LAUNCHED(ctx);
      mf_rows<MF_JACOBI>(ctx, s, v.sol, v.rhs, s.d_diag32, v.alt, omega);
      CD_LAUNCHED(ctx);
      std::swap(v.sol, v.alt);
      return CDGPU_OK;
    }
  }
  csr_jacobi<T>(ctx, s, v.sol, v.rhs, v.alt, omega);
  CD_LAUNCHED(ctx);
  std::swap(v.sol, v.alt);
  return CDGPU_OK;
}

template <typename T> static int jacobi_first(cdgpu_ctx *ctx, Level &L, T omega, int all_zero)
{
  LevelVec<T> &v = vecs<T>(L);
  const Space &s = *L.sp;
  (void)cd_launch(jacobi_first_kernel<T>, (s.n_dof + 255) / 256, 256, 0, ctx->stream, 
      s.n_dof, s.n_active, s.d_row_ptr, s.d_kcol, s.d_dir_start, mat<T>(s), dg<T>(s), v.sol, v.rhs,
      v.alt, omega, all_zero);
  CD_LAUNCHED(ctx);
  std::swap(v.sol, v.alt);
  return CDGPU_OK;
}

// ---------------------------------------------------------------------------
// V/W/F cycle
// ---------------------------------------------------------------------------
struct CycleState
{
  const cdgpu_solver_params *p;
  int rec[64];
  int pre_done[64];    // pre-smoothing sweeps already done (fused into the cycle's start)
  bool sol_zero[64];   // active part and Dirichlet part zero
  bool active_zero[64];
};

template <typename T> static int smooth(cdgpu_ctx *ctx, Hierarchy &h, CycleState &cs, int i, int count)
{
  Level &L = h.lev[i];
  T omega = (T)cs.p->omega;
  int rc;
  for (int k = 0; k < count; k++)
  {
    if (cs.active_zero[i])
      rc = jacobi_first<T>(ctx, L, omega, cs.sol_zero[i] ? 1 : 0);
    else
      rc = jacobi_sweep<T>(ctx, L, omega);
    if (rc) return rc;
    cs.active_zero[i] = cs.sol_zero[i] = false;
  }
  return CDGPU_OK;
}

template <typename T> static int coarse_solve(cdgpu_ctx *ctx, Hierarchy &h, CycleState &cs)
{
  Level &L = h.lev[0];
  const Space &s = *L.sp;
  LevelVec<T> &v = vecs<T>(L);
  if (cs.p->coarse_smoother == 17)
  {
    size_t sm = sizeof(double) * (s.n_dof + s.n_active);
    (void)cd_launch(coarse_exact_kernel<T>, 1, 1024, sm, ctx->stream, s.n_dof, s.n_active, s.d_row_ptr, s.d_kcol,
                                                         s.d_dir_start, s.d_a, h.d_cinv, v.rhs, v.sol);
    CD_LAUNCHED(ctx);
  }
  else
  {
    size_t sm = sizeof(double) * 2 * s.n_dof;
    (void)cd_launch(coarse_smooth_kernel<T>, 1, 256, sm, ctx->stream, s.n_dof, s.n_active, s.d_row_ptr, s.d_kcol,
                                                         mat<T>(s), v.rhs, v.sol, cs.p->omega,
                                                         cs.p->coarse_smoother, cs.p->coarse_maxit,
                                                         cs.p->coarse_red);
    CD_LAUNCHED(ctx);
  }
  cs.sol_zero[0] = cs.active_zero[0] = false;
  return CDGPU_OK;
}

template <typename T> static int cycle(cdgpu_ctx *ctx, Hierarchy &h, CycleState &cs, int i)
{
  if (i == 0) return coarse_solve<T>(ctx, h, cs);
  Level &L = h.lev[i], &C = h.lev[i - 1];
  const Space &s = *L.sp, &sc = *C.sp;
  LevelVec<T> &v = vecs<T>(L), &vc = vecs<T>(C);
  int rc;
  if ((rc = smooth<T>(ctx, h, cs, i, cs.p->pre - cs.pre_done[i]))) return rc;
  cs.pre_done[i] = 0;
  bool done = false;
  if constexpr (std::is_same<T, float>::value)
  {
    if (use_mf(s))
    {
      mf_apply_cells(ctx, s, v.sol);
      CD_LAUNCHED(ctx);
      mf_rows<MF_DEFECT>(ctx, s, v.sol, v.rhs, s.d_diag32, v.def, 0.f);
      done = true;
    }
  }
  if (!done) csr_defect<T>(ctx, s, v.sol, v.rhs, v.def, nullptr, defect_grid<T>(ctx, s));
  CD_LAUNCHED(ctx);
  csr_restrict<T>(ctx, L, sc, v.def, vc.rhs, vc.sol);
  CD_LAUNCHED(ctx);
  cs.sol_zero[i - 1] = cs.active_zero[i - 1] = true;
  for (int j = 0; j < cs.rec[i]; j++)
    if ((rc = cycle<T>(ctx, h, cs, i - 1))) return rc;
  if (cs.p->cycle < 1) cs.rec[i] = 1;
  csr_prolong<T>(ctx, L, s, vc.sol, v.sol, (T)cs.p->gmg_damp);
  CD_LAUNCHED(ctx);
  return smooth<T>(ctx, h, cs, i, cs.p->post);
}

// enqueue one preconditioner application z = M^{-1} r (TMultiGridScaIte::Iterate with zero
// start); r and z are read from the device pointer slot h.d_io
template <typename T> static int mg_record(cdgpu_ctx *ctx, Hierarchy &h, const cdgpu_solver_params &p)
{
  int L = (int)h.lev.size();
  // every level starts from its own first buffer, so the recorded pointers are the same on
  // every application
  for (auto &lv : h.lev) vecs<T>(lv) = canon<T>(lv);
  Level &F = h.lev[L - 1];
  LevelVec<T> &v = vecs<T>(F);
  int n = F.sp->n_dof;
  CycleState cs;
  cs.p = &p;
  // SetRecursion(levels = L-1), MultiGrid3D.C:691-703
  cs.rec[1] = 1;
  for (int k = 2; k <= L - 1; k++) cs.rec[k] = p.cycle > 0 ? p.cycle : 2;
  for (int k = 0; k < L; k++)
  {
    cs.sol_zero[k] = cs.active_zero[k] = false;
    cs.pre_done[k] = 0;
  }
  if (L > 1 && p.pre >= 1)
  {
    // zero start and the first pre-smoothing sweep of the finest level in one kernel
    const Space &s = *F.sp;
    const int nb1 = (n + 255) / 256, nb2 = (int)(((long)s.n_dir_rows * 8 + 255) / 256);
    (void)cd_launch(mg_start_first_kernel<T>, nb1 + nb2, 256, 0, ctx->stream, n, s.n_active, nb1, s.n_dir_rows, s.d_dir_rows,
                                                                s.d_row_ptr, s.d_kcol, s.d_dir_start,
                                                           mat<T>(s), dg<T>(s), h.d_io, v.rhs, v.alt,
                                                           (T)p.omega);
    CD_LAUNCHED(ctx);
    std::swap(v.sol, v.alt);
    cs.pre_done[L - 1] = 1;
  }
  else
  {
    (void)cd_launch(mg_start_kernel<T>, (n + 255) / 256, 256, 0, ctx->stream, n, F.sp->n_active, h.d_io, v.rhs, v.sol);
    CD_LAUNCHED(ctx);
    cs.active_zero[L - 1] = true;
  }
  int rc = cycle<T>(ctx, h, cs, L - 1);
  if (rc) return rc;
  (void)cd_launch(mg_finish_kernel<T>, (n + 255) / 256, 256, 0, ctx->stream, n, v.sol, h.d_io);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

static bool same_cycle_params(const cdgpu_solver_params &a, const cdgpu_solver_params &b)
{
  return a.precision == b.precision && a.pre == b.pre && a.post == b.post && a.cycle == b.cycle &&
         a.coarse_smoother == b.coarse_smoother && a.coarse_maxit == b.coarse_maxit &&
         a.coarse_red == b.coarse_red && a.omega == b.omega && a.gmg_damp == b.gmg_damp;
}

// The whole V/W/F cycle (about 7 kernels per level) is captured once into a CUDA graph
// and replayed for every basis vector; only the two pointers in h.d_io change.
// io_ready: the kernel before this call already set the graph's (in, out) slot to (r, z)
static int mg_apply(cdgpu_ctx *ctx, Hierarchy &h, const cdgpu_solver_params &p, const double *r, double *z,
                    bool io_ready = false)
{
  const int k = p.precision == 1 ? 1 : 0;
  int rc;
  if (!h.gexec[k] || !same_cycle_params(h.gparams[k], p))
  {
    if (h.gexec[k]) { cudaGraphExecDestroy(h.gexec[k]); h.gexec[k] = nullptr; }
    // dynamic shared memory of the coarse kernels is set outside the capture
    const int nc = h.lev[0].sp->n_dof;
    const int sm1 = (int)(sizeof(double) * (nc + h.lev[0].sp->n_active)), sm2 = (int)(2 * sizeof(double) * nc);
    CD_CUDA(ctx, cudaFuncSetAttribute(coarse_exact_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm1));
    CD_CUDA(ctx, cudaFuncSetAttribute(coarse_exact_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm1));
    CD_CUDA(ctx, cudaFuncSetAttribute(coarse_smooth_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2));
    CD_CUDA(ctx, cudaFuncSetAttribute(coarse_smooth_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2));
    cudaGraph_t g = nullptr;
    const long long before = ctx->launches;
    CD_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->pdl_pre = true; // kernels of the cycle load matrix data before waiting (CD_PDL_WAIT)
    rc = k == 1 ? mg_record<float>(ctx, h, p) : mg_record<double>(ctx, h, p);
    ctx->pdl_pre = false;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    h.graph_nodes[k] = ctx->launches - before; // kernels per replay; capturing runs none
    ctx->launches = before;
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture of the multigrid cycle");
    e = cudaGraphInstantiate(&h.gexec[k], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { h.gexec[k] = nullptr; return cuda_fail(ctx, e, "graph instantiate"); }
    h.gparams[k] = p;
  }
  // the application's (in, out) pointers into the graph's slot: a one-thread kernel in the
  // stream's launch chain (a host-to-device copy would hold the stream for the copy engine's
  // round trip)
  if (!io_ready)
  {
    (void)cd_launch(set_io_kernel, 1, 1, 0, ctx->stream, h.d_io, r, z);
    CD_LAUNCHED(ctx);
  }
  CD_CUDA(ctx, cudaGraphLaunch(h.gexec[k], ctx->stream));
  ctx->launches += h.graph_nodes[k];
  return CDGPU_OK;
}

// Tiles of the TMA product: consecutive rows, at most kTmaRows rows and `cap` nonzeros per
// tile, for matrices whose stream does not fit in L2 (smaller ones are latency-bound and keep
// the plain kernels).  A row longer than the smallest capacity leaves the matrix on the plain
// kernels.
constexpr long kTmaMinNnz = 4L << 20;

static bool make_tiles(const Space &s, int cap, int rows, std::vector<int2> &tiles)
{
  tiles.clear();
  const int *rp = s.h_row_ptr.data();
  int r = 0;
  while (r < s.n_dof)
  {
    if (rp[r + 1] - rp[r] > cap) return false;
    int e = r;
    while (e < s.n_dof && e - r < rows && rp[e + 1] - rp[r] <= cap) e++;
    tiles.push_back(make_int2(r, rp[r]));
    r = e;
  }
  tiles.push_back(make_int2(s.n_dof, rp[s.n_dof]));
  return true;
}

int build_csr_tiles(cdgpu_ctx *ctx, Space &s)
{
  if (s.d_tiles) { cudaFree(s.d_tiles); s.d_tiles = nullptr; }
  s.n_tiles = 0;
  s.tma_var = -1;
  s.tma_report.clear();
  if (s.nnz < kTmaMinNnz) return CDGPU_OK;
  std::vector<int2> tiles;
  if (!make_tiles(s, kTmaVariants[0].cap, tma_rows(0), tiles)) return CDGPU_OK;
  int rc;
  if ((rc = ensure_err_flag(ctx))) return rc;
  if ((rc = dev_alloc(ctx, &s.d_tiles, tiles.size()))) return rc;
  CD_CUDA(ctx, cudaMemcpy(s.d_tiles, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice));
  if (tma_ctas_per_sm(0) <= 0) return cuda_fail(ctx, cudaErrorInvalidConfiguration, "TMA product: no resident CTA");
  s.n_tiles = (int)tiles.size() - 1;
  return CDGPU_OK;
}

// Tile-shape autotuner of the TMA product, run once per pattern on the first solve with
// assembled values (outside any stream capture): every variant (tile capacity, stages,
// resident CTAs per SM from its shared memory) times five products y = A x on this matrix
// after one warm-up launch; the fastest is kept with its tiles.  The report lists the
// variants and their mean times.
static int tune_tma(cdgpu_ctx *ctx, Space &s)
{
  if (s.n_tiles <= 0 || s.tma_var >= 0) return CDGPU_OK;
  int rc;
  double *x = nullptr, *y = nullptr;
  if ((rc = dev_alloc(ctx, &x, s.n_dof)) || (rc = dev_alloc(ctx, &y, s.n_dof)))
  {
    if (x) cudaFree(x);
    return rc;
  }
  CD_CUDA(ctx, cudaMemsetAsync(x, 0, sizeof(double) * s.n_dof, ctx->stream));
  cudaEvent_t e0, e1;
  CD_CUDA(ctx, cudaEventCreate(&e0));
  CD_CUDA(ctx, cudaEventCreate(&e1));
  int best = -1, best_ctas = 0, best_n = 0;
  float best_ms = 1e30f;
  int2 *best_tiles = nullptr;
  std::string report;
  for (int v = 0; v < kNumTmaVariants; v++)
  {
    std::vector<int2> tiles;
    const int ctas = tma_ctas_per_sm(v);
    if (ctas <= 0 || !make_tiles(s, kTmaVariants[v].cap, tma_rows(v), tiles)) continue;
    int2 *dt = nullptr;
    if ((rc = dev_alloc(ctx, &dt, tiles.size()))) break;
    CD_CUDA(ctx, cudaMemcpy(dt, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice));
    const int nt = (int)tiles.size() - 1;
    const int grid = std::max(1, std::min(nt, ctx->sm_count * ctas));
    CsrArgs<double> p = csr_args<double>(s, x);
    p.y = y;
    auto k = tma_kernel<CM_SPMV>(v);
    (void)cd_launch(k, grid, (kTmaWarps + 1) * 32, tma_smem(v), ctx->stream, p, (const int2 *)dt, nt, ctx->d_err);
    CD_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
    for (int i = 0; i < 5; i++)
      (void)cd_launch(k, grid, (kTmaWarps + 1) * 32, tma_smem(v), ctx->stream, p, (const int2 *)dt, nt, ctx->d_err);
    CD_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
    CD_CUDA(ctx, cudaEventSynchronize(e1));
    CD_LAUNCHED(ctx);
    float ms = 0;
    CD_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
    ms /= 5;
    char line[128];
    snprintf(line, sizeof(line), "%scap %d rows %d stages %d ctas/SM %d: %.1f us", report.empty() ? "" : "; ",
             kTmaVariants[v].cap, tma_rows(v), kTmaVariants[v].stages, ctas, 1e3 * ms);
    report += line;
    if (ms < best_ms)
    {
      if (best_tiles) cudaFree(best_tiles);
      best_tiles = dt;
      best_ms = ms;
      best = v;
      best_ctas = ctas;
      best_n = nt;
    }
    else
      cudaFree(dt);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(x);
  cudaFree(y);
  if (rc) { if (best_tiles) cudaFree(best_tiles); return rc; }
  if ((rc = assemble_check(ctx))) { if (best_tiles) cudaFree(best_tiles); return rc; } // wait flag of the timed launches
  if (best < 0) return CDGPU_OK; // keep the default variant
  cudaFree(s.d_tiles);
  s.d_tiles = best_tiles;
  s.n_tiles = best_n;
  s.tma_var = best;
  s.tma_ctas = best_ctas;
  char sel[96];
  snprintf(sel, sizeof(sel), "chosen: cap %d rows %d stages %d ctas/SM %d; ", kTmaVariants[best].cap, tma_rows(best),
           kTmaVariants[best].stages, best_ctas);
  s.tma_report = sel + report;
  return CDGPU_OK;
}

int csr_tuning_report(cdgpu_ctx *ctx, Space &s, std::string &out)
{
  (void)ctx;
  out = s.n_tiles > 0 ? (s.tma_var >= 0 ? s.tma_report : std::string("default variant (not tuned yet)"))
                      : std::string("plain CSR kernels (no TMA tiles for this matrix)");
  return CDGPU_OK;
}

// ---------------------------------------------------------------------------
// hierarchy buffers and the exact coarse inverse
// ---------------------------------------------------------------------------
template <typename T> static int alloc_vecs(cdgpu_ctx *ctx, LevelVec<T> &v, int n)
{
  int rc;
  if ((rc = dev_alloc(ctx, &v.sol, n)) || (rc = dev_alloc(ctx, &v.alt, n)) ||
      (rc = dev_alloc(ctx, &v.rhs, n)) || (rc = dev_alloc(ctx, &v.def, n)))
    return rc;
  CD_CUDA(ctx, cudaMemset(v.sol, 0, sizeof(T) * n));
  CD_CUDA(ctx, cudaMemset(v.alt, 0, sizeof(T) * n));
  return CDGPU_OK;
}

int setup_hierarchy_buffers(cdgpu_ctx *ctx, Hierarchy &h, int m)
{
  int rc;
  for (auto &L : h.lev)
  {
    if (!L.c64.sol && (rc = alloc_vecs(ctx, L.c64, L.sp->n_dof))) return rc;
    if (!L.c32.sol && (rc = alloc_vecs(ctx, L.c32, L.sp->n_dof))) return rc;
    L.v64 = L.c64;
    L.v32 = L.c32;
  }
  int n = h.lev.back().sp->n_dof;
  if (h.m != m)
  {
    if ((rc = dev_alloc(ctx, &h.d_V, (size_t)(m + 1) * n)) || (rc = dev_alloc(ctx, &h.d_Z, (size_t)(m + 1) * n)))
      return rc;
    h.m = m;
  }
  if (!h.d_w)
  {
    h.partial_blocks = std::min(ctx->sm_count * 4, (n + kBlock - 1) / kBlock);
    if (h.partial_blocks < 1) h.partial_blocks = 1;
    if ((rc = dev_alloc(ctx, &h.d_w, n)) || (rc = dev_alloc(ctx, &h.d_ctl, 256)) ||
        (rc = dev_alloc(ctx, &h.d_partial, (size_t)std::max(h.partial_blocks, ctx->sm_count * 8) * 33)) ||
        (rc = dev_alloc(ctx, &h.d_x, n)) || (rc = dev_alloc(ctx, &h.d_b, n)))
      return rc;
    CD_CUDA(ctx, cudaMallocHost((void **)&h.h_ctl, 256 * sizeof(double)));
    CD_CUDA(ctx, cudaMallocHost((void **)&h.h_slot, 2 * 80 * sizeof(double)));
    for (auto &e : h.ev_slot) CD_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : h.ev_ready) CD_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CD_CUDA(ctx, cudaEventCreateWithFlags(&h.ev_beta, cudaEventDisableTiming));
    CD_CUDA(ctx, cudaStreamCreateWithFlags(&h.cstream, cudaStreamNonBlocking));
    CD_CUDA(ctx, cudaMallocHost((void **)&h.h_io, 128 * sizeof(double *)));
    if ((rc = dev_alloc(ctx, &h.d_io, 2))) return rc;
    if ((rc = dev_alloc(ctx, &h.d_gs_count, 1))) return rc;
    CD_CUDA(ctx, cudaMemset(h.d_gs_count, 0, sizeof(unsigned)));
  }
  return CDGPU_OK;
}

// dense copy of the active block A_AA (rows and columns below na) of a CSR matrix
__global__ void csr_to_dense_kernel(int na, const int *__restrict__ rp, const int *__restrict__ kc,
                                    const double *__restrict__ a, double *__restrict__ dense)
{
  CD_PDL_ENTRY();
  int r = blockIdx.x;
  for (int c = threadIdx.x; c < na; c += blockDim.x) dense[(size_t)r * na + c] = 0.0;
  __syncthreads();
  for (int j = rp[r] + threadIdx.x; j < rp[r + 1]; j += blockDim.x)
    if (kc[j] < na) dense[(size_t)r * na + kc[j]] = a[j];
}

// In-place Gauss-Jordan inversion with partial (row) pivoting, one CTA; the matrix lives in
// shared memory when it fits, otherwise in the global buffer itself.  flag[0] = 1 when a
// zero pivot is met.
__global__ void __launch_bounds__(1024) gj_invert_kernel(int n, double *__restrict__ g, int use_smem,
                                                         int *__restrict__ piv, int *__restrict__ flag)
{
  CD_PDL_ENTRY();
  extern __shared__ double sm[];
  double *A = use_smem ? sm : g;
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int p_s;
  const int nt = blockDim.x, t = threadIdx.x, lane = t % 32, warp = t / 32;
  if (use_smem)
    for (int i = t; i < n * n; i += nt) A[i] = g[i];
  __syncthreads();
  for (int k = 0; k < n; k++)
  {
    // pivot search in column k, rows k..n-1 (largest magnitude, lowest row on ties)
    double bv = -1.0;
    int bi = n;
    for (int i = k + t; i < n; i += nt)
    {
      double v = fabs(A[(size_t)i * n + k]);
      if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1)
    {
      double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
    __syncthreads();
    if (t == 0)
    {
      double v = -1.0;
      int p = n;
      for (int w = 0; w < nt / 32; w++)
        if (red_v[w] > v || (red_v[w] == v && red_i[w] < p)) { v = red_v[w]; p = red_i[w]; }
      p_s = p;
      piv[k] = p;
      if (!(v > 0.0)) flag[0] = 1;
    }
    __syncthreads();
    const int p = p_s;
    if (p != k)
      for (int j = t; j < n; j += nt)
      {
        double tmp = A[(size_t)k * n + j];
        A[(size_t)k * n + j] = A[(size_t)p * n + j];
        A[(size_t)p * n + j] = tmp;
      }
    __syncthreads();
    const double pivot = A[(size_t)k * n + k];
    __syncthreads();
    for (int j = t; j < n; j += nt)
      A[(size_t)k * n + j] = (j == k ? 1.0 : A[(size_t)k * n + j]) / pivot;
    __syncthreads();
    // eliminate column k from the other rows: first every column but k (which holds the
    // multipliers), then column k itself
    for (int i = warp; i < n; i += nt / 32)
    {
      if (i == k) continue;
      const double f = A[(size_t)i * n + k];
      if (f == 0.0) continue;
      for (int j = lane; j < n; j += 32)
        if (j != k) A[(size_t)i * n + j] -= f * A[(size_t)k * n + j];
    }
    __syncthreads();
    for (int i = t; i < n; i += nt)
      if (i != k) A[(size_t)i * n + k] = -A[(size_t)i * n + k] * A[(size_t)k * n + k];
    __syncthreads();
  }
  // undo the row interchanges as column interchanges, last first
  for (int k = n - 1; k >= 0; k--)
  {
    int p = piv[k];
    if (p != k)
      for (int i = t; i < n; i += nt)
      {
        double tmp = A[(size_t)i * n + k];
        A[(size_t)i * n + k] = A[(size_t)i * n + p];
        A[(size_t)i * n + p] = tmp;
      }
    __syncthreads();
  }
  if (use_smem)
    for (int i = t; i < n * n; i += nt) g[i] = A[i];
}

int refresh_coarse_inverse(cdgpu_ctx *ctx, Hierarchy &h)
{
  Space &s = *h.lev[0].sp;
  if (h.d_cinv && h.cinv_version == s.assembly_version) return CDGPU_OK;
  const int na = s.n_active;
  if (na > 4096)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "exact coarse solve: more than 4096 active DOFs on the coarsest level");
  int rc;
  if (!h.d_cinv)
  {
    if ((rc = dev_alloc(ctx, &h.d_cinv, (size_t)na * na)) || (rc = dev_alloc(ctx, &h.d_cpiv, na + 1)))
      return rc;
  }
  CD_CUDA(ctx, cudaMemsetAsync(h.d_cpiv + na, 0, sizeof(int), ctx->stream));
  if (na > 0)
  {
    (void)cd_launch(csr_to_dense_kernel, na, 128, 0, ctx->stream, na, s.d_row_ptr, s.d_kcol, s.d_a, h.d_cinv);
    CD_LAUNCHED(ctx);
    size_t sm = sizeof(double) * (size_t)na * na;
    int use_smem = sm <= 200 * 1024;
    if (use_smem)
      CD_CUDA(ctx, cudaFuncSetAttribute(gj_invert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    // one warp per four rows (at most 32 warps): short barriers for small coarse levels
    const int nt = std::min(1024, 32 * std::max(1, (na + 3) / 4));
    (void)cd_launch(gj_invert_kernel, 1, nt, use_smem ? sm : 0, ctx->stream, na, h.d_cinv, use_smem, h.d_cpiv, h.d_cpiv + na);
    CD_LAUNCHED(ctx);
  }
  // the zero-pivot flag is copied back behind the inversion and checked after the solve,
  // which synchronises anyway
  if (!h.h_cflag) CD_CUDA(ctx, cudaMallocHost((void **)&h.h_cflag, sizeof(int)));
  CD_CUDA(ctx, cudaMemcpyAsync(h.h_cflag, h.d_cpiv + na, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  h.cflag_pending = true;
  h.cinv_version = s.assembly_version;
  return CDGPU_OK;
}

// ---------------------------------------------------------------------------
// FP64 building blocks on the finest level
// ---------------------------------------------------------------------------
int spmv64(cdgpu_ctx *ctx, const Space &s, const double *x, double *y)
{
  csr_spmv<double>(ctx, s, x, y);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

// the matrix-free FP64 operator (mf64.cuh) applies to Q2 hexahedra assembled by the affine
// constant-coefficient path: the cell coefficients of the last assembly are on the device
static bool use_mf64(const Space &s)
{
  return s.assembled && s.mf_T > 0 && s.d_cellcoef && mf_shape_ok(s.nbf, s.mf_T) && s.dim == 3;
}

// the 8-wide incidence records of the matrix-free row kernels, built once per space (kept
// only when every active row has at most 8 cells); synchronises on the first call
static int ensure_inc8(cdgpu_ctx *ctx, Space &s)
{
  if (s.inc8_tried) return CDGPU_OK;
  s.inc8_tried = true;
  if (s.n_active <= 0 || (long)s.nbf * s.n_cells >= (long)INT_MAX) return CDGPU_OK;
  int rc, *flag = nullptr;
  if ((rc = dev_alloc(ctx, &s.d_inc8, (size_t)s.n_active * 8)) || (rc = dev_alloc(ctx, &flag, 1))) return rc;
  CD_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream));
  mf_inc8_kernel<<<(s.n_active + 255) / 256, 256, 0, ctx->stream>>>(s.n_active, s.nbf, s.n_cells, s.d_inc_ptr, s.d_inc,
                                                                   s.d_inc8, flag);
  CD_LAUNCHED(ctx);
  int h = 0;
  CD_CUDA(ctx, cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(flag);
  if (h)
  {
    cudaFree(s.d_inc8);
    s.d_inc8 = nullptr;
  }
  return CDGPU_OK;
}

static int ensure_mf64(cdgpu_ctx *ctx, Space &s)
{
  int rc;
  if (!s.d_ybuf64 && (rc = dev_alloc(ctx, &s.d_ybuf64, (size_t)s.nbf * s.n_cells))) return rc;
  return ensure_inc8(ctx, s);
}

// phase 1 of the matrix-free FP64 product: the per-cell products A_c x_c into d_ybuf64
static void mf64_cells(cdgpu_ctx *ctx, const Space &s, const double *x)
{
  static const Mf64Tab tab = mf64_tables();
  const int groups = (s.n_cells + kMf64Cells - 1) / kMf64Cells;
  const int grid = std::max(1, std::min(groups, ctx->sm_count * 3));
  const int cstride = s.mf_T + n_rhs_tensors(s.dim, s.ref_disctype);
  // the cell data is read before the wait once a launch of this assembly has waited
  const int pre = s.mf64_safe_version == s.assembly_version ? 1 : 0;
  if (!pre) s.mf64_safe_version = s.assembly_version;
  if (s.mf_T == 10)
    (void)cd_launch(mf64_cell27_kernel<10>, grid, kMf64Warps * 32, 0, ctx->stream, s.n_cells, (const int *)s.d_gn,
                    (const double *)s.d_cellcoef, cstride, tab, x, s.d_ybuf64, pre);
  else
    (void)cd_launch(mf64_cell27_kernel<13>, grid, kMf64Warps * 32, 0, ctx->stream, s.n_cells, (const int *)s.d_gn,
                    (const double *)s.d_cellcoef, cstride, tab, x, s.d_ybuf64, pre);
}

// phase 2: y = A x, or d = f - A x with per-block sums of d^2 in partial (grid <= 8 per SM)
static int mf64_rows_grid(const cdgpu_ctx *ctx, const Space &s)
{
  return std::max(1, std::min((s.n_dof + 255) / 256, ctx->sm_count * 8));
}
template <int MODE>
static void mf64_rows(cdgpu_ctx *ctx, const Space &s, const double *x, const double *f, double *out, double *partial)
{
  (void)cd_launch(mf64_row_kernel<MODE>, mf64_rows_grid(ctx, s), 256, 0, ctx->stream, s.n_dof, s.n_active,
                  s.n_cells, (const int *)s.d_inc_ptr, (const int *)s.d_inc, (const int *)s.d_inc8,
                  (const double *)s.d_ybuf64, x, f, out, partial);
}

// y = A x on the finest level: matrix-free in FP64 where the solve chose it, else the CSR entries
static int finest_spmv(cdgpu_ctx *ctx, Hierarchy &h, const double *x, double *y)
{
  const Space &s = *h.lev.back().sp;
  if (!h.mf64) return spmv64(ctx, s, x, y);
  mf64_cells(ctx, s, x);
  CD_LAUNCHED(ctx);
  mf64_rows<MF64_SPMV>(ctx, s, x, nullptr, y, nullptr);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

static int finest_defect_norm(cdgpu_ctx *ctx, Hierarchy &h, const double *x, const double *f, double *d,
                              double *norm_out_dev)
{
  const Space &s = *h.lev.back().sp;
  if (h.mf64)
  {
    mf64_cells(ctx, s, x);
    CD_LAUNCHED(ctx);
    mf64_rows<MF64_DEFECT>(ctx, s, x, f, d, h.d_partial);
    CD_LAUNCHED(ctx);
    (void)cd_launch(sum_blocks_kernel, 1, 256, 0, ctx->stream, mf64_rows_grid(ctx, s), h.d_partial,
                    norm_out_dev);
    CD_LAUNCHED(ctx);
    return CDGPU_OK;
  }
  const int grid = defect_grid<double>(ctx, s); // <= 8 blocks per SM, within d_partial
  csr_defect<double>(ctx, s, x, f, d, h.d_partial, grid);
  CD_LAUNCHED(ctx);
  (void)cd_launch(sum_blocks_kernel, 1, 256, 0, ctx->stream, grid, h.d_partial, norm_out_dev);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}


int defect64(cdgpu_ctx *ctx, const Space &s, const double *x, const double *f, double *d, double *res)
{
  int rc;
  const int grid = defect_grid<double>(ctx, s);
  double *partial = nullptr, *out = nullptr;
  if ((rc = dev_alloc(ctx, &partial, grid)) || (rc = dev_alloc(ctx, &out, 1))) return rc;
  csr_defect<double>(ctx, s, x, f, d, partial, grid);
  CD_LAUNCHED(ctx);
  (void)cd_launch(sum_blocks_kernel, 1, 256, 0, ctx->stream, grid, partial, out);
  CD_LAUNCHED(ctx);
  double r2 = 0;
  CD_CUDA(ctx, cudaMemcpyAsync(&r2, out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(partial);
  cudaFree(out);
  if (res) *res = std::sqrt(r2);
  return CDGPU_OK;
}

static int precondition(cdgpu_ctx *ctx, Hierarchy &h, const cdgpu_solver_params &p, const double *r, double *z,
                        bool io_ready = false)
{
  return mg_apply(ctx, h, p, r, z, io_ready);
}

// the host copy of the FGMRES control block: [0..k) h1, [33..33+k) h2, [66] ||w||^2
static int read_ctl(cdgpu_ctx *ctx, Hierarchy &h, int count, const double *src = nullptr)
{
  CD_CUDA(ctx, cudaMemcpyAsync(h.h_ctl, src ? src : h.d_ctl, sizeof(double) * count, cudaMemcpyDeviceToHost,
                               ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CDGPU_OK;
}

// Givens helpers exactly as FgmresIte.C:149-181
static void gen_rot(double dx, double dy, double &cs, double &sn)
{
  if (dy == 0.0) { cs = 1.0; sn = 0.0; }
  else if (std::fabs(dy) > std::fabs(dx))
  {
    double t = dx / dy;
    sn = 1.0 / std::sqrt(1.0 + t * t);
    cs = t * sn;
  }
  else
  {
    double t = dy / dx;
    cs = 1.0 / std::sqrt(1.0 + t * t);
    sn = t * cs;
  }
}
static void app_rot(double &dx, double &dy, double cs, double sn)
{
  double t = cs * dx + sn * dy;
  dy = -sn * dx + cs * dy;
  dx = t;
}

static int fgmres(cdgpu_ctx *ctx, Hierarchy &h, const cdgpu_solver_params &p, const double *f, double *x,
                  cdgpu_solve_info *info)
{
  const Space &s = *h.lev.back().sp;
  const int n = s.n_dof;
  int m = std::min(p.restart, p.maxit);
  if (m <= 0) m = 10;
  if (m > 32) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "FGMRES: restart above 32 is not supported");
  int rc;
  if ((rc = setup_hierarchy_buffers(ctx, h, m))) return rc;
  std::vector<double> H((size_t)(m + 1) * m, 0.0), sv(m + 1), cs(m + 1), sn(m + 1), y(m + 1);
  const int blocks = (n + 255) / 256;
  auto V = [&](int k) { return h.d_V + (size_t)k * n; };
  auto Z = [&](int k) { return h.d_Z + (size_t)k * n; };
  // control blocks: an iteration's Gram-Schmidt results (dots at +0 and +33, ||w||^2 at +66)
  // alternate between two blocks by the iteration's parity, the residual norm has its own
  // slot; the back-substitution coefficients are at +100
  auto ctl_it = [&](int i) { return h.d_ctl + (i & 1) * 160; };
  double *const nrm = h.d_ctl + 240;
  // r0 = f - A x, beta = ||r0|| (FgmresIte.C:275-284); v_0 = r0 / beta is formed on the device
  // and the first iteration enqueued while ||r0||^2 travels to the host on the copy stream
  if ((rc = finest_defect_norm(ctx, h, x, f, V(0), nrm))) return rc;
  CD_CUDA(ctx, cudaEventRecord(h.ev_ready[0], ctx->stream));
  CD_CUDA(ctx, cudaStreamWaitEvent(h.cstream, h.ev_ready[0], 0));
  CD_CUDA(ctx, cudaMemcpyAsync(h.h_ctl, nrm, sizeof(double), cudaMemcpyDeviceToHost, h.cstream));
  CD_CUDA(ctx, cudaEventRecord(h.ev_beta, h.cstream));
  // Iteration i on the device: the preconditioner on v_i, w = A z_i, the Gram-Schmidt passes,
  // a copy of the control block to pinned slot i % 2 (on the copy stream, behind an event, so
  // the iteration does not wait for it) and v_{i+1} = w / ||w||, which needs no host value.
  // The host then applies the Givens rotations and the stopping tests.  While it waits for
  // iteration i it has, as a rule, already enqueued iteration i + 1, so the device does not
  // idle during the host's part; it does not when the residual predicted from the convergence
  // so far is within a factor of 4 of the stopping threshold, because an iteration enqueued
  // after the one that converges is wasted.  Which iterations are enqueued early changes no
  // arithmetic.
  auto enqueue = [&](int i) -> int {
    int rc2;
    // the kernel that formed v_i (scale_norm_kernel or axpy_scale_kernel) set the cycle's slot
    if ((rc2 = precondition(ctx, h, p, V(i), Z(i), true))) return rc2;
    int k = i + 1, pb = h.partial_blocks;
    double *c = ctl_it(i);
    if (h.mf64 && s.d_inc8)
    {
      // w = A z_i matrix-free, its second phase fused with pass 1: h1 = V^T w
      mf64_cells(ctx, s, Z(i));
      CD_LAUNCHED(ctx);
      launch_row_dots(k, pb, ctx->stream, n, s.n_active, s.d_inc8, s.d_ybuf64, Z(i), h.d_w, h.d_V, h.d_partial, c,
                      h.d_gs_count);
      CD_LAUNCHED(ctx);
    }
    else
    {
      if ((rc2 = finest_spmv(ctx, h, Z(i), h.d_w))) return rc2;
      // pass 1: h1 = V^T w
      launch_gs<GS_DOTS>(k, pb, ctx->stream, n, h.d_V, h.d_w, nullptr, h.d_partial, c, h.d_gs_count);
      CD_LAUNCHED(ctx);
    }
    // pass 2: w -= V h1, h2 = V^T w, and ||w - V h2||^2 = ||w||^2 - ||h2||^2
    launch_gs<GS_AXPY_DOTS_NORM>(k, pb, ctx->stream, n, h.d_V, h.d_w, c, h.d_partial, c + 33, h.d_gs_count,
                                 c + 66);
    CD_LAUNCHED(ctx);
    CD_CUDA(ctx, cudaEventRecord(h.ev_ready[i & 1], ctx->stream));
    CD_CUDA(ctx, cudaStreamWaitEvent(h.cstream, h.ev_ready[i & 1], 0));
    CD_CUDA(ctx, cudaMemcpyAsync(h.h_slot + (i & 1) * 80, c, sizeof(double) * 67, cudaMemcpyDeviceToHost, h.cstream));
    CD_CUDA(ctx, cudaEventRecord(h.ev_slot[i & 1], h.cstream));
    // v_{i+1} = (w - V h2) / ||w - V h2||
    launch_axpy_scale(k, blocks, ctx->stream, n, h.d_V, h.d_w, c + 33, c + 66, V(i + 1), h.d_io, Z(i + 1));
    CD_LAUNCHED(ctx);
    return CDGPU_OK;
  };
  // the first restart cycle's v_0 and iteration 0, before ||r0|| is known on the host (if the
  // start already satisfies the stopping test they are discarded: x is not touched)
  (void)cd_launch(scale_norm_kernel, blocks, 256, 0, ctx->stream, n, (const double *)nrm, V(0), V(0), h.d_io,
                  Z(0));
  CD_LAUNCHED(ctx);
  if ((rc = enqueue(0))) return rc;
  CD_CUDA(ctx, cudaEventSynchronize(h.ev_beta));
  double res = std::sqrt(h.h_ctl[0]), res0 = res, beta = res;
  info->initial_residual = res;
  int maxite = p.maxit, ret = 0, status = CDGPU_OK;
  if (beta <= p.res_norm_min)
  {
    if (p.minit == 0 || beta < 1e-20)
    {
      CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      CD_CUDA(ctx, cudaStreamSynchronize(h.cstream));
      info->iterations = 0;
      info->final_residual = res;
      info->status = CDGPU_OK;
      return CDGPU_OK;
    }
    maxite = p.minit;
  }
  int j = 1;
  bool done = false, first_cycle = true;
  while (j <= maxite && !done)
  {
    if (!first_cycle)
    {
      (void)cd_launch(scale_norm_kernel, blocks, 256, 0, ctx->stream, n, (const double *)nrm, V(0), V(0), h.d_io,
                  Z(0));
      CD_LAUNCHED(ctx);
    }
    std::fill(sv.begin(), sv.end(), 0.0);
    sv[0] = beta;
    const double thr = std::max(p.res_norm_min, p.red_factor * res0);
    double last = beta, rate = 0.5;
    int i;
    if (!first_cycle && (rc = enqueue(0))) return rc;
    first_cycle = false;
    for (i = 0; i < m && j <= maxite; i++, j++)
    {
      bool next_enqueued = false;
      if (i + 1 < m && j + 1 <= maxite && (j < p.minit || last * rate > 4.0 * thr))
      {
        if ((rc = enqueue(i + 1))) return rc;
        next_enqueued = true;
      }
      CD_CUDA(ctx, cudaEventSynchronize(h.ev_slot[i & 1]));
      const double *c = h.h_slot + (i & 1) * 80;
      const int k = i + 1;
      // the slot-0 reduction of the last pass holds ||w||^2 (slot 32 of the partials)
      for (int t = 0; t < k; t++) H[(size_t)t * m + i] = c[t] + c[33 + t];
      double hn = std::sqrt(c[66]);
      H[(size_t)(i + 1) * m + i] = hn;
      for (int t = 0; t < i; t++) app_rot(H[(size_t)t * m + i], H[(size_t)(t + 1) * m + i], cs[t], sn[t]);
      gen_rot(H[(size_t)i * m + i], H[(size_t)(i + 1) * m + i], cs[i], sn[i]);
      app_rot(H[(size_t)i * m + i], H[(size_t)(i + 1) * m + i], cs[i], sn[i]);
      app_rot(sv[i], sv[i + 1], cs[i], sn[i]);
      res = std::fabs(sv[i + 1]);
      if (j >= p.minit && (res < p.res_norm_min || res < p.red_factor * res0))
      {
        // back substitution and x += Z y (UpdateGmresIterate, FgmresIte.C:198-216)
        for (int a = 0; a <= i; a++) y[a] = sv[a];
        for (int a = i; a >= 0; a--)
        {
          y[a] /= H[(size_t)a * m + a];
          for (int b = a - 1; b >= 0; b--) y[b] -= H[(size_t)b * m + a] * y[a];
        }
        // staged in the pinned control mirror (positions 100..131), so the copy is asynchronous
        std::copy(y.begin(), y.begin() + (i + 1), h.h_ctl + 100);
        CD_CUDA(ctx, cudaMemcpyAsync(h.d_ctl + 100, h.h_ctl + 100, sizeof(double) * (i + 1), cudaMemcpyHostToDevice,
                                     ctx->stream));
        (void)cd_launch(update_kernel, blocks, 256, 0, ctx->stream, n, i + 1, h.d_ctl + 100, h.d_Z, x);
        CD_LAUNCHED(ctx);
        ret = j;
        done = true;
        break;
      }
      if (res > p.div_factor * res0)
      {
        ret = j;
        status = CDGPU_ERR_DIVERGED;
        done = true;
        break;
      }
      // convergence rate so far in this restart cycle, for the next prediction
      if (beta > 0 && res > 0) rate = std::pow(res / beta, 1.0 / (i + 1));
      last = res;
      if (!next_enqueued && i + 1 < m && j + 1 <= maxite && (rc = enqueue(i + 1))) return rc;
    }
    if (done) break;
    // restart: x += Z y over the full basis, new residual (FgmresIte.C:536-560)
    for (int a = 0; a < m; a++) y[a] = sv[a];
    for (int a = m - 1; a >= 0; a--)
    {
      y[a] /= H[(size_t)a * m + a];
      for (int b = a - 1; b >= 0; b--) y[b] -= H[(size_t)b * m + a] * y[a];
    }
    std::copy(y.begin(), y.begin() + m, h.h_ctl + 100);
    CD_CUDA(ctx, cudaMemcpyAsync(h.d_ctl + 100, h.h_ctl + 100, sizeof(double) * m, cudaMemcpyHostToDevice, ctx->stream));
    (void)cd_launch(update_kernel, blocks, 256, 0, ctx->stream, n, m, h.d_ctl + 100, h.d_Z, x);
    CD_LAUNCHED(ctx);
    if ((rc = finest_defect_norm(ctx, h, x, f, V(0), nrm))) return rc;
    if ((rc = read_ctl(ctx, h, 1, nrm))) return rc;
    res = beta = std::sqrt(h.h_ctl[0]);
    if (p.stop_rule == 0) res0 = res; // the reference measures the next cycle against this residual
  }
  if (!done)
  {
    ret = j > maxite ? maxite : j;
    if (res > p.res_norm_min && res > res0 * p.red_factor) status = CDGPU_ERR_NOT_CONVERGED;
  }
  if (ctx->d_err && ctx->h_err)
    CD_CUDA(ctx, cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(h.cstream));
  info->iterations = ret;
  info->final_residual = res;
  info->status = status;
  return CDGPU_OK;
}

static int fixed_point(cdgpu_ctx *ctx, Hierarchy &h, const cdgpu_solver_params &p, const double *f,
                       double *x, cdgpu_solve_info *info)
{
  const Space &s = *h.lev.back().sp;
  const int n = s.n_dof;
  int rc;
  if ((rc = setup_hierarchy_buffers(ctx, h, std::max(h.m, 1)))) return rc;
  double *d = h.d_w, *z = h.d_V;
  if ((rc = finest_defect_norm(ctx, h, x, f, d, h.d_ctl))) return rc;
  if ((rc = read_ctl(ctx, h, 1))) return rc;
  double res = std::sqrt(h.h_ctl[0]), res0 = res;
  info->initial_residual = res;
  int maxite = p.maxit, i, status = CDGPU_OK;
  if (res <= p.res_norm_min) maxite = p.minit;
  for (i = 1; i <= maxite; i++)
  {
    if ((rc = precondition(ctx, h, p, d, z))) return rc;
    (void)cd_launch(axpy_kernel, (n + 255) / 256, 256, 0, ctx->stream, n, 1.0, z, x);
    CD_LAUNCHED(ctx);
    if ((rc = finest_defect_norm(ctx, h, x, f, d, h.d_ctl))) return rc;
    if ((rc = read_ctl(ctx, h, 1))) return rc;
    res = std::sqrt(h.h_ctl[0]);
    if (i < p.minit) continue;
    if (res <= res0 * p.red_factor) break;
    if (res <= p.res_norm_min) break;
    if (res > p.div_factor * res0) { status = CDGPU_ERR_DIVERGED; break; }
  }
  if (i > maxite && res > p.res_norm_min && res > res0 * p.red_factor) status = CDGPU_ERR_NOT_CONVERGED;
  info->iterations = i;
  info->final_residual = res;
  info->status = status;
  return CDGPU_OK;
}

// FP32 cell coefficients and tensors of a space's matrix-free operator, made from its last
// assembly, plus the tensor-core kernel's shared-memory attribute and the error flag (all set
// outside any capture)
static int prepare_mf(cdgpu_ctx *ctx, Space &s)
{
  int rc;
  if ((rc = ensure_inc8(ctx, s))) return rc;
  if (!s.d_ybuf)
  {
    if ((rc = dev_alloc(ctx, &s.d_cf32, (size_t)s.n_cells * CD_MAXT)) ||
        (rc = dev_alloc(ctx, &s.d_R32, (size_t)CD_MAXT * s.nbf * s.nbf)) ||
        (rc = dev_alloc(ctx, &s.d_R32img, (size_t)CD_MAXT * 32 * 32)) ||
        (rc = dev_alloc(ctx, &s.d_ybuf, (size_t)s.nbf * s.n_cells)))
      return rc;
  }
  if (s.mf_version != s.assembly_version)
  {
    const int T = s.mf_T, Tr = n_rhs_tensors(s.dim, s.ref_disctype);
    const long total = (long)s.n_cells * T + (long)T * s.nbf * s.nbf;
    const int grid = (int)std::min<long>((total + 255) / 256, (long)ctx->sm_count * 8);
    (void)cd_launch(mf_convert_kernel, grid, 256, 0, ctx->stream, s.n_cells, T, Tr, s.nbf, s.d_cellcoef, s.d_ref,
                    s.d_cf32, s.d_R32);
    CD_LAUNCHED(ctx);
    if (s.nbf == 27 && T <= CD_MAXT)
    {
      (void)cd_launch(mf_tc_tensor_image_kernel, (32 * T * 32 + 255) / 256, 256, 0, ctx->stream, T,
                      (const float *)s.d_R32, s.d_R32img);
      CD_LAUNCHED(ctx);
    }
    s.mf_version = s.assembly_version;
  }
  if (!ctx->mf_attr_set)
  {
    CD_CUDA(ctx, cudaFuncSetAttribute(mf_cell27_tc_kernel<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMfTcSmem));
    CD_CUDA(ctx, cudaFuncSetAttribute(mf_cell27_tc_kernel<13>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMfTcSmem));
    ctx->mf_attr_set = true;
  }
  if (!ctx->d_err)
  {
    if ((rc = dev_alloc(ctx, &ctx->d_err, 1))) return rc;
    CD_CUDA(ctx, cudaMallocHost((void **)&ctx->h_err, sizeof(int)));
    CD_CUDA(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
  }
  return CDGPU_OK;
}

// FP32 copies for the matrix-free operator of every level that has one; the captured FP32
// cycle is recaptured when the set of such levels changes
static int refresh_mf(cdgpu_ctx *ctx, Hierarchy &h)
{
  unsigned mask = 0;
  for (size_t l = 0; l < h.lev.size(); l++)
  {
    Space &s = *h.lev[l].sp;
    if (s.mf_T <= 0 || s.n_cells < kMfMinCells || !mf_shape_ok(s.nbf, s.mf_T)) continue;
    int rc = prepare_mf(ctx, s);
    if (rc) return rc;
    mask |= 1u << l;
  }
  if (mask != h.mf_mask && h.gexec[1])
  {
    cudaGraphExecDestroy(h.gexec[1]);
    h.gexec[1] = nullptr;
  }
  h.mf_mask = mask;
  return CDGPU_OK;
}

int run_solve(cdgpu_ctx *ctx, Hierarchy &h, const cdgpu_solver_params &p, const double *d_rhs, double *d_sol,
              cdgpu_solve_info *info)
{
  for (auto &L : h.lev)
    if (!L.sp->assembled) return fail(ctx, CDGPU_ERR_INVALID, "solve: every level must be assembled");
  if (p.smoother != 1) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "solve: only the damped Jacobi smoother (1) runs on the GPU");
  if (p.slc) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "solve: step-length control is not supported on the GPU");
  if (p.coarse_smoother != 1 && p.coarse_smoother != 2 && p.coarse_smoother != 3 && p.coarse_smoother != 17)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "solve: coarse smoother must be 1, 2, 3 or 17");
  if (p.precision != 0 && p.precision != 1) return fail(ctx, CDGPU_ERR_INVALID, "solve: precision must be 0 or 1");
  if (p.coarse_smoother != 17 && h.lev[0].sp->n_dof > 6000)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "solve: coarse smoother loop needs a coarsest level below 6000 DOFs");
  int rc;
  // the mixed form applies the finest operator of its FGMRES iteration matrix-free in FP64 on
  // levels large enough for the per-cell form to pay off; the FP64 form keeps the CSR entries,
  // whose bulk-copy kernels are tuned once per pattern, before any capture
  Space &fs = *h.lev.back().sp;
  h.mf64 = p.precision == 1 && use_mf64(fs) && fs.n_cells >= kMfMinCells;
  if (h.mf64 && (rc = ensure_mf64(ctx, fs))) return rc;
  if (!h.mf64 && (rc = tune_tma(ctx, fs))) return rc;
  if (p.coarse_smoother == 17 && (rc = refresh_coarse_inverse(ctx, h))) return rc;
  if (p.precision == 1 && (rc = refresh_mf(ctx, h))) return rc;
  cdgpu_solve_info local{};
  if (!info) info = &local;
  if (p.solver == 11) rc = fixed_point(ctx, h, p, d_rhs, d_sol, info);
  else if (p.solver == 16) rc = fgmres(ctx, h, p, d_rhs, d_sol, info);
  else return fail(ctx, CDGPU_ERR_UNSUPPORTED, "solve: SC_SOLVER_SCALAR must be 16 (FGMRES) or 11 (fixed point)");
  if (h.cflag_pending)
  {
    h.cflag_pending = false;
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (*h.h_cflag)
    {
      h.cinv_version = -2; // invert again on the next solve
      return fail(ctx, CDGPU_ERR_INVALID, "exact coarse solve: singular coarse matrix");
    }
  }
  // wait flags of the tensor-core and bulk-copy kernels: FGMRES copied the flag back with its
  // last synchronisation
  if (rc == CDGPU_OK && ctx->d_err && ctx->h_err)
    rc = p.solver == 16 ? err_flag_status(ctx) : assemble_check(ctx);
  return rc;
}

// y = A x with one of the FP64 forms of a space's operator: form 0 the assembled CSR entries,
// 1 the matrix-free sum-factorised per-cell products the mixed form's FGMRES iteration applies
// on its finest level.  Dirichlet rows are identity rows in both.  Form 1 needs a Q2
// hexahedral space assembled by the affine constant-coefficient path.  check: read back the
// bulk-copy product's wait flag (synchronises).
int apply_fp64_form(cdgpu_ctx *ctx, Space &s, int form, const double *d_x, double *d_y, bool check)
{
  if (form == 0)
  {
    csr_spmv<double>(ctx, s, d_x, d_y);
    CD_LAUNCHED(ctx);
    return check && ctx->d_err ? assemble_check(ctx) : CDGPU_OK;
  }
  if (!use_mf64(s))
    return fail(ctx, CDGPU_ERR_UNSUPPORTED,
                "apply_fp64: the matrix-free form needs Q2 hexahedra assembled from affine cells with constant coefficients");
  int rc = ensure_mf64(ctx, s);
  if (rc) return rc;
  mf64_cells(ctx, s, d_x);
  CD_LAUNCHED(ctx);
  mf64_rows<MF64_SPMV>(ctx, s, d_x, nullptr, d_y, nullptr);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

// y = A x with one of the FP32 forms of a space's operator that the mixed multigrid cycle uses:
// form 0 the FP32 copy of the assembled CSR matrix, 1 the matrix-free per-cell products on CUDA
// cores, 2 the same products on the tensor cores (tcgen05, TF32 inputs).  Dirichlet rows are
// identity rows in every form.  Forms 1 and 2 need a Q2 hexahedral space assembled by the
// affine constant-coefficient path.
int apply_fp32_form(cdgpu_ctx *ctx, Space &s, int form, const float *d_x, float *d_y)
{
  if (form == 0)
  {
    csr_spmv<float>(ctx, s, d_x, d_y);
    CD_LAUNCHED(ctx);
    return CDGPU_OK;
  }
  if (s.mf_T <= 0 || !mf_shape_ok(s.nbf, s.mf_T))
    return fail(ctx, CDGPU_ERR_UNSUPPORTED,
                "apply_fp32: the matrix-free forms need Q2 hexahedra assembled from affine cells with constant coefficients");
  int rc = prepare_mf(ctx, s);
  if (rc) return rc;
  mf_apply_cells(ctx, s, d_x, form == 2);
  CD_LAUNCHED(ctx);
  mf_rows<MF_SPMV>(ctx, s, d_x, nullptr, nullptr, d_y, 0.f);
  CD_LAUNCHED(ctx);
  return assemble_check(ctx); // the tensor-core wait flag
}
