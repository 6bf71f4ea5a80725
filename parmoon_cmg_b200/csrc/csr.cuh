// CSR kernels of the solver: matrix-vector product, defect, damped Jacobi sweep,
// restriction and prolongation, one template with an epilogue per operation.
//
// A group of GS threads takes one row; each thread issues all of its U column and value
// loads of the row (predicated on the row length) before the first x gather, so a warp
// keeps 32*U independent loads of the matrix stream in flight regardless of where the row
// starts.  GS follows the longest row of the matrix (csr_shape), U = 8 (16 with GS = 8); a
// tail loop takes the entries beyond GS*U.  On the 32^3 Q2 hexahedral matrix (rows of
// 27..125 entries) GS = 8, U = 16 gave the fastest multigrid step among warp-per-row,
// row-tiled shared-memory and sliced-ELL forms (product alone: FP64 49 us, FP32 37 us).  Rows are visited warp by
// warp, so every lane of a warp reaches every shuffle.  Sums are deterministic: fixed
// order within a row, per-block partials of the defect norm in block order.
#pragma once

#include "internal.h"

enum { CM_SPMV = 0, CM_DEFECT = 1, CM_JACOBI = 2, CM_RESTRICT = 3, CM_PROLONG = 4 };

template <typename T> struct CsrArgs
{
  int n = 0, n_active = 0;
  const int *rp = nullptr, *kc = nullptr;
  const T *a = nullptr, *x = nullptr, *f = nullptr, *diag = nullptr;
  T *y = nullptr, *y2 = nullptr;
  T omega = 0;
  double *partial = nullptr;
  // 1: the kernel loads its first rows' pointers, columns and values before waiting for its
  // predecessor (set for the kernels of the captured multigrid cycle, where no kernel writes
  // a matrix; see CD_PDL_WAIT)
  int pre = 0;
};

template <int G, typename T> __device__ __forceinline__ T csr_group_sum(T v)
{
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
  return v;
}

// epilogue of row r with row sum s = (A x)_r (acc collects this thread's defect norm)
template <typename T, int MODE>
__device__ __forceinline__ void csr_epilogue(const CsrArgs<T> &p, int r, T s, double &acc)
{
  if (MODE == CM_SPMV)
    p.y[r] = s;
  else if (MODE == CM_DEFECT)
  {
    T v = p.f[r] - s;
    p.y[r] = v;
    acc += (double)v * (double)v;
  }
  else if (MODE == CM_JACOBI)
  {
    // x + omega D^{-1} (f - A x) = (1 - omega) x + omega (f - sum_{j != r} a_rj x_j) / a_rr
    // (MGLevel3D.C:443-537, MGLevel2D.C:318-368); Dirichlet rows take the right-hand side
    if (r < p.n_active)
      p.y[r] = p.x[r] + p.omega * (p.f[r] - s) / p.diag[r];
    else
      p.y[r] = p.f[r];
  }
  else if (MODE == CM_RESTRICT)
  {
    // coarse rhs = R d on active rows, zero elsewhere (CorrectDefect, MGLevel3D.C:588);
    // coarse solution reset (MGLevel3D.C:557)
    p.y[r] = r < p.n_active ? s : T(0);
    p.y2[r] = T(0);
  }
  else // CM_PROLONG: sol += damp * (P xc) on active fine rows (Update, MGLevel3D.C:539)
  {
    if (r < p.n_active) p.y[r] += p.omega * s;
  }
}

// the pointers, columns and values of row r for a group of GS threads (U per thread,
// predicated on the row length)
template <typename T, int GS, int U> struct CsrRow
{
  int b, e;
  int c[U];
  T v[U];
};
template <typename T, int GS, int U>
__device__ __forceinline__ void csr_load_row(const CsrArgs<T> &p, int r, int rows_end, int lane, CsrRow<T, GS, U> &w)
{
  w.b = 0;
  w.e = 0;
  if (r < rows_end)
  {
    w.b = p.rp[r];
    w.e = p.rp[r + 1];
  }
#pragma unroll
  for (int i = 0; i < U; i++)
  {
    const int j = w.b + lane + i * GS;
    w.c[i] = j < w.e ? __ldcs(p.kc + j) : -1;
    w.v[i] = j < w.e ? __ldcs(p.a + j) : T(0);
  }
}

// gathers, group sum and epilogue of row r (every lane of the warp calls it)
template <typename T, int GS, int U, int MODE>
__device__ __forceinline__ void csr_do_row(const CsrArgs<T> &p, int r, int rows_end, int lane,
                                           const CsrRow<T, GS, U> &w, double &acc)
{
  T s = 0;
  if (r < rows_end)
  {
#pragma unroll
    for (int i = 0; i < U; i++)
      if (w.c[i] >= 0) s += w.v[i] * __ldg(p.x + w.c[i]);
    for (int j = w.b + lane + U * GS; j < w.e; j += GS) s += p.a[j] * __ldg(p.x + p.kc[j]);
  }
  s = csr_group_sum<GS>(s);
  if (r < rows_end && lane == 0) csr_epilogue<T, MODE>(p, r, s, acc);
}

template <typename T, int GS, int U, int MODE, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) csr_kernel(CsrArgs<T> p)
{
  constexpr int NT = 256;
  __shared__ double red[NT / 32];
  const int lane = threadIdx.x % GS, sub = (threadIdx.x % 32) / GS;
  const long nwarp = (long)gridDim.x * NT / 32;
  const int rows_end = MODE == CM_PROLONG ? p.n_active : p.n;
  const long step = nwarp * (32 / GS);
  long base = ((long)blockIdx.x * NT + threadIdx.x) / 32 * (32 / GS);
  double acc = 0;
  if (p.pre && base < rows_end)
  {
    // the first row's matrix data before the wait, its gathers after
    CsrRow<T, GS, U> w;
    csr_load_row<T, GS, U>(p, (int)base + sub, rows_end, lane, w);
    CD_PDL_ENTRY();
    csr_do_row<T, GS, U, MODE>(p, (int)base + sub, rows_end, lane, w, acc);
    base += step;
  }
  else
    CD_PDL_ENTRY();
  for (; base < rows_end; base += step)
  {
    CsrRow<T, GS, U> w;
    csr_load_row<T, GS, U>(p, (int)base + sub, rows_end, lane, w);
    csr_do_row<T, GS, U, MODE>(p, (int)base + sub, rows_end, lane, w, acc);
  }
  if (MODE == CM_DEFECT && p.partial)
  {
    acc = csr_group_sum<32>(acc);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
    __syncthreads();
    if (threadIdx.x == 0)
    {
      double tot = 0;
      for (int wi = 0; wi < NT / 32; wi++) tot += red[wi];
      p.partial[blockIdx.x] = tot;
    }
  }
}

// The same operations with the row loop software-pipelined: the row pointers and the
// column/value loads of a warp's next row chunk are issued before the x gathers of the
// current chunk, so each row's dependent load chain overlaps the previous row's.  Used for
// the FP32 multigrid levels with 8 threads per row, where it measured 31 us against 36 us
// for the 32^3 Q2 product (FP64 gained nothing).
template <typename T, int GS, int U, int MODE, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) csr_pipe_kernel(CsrArgs<T> p)
{
  if (!p.pre) CD_PDL_ENTRY();
  constexpr int NT = 256;
  __shared__ double red[NT / 32];
  const int lane = threadIdx.x % GS, sub = (threadIdx.x % 32) / GS;
  const long nwarp = (long)gridDim.x * NT / 32;
  const long step = nwarp * (32 / GS);
  const int rows_end = MODE == CM_PROLONG ? p.n_active : p.n;
  long base = ((long)blockIdx.x * NT + threadIdx.x) / 32 * (32 / GS);
  int r = (int)base + sub;
  int b = 0, e = 0;
  if (base < rows_end && r < rows_end) { b = p.rp[r]; e = p.rp[r + 1]; }
  int c[U];
  T v[U];
#pragma unroll
  for (int i = 0; i < U; i++)
  {
    const int j = b + lane + i * GS;
    c[i] = j < e ? __ldcs(p.kc + j) : -1;
    v[i] = j < e ? __ldcs(p.a + j) : T(0);
  }
  if (p.pre) CD_PDL_ENTRY(); // the first rows' matrix data is in flight
  double acc = 0;
  for (; base < rows_end; base += step)
  {
    const long nb = base + step;
    const int rn = (int)nb + sub;
    int bn = 0, en = 0;
    if (nb < rows_end && rn < rows_end) { bn = p.rp[rn]; en = p.rp[rn + 1]; }
    T s = 0;
#pragma unroll
    for (int i = 0; i < U; i++)
      if (c[i] >= 0) s += v[i] * __ldg(p.x + c[i]);
    for (int j = b + lane + U * GS; j < e; j += GS) s += p.a[j] * __ldg(p.x + p.kc[j]);
#pragma unroll
    for (int i = 0; i < U; i++)
    {
      const int j = bn + lane + i * GS;
      c[i] = j < en ? __ldcs(p.kc + j) : -1;
      v[i] = j < en ? __ldcs(p.a + j) : T(0);
    }
    s = csr_group_sum<GS>(s);
    if (r < rows_end && lane == 0) csr_epilogue<T, MODE>(p, r, s, acc);
    r = rn;
    b = bn;
    e = en;
  }
  if (MODE == CM_DEFECT && p.partial)
  {
    acc = csr_group_sum<32>(acc);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
    __syncthreads();
    if (threadIdx.x == 0)
    {
      double tot = 0;
      for (int w = 0; w < NT / 32; w++) tot += red[w];
      p.partial[blockIdx.x] = tot;
    }
  }
}

// grid of a CSR launch: one pass over the rows, at most 8 blocks of 256 threads per SM
inline int csr_grid(const cdgpu_ctx *ctx, const CsrShape &sh, int rows)
{
  const long per_block = 256 / sh.gs;
  const long need = (rows + per_block - 1) / per_block;
  return (int)std::max<long>(1, std::min<long>(need, (long)ctx->sm_count * 8));
}

template <typename T, int MODE>
inline void launch_csr(cdgpu_ctx *ctx, const CsrShape &sh, const CsrArgs<T> &pa, int grid)
{
  CsrArgs<T> p = pa;
  p.pre = ctx->pdl_pre ? 1 : 0;
  switch (sh.gs)
  {
    case 1: (void)cd_launch(csr_kernel<T, 1, 8, MODE>, grid, 256, 0, ctx->stream, p); break;
    case 2: (void)cd_launch(csr_kernel<T, 2, 8, MODE>, grid, 256, 0, ctx->stream, p); break;
    case 4: (void)cd_launch(csr_kernel<T, 4, 8, MODE>, grid, 256, 0, ctx->stream, p); break;
    case 8:
      // FP64: at most 64 registers, so that 4 CTAs (32 warps) share an SM instead of 3; the
      // 32^3 Q2 product went from 73 to 54 us with a cold L2
      if (sizeof(T) == 4 && (MODE == CM_JACOBI || MODE == CM_DEFECT))
        (void)cd_launch(csr_pipe_kernel<T, 8, 8, MODE>, grid, 256, 0, ctx->stream, p);
      else if (sizeof(T) == 8)
        (void)cd_launch(csr_kernel<T, 8, 16, MODE, 4>, grid, 256, 0, ctx->stream, p);
      else
        (void)cd_launch(csr_kernel<T, 8, 16, MODE>, grid, 256, 0, ctx->stream, p);
      break;
    default: (void)cd_launch(csr_kernel<T, 32, 8, MODE>, grid, 256, 0, ctx->stream, p); break;
  }
}
