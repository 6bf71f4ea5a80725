// Matrix-free FP32 operator of the multigrid cycle on affine cells with constant
// coefficients: A x = sum over cells of A_c x_c with A_c = sum_t coef_{c,t} R_t, the same
// reference tensors R_t and cell coefficients the assembly uses (ConvDiff3D.C:61-120 /
// ConvDiff2D.C:32-162 restated as fixed tensors on affine cells), so no matrix is read.
//   phase 1 (mf_cell_kernel): one thread per cell gathers its nbf values of x, forms the rows
//     of A_c on the fly (tensors broadcast from shared memory, coefficients in registers) and
//     writes A_c x_c to a per-cell buffer laid out [local index][cell] (coalesced);
//   phase 2 (mf_row_kernel): one thread per DOF sums its cells' contributions in ascending
//     cell order (the DOF -> cell incidence of the assembly) and applies the damped-Jacobi
//     update or the defect; Dirichlet rows are identity rows.
// Per cell nbf^2 (T + 1) FP32 FMAs (Q2 hexahedron, Galerkin: 8,019) and ~nbf values in and
// out instead of the cell's share of the CSR matrix (Q2 hexahedron: ~480 values + columns).
// Used for levels of at least kMfMinCells cells; rounding differs from the FP32 copy of the
// assembled matrix only in the order of the sums, and only the preconditioner sees it.
#pragma once

#include "internal.h"

constexpr int kMfMinCells = 16384;

template <int NBF, int T>
__global__ void __launch_bounds__(128) mf_cell_kernel(int n_cells, const int *__restrict__ gn,
                                                      const float *__restrict__ cf32,
                                                      const float *__restrict__ R32, const float *__restrict__ x,
                                                      float *__restrict__ ybuf)
{
  __shared__ float Rs[T * NBF * NBF];
  for (int i = threadIdx.x; i < T * NBF * NBF; i += blockDim.x) Rs[i] = R32[i];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  float xv[NBF], cf[T];
#pragma unroll
  for (int j = 0; j < NBF; j++) xv[j] = __ldg(x + __ldg(gn + (size_t)c * NBF + j));
#pragma unroll
  for (int t = 0; t < T; t++) cf[t] = __ldg(cf32 + (size_t)c * T + t);
  for (int i = 0; i < NBF; i++)
  {
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < NBF; j++)
    {
      float a = 0.f;
#pragma unroll
      for (int t = 0; t < T; t++) a += cf[t] * Rs[(t * NBF + i) * NBF + j];
      acc += a * xv[j];
    }
    ybuf[(size_t)i * n_cells + c] = acc;
  }
}

// Q2 hexahedra (27 local DOFs): the per-cell products as one register-tiled product
// Z[c][t][i] = sum_k R_t[i][k] x_c[k] over a block of 64 cells, then y_c[i] =
// sum_t coef_{c,t} Z[c][t][i].  Thread (g, q) of the 16 x 14 block owns cells 4g..4g+3 and
// local rows 2q, 2q+1 for every tensor: per k it loads 4 cell values and 2T tensor entries
// from shared memory for 8T FMAs.
template <int T>
__global__ void __launch_bounds__(224) mf_cell27_kernel(int n_cells, const int *__restrict__ gn,
                                                        const float *__restrict__ cf32,
                                                        const float *__restrict__ R32, const float *__restrict__ x,
                                                        float *__restrict__ ybuf)
{
  constexpr int CB = 64, NB = 27;
  __shared__ float Rs[T * NB * NB];
  __shared__ float Xs[CB * NB];
  const int c_base = blockIdx.x * CB;
  for (int e = threadIdx.x; e < T * NB * NB; e += blockDim.x) Rs[e] = __ldg(R32 + e);
  for (int e = threadIdx.x; e < CB * NB; e += blockDim.x)
  {
    const int c = c_base + e / NB;
    Xs[e] = c < n_cells ? __ldg(x + __ldg(gn + (size_t)c_base * NB + e)) : 0.f;
  }
  __syncthreads();
  const int g = threadIdx.x / 14, q = threadIdx.x % 14;
  const int i0 = 2 * q, i1 = min(2 * q + 1, NB - 1);
  float acc[4][T][2];
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int t = 0; t < T; t++) acc[m][t][0] = acc[m][t][1] = 0.f;
#pragma unroll 3
  for (int k = 0; k < NB; k++)
  {
    float xk[4];
#pragma unroll
    for (int m = 0; m < 4; m++) xk[m] = Xs[(4 * g + m) * NB + k];
#pragma unroll
    for (int t = 0; t < T; t++)
    {
      const float r0 = Rs[(t * NB + i0) * NB + k], r1 = Rs[(t * NB + i1) * NB + k];
#pragma unroll
      for (int m = 0; m < 4; m++)
      {
        acc[m][t][0] += r0 * xk[m];
        acc[m][t][1] += r1 * xk[m];
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 4; m++)
  {
    const int c = c_base + 4 * g + m;
    if (c >= n_cells) continue;
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int t = 0; t < T; t++)
    {
      const float cf = __ldg(cf32 + (size_t)c * T + t);
      y0 += cf * acc[m][t][0];
      y1 += cf * acc[m][t][1];
    }
    ybuf[(size_t)i0 * n_cells + c] = y0;
    if (2 * q + 1 < NB) ybuf[(size_t)i1 * n_cells + c] = y1;
  }
}

enum { MF_JACOBI = 0, MF_DEFECT = 1 };

template <int NBF, int MODE>
__global__ void mf_row_kernel(int n, int na, int n_cells, const int *__restrict__ inc_ptr,
                              const int *__restrict__ inc, const float *__restrict__ ybuf,
                              const float *__restrict__ x, const float *__restrict__ f,
                              const float *__restrict__ diag, float *__restrict__ out, float omega)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  if (r >= na)
  {
    out[r] = MODE == MF_JACOBI ? f[r] : f[r] - x[r];
    return;
  }
  float s = 0.f;
  for (int t = inc_ptr[r]; t < inc_ptr[r + 1]; t++)
  {
    const int e = inc[t], K = e / NBF, li = e - K * NBF;
    s += ybuf[(size_t)li * n_cells + K];
  }
  out[r] = MODE == MF_JACOBI ? x[r] + omega * (f[r] - s) / diag[r] : f[r] - s;
}

// FP32 copies of the cell coefficients (first T of each cell's T + Tr) and of the tensors
// R[(i*nbf + j)*T + t] -> R32[(t*nbf + i)*nbf + j]
__global__ void mf_convert_kernel(int n_cells, int T, int Tr, int nbf, const double *__restrict__ cellcoef,
                                  const double *__restrict__ R, float *__restrict__ cf32, float *__restrict__ R32)
{
  const long total_c = (long)n_cells * T, total_r = (long)T * nbf * nbf;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total_c + total_r; e += (long)gridDim.x * blockDim.x)
  {
    if (e < total_c)
    {
      const long c = e / T, t = e - c * T;
      cf32[e] = (float)cellcoef[c * (T + Tr) + t];
    }
    else
    {
      const long q = e - total_c, t = q / (nbf * nbf), ij = q - t * nbf * nbf;
      R32[q] = (float)R[ij * T + t];
    }
  }
}

// is (nbf, T) one of the instantiated shapes
// the matrix-free operator pays off for Q2 hexahedra (27 local DOFs); other elements keep
// the CSR kernels, whose rows are short
inline bool mf_shape_ok(int nbf, int T) { return nbf == 27 && (T == 10 || T == 13); }

inline bool use_mf(const Space &s)
{
  return s.mf_T > 0 && s.d_ybuf && s.mf_version == s.assembly_version && s.n_cells >= kMfMinCells &&
         mf_shape_ok(s.nbf, s.mf_T);
}

// y = A x per cell (phase 1)
inline void mf_apply_cells(cdgpu_ctx *ctx, const Space &s, const float *x)
{
  if (s.nbf == 27)
  {
    const int g27 = (s.n_cells + 63) / 64;
    if (s.mf_T == 10) { mf_cell27_kernel<10><<<g27, 224, 0, ctx->stream>>>(s.n_cells, s.d_gn, s.d_cf32, s.d_R32, x, s.d_ybuf); return; }
    if (s.mf_T == 13) { mf_cell27_kernel<13><<<g27, 224, 0, ctx->stream>>>(s.n_cells, s.d_gn, s.d_cf32, s.d_R32, x, s.d_ybuf); return; }
  }
  const int grid = (s.n_cells + 127) / 128;
#define CD_MF_CASE(NB, TT)                                                                              \
  if (s.nbf == NB && s.mf_T == TT)                                                                      \
  {                                                                                                     \
    mf_cell_kernel<NB, TT><<<grid, 128, 0, ctx->stream>>>(s.n_cells, s.d_gn, s.d_cf32, s.d_R32, x, s.d_ybuf); \
    return;                                                                                             \
  }
  CD_MF_CASE(27, 10) CD_MF_CASE(27, 13) CD_MF_CASE(8, 10) CD_MF_CASE(8, 13)
  CD_MF_CASE(9, 6) CD_MF_CASE(9, 14) CD_MF_CASE(4, 6) CD_MF_CASE(4, 14)
#undef CD_MF_CASE
}

template <int MODE>
inline void mf_rows(cdgpu_ctx *ctx, const Space &s, const float *x, const float *f, const float *diag, float *out,
                    float omega)
{
  const int grid = (s.n_dof + 255) / 256;
  switch (s.nbf)
  {
    case 27: mf_row_kernel<27, MODE><<<grid, 256, 0, ctx->stream>>>(s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega); break;
    case 9: mf_row_kernel<9, MODE><<<grid, 256, 0, ctx->stream>>>(s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega); break;
    case 8: mf_row_kernel<8, MODE><<<grid, 256, 0, ctx->stream>>>(s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega); break;
    default: mf_row_kernel<4, MODE><<<grid, 256, 0, ctx->stream>>>(s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega); break;
  }
}
