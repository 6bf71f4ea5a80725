// Matrix-free FP64 operator of Q2 hexahedra on affine cells with constant coefficients, by sum
// factorisation: the product the mixed form's FGMRES iteration applies on the finest level
// (MatVect / Defect, Blas2.C:11-99, of the matrix TAssembleMat3D assembles) without reading
// that matrix.
//
// The local matrix of a cell is A_c = sum_t coef_{c,t} R_t with the reference tensors R_t of
// the affine fast path (integrals over [-1,1]^3 of products of the Q2 basis and its
// derivatives: I_ab, C_b, M and, for SUPG, D_a; ConvDiff3D.C:61-190).  Every R_t is an
// integral of a product of tensor-product polynomials of degree <= 2 per direction, so the
// 3-point Gauss rule in each direction integrates it exactly, and
//   (A_c x_c)_i = sum_q w_q [ sum_a d_a phi_i(q) F_a(q) + phi_i(q) S(q) ],
//   F_a = sum_b K_ab d_b u + delta_a u,   S = sum_b beta_b d_b u + c_M u,
// with u = sum_j x_j phi_j, K = [[c0 c3 c4] [c3 c1 c5] [c4 c5 c2]], beta = (c6, c7, c8),
// c_M = c9 and delta = (c10, c11, c12) (SUPG only).  Values and gradients at the 27 points
// come from three passes of 3 x 3 one-dimensional matrices (z, y, x), the test functions from
// three transposed passes: about 2,000 FMAs per cell instead of the dense 27 x 27 x T.  The
// result equals the assembled matrix's product up to rounding.
//
//   phase 1 (mf64_cell27_kernel): 32 cells per block pass, nine warps; warp w owns one of the
//     nine lines of a pass for 32 cells (lane = cell), keeps its 3 values per field in
//     registers and hands the lines to the next pass through shared memory ([field][point]
//     [cell], conflict-free); writes A_c x_c to the per-cell buffer [local index][cell];
//   phase 2 (mf64_row_kernel): one thread per DOF sums its cells' contributions in ascending
//     cell order (the assembly's DOF -> cell incidence), so the result is deterministic;
//     Dirichlet rows are identity rows, as in the assembled matrix; the defect form also
//     leaves per-block sums of d^2.
#pragma once

#include "internal.h"

// one-dimensional tables of the 3-point Gauss rule on [-1, 1] for the Lagrange basis on the
// nodes -1, 0, 1: B[q][a] = l_a(xi_q), G[q][a] = l_a'(xi_q), w[q] the weights
struct Mf64Tab
{
  double B[3][3], G[3][3], w[3];
};

inline Mf64Tab mf64_tables()
{
  Mf64Tab t;
  const double xi[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)};
  for (int q = 0; q < 3; q++)
  {
    const double s = xi[q];
    t.B[q][0] = 0.5 * s * (s - 1);
    t.B[q][1] = 1 - s * s;
    t.B[q][2] = 0.5 * s * (s + 1);
    t.G[q][0] = s - 0.5;
    t.G[q][1] = -2 * s;
    t.G[q][2] = s + 0.5;
  }
  t.w[0] = t.w[2] = 5.0 / 9.0;
  t.w[1] = 8.0 / 9.0;
  return t;
}

constexpr int kMf64Warps = 9, kMf64Cells = 32;

template <int T>
__global__ void __launch_bounds__(kMf64Warps * 32, 3)
    mf64_cell27_kernel(int n_cells, const int *__restrict__ gn, const double *__restrict__ cellcoef, int cstride,
                       const Mf64Tab tb, const double *__restrict__ x, double *__restrict__ ybuf, int pre)
{
  // two exchange buffers of 81 lines x 32 cells, used alternately by the five passes
  __shared__ double bufA[81 * kMf64Cells], bufB[81 * kMf64Cells];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w3 = w / 3, w1 = w - 3 * w3;
  const int n_groups = (n_cells + kMf64Cells - 1) / kMf64Cells;
  // the next group's DOF numbers (this warp's z line), loaded one group ahead; with pre the
  // first group's (written by no kernel of the solve) come before the wait
  int gi[3];
  auto fetch = [&](int grp) {
    const int c = grp * kMf64Cells + lane;
    const bool live = grp < n_groups && c < n_cells;
#pragma unroll
    for (int k = 0; k < 3; k++) gi[k] = live ? __ldg(gn + (size_t)c * 27 + 9 * k + w) : -1;
  };
  if (pre) fetch(blockIdx.x);
  CD_PDL_ENTRY();
  if (!pre) fetch(blockIdx.x);
  for (int grp = blockIdx.x; grp < n_groups; grp += gridDim.x)
  {
    const int c = grp * kMf64Cells + lane;
    double X[3], C[T];
#pragma unroll
    for (int k = 0; k < 3; k++) X[k] = gi[k] >= 0 ? __ldg(x + gi[k]) : 0.0;
    // the coefficients, first read in pass 3, are in flight during passes 1 and 2
#pragma unroll
    for (int t = 0; t < T; t++) C[t] = c < n_cells ? __ldg(cellcoef + (size_t)c * cstride + t) : 0.0;
    fetch(grp + gridDim.x);
    // pass 1, z: warp w = line (jy, jx); UB[qz] = sum_jz B[qz][jz] X, UG[qz] = sum_jz G[qz][jz] X
#pragma unroll
    for (int q = 0; q < 3; q++)
    {
      bufA[((0 * 3 + q) * 9 + w) * 32 + lane] = tb.B[q][0] * X[0] + tb.B[q][1] * X[1] + tb.B[q][2] * X[2];
      bufA[((1 * 3 + q) * 9 + w) * 32 + lane] = tb.G[q][0] * X[0] + tb.G[q][1] * X[1] + tb.G[q][2] * X[2];
    }
    __syncthreads();
    // pass 2, y: warp w = (qz, jx); BB = B_y UB, GB = G_y UB (d/dy), BG = B_y UG (d/dz)
    {
      const int qz = w3, jx = w1;
      double ub[3], ug[3];
#pragma unroll
      for (int j = 0; j < 3; j++)
      {
        ub[j] = bufA[((0 * 3 + qz) * 9 + 3 * j + jx) * 32 + lane];
        ug[j] = bufA[((1 * 3 + qz) * 9 + 3 * j + jx) * 32 + lane];
      }
#pragma unroll
      for (int q = 0; q < 3; q++)
      {
        const int o = (qz * 9 + 3 * q + jx) * 32 + lane;
        bufB[o] = tb.B[q][0] * ub[0] + tb.B[q][1] * ub[1] + tb.B[q][2] * ub[2];
        bufB[27 * 32 + o] = tb.G[q][0] * ub[0] + tb.G[q][1] * ub[1] + tb.G[q][2] * ub[2];
        bufB[54 * 32 + o] = tb.B[q][0] * ug[0] + tb.B[q][1] * ug[1] + tb.B[q][2] * ug[2];
      }
    }
    __syncthreads();
    // pass 3, x, the point-wise fluxes and the first transposed pass: warp w = (qz, qy)
    {
      const int qz = w3, qy = w1;
      double bb[3], gb[3], bg[3];
#pragma unroll
      for (int j = 0; j < 3; j++)
      {
        const int o = (qz * 9 + 3 * qy + j) * 32 + lane;
        bb[j] = bufB[o];
        gb[j] = bufB[27 * 32 + o];
        bg[j] = bufB[54 * 32 + o];
      }
      // (w[0] = w[2]: selected, not indexed, so the tables stay in the parameter bank)
      const double wyz = (qy == 1 ? tb.w[1] : tb.w[0]) * (qz == 1 ? tb.w[1] : tb.w[0]);
      double P1[3] = {0, 0, 0}, P2[3] = {0, 0, 0}, P3[3] = {0, 0, 0};
#pragma unroll
      for (int q = 0; q < 3; q++)
      {
        const double u = tb.B[q][0] * bb[0] + tb.B[q][1] * bb[1] + tb.B[q][2] * bb[2];
        const double ux = tb.G[q][0] * bb[0] + tb.G[q][1] * bb[1] + tb.G[q][2] * bb[2];
        const double uy = tb.B[q][0] * gb[0] + tb.B[q][1] * gb[1] + tb.B[q][2] * gb[2];
        const double uz = tb.B[q][0] * bg[0] + tb.B[q][1] * bg[1] + tb.B[q][2] * bg[2];
        const double wq = wyz * tb.w[q];
        double Fx = C[0] * ux + C[3] * uy + C[4] * uz;
        double Fy = C[3] * ux + C[1] * uy + C[5] * uz;
        double Fz = C[4] * ux + C[5] * uy + C[2] * uz;
        if constexpr (T == 13)
        {
          Fx += C[10] * u;
          Fy += C[11] * u;
          Fz += C[12] * u;
        }
        const double S = wq * (C[6] * ux + C[7] * uy + C[8] * uz + C[9] * u);
        Fx *= wq;
        Fy *= wq;
        Fz *= wq;
#pragma unroll
        for (int i = 0; i < 3; i++)
        {
          P1[i] += tb.G[q][i] * Fx + tb.B[q][i] * S;
          P2[i] += tb.B[q][i] * Fy;
          P3[i] += tb.B[q][i] * Fz;
        }
      }
#pragma unroll
      for (int i = 0; i < 3; i++)
      {
        const int o = (qz * 9 + 3 * qy + i) * 32 + lane;
        bufA[o] = P1[i];
        bufA[27 * 32 + o] = P2[i];
        bufA[54 * 32 + o] = P3[i];
      }
    }
    __syncthreads();
    // pass 4, y transposed: warp w = (qz, ix); Q1 = B_y^T P1 + G_y^T P2, Q2 = B_y^T P3
    {
      const int qz = w3, ix = w1;
      double p1[3], p2[3], p3[3];
#pragma unroll
      for (int q = 0; q < 3; q++)
      {
        const int o = (qz * 9 + 3 * q + ix) * 32 + lane;
        p1[q] = bufA[o];
        p2[q] = bufA[27 * 32 + o];
        p3[q] = bufA[54 * 32 + o];
      }
#pragma unroll
      for (int i = 0; i < 3; i++)
      {
        const int o = (qz * 9 + 3 * i + ix) * 32 + lane;
        bufB[o] = tb.B[0][i] * p1[0] + tb.B[1][i] * p1[1] + tb.B[2][i] * p1[2] + tb.G[0][i] * p2[0] +
                  tb.G[1][i] * p2[1] + tb.G[2][i] * p2[2];
        bufB[27 * 32 + o] = tb.B[0][i] * p3[0] + tb.B[1][i] * p3[1] + tb.B[2][i] * p3[2];
      }
    }
    __syncthreads();
    // pass 5, z transposed: warp w = (iy, ix); y[iz] = B_z^T Q1 + G_z^T Q2
    {
      double q1[3], q2[3];
#pragma unroll
      for (int q = 0; q < 3; q++)
      {
        q1[q] = bufB[(q * 9 + w) * 32 + lane];
        q2[q] = bufB[27 * 32 + (q * 9 + w) * 32 + lane];
      }
      if (c < n_cells)
      {
#pragma unroll
        for (int i = 0; i < 3; i++)
          ybuf[(size_t)(9 * i + w) * n_cells + c] = tb.B[0][i] * q1[0] + tb.B[1][i] * q1[1] + tb.B[2][i] * q1[2] +
                                                    tb.G[0][i] * q2[0] + tb.G[1][i] * q2[1] + tb.G[2][i] * q2[2];
      }
    }
    // the next group's pass 1 writes bufA, last read in pass 4 (before the barrier above); its
    // pass 2 writes bufB after the barrier that follows its pass 1
  }
}

enum { MF64_SPMV = 0, MF64_DEFECT = 1 };

// y = sum over a DOF's cells of their contributions (ascending cell order), or d = f - y;
// Dirichlet rows: y = x, d = f - x.  With partial (defect form), per-block sums of d^2 over
// all rows, as the CSR defect leaves them.  Grid-stride over rows.
// With inc8 (the 8-wide incidence records of mf_inc8_kernel) a row reads one record and then
// its cells' contributions; without, its incidence pointers and entries.
template <int MODE>
__global__ void __launch_bounds__(256) mf64_row_kernel(int n, int na, int n_cells, const int *__restrict__ inc_ptr,
                                                       const int *__restrict__ inc, const int *__restrict__ inc8,
                                                       const double *__restrict__ ybuf,
                                                       const double *__restrict__ x, const double *__restrict__ f,
                                                       double *__restrict__ out, double *__restrict__ partial)
{
  CD_PDL_ENTRY();
  double acc = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
  {
    double s;
    if (r >= na)
      s = x[r];
    else if (inc8)
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
    else
    {
      const int b = inc_ptr[r], e = inc_ptr[r + 1];
      int ei[8];
#pragma unroll
      for (int j = 0; j < 8; j++) ei[j] = b + j < e ? __ldg(inc + b + j) : -1;
      double yv[8];
#pragma unroll
      for (int j = 0; j < 8; j++)
      {
        const int K = ei[j] / 27, li = ei[j] - K * 27;
        yv[j] = ei[j] >= 0 ? ybuf[(size_t)li * n_cells + K] : 0.0;
      }
      s = 0;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (b + j < e) s += yv[j];
      for (int t = b + 8; t < e; t++)
      {
        const int K = inc[t] / 27, li = inc[t] - K * 27;
        s += ybuf[(size_t)li * n_cells + K];
      }
    }
    if (MODE == MF64_DEFECT)
    {
      const double d = f[r] - s;
      out[r] = d;
      acc += d * d;
    }
    else
      out[r] = s;
  }
  if (MODE == MF64_DEFECT && partial)
  {
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0)
    {
      double t = 0;
      for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
      partial[blockIdx.x] = t;
    }
  }
}
