// The FP32 V-cycle below the finest level as ONE cooperative kernel.
//
// On the benchmark hierarchy the levels 16^3 ... 2^3 hold 36k DOFs and fewer; each of their
// ~22 operations (Jacobi sweeps, defect, restriction, prolongation, the exact coarse solve) is
// a few microseconds of work, so as separate launches they are bound by the launch and
// dependency latency between kernels.  Here one persistent grid (every CTA resident:
// cooperative launch) runs them in the cycle's order (TMultiGrid3D::Cycle,
// src/FE/MultiGrid3D.C:423-669, gamma = 1) with a grid-wide barrier between dependent
// operations.  The arithmetic of every row is the CSR kernels' (csr.cuh), in the same order,
// so the result equals the per-kernel cycle bit for bit.
//
// The barrier is a generation counter in global memory; every wait is bounded: a CTA that
// waits too long sets err = 5 and the abort flag, after which every later barrier returns at
// once and the remaining operations are skipped (the host reports the error after the solve).
#pragma once

#include "csr.cuh"

constexpr int kCoopMaxLevels = 16;
constexpr int kCoopThreads = 256;
constexpr long kCoopSpin = 1L << 22;

struct CoopLevel
{
  int n, n_active, gs;              // rows, active rows, threads per row of A
  const int *rp, *kc;               // A (FP32 copy)
  const float *a, *diag;
  float *sol, *alt, *rhs, *def;     // buffers at the start of the cycle (sol, alt swap per sweep)
  // transfer to the next coarser level: R = P^T over the coarser level's rows, P over this
  // level's rows
  const int *r_row, *r_col, *p_row, *p_col;
  const float *r_val, *p_val;
  int r_gs, p_gs;
};

struct CoopArgs
{
  int top;           // the level the kernel starts on (its rhs and zero sol come from the finest restriction)
  int pre, post;     // sweeps
  float omega, damp; // SC_SMOOTH_DAMP_FACTOR_SCALAR, SC_GMG_DAMP_FACTOR_SCALAR
  CoopLevel lev[kCoopMaxLevels];
  // exact coarse solve of level 0: explicit inverse of its active block (FP64)
  const double *a0;  // level 0 FP64 entries (for A_AD)
  const int *dir_start0;
  const double *cinv;
  unsigned *bar;     // [0] arrivals, [1] generation, [2] abort
  int *err;
};

__device__ __forceinline__ bool coop_barrier(unsigned *bar, int *err)
{
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    volatile unsigned *vb = bar;
    int ok = vb[2] == 0u;
    if (ok)
    {
      const unsigned g = vb[1];
      __threadfence();
      if (atomicAdd(&bar[0], 1u) == gridDim.x - 1)
      {
        bar[0] = 0u;
        __threadfence();
        atomicAdd(&bar[1], 1u);
      }
      else
      {
        long it = 0;
        while (vb[1] == g && vb[2] == 0u && it < kCoopSpin) it++;
        if (vb[1] == g)
        {
          if (vb[2] == 0u) atomicExch(err, 5);
          atomicExch(&bar[2], 1u);
          ok = 0;
        }
      }
      __threadfence();
    }
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// one CSR operation over all rows of a matrix, spread over the whole grid (every lane of a
// warp runs the same trips, as csr_kernel requires)
template <int GS, int U, int MODE> __device__ __forceinline__ void coop_rows_gs(const CsrArgs<float> &p)
{
  const int rows_end = MODE == CM_PROLONG ? p.n_active : p.n;
  const int lane = threadIdx.x % GS, sub = (threadIdx.x % 32) / GS;
  const long nwarp = (long)gridDim.x * blockDim.x / 32;
  const long step = nwarp * (32 / GS);
  double acc = 0;
  for (long base = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32 * (32 / GS); base < rows_end; base += step)
  {
    CsrRow<float, GS, U> w;
    csr_load_row<float, GS, U>(p, (int)base + sub, rows_end, lane, w);
    csr_do_row<float, GS, U, MODE>(p, (int)base + sub, rows_end, lane, w, acc);
  }
}

template <int MODE> __device__ __forceinline__ void coop_rows(const CsrArgs<float> &p, int gs)
{
  switch (gs)
  {
    case 1: coop_rows_gs<1, 8, MODE>(p); break;
    case 2: coop_rows_gs<2, 8, MODE>(p); break;
    case 4: coop_rows_gs<4, 8, MODE>(p); break;
    case 8: coop_rows_gs<8, 16, MODE>(p); break;
    default: coop_rows_gs<32, 8, MODE>(p); break;
  }
}

__global__ void __launch_bounds__(kCoopThreads) mg_coop_cycle_kernel(CoopArgs a)
{
  extern __shared__ double coop_sm[];
  const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
  float *x[kCoopMaxLevels], *xa[kCoopMaxLevels];
  for (int i = 0; i <= a.top; i++)
  {
    x[i] = a.lev[i].sol;
    xa[i] = a.lev[i].alt;
  }
  auto jacobi = [&](int i) {
    const CoopLevel &L = a.lev[i];
    CsrArgs<float> p;
    p.n = L.n; p.n_active = L.n_active; p.rp = L.rp; p.kc = L.kc; p.a = L.a; p.x = x[i]; p.f = L.rhs;
    p.diag = L.diag; p.y = xa[i]; p.omega = a.omega;
    coop_rows<CM_JACOBI>(p, L.gs);
    float *t = x[i]; x[i] = xa[i]; xa[i] = t;
  };
  // down: levels top .. 1
  for (int i = a.top; i >= 1; i--)
  {
    const CoopLevel &L = a.lev[i];
    // first pre-smoothing sweep from the zero start (jacobi_first_kernel with x = 0)
    if (a.pre > 0)
    {
      for (long r = tid; r < L.n; r += nth)
        xa[i][r] = r < L.n_active ? a.omega * L.rhs[r] / L.diag[r] : L.rhs[r];
      float *t = x[i]; x[i] = xa[i]; xa[i] = t;
      if (!coop_barrier(a.bar, a.err)) return;
    }
    for (int k = 1; k < a.pre; k++)
    {
      jacobi(i);
      if (!coop_barrier(a.bar, a.err)) return;
    }
    {
      CsrArgs<float> p;
      p.n = L.n; p.n_active = L.n_active; p.rp = L.rp; p.kc = L.kc; p.a = L.a; p.x = x[i]; p.f = L.rhs; p.y = L.def;
      coop_rows<CM_DEFECT>(p, L.gs);
      if (!coop_barrier(a.bar, a.err)) return;
    }
    {
      const CoopLevel &C = a.lev[i - 1];
      CsrArgs<float> p;
      p.n = C.n; p.n_active = C.n_active; p.rp = L.r_row; p.kc = L.r_col; p.a = L.r_val; p.x = L.def;
      p.y = C.rhs; p.y2 = x[i - 1];
      coop_rows<CM_RESTRICT>(p, L.r_gs);
      if (!coop_barrier(a.bar, a.err)) return;
    }
  }
  // exact coarse solve on level 0 by block 0 (coarse_exact_kernel): sol_D = rhs_D,
  // sol_A = inv(A_AA) (rhs_A - A_AD rhs_D)
  if (blockIdx.x == 0)
  {
    const CoopLevel &L = a.lev[0];
    const int n = L.n, na = L.n_active;
    double *b = coop_sm;
    for (int i = threadIdx.x; i < n; i += blockDim.x) b[i] = (double)L.rhs[i];
    __syncthreads();
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nw = blockDim.x / 32;
    for (int i = warp; i < na; i += nw)
    {
      double v = 0.0;
      for (int j = a.dir_start0[i] + lane; j < L.rp[i + 1]; j += 32) v += a.a0[j] * b[L.kc[j]];
      v = csr_group_sum<32>(v);
      if (lane == 0) b[n + i] = b[i] - v;
    }
    for (int i = na + threadIdx.x; i < n; i += blockDim.x) x[0][i] = (float)b[i];
    __syncthreads();
    for (int r = warp; r < na; r += nw)
    {
      double s = 0;
      for (int j = lane; j < na; j += 32) s += a.cinv[(size_t)r * na + j] * b[n + j];
      s = csr_group_sum<32>(s);
      if (lane == 0) x[0][r] = (float)s;
    }
  }
  if (!coop_barrier(a.bar, a.err)) return;
  // up: levels 1 .. top
  for (int i = 1; i <= a.top; i++)
  {
    const CoopLevel &L = a.lev[i];
    {
      CsrArgs<float> p;
      p.n = L.n; p.n_active = L.n_active; p.rp = L.p_row; p.kc = L.p_col; p.a = L.p_val; p.x = x[i - 1];
      p.y = x[i]; p.omega = a.damp;
      coop_rows<CM_PROLONG>(p, L.p_gs);
      if (!coop_barrier(a.bar, a.err)) return;
    }
    for (int k = 0; k < a.post; k++)
    {
      jacobi(i);
      if (i < a.top || k + 1 < a.post)
        if (!coop_barrier(a.bar, a.err)) return;
    }
  }
}
