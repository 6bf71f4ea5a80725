// The coarse end of the FP32 V-cycle in one launch: the levels below ~8k rows (for the 32^3
// bench hierarchy the 8^3, 4^3 and 2^3 levels) run on one thread-block cluster whose CTAs
// split every level's rows and meet at the cluster's hardware barrier between the steps --
// pre-smoothing, defect, restriction, the exact coarse solve, prolongation, post-smoothing
// (MultiGrid3D.C:423-669 for one V-cycle; MGLevel3D.C:443-537 for the damped-Jacobi sweep,
// 539-588 for the transfers) -- instead of one grid-wide launch per step.  The arithmetic
// per row is that of the per-level kernels (csr_kernel's Jacobi, defect, restriction and
// prolongation epilogues, jacobi_first_kernel, coarse_exact_kernel); only the summation
// order inside a row differs.  Level vectors live in global memory (L2) and are read with
// L2-only loads, so no CTA sees a stale L1 line of a vector another CTA wrote before the
// barrier; matrices and transfer operators are read-only.  The barriers are the cluster's
// (barrier.cluster, release/acquire), every thread reaches each of them, and no wait spins.
#pragma once

#include <cooperative_groups.h>

#include "internal.h"

constexpr int kClusterMaxLevels = 4;
constexpr int kClusterMaxRows = 8192; // levels with at most this many rows go to the cluster
constexpr int kClusterThreads = 1024;
// off: with the vectors and matrices read from L2 in every step the cluster launch took
// ~127 us per V-cycle against ~85 us for the per-level launches on all SMs (170.6 against
// 194.1 solves/s)
constexpr bool kClusterCycleOn = false;

struct ClusterLevel
{
  int n = 0, na = 0;
  const int *rp = nullptr, *kc = nullptr, *dir_start = nullptr;
  const float *a = nullptr, *diag = nullptr;
  float *sol = nullptr, *alt = nullptr, *rhs = nullptr, *def = nullptr;
  // restriction to the next coarser level (rows = coarser DOFs) and prolongation from it
  // (rows = this level's DOFs); unused on level 0
  const int *r_rp = nullptr, *r_kc = nullptr, *p_rp = nullptr, *p_kc = nullptr;
  const float *r_val = nullptr, *p_val = nullptr;
};

struct ClusterCycle
{
  int nl = 0; // levels 0 .. nl-1, nl-1 the top one (its rhs written by the restriction above)
  ClusterLevel lev[kClusterMaxLevels];
  int pre = 2, post = 2;
  float omega = 0.8f, damp = 1.0f;
  // level 0: exact solve with the FP64 matrix's Dirichlet columns and the explicit inverse
  const double *a64 = nullptr, *cinv = nullptr;
};

// sum of a row of A times x over entries [jb, je), 4 threads per row (lane4 = 0..3): in rounds
// of 32 entries, each thread issues its 8 column and value loads, then its 8 gathers of x,
// before the first product, so a round costs two L2 latencies whatever its length
__device__ __forceinline__ float cl_row(const int *__restrict__ kc, const float *__restrict__ a,
                                        const float *x, int jb, int je, int lane4)
{
  float s = 0.f;
  for (int j0 = jb + lane4; j0 < je; j0 += 32)
  {
    int c[8];
    float v[8], xv[8];
#pragma unroll
    for (int u = 0; u < 8; u++)
    {
      const int j = j0 + 4 * u;
      c[u] = j < je ? __ldg(kc + j) : -1;
      v[u] = j < je ? __ldg(a + j) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) xv[u] = c[u] >= 0 ? __ldcg(x + c[u]) : 0.f;
#pragma unroll
    for (int u = 0; u < 8; u++) s += v[u] * xv[u];
  }
  s += __shfl_xor_sync(0xffffffffu, s, 1, 4);
  s += __shfl_xor_sync(0xffffffffu, s, 2, 4);
  return s;
}

__global__ void __launch_bounds__(kClusterThreads, 1) mg_cluster_kernel(ClusterCycle c)
{
  CD_PDL_ENTRY();
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), nb = (int)cl.num_blocks();
  const int tid = threadIdx.x, lane4 = tid & 3, grp = tid >> 2;
  constexpr int kGroups = kClusterThreads / 4;
  extern __shared__ double cl_sm[];
  // rows [r0, r1) of an n-row level for this CTA
  auto range = [&](int n, int &r0, int &r1) {
    const int per = (n + nb - 1) / nb;
    r0 = min(n, rank * per);
    r1 = min(n, r0 + per);
  };
  // one damped-Jacobi sweep x -> y; first: x is zero on every row (jacobi_first_kernel with
  // x_all_zero), else the csr_kernel Jacobi epilogue
  auto sweep = [&](const ClusterLevel &L, const float *x, float *y, bool first) {
    int r0, r1;
    range(L.n, r0, r1);
    for (int base = r0; base < r1; base += kGroups)
    {
      const int r = base + grp;
      const bool in = r < r1;
      float s = 0.f;
      if (!first && in) s = cl_row(L.kc, L.a, x, __ldg(L.rp + r), __ldg(L.rp + r + 1), lane4);
      else if (!first) s = cl_row(L.kc, L.a, x, 0, 0, lane4); // keeps every lane in the shuffles
      if (in && lane4 == 0)
      {
        const float f = __ldcg(L.rhs + r);
        if (r >= L.na)
          y[r] = f;
        else if (first)
          y[r] = c.omega * f / __ldg(L.diag + r);
        else
          y[r] = __ldcg(x + r) + c.omega * (f - s) / __ldg(L.diag + r);
      }
    }
  };
  auto defect = [&](const ClusterLevel &L, const float *x) {
    int r0, r1;
    range(L.n, r0, r1);
    for (int base = r0; base < r1; base += kGroups)
    {
      const int r = base + grp;
      const bool in = r < r1;
      const float s = in ? cl_row(L.kc, L.a, x, __ldg(L.rp + r), __ldg(L.rp + r + 1), lane4)
                         : cl_row(L.kc, L.a, x, 0, 0, lane4);
      if (in && lane4 == 0) L.def[r] = __ldcg(L.rhs + r) - s;
    }
  };
  // coarse rhs = R d on active coarse rows, 0 elsewhere; coarse solution reset
  auto restrict_to = [&](const ClusterLevel &F, ClusterLevel &C) {
    int r0, r1;
    range(C.n, r0, r1);
    for (int base = r0; base < r1; base += kGroups)
    {
      const int r = base + grp;
      const bool in = r < r1;
      const float s = in ? cl_row(F.r_kc, F.r_val, F.def, __ldg(F.r_rp + r), __ldg(F.r_rp + r + 1), lane4)
                         : cl_row(F.r_kc, F.r_val, F.def, 0, 0, lane4);
      if (in && lane4 == 0)
      {
        C.rhs[r] = r < C.na ? s : 0.f;
        C.sol[r] = 0.f;
      }
    }
  };
  // sol += damp * P xc on active fine rows
  auto prolong = [&](const ClusterLevel &F, float *sol, const float *xc) {
    int r0, r1;
    range(F.na, r0, r1);
    for (int base = r0; base < r1; base += kGroups)
    {
      const int r = base + grp;
      const bool in = r < r1;
      const float s = in ? cl_row(F.p_kc, F.p_val, xc, __ldg(F.p_rp + r), __ldg(F.p_rp + r + 1), lane4)
                         : cl_row(F.p_kc, F.p_val, xc, 0, 0, lane4);
      if (in && lane4 == 0) sol[r] = __ldcg(sol + r) + c.damp * s;
    }
  };
  // the working pointers of every level (swapped after every sweep, as the host does)
  float *sol[kClusterMaxLevels], *alt[kClusterMaxLevels];
  for (int l = 0; l < c.nl; l++) { sol[l] = c.lev[l].sol; alt[l] = c.lev[l].alt; }
  // down: the top level's rhs is given and its solution zero
  for (int l = c.nl - 1; l >= 1; l--)
  {
    const ClusterLevel &L = c.lev[l];
    for (int k = 0; k < c.pre; k++)
    {
      sweep(L, sol[l], alt[l], k == 0);
      float *t = sol[l]; sol[l] = alt[l]; alt[l] = t;
      cl.sync();
    }
    defect(L, sol[l]);
    cl.sync();
    restrict_to(L, c.lev[l - 1]);
    cl.sync();
  }
  // level 0: exact solve (coarse_exact_kernel) on the first CTA
  if (rank == 0)
  {
    const ClusterLevel &L = c.lev[0];
    double *b = cl_sm;
    for (int i = tid; i < L.n; i += blockDim.x) b[i] = (double)__ldcg(L.rhs + i);
    __syncthreads();
    const int warp = tid / 32, lane = tid % 32, nw = blockDim.x / 32;
    for (int i = warp; i < L.na; i += nw)
    {
      double v = 0.0;
      for (int j = __ldg(L.dir_start + i) + lane; j < __ldg(L.rp + i + 1); j += 32) v += __ldg(c.a64 + j) * b[__ldg(L.kc + j)];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) b[L.n + i] = b[i] - v;
    }
    for (int i = L.na + tid; i < L.n; i += blockDim.x) sol[0][i] = (float)b[i];
    __syncthreads();
    for (int r = warp; r < L.na; r += nw)
    {
      double s = 0;
      for (int j = lane; j < L.na; j += 32) s += __ldg(c.cinv + (size_t)r * L.na + j) * b[L.n + j];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) sol[0][r] = (float)s;
    }
  }
  cl.sync();
  // up
  for (int l = 1; l < c.nl; l++)
  {
    const ClusterLevel &L = c.lev[l];
    prolong(L, sol[l], sol[l - 1]);
    cl.sync();
    for (int k = 0; k < c.post; k++)
    {
      sweep(L, sol[l], alt[l], false);
      float *t = sol[l]; sol[l] = alt[l]; alt[l] = t;
      cl.sync();
    }
  }
}
