// The coarse end of the FP32 V-cycle in one launch: the levels below ~8k rows (for the 32^3
// bench hierarchy the 8^3, 4^3 and 2^3 levels) run on one 16-CTA thread-block cluster
// (MultiGrid3D.C:423-669 for one V-cycle; MGLevel3D.C:443-537 for the damped-Jacobi sweep,
// 539-588 for the transfers).  The CTAs split every level's rows; at the start each CTA copies
// its rows of every level's matrix, restriction and prolongation into its shared memory
// (columns as 16-bit indices), and every CTA keeps a full copy of every level's iterate and
// defect there.  A step (sweep, defect, restriction, prolongation) computes the CTA's rows from
// shared memory alone and writes each new value into the copies of all CTAs of the cluster
// (distributed shared memory); the cluster barrier (barrier.cluster, release/acquire) then
// makes them visible.  The exact coarse solve runs on the first CTA.  The arithmetic per row
// is that of the per-level kernels (jacobi_first_kernel, csr_kernel's Jacobi, defect,
// restriction and prolongation epilogues, coarse_exact_kernel); only the summation order
// inside a row differs.  Every thread reaches every barrier, no wait spins, and a final
// barrier keeps each CTA's shared memory alive until no other CTA writes into it.
#pragma once

#include <cooperative_groups.h>

#include "internal.h"

// ClusterLevel, ClusterCycle and the kCluster* constants are in internal.h

template <typename P> __device__ __forceinline__ P *cl_at(unsigned char *sm, int off) { return (P *)(sm + off); }

// a row of a CSR slice in shared memory (row pointers rebased at the CTA's first row) times
// x, 4 threads per row
__device__ __forceinline__ float cl_row_sm(const int *rp, const unsigned short *kc, const float *a, const float *x,
                                           int lr, int lane4)
{
  float s = 0.f;
  for (int j = rp[lr] + lane4; j < rp[lr + 1]; j += 4) s += a[j] * x[kc[j]];
  s += __shfl_xor_sync(0xffffffffu, s, 1, 4);
  s += __shfl_xor_sync(0xffffffffu, s, 2, 4);
  return s;
}

__global__ void __launch_bounds__(kClusterThreads, 1) mg_cluster_kernel(ClusterCycle c)
{
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), nb = (int)cl.num_blocks();
  const int tid = threadIdx.x, lane4 = tid & 3, grp = tid >> 2;
  constexpr int kGroups = kClusterThreads / 4;
  extern __shared__ __align__(16) unsigned char cl_sm[];
  // ---- the CTA's slices of every level's operators and its diagonal (written by no kernel
  // of the cycle, so copied before the wait for the predecessor); iterates zero ----
  auto load_csr = [&](const int *rp, const int *kc, const float *a, int r0, int r1, int o_rp, int o_kc, int o_a) {
    if (r1 <= r0) return;
    const int base = __ldg(rp + r0);
    int *srp = cl_at<int>(cl_sm, o_rp);
    for (int i = tid; i <= r1 - r0; i += blockDim.x) srp[i] = __ldg(rp + r0 + i) - base;
    const int ne = __ldg(rp + r1) - base;
    unsigned short *skc = cl_at<unsigned short>(cl_sm, o_kc);
    float *sa = cl_at<float>(cl_sm, o_a);
    for (int i = tid; i < ne; i += blockDim.x)
    {
      skc[i] = (unsigned short)__ldg(kc + base + i);
      sa[i] = __ldg(a + base + i);
    }
  };
  for (int l = 0; l < c.nl; l++)
  {
    const ClusterLevel &L = c.lev[l];
    float *x0 = cl_at<float>(cl_sm, L.o_x0);
    for (int i = tid; i < L.n; i += blockDim.x) x0[i] = 0.f;
    if (l == 0) continue;
    const int r0 = L.rb[rank], r1 = L.rb[rank + 1];
    load_csr(L.rp, L.kc, L.a, r0, r1, L.o_rp, L.o_kc, L.o_a);
    load_csr(L.p_rp, L.p_kc, L.p_val, L.pb[rank], L.pb[rank + 1], L.o_prp, L.o_pkc, L.o_pval);
    const int c0 = L.cb[rank], c1 = L.cb[rank + 1];
    load_csr(L.r_rp, L.r_kc, L.r_val, c0, c1, L.o_rrp, L.o_rkc, L.o_rval);
    float *dg = cl_at<float>(cl_sm, L.o_diag);
    for (int i = tid; i < r1 - r0; i += blockDim.x) dg[i] = __ldg(L.diag + r0 + i);
  }
  CD_PDL_WAIT();
  CD_PDL_TRIGGER();
  {
    const ClusterLevel &L = c.lev[c.nl - 1];
    const int r0 = L.rb[rank], r1 = L.rb[rank + 1];
    float *rhs = cl_at<float>(cl_sm, L.o_rhs);
    for (int i = tid; i < r1 - r0; i += blockDim.x) rhs[i] = __ldcg(c.top_rhs + r0 + i);
  }
  // no CTA writes into another's copies before every CTA has zeroed its own
  cl.sync();
  // write value v of row r of the array at byte offset off into every CTA's copy (the four
  // lanes of a row group share the CTAs)
  auto bcast = [&](int off, int r, float v) {
    for (int k = lane4; k < nb; k += 4) cl.map_shared_rank(cl_at<float>(cl_sm, off), k)[r] = v;
  };
  // the iterate buffers of every level (swapped after every sweep)
  int xo[kClusterMaxLevels], xa[kClusterMaxLevels];
  for (int l = 0; l < c.nl; l++) { xo[l] = c.lev[l].o_x0; xa[l] = c.lev[l].o_x1; }
  // one damped-Jacobi sweep of level l from buffer xo[l] into xa[l] (all copies); first: the
  // iterate is zero (jacobi_first_kernel with x_all_zero)
  auto sweep = [&](int l, bool first) {
    const ClusterLevel &L = c.lev[l];
    const int r0 = L.rb[rank], r1 = L.rb[rank + 1];
    const int *rp = cl_at<int>(cl_sm, L.o_rp);
    const unsigned short *kc = cl_at<unsigned short>(cl_sm, L.o_kc);
    const float *a = cl_at<float>(cl_sm, L.o_a), *dg = cl_at<float>(cl_sm, L.o_diag);
    const float *rhs = cl_at<float>(cl_sm, L.o_rhs), *x = cl_at<float>(cl_sm, xo[l]);
    for (int base = r0; base < r1; base += kGroups)
    {
      const int r = base + grp, lr = r - r0;
      const bool in = r < r1;
      float s = 0.f;
      if (!first) s = cl_row_sm(rp, kc, a, x, in ? lr : 0, lane4); // every lane in the shuffles
      if (in)
      {
        const float f = rhs[lr];
        float y;
        if (r >= L.na)
          y = f;
        else if (first)
          y = c.omega * f / dg[lr];
        else
          y = x[r] + c.omega * (f - s) / dg[lr];
        bcast(xa[l], r, y);
      }
    }
    const int t = xo[l];
    xo[l] = xa[l];
    xa[l] = t;
  };
  auto defect = [&](int l) {
    const ClusterLevel &L = c.lev[l];
    const int r0 = L.rb[rank], r1 = L.rb[rank + 1];
    const int *rp = cl_at<int>(cl_sm, L.o_rp);
    const unsigned short *kc = cl_at<unsigned short>(cl_sm, L.o_kc);
    const float *a = cl_at<float>(cl_sm, L.o_a), *rhs = cl_at<float>(cl_sm, L.o_rhs);
    const float *x = cl_at<float>(cl_sm, xo[l]);
    for (int base = r0; base < r1; base += kGroups)
    {
      const int r = base + grp, lr = r - r0;
      const bool in = r < r1;
      const float s = cl_row_sm(rp, kc, a, x, in ? lr : 0, lane4);
      if (in) bcast(L.o_def, r, rhs[lr] - s);
    }
  };
  // restriction from level l into level l-1 >= 1: rhs = R d on active rows, 0 elsewhere (the
  // coarser iterate is zero already: zeroed at the start, and a V-cycle visits it once).  The
  // CTA computes its rows of R (split cb) and stores each value in the right-hand-side slice of
  // the CTA that owns the row on the coarser level (split rb there)
  auto restrict_to = [&](int l) {
    const ClusterLevel &L = c.lev[l], &C = c.lev[l - 1];
    const int c0 = L.cb[rank], c1 = L.cb[rank + 1];
    const int *rp = cl_at<int>(cl_sm, L.o_rrp);
    const unsigned short *kc = cl_at<unsigned short>(cl_sm, L.o_rkc);
    const float *rv = cl_at<float>(cl_sm, L.o_rval), *d = cl_at<float>(cl_sm, L.o_def);
    for (int base = c0; base < c1; base += kGroups)
    {
      const int r = base + grp, lr = r - c0;
      const bool in = r < c1;
      const float s = cl_row_sm(rp, kc, rv, d, in ? lr : 0, lane4);
      if (in && lane4 == 0)
      {
        int k = 0;
        while (k + 1 < nb && C.rb[k + 1] <= r) k++;
        cl.map_shared_rank(cl_at<float>(cl_sm, C.o_rhs), k)[r - C.rb[k]] = r < C.na ? s : 0.f;
      }
    }
  };
  // x_l += damp * P x_{l-1} on active rows (all copies)
  auto prolong = [&](int l) {
    const ClusterLevel &L = c.lev[l];
    const int r0 = L.pb[rank], r1 = L.pb[rank + 1];
    const int *rp = cl_at<int>(cl_sm, L.o_prp);
    const unsigned short *kc = cl_at<unsigned short>(cl_sm, L.o_pkc);
    const float *pv = cl_at<float>(cl_sm, L.o_pval), *xc = cl_at<float>(cl_sm, xo[l - 1]);
    const float *x = cl_at<float>(cl_sm, xo[l]);
    for (int base = r0; base < r1; base += kGroups)
    {
      const int r = base + grp, lr = r - r0;
      const bool in = r < r1;
      const float s = cl_row_sm(rp, kc, pv, xc, in ? lr : 0, lane4);
      if (in) bcast(xo[l], r, x[r] + c.damp * s);
    }
  };
  // ---- down ----
  for (int l = c.nl - 1; l >= 1; l--)
  {
    for (int k = 0; k < c.pre; k++)
    {
      sweep(l, k == 0);
      cl.sync();
    }
    defect(l);
    cl.sync();
    if (l >= 2)
    {
      restrict_to(l);
      cl.sync();
    }
  }
  // ---- level 0 on the first CTA: rhs = R d_1 on active rows (FP32, as the restriction
  // kernel writes it), then coarse_exact_kernel's steps, the result into every CTA's copy ----
  if (rank == 0)
  {
    const ClusterLevel &L1 = c.lev[1], &L = c.lev[0];
    double *b = cl_at<double>(cl_sm, c.o_b);
    const float *d1 = cl_at<float>(cl_sm, L1.o_def);
    const int warp = tid / 32, lane = tid % 32, nw = blockDim.x / 32;
    for (int i = warp; i < L.n; i += nw)
    {
      float v = 0.f;
      if (i < L.na)
        for (int j = __ldg(L1.r_rp + i) + lane; j < __ldg(L1.r_rp + i + 1); j += 32) v += __ldg(L1.r_val + j) * d1[__ldg(L1.r_kc + j)];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) b[i] = (double)v;
    }
    __syncthreads();
    for (int i = warp; i < L.na; i += nw)
    {
      double v = 0.0;
      for (int j = __ldg(c.dir_start0 + i) + lane; j < __ldg(L.rp + i + 1); j += 32) v += __ldg(c.a64 + j) * b[__ldg(L.kc + j)];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) b[L.n + i] = b[i] - v;
    }
    __syncthreads();
    for (int i = L.na + tid; i < L.n; i += blockDim.x)
      for (int k = 0; k < nb; k++) cl.map_shared_rank(cl_at<float>(cl_sm, xo[0]), k)[i] = (float)b[i];
    for (int r = warp; r < L.na; r += nw)
    {
      double s = 0;
      for (int j = lane; j < L.na; j += 32) s += __ldg(c.cinv + (size_t)r * L.na + j) * b[L.n + j];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane < nb) cl.map_shared_rank(cl_at<float>(cl_sm, xo[0]), lane)[r] = (float)s;
    }
  }
  cl.sync();
  // ---- up ----
  for (int l = 1; l < c.nl; l++)
  {
    prolong(l);
    cl.sync();
    for (int k = 0; k < c.post; k++)
    {
      sweep(l, false);
      cl.sync();
    }
  }
  // the top level's iterate back to global memory (this CTA's rows)
  {
    const ClusterLevel &L = c.lev[c.nl - 1];
    const int r0 = L.rb[rank], r1 = L.rb[rank + 1];
    const float *x = cl_at<float>(cl_sm, xo[c.nl - 1]);
    for (int r = r0 + tid; r < r1; r += blockDim.x) c.top_out[r] = x[r];
  }
  cl.sync();
}
