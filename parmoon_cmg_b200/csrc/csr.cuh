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

// ---------------------------------------------------------------------------
// FP64 CSR product / defect / Jacobi sweep with the matrix streamed into shared memory by the
// bulk-copy engine (TMA, cp.async.bulk) for matrices too large for L2 (the finest level).
//
// The rows are cut once per pattern into tiles of at most kTmaRows rows and kTmaCap nonzeros
// (CsrTiles, built on the host).  A persistent CTA takes tiles b, b + G, b + 2G, ...; one
// producer thread copies each tile's row pointers, column indices and values into one of
// kTmaStages shared-memory stages (three bulk copies completing on the stage's "full"
// mbarrier), running up to kTmaStages - 1 tiles ahead; kTmaWarps consumer warps take 8 rows
// each (4 threads per row), gather x, reduce, run the epilogue of csr_kernel, and release the
// stage on its "empty" mbarrier.  The DRAM stream is the bulk copies alone, so it no longer
// waits on the gathers' dependent loads.  A bulk copy must start on a 16-byte boundary and
// move a multiple of 16 bytes: each copy starts at the tile's first element rounded down to a
// multiple of 4 elements and ends rounded up (the arrays are allocated 8 elements longer).
// Every mbarrier wait is bounded; on a timeout the kernel sets err = 4, stops, waits (bounded)
// for the copies it issued and returns.
// ---------------------------------------------------------------------------
// CAP (nonzeros per tile) and STAGES are template parameters: the variants a tile-shape
// autotuner chooses from per matrix (solve.cu, tune_tma); kTmaRows = 8 consumer warps x 8 rows
constexpr int kTmaRows = 64, kTmaWarps = 8;
constexpr int kTmaRpBytes = ((kTmaRows + 1 + 8) * 4 + 127) / 128 * 128;
__host__ __device__ constexpr int tma_vals_bytes(int cap) { return (cap + 8) * 8; }
__host__ __device__ constexpr int tma_cols_bytes(int cap) { return (cap + 8) * 4; }
__host__ __device__ constexpr int tma_stage_bytes(int cap) { return tma_vals_bytes(cap) + tma_cols_bytes(cap) + kTmaRpBytes; }
__host__ __device__ constexpr int tma_smem_bytes(int cap, int stages) { return stages * tma_stage_bytes(cap) + 256; }
constexpr long kTmaSpin = 1L << 22; // polls of one wait before it is declared timed out

__device__ __forceinline__ uint32_t tma_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool tma_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t done;
  asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
               "selp.b32 %0, 1, 0, P1;\n\t}"
               : "=r"(done)
               : "r"(tma_smem_u32(bar)), "r"(parity)
               : "memory");
  return done != 0;
}

// bounded wait; gives up early once another thread of the CTA has aborted
__device__ __forceinline__ bool tma_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag)
{
  for (long it = 0; it < kTmaSpin; it++)
  {
    if (tma_try_wait(bar, parity)) return true;
    if ((it & 255) == 255 && *abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tma_smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(tma_smem_u32(bar))
               : "memory");
}

struct TmaMeta
{
  int rb, re, rb0, nb0; // rows [rb, re); row-pointer and nonzero copies start at rb0, nb0
};

// TPR threads per row (4: 64-row tiles, 16 gathers per thread and round; 8: 32-row tiles,
// 8 gathers per thread and round -- the same 64 entries of a row in flight per round)
template <int MODE, int CAP, int STAGES, int TPR = 4>
__global__ void __launch_bounds__((kTmaWarps + 1) * 32) csr_tma_kernel(CsrArgs<double> p, const int2 *__restrict__ tiles,
                                                                         int n_tiles, int *__restrict__ err)
{
  constexpr int kTmaStages = STAGES, kTmaCap = CAP;
  constexpr int kTmaValsBytes = tma_vals_bytes(CAP), kTmaColsBytes = tma_cols_bytes(CAP);
  constexpr int kTmaStageBytes = tma_stage_bytes(CAP);
  static_assert(kTmaValsBytes % 16 == 0 && kTmaColsBytes % 16 == 0 && kTmaStageBytes % 16 == 0,
                "bulk-copy destinations must stay 16-byte aligned");
  (void)kTmaCap;
  extern __shared__ __align__(128) unsigned char tma_sm[];
  __shared__ __align__(8) uint64_t full[kTmaStages], empty[kTmaStages];
  __shared__ TmaMeta meta[kTmaStages];
  __shared__ int abort_s;
  __shared__ double red[kTmaWarps];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int G = gridDim.x;
  const int my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / G + 1 : 0;
  if (threadIdx.x == 0)
  {
    for (int s = 0; s < kTmaStages; s++)
    {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tma_smem_u32(&full[s])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tma_smem_u32(&empty[s])), "r"(kTmaWarps));
    }
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto stage_vals = [&](int s) { return (double *)(tma_sm + (size_t)s * kTmaStageBytes); };
  auto stage_cols = [&](int s) { return (int *)(tma_sm + (size_t)s * kTmaStageBytes + kTmaValsBytes); };
  auto stage_rp = [&](int s) { return (int *)(tma_sm + (size_t)s * kTmaStageBytes + kTmaValsBytes + kTmaColsBytes); };
  double acc = 0;
  if (warp == kTmaWarps)
  {
    // producer: one thread issues the copies of this CTA's tiles
    if (lane == 0)
    {
      // the matrix is written by no kernel of a solve; with p.pre the first stages are issued
      // before the wait for the predecessor (whose output x is only gathered by the consumers)
      if (!p.pre) CD_PDL_WAIT();
      int issued = 0;
      for (int k = 0; k < my_tiles; k++)
      {
        const int s = k % kTmaStages, f = k / kTmaStages;
        if (f > 0 && !tma_wait(&empty[s], (f - 1) & 1, &abort_s))
        {
          atomicExch(err, 4);
          abort_s = 1;
          break;
        }
        if (*(volatile int *)&abort_s) break;
        const int t = blockIdx.x + k * G;
        const int2 a = tiles[t], b = tiles[t + 1];
        TmaMeta m;
        m.rb = a.x;
        m.re = b.x;
        m.rb0 = a.x & ~3;
        m.nb0 = a.y & ~3;
        const int rp_n = ((b.x + 1 + 3) & ~3) - m.rb0; // row pointers rb0 .. re, rounded up
        const int nz_n = ((b.y + 3) & ~3) - m.nb0;     // nonzeros nb0 .. ne, rounded up
        meta[s] = m;
        const uint32_t bytes = (uint32_t)(rp_n * 4 + nz_n * 12);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_smem_u32(&full[s])), "r"(bytes)
                     : "memory");
        tma_bulk_g2s(stage_rp(s), p.rp + m.rb0, rp_n * 4, &full[s]);
        tma_bulk_g2s(stage_cols(s), p.kc + m.nb0, nz_n * 4, &full[s]);
        tma_bulk_g2s(stage_vals(s), p.a + m.nb0, nz_n * 8, &full[s]);
        issued = k + 1;
        if (k == kTmaStages - 1 && p.pre) CD_PDL_WAIT();
      }
      if (p.pre && issued < kTmaStages) CD_PDL_WAIT();
      CD_PDL_TRIGGER();
      // no copy may still be in flight when the CTA exits: wait (bounded) for the last fill of
      // every stage (returns at once for fills the consumers have already seen)
      for (int s = 0; s < kTmaStages && s < issued; s++)
      {
        const int k_last = s + ((issued - 1 - s) / kTmaStages) * kTmaStages;
        for (long it = 0; it < kTmaSpin && !tma_try_wait(&full[s], (k_last / kTmaStages) & 1); it++)
          ;
      }
    }
  }
  else
  {
    CD_PDL_WAIT(); // x (and, in the Jacobi sweep, f) are read only after the predecessor completed
    constexpr int G = 64 / TPR, RW = 32 / TPR; // gathers per thread and round, rows per warp
    const int g = lane / TPR, lt = lane % TPR;
    for (int k = 0; k < my_tiles; k++)
    {
      const int s = k % kTmaStages, f = k / kTmaStages;
      // every lane waits (each needs the acquire of the stage's data); the outcome is made
      // warp-uniform, so a timeout never leaves part of the warp before the shuffles below
      const bool arrived = tma_wait(&full[s], f & 1, &abort_s);
      if (!__all_sync(0xffffffffu, arrived))
      {
        if (lane == 0)
        {
          atomicExch(err, 4);
          abort_s = 1;
        }
        break;
      }
      const TmaMeta m = meta[s];
      const double *va = stage_vals(s);
      const int *co = stage_cols(s), *rs = stage_rp(s);
      const int r = m.rb + warp * RW + g;
      double sum = 0;
      if (r < m.re)
      {
        const int jb = rs[r - m.rb0] - m.nb0, je = rs[r + 1 - m.rb0] - m.nb0;
        // G entries per thread at once: every gather of a row of up to 64 entries is in
        // flight together (longer rows take a second round)
        for (int j0 = jb + lt; j0 < je; j0 += 64)
        {
          int c[G];
#pragma unroll
          for (int u = 0; u < G; u++)
          {
            const int j = j0 + TPR * u;
            c[u] = j < je ? co[j] : -1;
          }
          // the G gathers are issued in order before the first product (positions beyond
          // the row read x[0] and are multiplied by nothing)
          double xv[G];
#pragma unroll
          for (int u = 0; u < G; u++)
            asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(xv[u]) : "l"(p.x + (c[u] >= 0 ? c[u] : 0)));
          // all G values pass through this point before any product uses one, so the compiler
          // cannot put a product (and its wait) between two gathers
          if constexpr (G == 16)
            asm volatile("" : "+d"(xv[0]), "+d"(xv[1]), "+d"(xv[2]), "+d"(xv[3]), "+d"(xv[4]), "+d"(xv[5]),
                         "+d"(xv[6]), "+d"(xv[7]), "+d"(xv[8]), "+d"(xv[9]), "+d"(xv[10]), "+d"(xv[11]), "+d"(xv[12]),
                         "+d"(xv[13]), "+d"(xv[14]), "+d"(xv[15]));
          else
            asm volatile("" : "+d"(xv[0]), "+d"(xv[1]), "+d"(xv[2]), "+d"(xv[3]), "+d"(xv[4]), "+d"(xv[5]),
                         "+d"(xv[6]), "+d"(xv[7]));
#pragma unroll
          for (int u = 0; u < G; u++)
          {
            const int j = j0 + TPR * u;
            if (j < je) sum += va[j] * xv[u];
          }
        }
      }
      sum = csr_group_sum<TPR>(sum);
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tma_smem_u32(&empty[s])) : "memory");
      if (r < m.re && lt == 0) csr_epilogue<double, MODE>(p, r, sum, acc);
    }
  }
  if (MODE == CM_DEFECT && p.partial)
  {
    if (warp < kTmaWarps)
    {
      acc = csr_group_sum<32>(acc);
      if (lane == 0) red[warp] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
      double tot = 0;
      for (int w = 0; w < kTmaWarps; w++) tot += red[w];
      p.partial[blockIdx.x] = tot;
    }
  }
}
