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
  CD_PDL_ENTRY();
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
  CD_PDL_ENTRY();
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

// ---------------------------------------------------------------------------
// The same per-cell products on the 5th-generation tensor cores (tcgen05, kind::tf32):
// for a tile of 128 cells, D[cell][t*32 + i] = sum_k X[cell][k] R_t[i][k] is one
// 128 x 32T x 32 product (K = 27 local DOFs padded to 32), A = the gathered cell values and
// B = the reference tensors, both K-major in shared memory in the no-swizzle core-matrix
// layout (8 rows x 16 bytes per core matrix), the accumulator in tensor memory (TMEM).  One
// thread issues 2 x 4 MMAs (two N halves of 16T columns, four K steps of 8) and commits them
// to an mbarrier; after the (bounded) wait each of the 4 warps reads its 32 TMEM lanes (one
// cell per thread) tensor by tensor with tcgen05.ld and contracts them with the cell's
// coefficients: y[i] = sum_t coef_t D[t*32 + i].  Inputs are rounded to TF32 (10-bit
// mantissa); only the FP32 multigrid cycle uses this operator.  Persistent CTAs, one per SM
// (TMEM: 512 columns per CTA).
__device__ __forceinline__ uint32_t mf_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of an R-row, K = 32 K-major operand in core-matrix layout
__device__ __forceinline__ int mf_core_off(int r, int k, int R)
{
  return (((k >> 2) * (R >> 3) + (r >> 3)) * 8 + (r & 7)) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ uint64_t mf_sdesc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46; // descriptor version of sm_100; layout type 0 = no swizzle
  return d;
}

// poll the mbarrier for completion of the given phase at most `limit` times; 1 when it completed
__device__ __forceinline__ uint32_t mf_wait_parity(uint64_t *mbar, uint32_t phase, long limit)
{
  uint32_t done = 0;
  for (long it = 0; it < limit && !done; it++)
    asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}"
                 : "=r"(done)
                 : "r"(mf_smem_u32(mbar)), "r"(phase)
                 : "memory");
  return done;
}

// bulk copy (cp.async.bulk, 1D TMA) of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) from global to shared memory, completing on mbarrier `bar`
__device__ __forceinline__ void mf_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   mf_smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(mf_smem_u32(bar))
               : "memory");
}

// dynamic shared memory of mf_cell27_tc_kernel<T>: A (128 x 32 floats), B (32T x 32 floats),
// two stages of a tile's GlobalNumbers (128 x 27 ints) and cell coefficients (128 x T floats)
template <int T> constexpr int mf_tc_gn_bytes() { return 128 * 27 * 4; }
template <int T> constexpr int mf_tc_cf_bytes() { return 128 * T * 4; }
template <int T> constexpr int mf_tc_smem_bytes()
{
  return 128 * 32 * 4 + 32 * T * 32 * 4 + 2 * (mf_tc_gn_bytes<T>() + mf_tc_cf_bytes<T>());
}

// the B operand of mf_cell27_tc_kernel as its shared-memory image (32T x 32 floats in the
// core-matrix layout, rows i >= 27 and columns k >= 27 zero), written once per assembly so
// that the kernel stages it with one bulk copy
__global__ void mf_tc_tensor_image_kernel(int T, const float *__restrict__ R32, float *__restrict__ img)
{
  CD_PDL_ENTRY();
  constexpr int KP = 32, NB = 27;
  const int N = 32 * T;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N * KP; e += gridDim.x * blockDim.x)
  {
    const int n = e / KP, k = e % KP, t = n / 32, i = n % 32;
    img[mf_core_off(n, k, N) / 4] = (i < NB && k < NB) ? R32[(t * NB + i) * NB + k] : 0.f;
  }
}

template <int T>
__global__ void __launch_bounds__(128, 1) mf_cell27_tc_kernel(int n_cells, const int *__restrict__ gn,
                                                              const float *__restrict__ cf32,
                                                              const float *__restrict__ Bimg,
                                                              const float *__restrict__ x, float *__restrict__ ybuf,
                                                              int *__restrict__ err, int pre)
{
  // with pre, the tensors, the shared-memory set-up and the bulk copies of the first two
  // tiles' DOF numbers and coefficients (written by no kernel of the cycle) come before the
  // wait for the predecessor
  if (!pre) CD_PDL_ENTRY();
  constexpr int MT = 128, KP = 32, NB = 27, N = 32 * T, NH = N / 2;
  extern __shared__ __align__(1024) unsigned char mf_sm[];
  unsigned char *As = mf_sm;                    // 128 x 32 x 4 = 16 KB
  unsigned char *Bs = mf_sm + MT * KP * 4;      // N x 32 x 4
  unsigned char *St = Bs + N * KP * 4;          // 2 stages of (GlobalNumbers, coefficients)
  constexpr int GB = mf_tc_gn_bytes<T>(), CB = mf_tc_cf_bytes<T>();
  __shared__ __align__(8) uint64_t mbar;
  __shared__ __align__(8) uint64_t sbar[2];
  __shared__ __align__(8) uint64_t bbar; // the B image's bulk copy
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int n_tiles = (n_cells + MT - 1) / MT;
  if (tid == 0)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mf_smem_u32(&mbar)), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mf_smem_u32(&sbar[0])), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mf_smem_u32(&sbar[1])), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mf_smem_u32(&bbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // the copies of a tile's numbers and coefficients: sizes rounded up to 16 bytes (the
  // GlobalNumbers array carries 4 spare ints, the coefficient array n_cells * (14 - T) spare
  // floats); only the tile's own cells are read back
  // per stage: copies issued (thread 0) and waits passed, as scalars (no local memory)
  int issued0 = 0, issued1 = 0, waited0 = 0, waited1 = 0;
  auto issue = [&](int tile, int stage) {
    if (stage) issued1++; else issued0++;
    const int c0 = tile * MT, nc = min(MT, n_cells - c0);
    const uint32_t gb = ((uint32_t)nc * NB * 4 + 15u) & ~15u, cb = ((uint32_t)nc * T * 4 + 15u) & ~15u;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mf_smem_u32(&sbar[stage])),
                 "r"(gb + cb)
                 : "memory");
    unsigned char *dst = St + stage * (GB + CB);
    mf_bulk_g2s(dst, gn + (size_t)c0 * NB, gb, &sbar[stage]);
    mf_bulk_g2s(dst + GB, cf32 + (size_t)c0 * T, cb, &sbar[stage]);
  };
  __syncthreads();
  if (tid == 0)
  {
    // B = the tensors' shared-memory image (N x 32 floats, a multiple of 16 bytes), one copy
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mf_smem_u32(&bbar)),
                 "r"((uint32_t)(N * KP * 4))
                 : "memory");
    mf_bulk_g2s(Bs, Bimg, (uint32_t)(N * KP * 4), &bbar);
    if (blockIdx.x < n_tiles) issue(blockIdx.x, 0);
    if (blockIdx.x + gridDim.x < n_tiles) issue(blockIdx.x + gridDim.x, 1);
  }
  // A: the padding columns k >= 27 zero once (every tile writes columns 0..26 of all 128 rows,
  // zeros for absent cells)
#pragma unroll
  for (int k = NB; k < KP; k++) *(float *)(As + mf_core_off(tid, k, MT)) = 0.f;
  if (pre) CD_PDL_ENTRY();
  if (warp == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(mf_smem_u32(&tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NH >> 3) << 17) | ((uint32_t)(MT >> 4) << 24);
  uint32_t phase = 0, pend_phase = 0;
  bool ok = true, pending = false;
  // the next tile's cell values and coefficients, one cell per thread (thread r gathers and
  // later contracts cell c0 + r), read from the staged copy of the tile's numbers and
  // coefficients; gathered before the current tile's products are awaited, so the gather
  // latency overlaps the tensor-core work and the epilogue.  li = the CTA's tile counter.
  float vn[NB], cn[T];
  auto gather = [&](int li) {
    const int tile = blockIdx.x + li * gridDim.x;
    const bool have = tile < n_tiles;
    const int stage = li & 1;
    bool ready = true;
    if (have && ok)
    {
      const uint32_t got = mf_wait_parity(&sbar[stage], (uint32_t)(li >> 1) & 1u, 1L << 24);
      ready = __syncthreads_and(got != 0) != 0;
      if (ready)
      {
        if (stage) waited1++; else waited0++;
      }
      else
      {
        if (tid == 0) atomicExch(err, 3);
        ok = false;
      }
    }
    const int c = tile * MT + tid;
    const bool in = have && ready && ok && c < n_cells;
    const int *gq = (const int *)(St + stage * (GB + CB));
    const float *cq = (const float *)(St + stage * (GB + CB) + GB);
#pragma unroll
    for (int k = 0; k < NB; k++) vn[k] = in ? __ldg(x + gq[tid * NB + k]) : 0.f;
#pragma unroll
    for (int t = 0; t < T; t++) cn[t] = in ? cq[tid * T + t] : 0.f;
  };
  gather(0);
  // the B image must have landed before the first product (bounded, CTA-uniform)
  bool b_in_flight = false;
  if (ok && !__syncthreads_and(mf_wait_parity(&bbar, 0u, 1L << 24) != 0))
  {
    if (tid == 0) atomicExch(err, 3);
    ok = false;
    b_in_flight = true;
  }
  int li = 0;
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, li++)
  {
    const int c0 = tile * MT;
    float cf[T];
#pragma unroll
    for (int t = 0; t < T; t++) cf[t] = cn[t];
#pragma unroll
    for (int k = 0; k < NB; k++) *(float *)(As + mf_core_off(tid, k, MT)) = vn[k];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // every thread has gathered this tile from stage li & 1 (before the barrier above): refill
    // the stage with the tile after next
    if (tid == 0 && ok && tile + 2 * gridDim.x < n_tiles) issue(tile + 2 * gridDim.x, li & 1);
    if (tid == 0 && ok)
    {
      const uint32_t a0 = mf_smem_u32(As), b0 = mf_smem_u32(Bs);
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int s = 0; s < KP / 8; s++)
        {
          const uint64_t da = mf_sdesc(a0 + s * 2 * (MT / 8) * 128, (MT / 8) * 128, 128);
          const uint64_t db = mf_sdesc(b0 + s * 2 * (N / 8) * 128 + h * (NH / 8) * 128, (N / 8) * 128, 128);
          const uint32_t acc = s > 0 ? 1u : 0u;
          asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                       "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + h * NH),
                       "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       mf_smem_u32(&mbar))
                   : "memory");
    }
    gather(li + 1);
    // bounded wait for this tile's products (an error flag instead of a hang); the outcome is
    // made CTA-uniform, so the warp-collective TMEM loads below run with every lane or none
    const uint32_t done = ok ? mf_wait_parity(&mbar, phase, 1L << 24) : 0u;
    const int all_done = __syncthreads_and(done != 0);
    if (ok && !all_done)
    {
      if (tid == 0) atomicExch(err, 3);
      ok = false;
      pending = true; // the committed products may still write TMEM
      pend_phase = phase;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int c = c0 + warp * 32 + lane;
    if (ok)
    {
      float y[NB];
#pragma unroll
      for (int i = 0; i < NB; i++) y[i] = 0.f;
      // two tensors (64 columns) per TMEM load, one wait per load
#pragma unroll
      for (int t = 0; t + 1 < T; t += 2)
      {
        uint32_t v[64];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + t * 32;
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                     "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,"
                     "%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,"
                     "%61,%62,%63}, [%64];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                       "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                       "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                       "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                       "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]),
                       "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]),
                       "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]),
                       "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]),
                       "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]),
                       "=r"(v[63])
                     : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const float c_a = cf[t], c_b = cf[t + 1];
#pragma unroll
        for (int i = 0; i < NB; i++) y[i] += c_a * __uint_as_float(v[i]);
#pragma unroll
        for (int i = 0; i < NB; i++) y[i] += c_b * __uint_as_float(v[32 + i]);
      }
      if (T % 2)
      {
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (T - 1) * 32;
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                     "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                       "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                       "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                       "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                       "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                     : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int i = 0; i < NB; i++) y[i] += cf[T - 1] * __uint_as_float(v[i]);
      }
      if (c < n_cells)
#pragma unroll
        for (int i = 0; i < NB; i++) ybuf[(size_t)i * n_cells + c] = y[i];
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  // after a timed-out wait, wait once more (bounded) for the products still in flight before
  // the accumulator columns are released, and for the staged copies still in flight before
  // the CTA's shared memory is given up
  if (pending)
  {
    const uint32_t late = tid == 0 ? mf_wait_parity(&mbar, pend_phase, 1L << 26) : 1u;
    __syncthreads_or(late == 0);
  }
  if (tid == 0)
  {
    // a copy still in flight (after a timeout): bounded wait for it
    if (issued0 > waited0) (void)mf_wait_parity(&sbar[0], (uint32_t)(issued0 - 1) & 1u, 1L << 24);
    if (issued1 > waited1) (void)mf_wait_parity(&sbar[1], (uint32_t)(issued1 - 1) & 1u, 1L << 24);
    if (b_in_flight) (void)mf_wait_parity(&bbar, 0u, 1L << 24);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

template <int T> inline size_t mf_tc_smem() { return (size_t)mf_tc_smem_bytes<T>(); }
// dynamic shared memory requested by every launch of the tensor-core kernel: more than either
// instance needs, so that a second CTA never shares an SM (each CTA allocates 512 TMEM columns)
constexpr int kMfTcSmem = 120 * 1024;
static_assert(mf_tc_smem_bytes<13>() <= kMfTcSmem && mf_tc_smem_bytes<10>() <= kMfTcSmem, "tensor-core kernel smem");

enum { MF_JACOBI = 0, MF_DEFECT = 1, MF_SPMV = 2 };

template <int NBF, int MODE>
__global__ void mf_row_kernel(int n, int na, int n_cells, const int *__restrict__ inc_ptr,
                              const int *__restrict__ inc, const float *__restrict__ ybuf,
                              const float *__restrict__ x, const float *__restrict__ f,
                              const float *__restrict__ diag, float *__restrict__ out, float omega, int pre)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  // the first 8 incidences (every DOF of a structured hexahedral or quadrilateral mesh) are
  // loaded at once, then added in ascending cell order; longer lists continue one by one.
  // With pre, the incidence list (written by no kernel of the cycle) is read before the wait.
  int b = 0, e = 0, ei[8];
  auto load_inc = [&]() {
    b = inc_ptr[r];
    e = inc_ptr[r + 1];
#pragma unroll
    for (int j = 0; j < 8; j++) ei[j] = b + j < e ? __ldg(inc + b + j) : -1;
  };
  if (pre && r < na) load_inc();
  CD_PDL_ENTRY();
  if (r >= na)
  {
    // Dirichlet rows are identity rows
    out[r] = MODE == MF_JACOBI ? f[r] : MODE == MF_DEFECT ? f[r] - x[r] : x[r];
    return;
  }
  if (!pre) load_inc();
  float yv[8];
#pragma unroll
  for (int j = 0; j < 8; j++)
  {
    const int K = ei[j] / NBF, li = ei[j] - K * NBF;
    yv[j] = ei[j] >= 0 ? __ldg(ybuf + (size_t)li * n_cells + K) : 0.f;
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (b + j < e) s += yv[j];
  for (int t = b + 8; t < e; t++)
  {
    const int K = inc[t] / NBF, li = inc[t] - K * NBF;
    s += ybuf[(size_t)li * n_cells + K];
  }
  out[r] = MODE == MF_JACOBI ? x[r] + omega * (f[r] - s) / diag[r] : MODE == MF_DEFECT ? f[r] - s : s;
}

// The DOF -> (cell, local index) incidence of every active row as up to 8 indices into the
// per-cell buffer, li * n_cells + cell, in ascending cell order and padded with -1: the row
// kernels then read one 32-byte record per row instead of the row's incidence pointers and,
// after them, its entries (one dependent load fewer).  Rows with more than 8 cells raise
// *overflow, and the space keeps the incidence lists.
__global__ void mf_inc8_kernel(int n_active, int nbf, int n_cells, const int *__restrict__ inc_ptr,
                               const int *__restrict__ inc, int *__restrict__ inc8, int *overflow)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_active) return;
  const int b = inc_ptr[r], e = inc_ptr[r + 1];
  if (e - b > 8) atomicExch(overflow, 1);
#pragma unroll
  for (int j = 0; j < 8; j++)
  {
    int v = -1;
    if (b + j < e)
    {
      const int t = inc[b + j], K = t / nbf, li = t - K * nbf;
      v = li * n_cells + K;
    }
    inc8[(size_t)r * 8 + j] = v;
  }
}

// mf_row_kernel with the 8-wide incidence records (same sums in the same order)
template <int MODE>
__global__ void mf_row8_kernel(int n, int na, const int *__restrict__ inc8, const float *__restrict__ ybuf,
                               const float *__restrict__ x, const float *__restrict__ f,
                               const float *__restrict__ diag, float *__restrict__ out, float omega, int pre)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  int4 i0 = make_int4(-1, -1, -1, -1), i1 = i0;
  if (pre && r < na)
  {
    i0 = __ldg((const int4 *)(inc8 + (size_t)r * 8));
    i1 = __ldg((const int4 *)(inc8 + (size_t)r * 8) + 1);
  }
  CD_PDL_ENTRY();
  if (r >= na)
  {
    // Dirichlet rows are identity rows
    out[r] = MODE == MF_JACOBI ? f[r] : MODE == MF_DEFECT ? f[r] - x[r] : x[r];
    return;
  }
  if (!pre)
  {
    i0 = __ldg((const int4 *)(inc8 + (size_t)r * 8));
    i1 = __ldg((const int4 *)(inc8 + (size_t)r * 8) + 1);
  }
  const int ix[8] = {i0.x, i0.y, i0.z, i0.w, i1.x, i1.y, i1.z, i1.w};
  float yv[8];
#pragma unroll
  for (int j = 0; j < 8; j++) yv[j] = ix[j] >= 0 ? __ldg(ybuf + ix[j]) : 0.f;
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (ix[j] >= 0) s += yv[j];
  out[r] = MODE == MF_JACOBI ? x[r] + omega * (f[r] - s) / diag[r] : MODE == MF_DEFECT ? f[r] - s : s;
}

// FP32 copies of the cell coefficients (first T of each cell's T + Tr) and of the tensors
// R[(i*nbf + j)*T + t] -> R32[(t*nbf + i)*nbf + j]
__global__ void mf_convert_kernel(int n_cells, int T, int Tr, int nbf, const double *__restrict__ cellcoef,
                                  const double *__restrict__ R, float *__restrict__ cf32, float *__restrict__ R32)
{
  CD_PDL_ENTRY();
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

// y = A x per cell (phase 1); tensor_cores = false keeps Q2 hexahedra on the CUDA-core kernel
inline void mf_apply_cells(cdgpu_ctx *ctx, const Space &s, const float *x, bool tensor_cores = true)
{
  if (s.nbf == 27 && ctx->d_err && tensor_cores)
  {
    // tensor cores: persistent CTAs, one per SM (the shared memory request keeps a second CTA
    // off the SM, so every CTA can allocate its 512 TMEM columns at once)
    const int grid = std::max(1, std::min((s.n_cells + 127) / 128, ctx->sm_count));
    if (s.mf_T == 10)
    {
      (void)cd_launch(mf_cell27_tc_kernel<10>, grid, 128, kMfTcSmem, ctx->stream, s.n_cells, s.d_gn, s.d_cf32,
                      s.d_R32img, x, s.d_ybuf, ctx->d_err, ctx->pdl_pre ? 1 : 0);
      return;
    }
    if (s.mf_T == 13)
    {
      (void)cd_launch(mf_cell27_tc_kernel<13>, grid, 128, kMfTcSmem, ctx->stream, s.n_cells, s.d_gn, s.d_cf32,
                      s.d_R32img, x, s.d_ybuf, ctx->d_err, ctx->pdl_pre ? 1 : 0);
      return;
    }
  }
  if (s.nbf == 27)
  {
    const int g27 = (s.n_cells + 63) / 64;
    if (s.mf_T == 10) { (void)cd_launch(mf_cell27_kernel<10>, g27, 224, 0, ctx->stream, s.n_cells, s.d_gn, s.d_cf32, s.d_R32, x, s.d_ybuf); return; }
    if (s.mf_T == 13) { (void)cd_launch(mf_cell27_kernel<13>, g27, 224, 0, ctx->stream, s.n_cells, s.d_gn, s.d_cf32, s.d_R32, x, s.d_ybuf); return; }
  }
  const int grid = (s.n_cells + 127) / 128;
#define CD_MF_CASE(NB, TT)                                                                              \
  if (s.nbf == NB && s.mf_T == TT)                                                                      \
  {                                                                                                     \
    (void)cd_launch(mf_cell_kernel<NB, TT>, grid, 128, 0, ctx->stream, s.n_cells, s.d_gn, s.d_cf32, s.d_R32, x, s.d_ybuf); \
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
  if (s.d_inc8)
  {
    (void)cd_launch(mf_row8_kernel<MODE>, grid, 256, 0, ctx->stream, s.n_dof, s.n_active, (const int *)s.d_inc8,
                    (const float *)s.d_ybuf, x, f, diag, out, omega, ctx->pdl_pre ? 1 : 0);
    return;
  }
  switch (s.nbf)
  {
    case 27: (void)cd_launch(mf_row_kernel<27, MODE>, grid, 256, 0, ctx->stream, s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega, ctx->pdl_pre ? 1 : 0); break;
    case 9: (void)cd_launch(mf_row_kernel<9, MODE>, grid, 256, 0, ctx->stream, s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega, ctx->pdl_pre ? 1 : 0); break;
    case 8: (void)cd_launch(mf_row_kernel<8, MODE>, grid, 256, 0, ctx->stream, s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega, ctx->pdl_pre ? 1 : 0); break;
    default: (void)cd_launch(mf_row_kernel<4, MODE>, grid, 256, 0, ctx->stream, s.n_dof, s.n_active, s.n_cells, s.d_inc_ptr, s.d_inc, s.d_ybuf, x, f, diag, out, omega, ctx->pdl_pre ? 1 : 0); break;
  }
}
