// CSR pattern construction on the device (TSquareStructure3D/2D(TFESpace*) + Sort,
// src/FE/SquareStructure3D.C:32, SquareStructure2D.C:46, SquareStructure.C:65).
//
// The same pattern as the host's build_pattern, bit for bit: an active row couples to every
// DOF of every cell that contains the row's DOF (Dirichlet columns included), columns sorted
// ascending without repeats; a Dirichlet row holds its diagonal only.  One warp per row:
// the candidate columns (the row's incident cells' DOF numbers, from the DOF -> cell
// incidence of upload_space) go to shared memory, a bitonic sort orders them and a ballot
// keeps the first of each run of equal values.  A counting pass gives the row lengths, an
// exclusive scan the row pointers, and a second pass writes the columns.  Rows with more than
// kPatMaxCand candidates (meshes with very many cells around one DOF) are left to the host
// build (the caller falls back).
#include <climits>

#include "internal.h"

namespace
{
constexpr int kPatMaxCand = 512; // per row; a Q2 hexahedron's row has 8 x 27 = 216
constexpr int kPatWarps = 8;
constexpr int kScanBlock = 1024;

enum { PAT_COUNT = 0, PAT_WRITE = 1 };

template <int MODE>
__global__ void __launch_bounds__(kPatWarps * 32) pattern_rows_kernel(int n_dof, int n_active, int nbf,
                                                                     const int *__restrict__ gn,
                                                                     const int *__restrict__ inc_ptr,
                                                                     const int *__restrict__ inc,
                                                                     const int *__restrict__ row_ptr,
                                                                     int *__restrict__ counts, int *__restrict__ kcol,
                                                                     int *__restrict__ overflow)
{
  CD_PDL_ENTRY();
  __shared__ int buf[kPatWarps][kPatMaxCand];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  int *b = buf[warp];
  for (int r = blockIdx.x * kPatWarps + warp; r < n_dof; r += gridDim.x * kPatWarps)
  {
    if (r >= n_active)
    {
      if (lane == 0)
      {
        if (MODE == PAT_COUNT) counts[r] = 1;
        else kcol[row_ptr[r]] = r;
      }
      continue;
    }
    const int ib = inc_ptr[r], ie = inc_ptr[r + 1];
    const int ncand = (ie - ib) * nbf;
    if (ncand > kPatMaxCand)
    {
      if (lane == 0) atomicExch(overflow, 1);
      continue; // warp-uniform
    }
    int P = 32;
    while (P < ncand) P <<= 1;
    for (int i = lane; i < P; i += 32)
    {
      int v = INT_MAX;
      if (i < ncand)
      {
        const int t = inc[ib + i / nbf] / nbf; // incident cell
        v = gn[(size_t)t * nbf + i % nbf];
      }
      b[i] = v;
    }
    __syncwarp();
    // bitonic sort of b[0, P) ascending
    for (int k = 2; k <= P; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1)
      {
        for (int i = lane; i < P; i += 32)
        {
          const int l = i ^ j;
          if (l > i)
          {
            const int a = b[i], c = b[l];
            const bool up = (i & k) == 0;
            if ((a > c) == up)
            {
              b[i] = c;
              b[l] = a;
            }
          }
        }
        __syncwarp();
      }
    // first element of every run of equal values
    int total = 0;
    const int base_out = MODE == PAT_WRITE ? row_ptr[r] : 0;
    for (int i0 = 0; i0 < P; i0 += 32)
    {
      const int i = i0 + lane;
      const int v = b[i];
      const bool keep = v != INT_MAX && (i == 0 || b[i - 1] != v);
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (MODE == PAT_WRITE && keep) kcol[base_out + total + __popc(m & ((1u << lane) - 1u))] = v;
      total += __popc(m);
    }
    if (MODE == PAT_COUNT && lane == 0) counts[r] = total;
    __syncwarp();
  }
}

// exclusive scan of in[0, n) into out[0, n], out[n] = total: per-block scans, a scan of the
// block totals by one block, then the block offsets added
__device__ __forceinline__ int warp_incl_scan(int v)
{
  const int lane = threadIdx.x % 32;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
  {
    const int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__global__ void __launch_bounds__(kScanBlock) scan_blocks_kernel(int n, const int *__restrict__ in, int *__restrict__ out,
                                                                 int *__restrict__ block_sum)
{
  CD_PDL_ENTRY();
  __shared__ int ws[kScanBlock / 32];
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  const int v = i < n ? in[i] : 0;
  int s = warp_incl_scan(v);
  if (threadIdx.x % 32 == 31) ws[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x < 32)
  {
    int w = ws[threadIdx.x];
    w = warp_incl_scan(w);
    ws[threadIdx.x] = w;
  }
  __syncthreads();
  if (threadIdx.x >= 32) s += ws[threadIdx.x / 32 - 1];
  if (i < n) out[i] = s - v; // exclusive within the block
  if (threadIdx.x == kScanBlock - 1) block_sum[blockIdx.x] = s;
}

// one block: exclusive scan of the block totals in place, the grand total to out_total
__global__ void __launch_bounds__(kScanBlock) scan_totals_kernel(int nb, int *__restrict__ block_sum, int *__restrict__ out_total)
{
  CD_PDL_ENTRY();
  __shared__ int ws[kScanBlock / 32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kScanBlock)
  {
    const int i = base + threadIdx.x;
    const int v = i < nb ? block_sum[i] : 0;
    int s = warp_incl_scan(v);
    if (threadIdx.x % 32 == 31) ws[threadIdx.x / 32] = s;
    __syncthreads();
    if (threadIdx.x < 32)
    {
      int w = ws[threadIdx.x];
      w = warp_incl_scan(w);
      ws[threadIdx.x] = w;
    }
    __syncthreads();
    if (threadIdx.x >= 32) s += ws[threadIdx.x / 32 - 1];
    const int c = carry;
    if (i < nb) block_sum[i] = c + s - v;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry = c + s;
    __syncthreads();
  }
  if (threadIdx.x == 0) *out_total = carry;
}

__global__ void scan_add_kernel(int n, const int *__restrict__ block_sum, int *__restrict__ out)
{
  CD_PDL_ENTRY();
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += block_sum[blockIdx.x];
}
} // namespace

// The pattern of space s built on the device: fills s.h_row_ptr and s.h_kcol (copied back for
// the host-side users of the pattern) and returns the device column array (nnz + kCsrPad
// entries) in *d_kcol_out.  *fallback = true (and nothing built) when a row has more
// candidates than the kernel's buffer.
int build_pattern_device(cdgpu_ctx *ctx, Space &s, int **d_kcol_out, bool *fallback)
{
  *fallback = false;
  *d_kcol_out = nullptr;
  const int n = s.n_dof;
  const int nb = (n + kScanBlock - 1) / kScanBlock;
  int *d_counts = nullptr, *d_rp = nullptr, *d_bsum = nullptr, *d_flag = nullptr, *d_kcol = nullptr;
  int rc;
  auto release = [&]() {
    for (int *p : {d_counts, d_rp, d_bsum, d_flag})
      if (p) cudaFree(p);
  };
  if ((rc = dev_alloc(ctx, &d_counts, n)) || (rc = dev_alloc(ctx, &d_rp, n + 1 + kCsrPad)) ||
      (rc = dev_alloc(ctx, &d_bsum, nb)) || (rc = dev_alloc(ctx, &d_flag, 1)))
  {
    release();
    return rc;
  }
  CD_CUDA(ctx, cudaMemsetAsync(d_flag, 0, sizeof(int), ctx->stream));
  const int grid = std::max(1, std::min((n + kPatWarps - 1) / kPatWarps, ctx->sm_count * 8));
  (void)cd_launch(pattern_rows_kernel<PAT_COUNT>, grid, kPatWarps * 32, 0, ctx->stream, n, s.n_active, s.nbf,
                  (const int *)s.d_gn, (const int *)s.d_inc_ptr, (const int *)s.d_inc, (const int *)nullptr,
                  d_counts, (int *)nullptr, d_flag);
  CD_LAUNCHED(ctx);
  (void)cd_launch(scan_blocks_kernel, nb, kScanBlock, 0, ctx->stream, n, (const int *)d_counts, d_rp, d_bsum);
  CD_LAUNCHED(ctx);
  (void)cd_launch(scan_totals_kernel, 1, kScanBlock, 0, ctx->stream, nb, d_bsum, d_rp + n);
  CD_LAUNCHED(ctx);
  (void)cd_launch(scan_add_kernel, nb, kScanBlock, 0, ctx->stream, n, (const int *)d_bsum, d_rp);
  CD_LAUNCHED(ctx);
  int flag = 0, nnz = 0;
  CD_CUDA(ctx, cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaMemcpyAsync(&nnz, d_rp + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (flag)
  {
    release();
    *fallback = true;
    return CDGPU_OK;
  }
  if ((rc = dev_alloc(ctx, &d_kcol, (size_t)nnz + kCsrPad)))
  {
    release();
    return rc;
  }
  (void)cd_launch(pattern_rows_kernel<PAT_WRITE>, grid, kPatWarps * 32, 0, ctx->stream, n, s.n_active, s.nbf,
                  (const int *)s.d_gn, (const int *)s.d_inc_ptr, (const int *)s.d_inc, (const int *)d_rp,
                  (int *)nullptr, d_kcol, d_flag);
  CD_LAUNCHED(ctx);
  s.h_row_ptr.resize(n + 1);
  s.h_kcol.resize(nnz);
  cudaError_t e = cudaMemcpyAsync(s.h_row_ptr.data(), d_rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.h_kcol.data(), d_kcol, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  release();
  if (e != cudaSuccess)
  {
    cudaFree(d_kcol);
    return cuda_fail(ctx, e, "build_pattern_device");
  }
  *d_kcol_out = d_kcol;
  return CDGPU_OK;
}
