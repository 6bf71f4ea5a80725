// cdgpu_defect_noalloc: the defect d = f - A x and its norm, like cdgpu_defect, for callers
// that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code running while another allocator (a framework's
// caching allocator, a pre-sized memory arena) has reserved the whole device, or host code
// that must not pay for the implicit device synchronisation of cudaFree.  This entry point
// needs no allocation: the caller passes device vectors for x, f and d, and the per-block
// partial sums of ||d||^2 live in a fixed array of this library
// (kScratchBlocks doubles + 1 for the total, 32 KB) that every GPU which loads the library
// keeps until the process exits.
//
// The array is shared by every call on a device and keeps the last call's contents; each
// call writes every slot it reads, so nothing has to start at zero.  Calls that overlap on
// the GPU (two streams, two host threads, two contexts on one device) race on the array.
//
// Set-up: cdgpu_create looks up the array's device address with cudaGetSymbolAddress, with the
// context's device current, once per device (noalloc_prepare below); under lazy module loading
// that lookup is what loads this file's kernels and the array, so it happens while the context
// is made, before another allocator can have taken the device.  Should that lookup have failed,
// the entry point's first call on the device repeats it; that call should then come before any
// stream capture.
#include <mutex>

#include "internal.h"

namespace
{
constexpr int kScratchBlocks = 4096;      // partial sums, one per thread block
constexpr int kRowsPerBlock = 2048;       // rows per block -> at most 8,388,608 rows
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;
}

static __device__ __align__(256) double g_defect_scratch[kScratchBlocks + 1];

static std::mutex g_scratch_mutex;
static double *g_scratch_ptr[kMaxDevices] = {nullptr};

template <int GS>
__global__ void __launch_bounds__(kThreads) defect_noalloc_kernel(int n, const int *__restrict__ rp,
                                                                  const int *__restrict__ kc,
                                                                  const double *__restrict__ a,
                                                                  const double *__restrict__ x,
                                                                  const double *__restrict__ f,
                                                                  double *__restrict__ d,
                                                                  double *__restrict__ partial)
{
  __shared__ double red[kThreads / 32];
  const int lane = threadIdx.x % GS;
  const int row0 = blockIdx.x * kRowsPerBlock;
  const int row1 = min(n, row0 + kRowsPerBlock);
  double acc = 0;
  // the rows of this block, one GS-thread group per row; every lane of a warp runs the same
  // number of trips so the shuffles below always see the whole warp
  for (int base = row0 + (threadIdx.x / 32) * (32 / GS); base < row1; base += (kThreads / 32) * (32 / GS))
  {
    const int r = base + (threadIdx.x % 32) / GS;
    double s = 0;
    if (r < row1)
      for (int j = rp[r] + lane; j < rp[r + 1]; j += GS) s += a[j] * x[kc[j]];
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, GS);
    if (r < row1 && lane == 0)
    {
      double v = f[r] - s;
      d[r] = v;
      acc += v * v;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += red[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void noalloc_total_kernel(int nblocks, double *__restrict__ partial)
{
  __shared__ double red[kThreads / 32];
  double t = 0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) t += partial[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = t;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double s = 0;
    for (int w = 0; w < kThreads / 32; w++) s += red[w];
    partial[kScratchBlocks] = s;
  }
}

// the device address of the scratch array on `device` (the current device), looked up once
static cudaError_t noalloc_scratch(int device, double **out)
{
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[device])
  {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_defect_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = (double *)p;
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

// called by cdgpu_create with the context's device current; a failure is left for the entry
// point to report
void noalloc_prepare(int device)
{
  if (device < 0 || device >= kMaxDevices) return;
  double *p = nullptr;
  if (noalloc_scratch(device, &p) != cudaSuccess) cudaGetLastError();
}

extern "C" int cdgpu_defect_noalloc(cdgpu_ctx *ctx, int space_id, const double *d_x, const double *d_f,
                                    double *d_d, double *h_res)
{
  if (!ctx || space_id < 0 || space_id >= (int)ctx->spaces.size() || !d_x || !d_f || !d_d)
    return fail(ctx, CDGPU_ERR_INVALID, "defect_noalloc: bad argument");
  Space &s = *ctx->spaces[space_id];
  if (!s.assembled) return fail(ctx, CDGPU_ERR_INVALID, "defect_noalloc: matrix not assembled");
  const long max_rows = (long)kScratchBlocks * kRowsPerBlock;
  if (s.n_dof > max_rows)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED,
                "defect_noalloc: at most 8388608 rows (fixed scratch of 4096 partial sums); use cdgpu_defect");
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "defect_noalloc: device index beyond 63");
  CD_CUDA(ctx, cudaSetDevice(ctx->device));
  if (s.n_dof <= 0)
  {
    if (h_res) *h_res = 0.0;
    return CDGPU_OK; // no rows: nothing to launch
  }
  double *scratch = nullptr;
  cudaError_t e = noalloc_scratch(ctx->device, &scratch);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "defect_noalloc: cudaGetSymbolAddress");
  const int blocks = (s.n_dof + kRowsPerBlock - 1) / kRowsPerBlock;
  if (s.dim == 3 && s.order == 2)
    defect_noalloc_kernel<32><<<blocks, kThreads, 0, ctx->stream>>>(s.n_dof, s.d_row_ptr, s.d_kcol, s.d_a, d_x,
                                                                   d_f, d_d, scratch);
  else
    defect_noalloc_kernel<16><<<blocks, kThreads, 0, ctx->stream>>>(s.n_dof, s.d_row_ptr, s.d_kcol, s.d_a, d_x,
                                                                   d_f, d_d, scratch);
  CD_LAUNCHED(ctx);
  noalloc_total_kernel<<<1, kThreads, 0, ctx->stream>>>(blocks, scratch);
  CD_LAUNCHED(ctx);
  if (h_res)
  {
    double r2 = 0;
    CD_CUDA(ctx, cudaMemcpyAsync(&r2, scratch + kScratchBlocks, sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *h_res = sqrt(r2);
  }
  return CDGPU_OK;
}
