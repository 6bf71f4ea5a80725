// Batched GMG-FGMRES: many independent convection-diffusion solves advanced together.
//
// Every kernel of an FGMRES iteration is one grouped launch over all running instances: a
// launch gets a table of (instance slot, first virtual block) pairs, and each virtual
// block finds its instance by binary search and works on a fixed row range of that
// instance's level.  Blocks loop over virtual blocks (grid <= 8 blocks per SM), so one
// launch covers any number of instances of any sizes.  The FGMRES control -- Gram-Schmidt
// coefficients, Givens rotations, stopping and divergence tests, restarts -- lives in a
// per-instance device control block (BCtl) and is updated by per-instance threads, so the
// host never waits on an instance: it launches iterations and polls a state array.
//
// Per instance the algorithm is the mixed form of cdgpu_solve: FGMRES(m) in FP64 on the
// finest level (TFgmresIte::Iterate, FgmresIte.C:219-582, classical Gram-Schmidt applied
// twice), preconditioned by one FP32 multigrid V-cycle (TMultiGrid3D::Cycle,
// MultiGrid3D.C:423-669; zero start and Dirichlet nodes as TMultiGridScaIte::Iterate,
// MultiGridScaIte.C:63-104) with the exact FP64 coarse solve on the active block.
// Smoothers: damped Jacobi (MGLevel3D.C:443-537), or SOR / SSOR sweeping the rows colour
// class by colour class of a greedy colouring (rows of one class share no matrix entry, so
// a class is updated in parallel with the Gauss-Seidel values of the earlier classes).
//
// Levels are addressed by depth below the finest level (depth 0 = finest) so that
// instances with different numbers of levels share every launch; an instance's coarsest
// depth gets the exact solve while deeper instances smooth and restrict.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace
{
constexpr int kMaxDepth = 12;
constexpr int kNT = 256;
constexpr int kCsrRows = 64;  // rows per virtual block of the CSR kernels (4 threads per row)
constexpr int kVecRows = 256; // rows per virtual block of the vector kernels
constexpr int kMaxM = 32;
constexpr int kSlots = 33;

enum { ST_EMPTY = 0, ST_RUN = 1, ST_DONE = 2 };
enum { A_START = 1, A_SCALE0 = 2, A_STEP = 3, A_NEXT = 4, A_UPD_DONE = 5, A_UPD_RESTART = 6 };
} // namespace

// one level of one instance, as the kernels see it
struct BLevel
{
  int n = 0, na = 0, nc = 0, nca = 0; // rows, active rows; coarser level rows, active rows
  const int *rp = nullptr, *kc = nullptr, *dirst = nullptr;
  const int *color_rows = nullptr;
  const float *a32 = nullptr, *d32 = nullptr;
  const double *a64 = nullptr;
  float *v[2] = {nullptr, nullptr};
  float *rhs = nullptr, *def = nullptr;
  const int *prp = nullptr, *pkc = nullptr; // P: rows of this level, columns of the coarser
  const float *pv = nullptr;
  const int *rrp = nullptr, *rkc = nullptr; // R = P^T: rows of the coarser level
  const float *rv = nullptr;
  const double *cinv = nullptr; // coarsest depth: inverse of the active block
};

// FGMRES control block of one instance
struct BCtl
{
  int state, action, j, its;
  int n, m, status, last; // last = index of the last basis vector in the update
  double beta, res, res0, tol, hn;
  double *V, *Z, *w, *x, *b, *H;
  const int *rp, *kc;
  const double *a64;
  double cs[kMaxM], sn[kMaxM], s[kMaxM + 1], y[kMaxM];
  double dots1[kSlots], dots2[kSlots], nrm2;
  // time-dependent instances: K = M - tau theta2 A (finest), f = (f, phi), c3/c4 = tau theta3/4
  int tcd, na;
  double c3, c4;
  const double *K, *f;
};

// a grouped launch: items (slots) and the prefix sums of their virtual blocks
struct BTab
{
  int K = 0, total = 0;
  const int *item = nullptr, *bstart = nullptr;
};

struct BInst
{
  bool used = false;
  int mg = -1, L = 0, state = ST_EMPTY;
  bool reported = false, tcd = false;
  size_t bytes = 0;
  std::vector<void *> allocs;
  // one allocation per instance, carved by balloc into its arrays (256-byte aligned); arrays
  // that do not fit get their own allocation
  char *arena = nullptr;
  size_t arena_off = 0, arena_size = 0;
};

struct Batch
{
  cdgpu_solver_params p{};
  int m = 30;
  std::vector<BInst> inst;
  int cap = 0;
  BCtl *d_ctl = nullptr;
  BLevel *d_lev = nullptr;
  int *d_state = nullptr, *h_state = nullptr; // compact copies of ctl.state for polling
  double *d_partial = nullptr;
  size_t partial_cap = 0;
  int *d_tab = nullptr;
  size_t tab_cap = 0;
  bool dirty = true, check_pending = false;
  std::vector<int> done_queue;
  size_t bytes = 0;
  // tables of the current running set
  std::vector<int> run;
  int depth = 0;
  BTab fine_vec, fine_csr, items;
  BTab tcd_csr, tcd_items; // every time-dependent instance, running or idle
  cudaGraphExec_t tcd_graph = nullptr;
  int tcd_graph_k = 0;
  bool tcd_looped = false; // tcd_graph ends in the device-side iteration loop
  // the device-side iteration loop: one graph whose WHILE node runs FGMRES iterations of the
  // running set until every solve has finished or the call's iteration budget is spent
  cudaGraphExec_t loop_graph = nullptr;
  int *d_loop = nullptr;        // iterations left in the current call
  int loop_mode = -1;           // -1 not tried, 0 host loop, 1 graph with PDL, 2 graph without
  long long loop_launches = 0, host_iterations = 0;
  std::vector<BTab> smooth, restrict_, coarse;
  std::vector<std::vector<BTab>> color;
  std::vector<int> ncolor_max;
};

static int free_inst(cdgpu_ctx *ctx, BInst &in)
{
  for (void *p : in.allocs) cudaFreeAsync(p, ctx->stream);
  in.allocs.clear();
  in.used = false;
  in.state = ST_EMPTY;
  return CDGPU_OK;
}

void free_batch(Batch *b)
{
  if (!b) return;
  for (auto &in : b->inst)
    for (void *p : in.allocs) cudaFree(p);
  if (b->tcd_graph) cudaGraphExecDestroy(b->tcd_graph);
  if (b->loop_graph) cudaGraphExecDestroy(b->loop_graph);
  void *ptrs[] = {b->d_ctl, b->d_lev, b->d_state, b->d_partial, b->d_tab, b->d_loop};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (b->h_state) cudaFreeHost(b->h_state);
  delete b;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int find_item(const BTab &t, int vb)
{
  int lo = 0, hi = t.K - 1;
  while (lo < hi)
  {
    int mid = (lo + hi + 1) >> 1;
    if (t.bstart[mid] <= vb) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int G, typename T> __device__ __forceinline__ T bsum(T v)
{
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
  return v;
}

// row r of a CSR matrix times x, 4 threads per row (8 predicated loads each + tail)
template <typename TA, typename TX>
__device__ __forceinline__ TX row4(const int *__restrict__ rp, const int *__restrict__ kc, const TA *__restrict__ a,
                                   const TX *__restrict__ x, int r, bool valid, int lane)
{
  TX s = 0;
  if (valid)
  {
    const int b = rp[r], e = rp[r + 1];
    int c[8];
    TA v[8];
#pragma unroll
    for (int i = 0; i < 8; i++)
    {
      const int j = b + lane + 4 * i;
      c[i] = j < e ? kc[j] : -1;
      v[i] = j < e ? a[j] : TA(0);
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
      if (c[i] >= 0) s += (TX)v[i] * x[c[i]];
    for (int j = b + lane + 32; j < e; j += 4) s += (TX)a[j] * x[kc[j]];
  }
  return bsum<4>(s);
}

__device__ __forceinline__ bool stepping(const BCtl &c) { return c.state == ST_RUN && c.action == A_STEP; }

// ---------------------------------------------------------------------------
// multigrid kernels (FP32)
// ---------------------------------------------------------------------------
// zero start + Dirichlet nodes on depth 0 from the current basis vector V_j
__global__ void b_mg_start(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev)
{
  CD_PDL_ENTRY();
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    const BCtl &c = ctl[slot];
    if (!stepping(c)) continue;
    const BLevel &L = lev[slot * kMaxDepth];
    const int r = (vb - t.bstart[k]) * kVecRows + threadIdx.x;
    if (r >= L.n) continue;
    const float v = (float)c.V[(size_t)c.j * c.n + r];
    L.rhs[r] = v;
    L.v[0][r] = r < L.na ? 0.f : v;
  }
}

// damped Jacobi sweep v[1-src] = v[src] + omega D^{-1} (f - A v[src]); first = active part
// of v[src] is zero, so only Dirichlet columns (from dirst) contribute
__global__ void b_jacobi(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev, int depth, int src,
                         int first, float omega)
{
  CD_PDL_ENTRY();
  const int lane = threadIdx.x % 4;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    if (!stepping(ctl[slot])) continue;
    const BLevel &L = lev[slot * kMaxDepth + depth];
    const int r = (vb - t.bstart[k]) * kCsrRows + threadIdx.x / 4;
    const bool valid = r < L.n;
    const float *x = L.v[src];
    float *y = L.v[1 - src];
    if (first)
    {
      if (valid && lane == 0)
      {
        if (r >= L.na) y[r] = L.rhs[r];
        else
        {
          float s = L.rhs[r];
          for (int j = L.dirst[r]; j < L.rp[r + 1]; j++) s -= L.a32[j] * x[L.kc[j]];
          y[r] = omega * s / L.d32[r];
        }
      }
      continue;
    }
    const float s = row4<float, float>(L.rp, L.kc, L.a32, x, r, valid && r < L.na, lane);
    if (valid && lane == 0) y[r] = r < L.na ? x[r] + omega * (L.rhs[r] - s) / L.d32[r] : L.rhs[r];
  }
}

// one colour class of an SOR sweep, in place on v[0]
__global__ void b_color(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev, int depth,
                        const int *__restrict__ cstart, float omega)
{
  CD_PDL_ENTRY();
  const int lane = threadIdx.x % 4;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    if (!stepping(ctl[slot])) continue;
    const BLevel &L = lev[slot * kMaxDepth + depth];
    // cstart[k]: first position of this colour in L.color_rows, cstart[K + k]: count
    const int i = (vb - t.bstart[k]) * kCsrRows + threadIdx.x / 4;
    const bool valid = i < cstart[t.K + k];
    const int r = valid ? L.color_rows[cstart[k] + i] : 0;
    float *x = L.v[0];
    const float s = row4<float, float>(L.rp, L.kc, L.a32, x, r, valid, lane);
    if (valid && lane == 0) x[r] += omega * (L.rhs[r] - s) / L.d32[r];
  }
}

// def = f - A v[src]
__global__ void b_defect(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev, int depth, int src)
{
  CD_PDL_ENTRY();
  const int lane = threadIdx.x % 4;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    if (!stepping(ctl[slot])) continue;
    const BLevel &L = lev[slot * kMaxDepth + depth];
    const int r = (vb - t.bstart[k]) * kCsrRows + threadIdx.x / 4;
    const bool valid = r < L.n;
    const float s = row4<float, float>(L.rp, L.kc, L.a32, L.v[src], r, valid, lane);
    if (valid && lane == 0) L.def[r] = L.rhs[r] - s;
  }
}

// coarse rhs = R def on active coarse rows (zero elsewhere), coarse v[0] = 0
__global__ void b_restrict(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev, int depth)
{
  CD_PDL_ENTRY();
  const int lane = threadIdx.x % 4;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    if (!stepping(ctl[slot])) continue;
    const BLevel &F = lev[slot * kMaxDepth + depth], &C = lev[slot * kMaxDepth + depth + 1];
    const int r = (vb - t.bstart[k]) * kCsrRows + threadIdx.x / 4;
    const bool valid = r < F.nc;
    const float s = row4<float, float>(F.rrp, F.rkc, F.rv, F.def, r, valid && r < F.nca, lane);
    if (valid && lane == 0)
    {
      C.rhs[r] = r < F.nca ? s : 0.f;
      C.v[0][r] = 0.f;
    }
  }
}

// fine v[fsrc] += damp * P coarse v[csrc] on active fine rows
__global__ void b_prolong(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev, int depth, int fsrc,
                          int csrc, float damp)
{
  CD_PDL_ENTRY();
  const int lane = threadIdx.x % 4;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    if (!stepping(ctl[slot])) continue;
    const BLevel &F = lev[slot * kMaxDepth + depth], &C = lev[slot * kMaxDepth + depth + 1];
    const int r = (vb - t.bstart[k]) * kCsrRows + threadIdx.x / 4;
    const bool valid = r < F.na;
    const float s = row4<float, float>(F.prp, F.pkc, F.pv, C.v[csrc], r, valid, lane);
    if (valid && lane == 0) F.v[fsrc][r] += damp * s;
  }
}

// exact coarse solve on the active block (one block per instance): v[out] = A^{-1} rhs with
// Dirichlet rows v = rhs and the active right-hand side corrected by A_AD rhs_D
__global__ void b_coarse(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev, int depth, int out)
{
  CD_PDL_ENTRY();
  extern __shared__ double sb[];
  for (int k = blockIdx.x; k < t.K; k += gridDim.x)
  {
    const int slot = t.item[k];
    if (!stepping(ctl[slot])) continue;
    const BLevel &L = lev[slot * kMaxDepth + depth];
    const int n = L.n, na = L.na;
    for (int i = threadIdx.x; i < n; i += blockDim.x) sb[i] = (double)L.rhs[i];
    __syncthreads();
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nw = blockDim.x / 32;
    for (int i = warp; i < na; i += nw)
    {
      double v = 0.0;
      for (int j = L.dirst[i] + lane; j < L.rp[i + 1]; j += 32) v += L.a64[j] * sb[L.kc[j]];
      v = bsum<32>(v);
      if (lane == 0) sb[n + i] = sb[i] - v;
    }
    for (int i = na + threadIdx.x; i < n; i += blockDim.x) L.v[out][i] = (float)sb[i];
    __syncthreads();
    for (int r = warp; r < na; r += nw)
    {
      double s = 0;
      for (int j = lane; j < na; j += 32) s += L.cinv[(size_t)r * na + j] * sb[n + j];
      s = bsum<32>(s);
      if (lane == 0) L.v[out][r] = (float)s;
    }
    __syncthreads();
  }
}

// Z_j = v[src] of depth 0, in FP64
__global__ void b_mg_finish(BTab t, const BCtl *__restrict__ ctl, const BLevel *__restrict__ lev, int src)
{
  CD_PDL_ENTRY();
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    const BCtl &c = ctl[slot];
    if (!stepping(c)) continue;
    const BLevel &L = lev[slot * kMaxDepth];
    const int r = (vb - t.bstart[k]) * kVecRows + threadIdx.x;
    if (r < L.n) c.Z[(size_t)c.j * c.n + r] = (double)L.v[src][r];
  }
}

// ---------------------------------------------------------------------------
// FGMRES kernels (FP64)
// ---------------------------------------------------------------------------
// w = A Z_j (stepping instances), or for restarting instances V_0 = b - A x with per-block
// partial sums of its square
__global__ void b_matvec(BTab t, const BCtl *__restrict__ ctl, int restart_phase, double *__restrict__ partial)
{
  CD_PDL_ENTRY();
  __shared__ double red[kNT / 32];
  const int lane = threadIdx.x % 4;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    const BCtl &c = ctl[slot];
    const bool act = restart_phase ? (c.state == ST_RUN && c.action == A_START) : stepping(c);
    if (!act) continue;
    const int r = (vb - t.bstart[k]) * kCsrRows + threadIdx.x / 4;
    const bool valid = r < c.n;
    const double *x = restart_phase ? c.x : c.Z + (size_t)c.j * c.n;
    const double s = row4<double, double>(c.rp, c.kc, c.a64, x, r, valid, lane);
    double sq = 0;
    if (valid && lane == 0)
    {
      if (restart_phase)
      {
        const double v = c.b[r] - s;
        c.V[r] = v;
        sq = v * v;
      }
      else
        c.w[r] = s;
    }
    if (restart_phase)
    {
      sq = bsum<32>(sq);
      if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = sq;
      __syncthreads();
      if (threadIdx.x == 0)
      {
        double tot = 0;
        for (int w = 0; w < kNT / 32; w++) tot += red[w];
        partial[(size_t)vb * kSlots] = tot;
      }
      __syncthreads();
    }
  }
}

// one fused classical Gram-Schmidt pass over V_0..V_j: mode 0 dots, 1 axpy (dots1) + dots,
// 2 axpy (dots2) + norm; per-virtual-block partials in partial[vb * 33 + t]
__global__ void b_gs(BTab t, const BCtl *__restrict__ ctl, int mode, double *__restrict__ partial)
{
  CD_PDL_ENTRY();
  __shared__ double red[kNT / 32][kSlots];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    const BCtl &c = ctl[slot];
    if (!stepping(c)) continue;
    const int kk = c.j + 1, n = c.n;
    const int r = (vb - t.bstart[k]) * kVecRows + threadIdx.x;
    const bool valid = r < n;
    double w = valid ? c.w[r] : 0.0;
    if (mode > 0)
    {
      const double *cf = mode == 1 ? c.dots1 : c.dots2;
      if (valid)
      {
        for (int q = 0; q < kk; q++) w -= cf[q] * c.V[(size_t)q * n + r];
        c.w[r] = w;
      }
    }
    if (mode == 2)
    {
      double sq = bsum<32>(w * w);
      if (lane == 0) red[warp][0] = sq;
      __syncthreads();
      if (threadIdx.x == 0)
      {
        double tot = 0;
        for (int q = 0; q < kNT / 32; q++) tot += red[q][0];
        partial[(size_t)vb * kSlots] = tot;
      }
    }
    else
    {
      for (int q = 0; q < kk; q++)
      {
        double p = bsum<32>(valid ? w * c.V[(size_t)q * n + r] : 0.0);
        if (lane == 0) red[warp][q] = p;
      }
      __syncthreads();
      if (threadIdx.x < kk)
      {
        double tot = 0;
        for (int q = 0; q < kNT / 32; q++) tot += red[q][threadIdx.x];
        partial[(size_t)vb * kSlots + threadIdx.x] = tot;
      }
    }
    __syncthreads();
  }
}

// per-instance sums of the partials of table t into ctl (which 0: dots1, 1: dots2, 2: nrm2);
// one block per instance, fixed order
__global__ void b_reduce(BTab t, BCtl *__restrict__ ctl, int which, int restart_phase,
                         const double *__restrict__ partial)
{
  CD_PDL_ENTRY();
  __shared__ double red[kNT / 32];
  for (int k = blockIdx.x; k < t.K; k += gridDim.x)
  {
    const int slot = t.item[k];
    BCtl &c = ctl[slot];
    const bool act = restart_phase ? (c.state == ST_RUN && c.action == A_START) : stepping(c);
    if (!act) continue;
    const int nslots = which == 2 ? 1 : c.j + 1;
    const int b0 = t.bstart[k], b1 = t.bstart[k + 1];
    for (int q = 0; q < nslots; q++)
    {
      double s = 0;
      for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) s += partial[(size_t)b * kSlots + q];
      s = bsum<32>(s);
      if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
      __syncthreads();
      if (threadIdx.x == 0)
      {
        double tot = 0;
        for (int w = 0; w < kNT / 32; w++) tot += red[w];
        if (which == 0) c.dots1[q] = tot;
        else if (which == 1) c.dots2[q] = tot;
        else c.nrm2 = tot;
      }
      __syncthreads();
    }
  }
}

__device__ void d_gen_rot(double dx, double dy, double &cs, double &sn)
{
  if (dy == 0.0) { cs = 1.0; sn = 0.0; }
  else if (fabs(dy) > fabs(dx)) { double t = dx / dy; sn = 1.0 / sqrt(1.0 + t * t); cs = t * sn; }
  else { double t = dy / dx; cs = 1.0 / sqrt(1.0 + t * t); sn = t * cs; }
}
__device__ void d_app_rot(double &dx, double &dy, double cs, double sn)
{
  double t = cs * dx + sn * dy;
  dy = -sn * dx + cs * dy;
  dx = t;
}

// y = H(0:k,0:k)^{-1} s(0:k) (back substitution, FgmresIte.C:198-216)
__device__ void d_solve_y(BCtl &c, int k)
{
  const int ld = c.m + 1;
  for (int a = 0; a < k; a++) c.y[a] = c.s[a];
  for (int a = k - 1; a >= 0; a--)
  {
    c.y[a] /= c.H[a * ld + a];
    for (int q = a - 1; q >= 0; q--) c.y[q] -= c.H[a * ld + q] * c.y[a];
  }
}

// Hessenberg column j, rotations, residual, stopping tests (FgmresIte.C:410-530)
__global__ void b_givens(BTab t, BCtl *__restrict__ ctl, int maxit, int minit, double div_factor)
{
  CD_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < t.K; k += gridDim.x * blockDim.x)
  {
    BCtl &c = ctl[t.item[k]];
    if (!stepping(c)) continue;
    const int j = c.j, ld = c.m + 1;
    double *h = c.H + (size_t)j * ld;
    for (int q = 0; q <= j; q++) h[q] = c.dots1[q] + c.dots2[q];
    const double hn = sqrt(c.nrm2);
    h[j + 1] = hn;
    c.hn = hn;
    for (int q = 0; q < j; q++) d_app_rot(h[q], h[q + 1], c.cs[q], c.sn[q]);
    d_gen_rot(h[j], h[j + 1], c.cs[j], c.sn[j]);
    d_app_rot(h[j], h[j + 1], c.cs[j], c.sn[j]);
    d_app_rot(c.s[j], c.s[j + 1], c.cs[j], c.sn[j]);
    c.res = fabs(c.s[j + 1]);
    c.its++;
    if (c.its >= minit && c.res < c.tol)
    {
      d_solve_y(c, j + 1);
      c.last = j;
      c.status = CDGPU_OK;
      c.action = A_UPD_DONE;
    }
    else if (c.res > div_factor * c.res0)
    {
      c.status = CDGPU_ERR_DIVERGED;
      c.state = ST_DONE;
    }
    else if (c.its >= maxit)
    {
      d_solve_y(c, j + 1);
      c.last = j;
      c.status = CDGPU_ERR_NOT_CONVERGED;
      c.action = A_UPD_DONE;
    }
    else if (j + 1 == c.m || hn == 0.0)
    {
      d_solve_y(c, j + 1);
      c.last = j;
      c.action = A_UPD_RESTART;
    }
    else
      c.action = A_NEXT;
  }
}

// V_{j+1} = w / h_{j+1,j} (A_NEXT), or x += Z y (A_UPD_*)
__global__ void b_next_update(BTab t, const BCtl *__restrict__ ctl)
{
  CD_PDL_ENTRY();
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    const BCtl &c = ctl[slot];
    if (c.state != ST_RUN) continue;
    const int r = (vb - t.bstart[k]) * kVecRows + threadIdx.x;
    if (r >= c.n) continue;
    if (c.action == A_NEXT)
      c.V[(size_t)(c.j + 1) * c.n + r] = c.w[r] / c.hn;
    else if (c.action == A_UPD_DONE || c.action == A_UPD_RESTART)
    {
      double s = 0;
      for (int q = 0; q <= c.last; q++) s += c.y[q] * c.Z[(size_t)q * c.n + r];
      c.x[r] += s;
    }
  }
}

// end of an iteration: advance j, finish, or schedule the restart
__global__ void b_post(BTab t, BCtl *__restrict__ ctl, int *__restrict__ state_out)
{
  CD_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < t.K; k += gridDim.x * blockDim.x)
  {
    const int slot = t.item[k];
    BCtl &c = ctl[slot];
    if (c.state == ST_RUN)
    {
      if (c.action == A_NEXT) { c.j++; c.action = A_STEP; }
      else if (c.action == A_UPD_DONE) c.state = ST_DONE;
      else if (c.action == A_UPD_RESTART) c.action = A_START;
    }
    state_out[slot] = c.state;
  }
}

// condition of the device-side iteration loop: another iteration while any solve of the set
// runs and the call's budget (loop[0]) lasts; consume = 1 after an iteration.  One block.
__global__ void b_loop_ctl(BTab t, const BCtl *__restrict__ ctl, int *__restrict__ loop,
                           cudaGraphConditionalHandle cond, int consume)
{
  CD_PDL_ENTRY();
  int any = 0;
  for (int k = threadIdx.x; k < t.K; k += blockDim.x) any |= ctl[t.item[k]].state == ST_RUN;
  any = __syncthreads_or(any);
  if (threadIdx.x == 0)
  {
    const int left = loop[0] - consume;
    loop[0] = left;
    cudaGraphSetConditional(cond, any && left > 0 ? 1u : 0u);
  }
}

__global__ void b_loop_budget(int *__restrict__ loop, int iterations)
{
  CD_PDL_ENTRY();
  loop[0] = iterations;
}

// restart: beta = ||b - A x||, stopping test on it, s = (beta, 0, ...), j = 0
__global__ void b_restart(BTab t, BCtl *__restrict__ ctl, int stop_rule, double red_factor, double res_norm_min)
{
  CD_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < t.K; k += gridDim.x * blockDim.x)
  {
    BCtl &c = ctl[t.item[k]];
    if (!(c.state == ST_RUN && c.action == A_START)) continue;
    const double beta = sqrt(c.nrm2);
    c.beta = beta;
    c.res = beta;
    if (c.its == 0 || stop_rule == 0) c.res0 = beta; // FgmresIte.C:557 (restart residual)
    c.tol = fmax(res_norm_min, red_factor * c.res0);
    if (c.its == 0 && (beta <= res_norm_min || beta < 1e-300))
    {
      c.status = CDGPU_OK;
      c.state = ST_DONE;
      continue;
    }
    for (int q = 0; q <= c.m; q++) c.s[q] = 0.0;
    c.s[0] = beta;
    c.j = 0;
    c.action = A_SCALE0;
  }
}

__global__ void b_scale0(BTab t, BCtl *__restrict__ ctl)
{
  CD_PDL_ENTRY();
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    const BCtl &c = ctl[slot];
    if (!(c.state == ST_RUN && c.action == A_SCALE0)) continue;
    const int r = (vb - t.bstart[k]) * kVecRows + threadIdx.x;
    if (r < c.n) c.V[r] /= c.beta;
  }
}

__global__ void b_begin_step(BTab t, BCtl *__restrict__ ctl)
{
  CD_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < t.K; k += gridDim.x * blockDim.x)
  {
    BCtl &c = ctl[t.item[k]];
    if (c.state == ST_RUN && c.action == A_SCALE0) c.action = A_STEP;
  }
}

// Gauss-Jordan inverse of the active block of an instance's coarsest level, one block, in
// global memory (partial pivoting; flag on a zero pivot)
__global__ void b_coarse_inverse(double *__restrict__ A, int n, int *__restrict__ piv, int *__restrict__ flag)
{
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int p_s;
  {
    const int nt = blockDim.x, t = threadIdx.x, lane = t % 32, warp = t / 32;
    for (int col = 0; col < n; col++)
    {
      double bv = -1.0;
      int bi = n;
      for (int i = col + t; i < n; i += nt)
      {
        double v = fabs(A[(size_t)i * n + col]);
        if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; }
      }
      for (int o = 16; o > 0; o >>= 1)
      {
        double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
      __syncthreads();
      if (t == 0)
      {
        double v = -1.0;
        int p = n;
        for (int w = 0; w < nt / 32; w++)
          if (red_v[w] > v || (red_v[w] == v && red_i[w] < p)) { v = red_v[w]; p = red_i[w]; }
        p_s = p;
        piv[col] = p;
        if (!(v > 0.0)) flag[0] = 1;
      }
      __syncthreads();
      const int p = p_s;
      if (p >= n) { __syncthreads(); continue; }
      if (p != col)
        for (int j = t; j < n; j += nt)
        {
          double tmp = A[(size_t)col * n + j];
          A[(size_t)col * n + j] = A[(size_t)p * n + j];
          A[(size_t)p * n + j] = tmp;
        }
      __syncthreads();
      const double pivot = A[(size_t)col * n + col];
      __syncthreads();
      for (int j = t; j < n; j += nt) A[(size_t)col * n + j] = (j == col ? 1.0 : A[(size_t)col * n + j]) / pivot;
      __syncthreads();
      for (int i = warp; i < n; i += nt / 32)
      {
        if (i == col) continue;
        const double f = A[(size_t)i * n + col];
        if (f == 0.0) continue;
        for (int j = lane; j < n; j += 32)
          if (j != col) A[(size_t)i * n + j] -= f * A[(size_t)col * n + j];
      }
      __syncthreads();
      for (int i = t; i < n; i += nt)
        if (i != col) A[(size_t)i * n + col] = -A[(size_t)i * n + col] * A[(size_t)col * n + col];
      __syncthreads();
    }
    for (int col = n - 1; col >= 0; col--)
    {
      int p = piv[col];
      if (p != col && p < n)
        for (int i = t; i < n; i += nt)
        {
          double tmp = A[(size_t)i * n + col];
          A[(size_t)i * n + col] = A[(size_t)i * n + p];
          A[(size_t)i * n + p] = tmp;
        }
      __syncthreads();
    }
  }
}

__global__ void b_dense_active(int na, const int *__restrict__ rp, const int *__restrict__ kc,
                               const double *__restrict__ a, double *__restrict__ dense)
{
  int r = blockIdx.x;
  for (int c = threadIdx.x; c < na; c += blockDim.x) dense[(size_t)r * na + c] = 0.0;
  __syncthreads();
  for (int j = rp[r] + threadIdx.x; j < rp[r + 1]; j += blockDim.x)
    if (kc[j] < na) dense[(size_t)r * na + kc[j]] = a[j];
}

__global__ void b_init_ctl(BCtl *__restrict__ ctl, int slot, BCtl init) { ctl[slot] = init; }

// theta-scheme matrices of one level from the mass matrix M and the stiffness matrix A, in
// the reference's order of in-place updates (SystemTCD2D.C:249-270, MatAdd on active rows):
// K = M - tau theta2 A, S = K + (tau theta2 + tau theta1) A; Dirichlet rows keep M's
// identity rows.  A is overwritten by S (FP64), S32 and the diagonals are filled; K is
// written when non-null (finest level).
__global__ void b_tcd_combine(int n, int na, const int *__restrict__ rp, const int *__restrict__ kc,
                              const double *__restrict__ M, double *__restrict__ AS, float *__restrict__ S32,
                              double *__restrict__ d64, float *__restrict__ d32, double mtt2, double tt12,
                              double *__restrict__ K)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  for (int j = rp[r]; j < rp[r + 1]; j++)
  {
    const double m = M[j], a = AS[j];
    double k = m, sv = m;
    if (r < na)
    {
      k = m + mtt2 * a;
      sv = k + tt12 * a;
    }
    if (K) K[j] = k;
    AS[j] = sv;
    S32[j] = (float)sv;
    if (kc[j] == r) { d64[r] = sv; d32[r] = (float)sv; }
  }
}

// right-hand side of a step (SystemTCD2D.C:237-262): b = tau theta3 f_old + tau theta4 f +
// K u_old on active rows (f_old = f: coefficients constant in time), b = f on Dirichlet rows
__global__ void b_tcd_rhs(BTab t, const BCtl *__restrict__ ctl)
{
  CD_PDL_ENTRY();
  const int lane = threadIdx.x % 4;
  for (int vb = blockIdx.x; vb < t.total; vb += gridDim.x)
  {
    const int k = find_item(t, vb), slot = t.item[k];
    const BCtl &c = ctl[slot];
    const int r = (vb - t.bstart[k]) * kCsrRows + threadIdx.x / 4;
    const bool valid = r < c.n;
    const double s = row4<double, double>(c.rp, c.kc, c.K, c.x, r, valid && r < c.na, lane);
    if (valid && lane == 0)
    {
      if (r < c.na)
      {
        double v = 0.0;
        v += c.c3 * c.f[r];
        v += c.c4 * c.f[r];
        c.b[r] = v + s;
      }
      else
        c.b[r] = c.f[r];
    }
  }
}

__global__ void b_tcd_begin(BTab t, BCtl *__restrict__ ctl)
{
  CD_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < t.K; k += gridDim.x * blockDim.x)
  {
    BCtl &c = ctl[t.item[k]];
    if (c.state == ST_EMPTY) continue;
    c.state = ST_RUN;
    c.action = A_START;
    c.its = 0;
    c.status = CDGPU_OK;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static Batch *get_batch(cdgpu_ctx *ctx, int id)
{
  if (!ctx || id < 0 || id >= (int)ctx->batches.size()) return nullptr;
  return ctx->batches[id];
}

// greedy distance-1 colouring of the active rows of every level of a hierarchy
static int ensure_colors(cdgpu_ctx *ctx, Hierarchy &h)
{
  for (auto &L : h.lev)
  {
    if (L.n_colors >= 0) continue;
    const Space &s = *L.sp;
    std::vector<int> col(s.n_dof, -1), mark;
    int nc = 0;
    for (int r = 0; r < s.n_active; r++)
    {
      mark.assign(nc + 1, 0);
      for (int j = s.h_row_ptr[r]; j < s.h_row_ptr[r + 1]; j++)
      {
        const int c = s.h_kcol[j];
        if (c != r && c < s.n_active && col[c] >= 0) mark[col[c]] = 1;
      }
      int c = 0;
      while (mark[c]) c++;
      col[r] = c;
      nc = std::max(nc, c + 1);
    }
    L.h_color_ptr.assign(nc + 1, 0);
    for (int r = 0; r < s.n_active; r++) L.h_color_ptr[col[r] + 1]++;
    for (int c = 0; c < nc; c++) L.h_color_ptr[c + 1] += L.h_color_ptr[c];
    std::vector<int> rows(std::max(1, s.n_active)), fill(L.h_color_ptr.begin(), L.h_color_ptr.end() - 1);
    for (int r = 0; r < s.n_active; r++) rows[fill[col[r]]++] = r;
    int rc = dev_alloc(ctx, &L.d_color_rows, rows.size());
    if (rc) return rc;
    CD_CUDA(ctx, cudaMemcpy(L.d_color_rows, rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice));
    L.n_colors = nc;
  }
  return CDGPU_OK;
}

template <typename T> static int balloc(cdgpu_ctx *ctx, BInst &in, T **p, size_t n)
{
  if (n == 0) n = 1;
  const size_t need = (n * sizeof(T) + 255) & ~(size_t)255;
  if (in.arena && in.arena_off + need <= in.arena_size)
  {
    *p = (T *)(in.arena + in.arena_off);
    in.arena_off += need;
    in.bytes += n * sizeof(T);
    return CDGPU_OK;
  }
  cudaError_t e = cudaMallocAsync((void **)p, n * sizeof(T), ctx->stream);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    *p = nullptr;
    return fail(ctx, CDGPU_ERR_OOM, "batch: device memory exhausted");
  }
  in.allocs.push_back(*p);
  in.bytes += n * sizeof(T);
  return CDGPU_OK;
}

static size_t instance_bytes(const Hierarchy &h, int m)
{
  size_t b = 0;
  for (size_t l = 0; l < h.lev.size(); l++)
  {
    const Space &s = *h.lev[l].sp;
    b += (size_t)s.nnz * (8 + 4) + (size_t)s.n_dof * (8 + 8 + 4 + 4 * 4);
  }
  const Space &f = *h.lev.back().sp;
  b += (size_t)(2 * (m + 1) + 3) * f.n_dof * 8 + (size_t)(m + 1) * m * 8;
  const Space &c = *h.lev[0].sp;
  b += (size_t)c.n_active * c.n_active * 8;
  return b;
}

static int grow(cdgpu_ctx *ctx, Batch &b, int need)
{
  if (need <= b.cap) return CDGPU_OK;
  int cap = std::max(need, std::max(64, b.cap * 2));
  BCtl *ctl = nullptr;
  BLevel *lev = nullptr;
  int *st = nullptr, *hst = nullptr;
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int rc;
  if ((rc = dev_alloc(ctx, &ctl, cap)) || (rc = dev_alloc(ctx, &lev, (size_t)cap * kMaxDepth)) ||
      (rc = dev_alloc(ctx, &st, cap)))
    return rc;
  CD_CUDA(ctx, cudaMallocHost((void **)&hst, sizeof(int) * cap));
  CD_CUDA(ctx, cudaMemset(ctl, 0, sizeof(BCtl) * cap));
  CD_CUDA(ctx, cudaMemset(lev, 0, sizeof(BLevel) * cap * kMaxDepth));
  CD_CUDA(ctx, cudaMemset(st, 0, sizeof(int) * cap));
  if (b.cap)
  {
    CD_CUDA(ctx, cudaMemcpy(ctl, b.d_ctl, sizeof(BCtl) * b.cap, cudaMemcpyDeviceToDevice));
    CD_CUDA(ctx, cudaMemcpy(lev, b.d_lev, sizeof(BLevel) * b.cap * kMaxDepth, cudaMemcpyDeviceToDevice));
    CD_CUDA(ctx, cudaMemcpy(st, b.d_state, sizeof(int) * b.cap, cudaMemcpyDeviceToDevice));
    cudaFree(b.d_ctl);
    cudaFree(b.d_lev);
    cudaFree(b.d_state);
    cudaFreeHost(b.h_state);
  }
  b.d_ctl = ctl;
  b.d_lev = lev;
  b.d_state = st;
  b.h_state = hst;
  b.cap = cap;
  return CDGPU_OK;
}

// the grouped-launch tables of the running set, packed into one device buffer
static int build_tables(cdgpu_ctx *ctx, Batch &b)
{
  b.run.clear();
  // time-dependent instances stay in the tables between steps (their kernels skip them
  // while they are idle), so the tables and the captured step do not change per step
  for (int i = 0; i < (int)b.inst.size(); i++)
    if (b.inst[i].used && (b.inst[i].state == ST_RUN || b.inst[i].tcd)) b.run.push_back(i);
  if (b.tcd_graph) { cudaGraphExecDestroy(b.tcd_graph); b.tcd_graph = nullptr; }
  if (b.loop_graph) { cudaGraphExecDestroy(b.loop_graph); b.loop_graph = nullptr; }
  int D = 0;
  for (int i : b.run) D = std::max(D, b.inst[i].L);
  b.depth = D;
  std::vector<int> pack;
  struct Pending { BTab *t; size_t item_off, bs_off; };
  std::vector<Pending> pend;
  auto add = [&](BTab &t, const std::vector<std::pair<int, int>> &items) {
    t.K = (int)items.size();
    size_t io = pack.size();
    for (auto &it : items) pack.push_back(it.first);
    size_t bo = pack.size();
    int acc = 0;
    for (auto &it : items) { pack.push_back(acc); acc += it.second; }
    pack.push_back(acc);
    t.total = acc;
    pend.push_back({&t, io, bo});
  };
  auto level_of = [&](int slot, int d) -> const Level & {
    const Hierarchy &h = *ctx->mgs[b.inst[slot].mg];
    return h.lev[h.lev.size() - 1 - d];
  };
  std::vector<std::pair<int, int>> v;
  auto fill = [&](int rows_per_block, auto rows_fn, auto keep_fn, int d) {
    v.clear();
    for (int i : b.run)
      if (keep_fn(i, d))
      {
        int rows = rows_fn(i, d);
        v.push_back({i, std::max(1, (rows + rows_per_block - 1) / rows_per_block)});
      }
  };
  auto nrows = [&](int i, int d) { return level_of(i, d).sp->n_dof; };
  auto all = [&](int, int) { return true; };
  fill(kVecRows, nrows, all, 0);
  add(b.fine_vec, v);
  fill(kCsrRows, nrows, all, 0);
  add(b.fine_csr, v);
  v.clear();
  for (int i : b.run) v.push_back({i, 1});
  add(b.items, v);
  fill(kCsrRows, nrows, [&](int i, int) { return b.inst[i].tcd; }, 0);
  add(b.tcd_csr, v);
  v.clear();
  for (int i : b.run)
    if (b.inst[i].tcd) v.push_back({i, 1});
  add(b.tcd_items, v);
  b.smooth.assign(D, BTab());
  b.restrict_.assign(D, BTab());
  b.coarse.assign(D, BTab());
  b.color.assign(D, std::vector<BTab>());
  b.ncolor_max.assign(D, 0);
  // the colour tables carry, after the usual item/bstart arrays, each item's first
  // position and count in its level's colour row list
  std::vector<std::vector<std::vector<std::pair<int, int>>>> cpos(D);
  for (int d = 0; d < D; d++)
  {
    auto deeper = [&](int i, int dd) { return b.inst[i].L - 1 > dd; };
    fill(kCsrRows, nrows, deeper, d);
    add(b.smooth[d], v);
    fill(kCsrRows, [&](int i, int dd) { return level_of(i, dd + 1).sp->n_dof; }, deeper, d);
    add(b.restrict_[d], v);
    v.clear();
    for (int i : b.run)
      if (b.inst[i].L - 1 == d) v.push_back({i, 1});
    add(b.coarse[d], v);
    if (b.p.smoother == 2 || b.p.smoother == 3)
    {
      int cm = 0;
      for (int i : b.run)
        if (deeper(i, d)) cm = std::max(cm, level_of(i, d).n_colors);
      b.ncolor_max[d] = cm;
      b.color[d].assign(cm, BTab());
      cpos[d].assign(cm, {});
      for (int c = 0; c < cm; c++)
      {
        v.clear();
        for (int i : b.run)
        {
          if (!deeper(i, d)) continue;
          const Level &L = level_of(i, d);
          if (c >= L.n_colors) continue;
          int cnt = L.h_color_ptr[c + 1] - L.h_color_ptr[c];
          if (cnt == 0) continue;
          v.push_back({i, (cnt + kCsrRows - 1) / kCsrRows});
          cpos[d][c].push_back({L.h_color_ptr[c], cnt});
        }
        add(b.color[d][c], v);
        // positions then counts, addressed through t.item + 2 * (K + 1) ... see colour_start()
        for (auto &pc : cpos[d][c]) pack.push_back(pc.first);
        for (auto &pc : cpos[d][c]) pack.push_back(pc.second);
      }
    }
  }
  if (pack.size() > b.tab_cap)
  {
    if (b.d_tab) { CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream)); cudaFree(b.d_tab); b.d_tab = nullptr; }
    int rc = dev_alloc(ctx, &b.d_tab, pack.size() * 2);
    if (rc) return rc;
    b.tab_cap = pack.size() * 2;
  }
  CD_CUDA(ctx, cudaMemcpyAsync(b.d_tab, pack.data(), sizeof(int) * pack.size(), cudaMemcpyHostToDevice, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream)); // pack is a host temporary
  for (auto &pd : pend)
  {
    pd.t->item = b.d_tab + pd.item_off;
    pd.t->bstart = b.d_tab + pd.bs_off;
  }
  // partial sums: one slot block per virtual block of the largest table that writes them
  size_t need = (size_t)std::max(b.fine_vec.total, b.fine_csr.total) * kSlots;
  if (need > b.partial_cap)
  {
    if (b.d_partial) { cudaFree(b.d_partial); b.d_partial = nullptr; }
    int rc = dev_alloc(ctx, &b.d_partial, need);
    if (rc) return rc;
    b.partial_cap = need;
  }
  b.dirty = false;
  return CDGPU_OK;
}

// device address of the colour positions of table (d, c): they follow its bstart array
static const int *colour_start(const BTab &t) { return t.bstart + t.K + 1; }

static int grid_of(cdgpu_ctx *ctx, int total)
{
  return std::max(1, std::min(total, ctx->sm_count * 8));
}

// one FP32 V-cycle of every stepping instance: Z_j = M^{-1} V_j
static int batch_cycle(cdgpu_ctx *ctx, Batch &b)
{
  const cdgpu_solver_params &p = b.p;
  const int D = b.depth;
  const bool jac = p.smoother == 1;
  const int pre = std::max(0, p.pre), post = std::max(0, p.post);
  const int after_pre = jac ? pre % 2 : 0, after_post = jac ? (pre + post) % 2 : 0;
  const float omega = (float)p.omega, damp = (float)p.gmg_damp;
  cudaStream_t st = ctx->stream;
  (void)cd_launch(b_mg_start, grid_of(ctx, b.fine_vec.total), kNT, 0, st, b.fine_vec, b.d_ctl, b.d_lev);
  CD_LAUNCHED(ctx);
  auto sweeps = [&](int d, int count, bool first_zero) -> int {
    const BTab &t = b.smooth[d];
    if (jac)
    {
      int src = first_zero ? 0 : after_pre;
      for (int s = 0; s < count; s++)
      {
        (void)cd_launch(b_jacobi, grid_of(ctx, t.total), kNT, 0, st, t, b.d_ctl, b.d_lev, d, src, first_zero && s == 0 ? 1 : 0,
                                                        omega);
        CD_LAUNCHED(ctx);
        src = 1 - src;
      }
    }
    else
      for (int s = 0; s < count; s++)
      {
        const int nc = b.ncolor_max[d];
        for (int pass = 0; pass < (p.smoother == 3 ? 2 : 1); pass++)
          for (int q = 0; q < nc; q++)
          {
            const int c = pass == 0 ? q : nc - 1 - q;
            const BTab &ct = b.color[d][c];
            if (ct.K == 0) continue;
            (void)cd_launch(b_color, grid_of(ctx, ct.total), kNT, 0, st, ct, b.d_ctl, b.d_lev, d, colour_start(ct), omega);
            CD_LAUNCHED(ctx);
          }
      }
    return CDGPU_OK;
  };
  for (int d = 0; d < D; d++)
  {
    if (b.coarse[d].K)
    {
      const Level *Lc = nullptr;
      int nmax = 0;
      for (int i : b.run)
        if (b.inst[i].L - 1 == d)
        {
          const Hierarchy &h = *ctx->mgs[b.inst[i].mg];
          Lc = &h.lev[0];
          nmax = std::max(nmax, Lc->sp->n_dof + Lc->sp->n_active);
        }
      size_t sm = sizeof(double) * nmax;
      if (sm > 48 * 1024)
        CD_CUDA(ctx, cudaFuncSetAttribute(b_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      (void)cd_launch(b_coarse, grid_of(ctx, b.coarse[d].K), 512, sm, st, b.coarse[d], b.d_ctl, b.d_lev, d, after_post);
      CD_LAUNCHED(ctx);
    }
    if (b.smooth[d].K == 0) continue;
    int rc = sweeps(d, pre, true);
    if (rc) return rc;
    (void)cd_launch(b_defect, grid_of(ctx, b.smooth[d].total), kNT, 0, st, b.smooth[d], b.d_ctl, b.d_lev, d, after_pre);
    CD_LAUNCHED(ctx);
    (void)cd_launch(b_restrict, grid_of(ctx, b.restrict_[d].total), kNT, 0, st, b.restrict_[d], b.d_ctl, b.d_lev, d);
    CD_LAUNCHED(ctx);
  }
  for (int d = D - 2; d >= 0; d--)
  {
    if (b.smooth[d].K == 0) continue;
    (void)cd_launch(b_prolong, grid_of(ctx, b.smooth[d].total), kNT, 0, st, b.smooth[d], b.d_ctl, b.d_lev, d, after_pre,
                                                               after_post, damp);
    CD_LAUNCHED(ctx);
    if (jac)
    {
      int src = after_pre;
      for (int s = 0; s < post; s++)
      {
        (void)cd_launch(b_jacobi, grid_of(ctx, b.smooth[d].total), kNT, 0, st, b.smooth[d], b.d_ctl, b.d_lev, d, src, 0, omega);
        CD_LAUNCHED(ctx);
        src = 1 - src;
      }
    }
    else
    {
      int rc = sweeps(d, post, false);
      if (rc) return rc;
    }
  }
  (void)cd_launch(b_mg_finish, grid_of(ctx, b.fine_vec.total), kNT, 0, st, b.fine_vec, b.d_ctl, b.d_lev, after_post);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

static int batch_iteration(cdgpu_ctx *ctx, Batch &b)
{
  const cdgpu_solver_params &p = b.p;
  cudaStream_t st = ctx->stream;
  const int gi = std::max(1, std::min((b.items.K + 127) / 128, ctx->sm_count * 4));
  // restarts (and first starts): V_0 = b - A x, beta, V_0 /= beta
  (void)cd_launch(b_matvec, grid_of(ctx, b.fine_csr.total), kNT, 0, st, b.fine_csr, b.d_ctl, 1, b.d_partial);
  CD_LAUNCHED(ctx);
  (void)cd_launch(b_reduce, grid_of(ctx, b.fine_csr.K), kNT, 0, st, b.fine_csr, b.d_ctl, 2, 1, b.d_partial);
  CD_LAUNCHED(ctx);
  (void)cd_launch(b_restart, gi, 128, 0, st, b.items, b.d_ctl, p.stop_rule, p.red_factor, p.res_norm_min);
  CD_LAUNCHED(ctx);
  (void)cd_launch(b_scale0, grid_of(ctx, b.fine_vec.total), kNT, 0, st, b.fine_vec, b.d_ctl);
  CD_LAUNCHED(ctx);
  (void)cd_launch(b_begin_step, gi, 128, 0, st, b.items, b.d_ctl);
  CD_LAUNCHED(ctx);
  // one Arnoldi step: z = M^{-1} v_j, w = A z, CGS2, Givens
  int rc = batch_cycle(ctx, b);
  if (rc) return rc;
  (void)cd_launch(b_matvec, grid_of(ctx, b.fine_csr.total), kNT, 0, st, b.fine_csr, b.d_ctl, 0, b.d_partial);
  CD_LAUNCHED(ctx);
  for (int mode = 0; mode < 3; mode++)
  {
    (void)cd_launch(b_gs, grid_of(ctx, b.fine_vec.total), kNT, 0, st, b.fine_vec, b.d_ctl, mode, b.d_partial);
    CD_LAUNCHED(ctx);
    (void)cd_launch(b_reduce, grid_of(ctx, b.fine_vec.K), kNT, 0, st, b.fine_vec, b.d_ctl, mode, 0, b.d_partial);
    CD_LAUNCHED(ctx);
  }
  (void)cd_launch(b_givens, gi, 128, 0, st, b.items, b.d_ctl, p.maxit, p.minit, p.div_factor);
  CD_LAUNCHED(ctx);
  (void)cd_launch(b_next_update, grid_of(ctx, b.fine_vec.total), kNT, 0, st, b.fine_vec, b.d_ctl);
  CD_LAUNCHED(ctx);
  (void)cd_launch(b_post, gi, 128, 0, st, b.items, b.d_ctl, b.d_state);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

// assemble one form of a shared space into the given arrays (the space's own value arrays
// and coefficients are restored afterwards)
static int assemble_to(cdgpu_ctx *ctx, Space &s, int disctype, const cdgpu_coeffs &co, double *a64, float *a32,
                       double *d64, float *d32, double *rhs64)
{
  int rc;
  if (!s.d_a)
  {
    // the space's own arrays are only scratch for a first assembly
    if ((rc = dev_alloc(ctx, &s.d_a, s.nnz)) || (rc = dev_alloc(ctx, &s.d_a32, s.nnz)) ||
        (rc = dev_alloc(ctx, &s.d_rhs, s.n_dof)) || (rc = dev_alloc(ctx, &s.d_diag, s.n_dof)) ||
        (rc = dev_alloc(ctx, &s.d_diag32, s.n_dof)))
      return rc;
  }
  double *sa = s.d_a, *srhs = s.d_rhs, *sd = s.d_diag;
  float *sa32 = s.d_a32, *sd32 = s.d_diag32;
  cdgpu_coeffs sco = s.co;
  bool sset = s.co_set, sasm = s.assembled;
  s.d_a = a64; s.d_rhs = rhs64; s.d_diag = d64; s.d_a32 = a32; s.d_diag32 = d32;
  s.co = co;
  s.co_set = true;
  rc = assemble_space(ctx, s, disctype, nullptr, false);
  s.d_a = sa; s.d_rhs = srhs; s.d_diag = sd; s.d_a32 = sa32; s.d_diag32 = sd32;
  s.co = sco; s.co_set = sset; s.assembled = sasm;
  s.mf_T = 0; // the cell coefficients now belong to the batch instance
  return rc;
}

// The device-side iteration loop as one graph: a kernel that sets the WHILE node's condition,
// then the WHILE node whose body is one FGMRES iteration of every running solve (the kernels
// of batch_iteration) followed by the kernel that consumes one iteration of the budget and
// sets the condition again.  Captured once per running set.  A driver that refuses the
// body's programmatic dependencies gets the body without them; one that refuses conditional
// nodes leaves the host loop (loop_mode 0).  Only API calls can fail here: nothing runs.
static int build_loop_graph(cdgpu_ctx *ctx, Batch &b, bool pdl, cudaGraph_t prefix, cudaGraphExec_t *out)
{
  int rc;
  if (!b.d_loop && (rc = dev_alloc(ctx, &b.d_loop, 1))) return rc;
  cudaGraph_t g = nullptr;
  cudaGraphConditionalHandle cond;
  cudaGraphNode_t pre = nullptr, init = nullptr, wnode = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, g, 0, 0);
  // work that runs once before the loop (a child graph)
  if (e == cudaSuccess && prefix) e = cudaGraphAddChildGraphNode(&pre, g, nullptr, 0, prefix);
  if (e == cudaSuccess)
  {
    cudaKernelNodeParams kp = {};
    BTab items = b.items;
    BCtl *ctl = b.d_ctl;
    int *loop = b.d_loop;
    int consume = 0;
    void *args[] = {&items, &ctl, &loop, &cond, &consume};
    kp.func = (void *)b_loop_ctl;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(256);
    kp.kernelParams = args;
    e = cudaGraphAddKernelNode(&init, g, pre ? &pre : nullptr, pre ? 1 : 0, &kp);
  }
  cudaGraph_t body = nullptr;
  if (e == cudaSuccess)
  {
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    e = cudaGraphAddNode(&wnode, g, &init, 1, &np);
    if (e == cudaSuccess) body = np.conditional.phGraph_out[0];
  }
  if (e != cudaSuccess)
  {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return CDGPU_ERR_UNSUPPORTED;
  }
  const long long before = ctx->launches;
  const bool pdl_was = cd_pdl_enabled();
  cd_pdl_enabled() = pdl;
  e = cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  rc = CDGPU_OK;
  if (e == cudaSuccess)
  {
    rc = batch_iteration(ctx, b);
    if (!rc)
    {
      (void)cd_launch(b_loop_ctl, 1, 256, 0, ctx->stream, b.items, (const BCtl *)b.d_ctl, b.d_loop, cond, 1);
      if (cudaGetLastError() != cudaSuccess) rc = CDGPU_ERR_CUDA;
    }
    cudaGraph_t captured = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &captured);
    if (e == cudaSuccess) e = e2;
  }
  cd_pdl_enabled() = pdl_was;
  ctx->launches = before;
  *out = nullptr;
  if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess || rc)
  {
    // a launch or capture refused inside the body (the driver's rules for conditional
    // bodies): nothing ran; the caller tries the next form
    *out = nullptr;
    cudaGetLastError();
    return CDGPU_ERR_UNSUPPORTED;
  }
  return CDGPU_OK;
}

static int running_count(const Batch &b)
{
  int r = 0;
  for (auto &in : b.inst)
    if (in.used && in.state == ST_RUN) r++;
  return r;
}

// theta-scheme parameters of a time-dependent instance
struct TcdSpec
{
  double tau, th1, th2, th3, th4;
};

static int submit_impl(cdgpu_ctx *ctx, Batch &b, int mg_id, const cdgpu_coeffs *co, int disctype,
                       int coarse_disctype, const TcdSpec *tcd, const double *h_u0, int *slot);

extern "C" {

int cdgpu_batch_create(cdgpu_ctx *ctx, const cdgpu_solver_params *params, int *batch_id)
{
  if (!ctx || !params || !batch_id) return fail(ctx, CDGPU_ERR_INVALID, "batch_create: bad argument");
  const cdgpu_solver_params &p = *params;
  if (p.solver != 16) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch: only FGMRES (solver 16) is batched");
  if (p.smoother < 1 || p.smoother > 3)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch: smoother must be 1 (Jacobi), 2 (SOR) or 3 (SSOR)");
  if (p.coarse_smoother != 17) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch: coarse_smoother must be 17 (exact)");
  if (p.cycle != 1) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch: V-cycles only");
  int m = std::min(p.restart, p.maxit);
  if (m <= 0) m = 10;
  if (m > kMaxM) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch: restart above 32 is not supported");
  cudaSetDevice(ctx->device);
  Batch *b = new Batch();
  b->p = p;
  b->m = m;
  // keep freed instance memory in the stream-ordered pool for the next submissions
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess)
  {
    unsigned long long thr = ~0ULL;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  ctx->batches.push_back(b);
  *batch_id = (int)ctx->batches.size() - 1;
  return CDGPU_OK;
}

int cdgpu_batch_instance_bytes(cdgpu_ctx *ctx, int batch_id, int mg_id, unsigned long long *bytes)
{
  Batch *b = get_batch(ctx, batch_id);
  if (!b || mg_id < 0 || mg_id >= (int)ctx->mgs.size() || !bytes)
    return fail(ctx, CDGPU_ERR_INVALID, "batch_instance_bytes: bad argument");
  *bytes = instance_bytes(*ctx->mgs[mg_id], b->m);
  return CDGPU_OK;
}

int cdgpu_batch_submit(cdgpu_ctx *ctx, int batch_id, int mg_id, const cdgpu_coeffs *co, int disctype,
                       int coarse_disctype, int *slot)
{
  Batch *bp = get_batch(ctx, batch_id);
  if (!bp || mg_id < 0 || mg_id >= (int)ctx->mgs.size() || !co || !slot)
    return fail(ctx, CDGPU_ERR_INVALID, "batch_submit: bad argument");
  return submit_impl(ctx, *bp, mg_id, co, disctype, coarse_disctype, nullptr, nullptr, slot);
}

int cdgpu_batch_submit_tcd(cdgpu_ctx *ctx, int batch_id, int mg_id, const cdgpu_coeffs *co, int disctype,
                           double tau, double theta1, double theta2, double theta3, double theta4,
                           const double *h_u0, int *slot)
{
  Batch *bp = get_batch(ctx, batch_id);
  if (!bp || mg_id < 0 || mg_id >= (int)ctx->mgs.size() || !co || !slot || !h_u0 || !(tau > 0))
    return fail(ctx, CDGPU_ERR_INVALID, "batch_submit_tcd: bad argument");
  TcdSpec t{tau, theta1, theta2, theta3, theta4};
  return submit_impl(ctx, *bp, mg_id, co, disctype, disctype, &t, h_u0, slot);
}

int cdgpu_batch_advance(cdgpu_ctx *ctx, int batch_id, int iterations, int *running)
{
  Batch *bp = get_batch(ctx, batch_id);
  if (!bp || iterations < 0) return fail(ctx, CDGPU_ERR_INVALID, "batch_advance: bad argument");
  Batch &b = *bp;
  cudaSetDevice(ctx->device);
  int rc;
  if (b.check_pending)
  {
    if ((rc = assemble_check(ctx))) return rc;
    b.check_pending = false;
  }
  if (b.dirty && (rc = build_tables(ctx, b))) return rc;
  if (iterations > 0 && running_count(b) > 0)
  {
    // the iterations run in a device-side loop (one graph launch) where the driver takes a
    // conditional node, else from this host loop
    if (!b.loop_graph && b.loop_mode != 0)
    {
      const int first = b.loop_mode < 0 ? 1 : b.loop_mode;
      for (int mode = first; mode <= 2 && !b.loop_graph; mode++)
      {
        rc = build_loop_graph(ctx, b, mode == 1, nullptr, &b.loop_graph);
        if (rc && rc != CDGPU_ERR_UNSUPPORTED) return rc;
        if (!rc) b.loop_mode = mode;
      }
      if (!b.loop_graph) b.loop_mode = 0;
    }
    if (b.loop_graph)
    {
      (void)cd_launch(b_loop_budget, 1, 1, 0, ctx->stream, b.d_loop, iterations);
      CD_LAUNCHED(ctx);
      CD_CUDA(ctx, cudaGraphLaunch(b.loop_graph, ctx->stream));
      b.loop_launches++;
    }
    else
      for (int it = 0; it < iterations && running_count(b) > 0; it++)
      {
        if ((rc = batch_iteration(ctx, b))) return rc;
        b.host_iterations++;
      }
  }
  // collect the states
  if (!b.run.empty())
  {
    CD_CUDA(ctx, cudaMemcpyAsync(b.h_state, b.d_state, sizeof(int) * b.cap, cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    bool changed = false;
    for (int i : b.run)
      if (b.h_state[i] == ST_DONE && b.inst[i].state == ST_RUN)
      {
        b.inst[i].state = ST_DONE;
        if (!b.inst[i].tcd)
        {
          b.done_queue.push_back(i);
          changed = true;
        }
      }
    if (changed) b.dirty = true;
  }
  int r = 0;
  for (auto &in : b.inst)
    if (in.used && in.state == ST_RUN) r++;
  if (running) *running = r;
  return CDGPU_OK;
}

int cdgpu_batch_tcd_step(cdgpu_ctx *ctx, int batch_id, int iterations, int *max_iterations)
{
  Batch *bp = get_batch(ctx, batch_id);
  if (!bp || iterations < 1) return fail(ctx, CDGPU_ERR_INVALID, "batch_tcd_step: bad argument");
  Batch &b = *bp;
  cudaSetDevice(ctx->device);
  int rc;
  if (b.check_pending)
  {
    if ((rc = assemble_check(ctx))) return rc;
    b.check_pending = false;
  }
  if (b.dirty && (rc = build_tables(ctx, b))) return rc;
  if (b.tcd_items.K == 0) return fail(ctx, CDGPU_ERR_INVALID, "batch_tcd_step: no time-dependent instance");
  for (auto &in : b.inst)
    if (in.used && in.tcd) in.state = ST_RUN;
  // the step -- right-hand sides, restart of every time-dependent solve from its previous
  // solution, FGMRES iterations of everything running -- is one CUDA graph, captured on first
  // use and replayed for every step while the instance set is unchanged.  Where the driver
  // takes conditional nodes the iterations are the device-side loop (until every solve has
  // finished, at most maxit + 1 iterations); otherwise the graph holds `iterations` of them
  // and solves that need more continue in rounds of `iterations` from the host.
  const int budget = b.p.maxit + 1;
  if (!b.tcd_graph || b.tcd_graph_k != iterations)
  {
    if (b.tcd_graph) { cudaGraphExecDestroy(b.tcd_graph); b.tcd_graph = nullptr; }
    // coarse-solve shared memory is configured outside the capture
    size_t sm = 0;
    for (int i : b.run)
    {
      const Space &c = *ctx->mgs[b.inst[i].mg]->lev[0].sp;
      sm = std::max(sm, sizeof(double) * (c.n_dof + c.n_active));
    }
    if (sm > 48 * 1024)
      CD_CUDA(ctx, cudaFuncSetAttribute(b_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    if (!b.d_loop && (rc = dev_alloc(ctx, &b.d_loop, 1))) return rc;
    const long long before = ctx->launches;
    bool looped = false;
    if (b.loop_mode != 0)
    {
      const int first = b.loop_mode < 0 ? 1 : b.loop_mode;
      for (int mode = first; mode <= 2 && !looped; mode++)
      {
        // the work before the loop, as a child graph (without programmatic dependencies in
        // the form that leaves them out of the loop body too)
        cudaGraph_t pg = nullptr;
        const bool pdl_was = cd_pdl_enabled();
        cd_pdl_enabled() = mode == 1;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess)
        {
          (void)cd_launch(b_tcd_rhs, std::max(1, std::min(b.tcd_csr.total, ctx->sm_count * 8)), kNT, 0, ctx->stream,
                          b.tcd_csr, b.d_ctl);
          (void)cd_launch(b_tcd_begin, 1, 256, 0, ctx->stream, b.tcd_items, b.d_ctl);
          (void)cd_launch(b_loop_budget, 1, 1, 0, ctx->stream, b.d_loop, budget);
          e = cudaGetLastError();
          cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &pg);
          if (e == cudaSuccess) e = e2;
        }
        cd_pdl_enabled() = pdl_was;
        if (e != cudaSuccess)
        {
          if (pg) cudaGraphDestroy(pg);
          return cuda_fail(ctx, e, "capture of the time step's right-hand sides");
        }
        rc = build_loop_graph(ctx, b, mode == 1, pg, &b.tcd_graph);
        cudaGraphDestroy(pg);
        if (rc && rc != CDGPU_ERR_UNSUPPORTED) return rc;
        if (!rc) { looped = true; b.loop_mode = mode; }
      }
      if (!looped && b.loop_mode < 0) b.loop_mode = 0;
    }
    if (!looped)
    {
      CD_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      (void)cd_launch(b_tcd_rhs, std::max(1, std::min(b.tcd_csr.total, ctx->sm_count * 8)), kNT, 0, ctx->stream, b.tcd_csr,
                      b.d_ctl);
      rc = cudaGetLastError() == cudaSuccess ? CDGPU_OK : CDGPU_ERR_CUDA;
      if (!rc)
      {
        (void)cd_launch(b_tcd_begin, 1, 256, 0, ctx->stream, b.tcd_items, b.d_ctl);
        for (int it = 0; it < iterations && !rc; it++) rc = batch_iteration(ctx, b);
      }
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      ctx->launches = before;
      if (rc) { if (g) cudaGraphDestroy(g); return rc; }
      if (e != cudaSuccess) return cuda_fail(ctx, e, "capture of the time step");
      e = cudaGraphInstantiate(&b.tcd_graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { b.tcd_graph = nullptr; return cuda_fail(ctx, e, "graph instantiate"); }
    }
    ctx->launches = before;
    b.tcd_graph_k = iterations;
    b.tcd_looped = looped;
  }
  CD_CUDA(ctx, cudaGraphLaunch(b.tcd_graph, ctx->stream));
  if (b.tcd_looped) b.loop_launches++;
  // solves that need more iterations continue outside the graph
  int r = 1, rounds = 0, extra = 0;
  while (true)
  {
    CD_CUDA(ctx, cudaMemcpyAsync(b.h_state, b.d_state, sizeof(int) * b.cap, cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    r = 0;
    for (int i : b.run)
    {
      BInst &in = b.inst[i];
      if (in.state == ST_RUN && b.h_state[i] == ST_DONE)
      {
        in.state = ST_DONE;
        if (!in.tcd) { b.done_queue.push_back(i); b.dirty = true; }
      }
      if (in.tcd && in.state == ST_RUN) r++;
    }
    if (r == 0) break;
    for (int it = 0; it < iterations; it++)
    {
      if ((rc = batch_iteration(ctx, b))) return rc;
      b.host_iterations++;
    }
    extra += iterations;
    rounds++;
  }
  if (max_iterations)
  {
    if (b.tcd_looped)
    {
      int left = 0;
      CD_CUDA(ctx, cudaMemcpy(&left, b.d_loop, sizeof(int), cudaMemcpyDeviceToHost));
      *max_iterations = (budget - std::max(0, left)) + extra;
    }
    else
      *max_iterations = iterations * (rounds + 1);
  }
  return CDGPU_OK;
}

int cdgpu_batch_tcd_solution(cdgpu_ctx *ctx, int batch_id, int slot, double *h_sol, cdgpu_solve_info *info)
{
  return cdgpu_batch_fetch(ctx, batch_id, slot, h_sol, info);
}

int cdgpu_batch_poll(cdgpu_ctx *ctx, int batch_id, int *slots, int max_slots, int *count)
{
  Batch *b = get_batch(ctx, batch_id);
  if (!b || !count || (max_slots > 0 && !slots)) return fail(ctx, CDGPU_ERR_INVALID, "batch_poll: bad argument");
  int k = std::min<int>(max_slots, (int)b->done_queue.size());
  for (int i = 0; i < k; i++) slots[i] = b->done_queue[i];
  b->done_queue.erase(b->done_queue.begin(), b->done_queue.begin() + k);
  *count = k;
  return CDGPU_OK;
}

int cdgpu_batch_fetch(cdgpu_ctx *ctx, int batch_id, int slot, double *h_sol, cdgpu_solve_info *info)
{
  Batch *b = get_batch(ctx, batch_id);
  if (!b || slot < 0 || slot >= (int)b->inst.size() || !b->inst[slot].used)
    return fail(ctx, CDGPU_ERR_INVALID, "batch_fetch: bad slot");
  cudaSetDevice(ctx->device);
  BCtl c;
  CD_CUDA(ctx, cudaMemcpyAsync(&c, b->d_ctl + slot, sizeof(BCtl), cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h_sol)
  {
    CD_CUDA(ctx, cudaMemcpyAsync(h_sol, c.x, sizeof(double) * c.n, cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (info)
  {
    info->iterations = c.its;
    info->status = c.state == ST_DONE ? c.status : CDGPU_ERR_NOT_CONVERGED;
    info->initial_residual = c.res0;
    info->final_residual = c.res;
  }
  return CDGPU_OK;
}

int cdgpu_batch_release(cdgpu_ctx *ctx, int batch_id, int slot)
{
  Batch *b = get_batch(ctx, batch_id);
  if (!b || slot < 0 || slot >= (int)b->inst.size() || !b->inst[slot].used)
    return fail(ctx, CDGPU_ERR_INVALID, "batch_release: bad slot");
  cudaSetDevice(ctx->device);
  BInst &in = b->inst[slot];
  const bool was_running = in.state == ST_RUN;
  // a running instance leaves the launches first: mark it done on the device
  int st = ST_EMPTY;
  CD_CUDA(ctx, cudaMemcpyAsync(&b->d_ctl[slot].state, &st, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CD_CUDA(ctx, cudaMemcpyAsync(b->d_state + slot, &st, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  b->bytes -= in.bytes;
  free_inst(ctx, in);
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream)); // st is a host temporary
  auto &q = b->done_queue;
  q.erase(std::remove(q.begin(), q.end(), slot), q.end());
  if (was_running) b->dirty = true;
  return CDGPU_OK;
}

int cdgpu_batch_loop_info(cdgpu_ctx *ctx, int batch_id, int *mode, long long *graph_launches,
                          long long *host_iterations)
{
  Batch *b = get_batch(ctx, batch_id);
  if (!b) return fail(ctx, CDGPU_ERR_INVALID, "batch_loop_info: bad id");
  if (mode) *mode = b->loop_mode;
  if (graph_launches) *graph_launches = b->loop_launches;
  if (host_iterations) *host_iterations = b->host_iterations;
  return CDGPU_OK;
}

int cdgpu_batch_memory(cdgpu_ctx *ctx, int batch_id, unsigned long long *bytes)
{
  Batch *b = get_batch(ctx, batch_id);
  if (!b || !bytes) return fail(ctx, CDGPU_ERR_INVALID, "batch_memory: bad argument");
  *bytes = b->bytes;
  return CDGPU_OK;
}

} // extern "C"

static int submit_impl(cdgpu_ctx *ctx, Batch &b, int mg_id, const cdgpu_coeffs *co, int disctype,
                       int coarse_disctype, const TcdSpec *tcd, const double *h_u0, int *slot)
{
  if (co->kind == CDGPU_COEFF_TABLE)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch_submit: coefficient tables are not batched");
  Hierarchy &h = *ctx->mgs[mg_id];
  const int L = (int)h.lev.size();
  if (L > kMaxDepth) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch_submit: more than 12 levels");
  const Space &cs = *h.lev[0].sp;
  if (cs.n_active > 4096) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch_submit: coarsest level above 4096 active DOFs");
  if ((size_t)(cs.n_dof + cs.n_active) * sizeof(double) > 200 * 1024)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "batch_submit: coarsest level too large for the exact solve");
  cudaSetDevice(ctx->device);
  int rc;
  if (b.p.smoother != 1 && (rc = ensure_colors(ctx, h))) return rc;
  // a free slot
  int sl = -1;
  for (int i = 0; i < (int)b.inst.size(); i++)
    if (!b.inst[i].used) { sl = i; break; }
  if (sl < 0) { sl = (int)b.inst.size(); b.inst.emplace_back(); }
  if ((rc = grow(ctx, b, (int)b.inst.size()))) return rc;
  BInst &in = b.inst[sl];
  in = BInst();
  in.used = true;
  in.mg = mg_id;
  in.L = L;
  const int m = b.m;
  {
    // the instance's arrays in one allocation (the estimate of instance_bytes plus the
    // alignment of every array); without it, one allocation per array
    const size_t size = instance_bytes(h, m) + (size_t)(L * 16 + 16) * 256;
    if (cudaMallocAsync((void **)&in.arena, size, ctx->stream) == cudaSuccess)
    {
      in.allocs.push_back(in.arena);
      in.arena_size = size;
    }
    else
    {
      cudaGetLastError();
      in.arena = nullptr;
    }
  }
  std::vector<BLevel> lv(kMaxDepth);
  double *tcd_K = nullptr;
  // per level: values, vectors; assemble with this instance's coefficients
  for (int l = 0; l < L; l++)
  {
    Level &Lv = h.lev[l];
    Space &s = *Lv.sp;
    if (s.nnz < 0) { free_inst(ctx, in); return fail(ctx, CDGPU_ERR_INVALID, "batch_submit: level without pattern"); }
    const int d = L - 1 - l;
    BLevel &B = lv[d];
    double *a64, *d64, *rhs64;
    float *a32, *d32;
    if ((rc = balloc(ctx, in, &a64, s.nnz)) || (rc = balloc(ctx, in, &d64, s.n_dof)) ||
        (rc = balloc(ctx, in, &rhs64, s.n_dof)) || (rc = balloc(ctx, in, &a32, s.nnz)) ||
        (rc = balloc(ctx, in, &d32, s.n_dof)) || (rc = balloc(ctx, in, &B.v[0], s.n_dof)) ||
        (rc = balloc(ctx, in, &B.v[1], s.n_dof)) || (rc = balloc(ctx, in, (float **)&B.rhs, s.n_dof)) ||
        (rc = balloc(ctx, in, &B.def, s.n_dof)))
    {
      free_inst(ctx, in);
      return rc;
    }
    // assemble into this instance's arrays through the shared space
    const int form = l == L - 1 ? disctype : coarse_disctype;
    if (!tcd)
      rc = assemble_to(ctx, s, form, *co, a64, a32, d64, d32, rhs64);
    else
    {
      // mass matrix into temporaries, stiffness matrix into the instance's arrays, then the
      // theta-scheme combinations
      double *Mt = nullptr, *dt = nullptr, *rt = nullptr, *K = nullptr;
      float *a32t = nullptr, *d32t = nullptr;
      cudaError_t e = cudaMallocAsync((void **)&Mt, sizeof(double) * s.nnz, ctx->stream);
      if (e == cudaSuccess) e = cudaMallocAsync((void **)&a32t, sizeof(float) * s.nnz, ctx->stream);
      if (e == cudaSuccess) e = cudaMallocAsync((void **)&dt, sizeof(double) * s.n_dof, ctx->stream);
      if (e == cudaSuccess) e = cudaMallocAsync((void **)&d32t, sizeof(float) * s.n_dof, ctx->stream);
      if (e == cudaSuccess) e = cudaMallocAsync((void **)&rt, sizeof(double) * s.n_dof, ctx->stream);
      if (e != cudaSuccess) { cudaGetLastError(); free_inst(ctx, in); return fail(ctx, CDGPU_ERR_OOM, "batch: device memory exhausted"); }
      rc = assemble_to(ctx, s, CDGPU_MASS, *co, Mt, a32t, dt, d32t, rt);
      if (!rc) rc = assemble_to(ctx, s, form, *co, a64, a32, d64, d32, rhs64);
      if (!rc && l == L - 1) rc = balloc(ctx, in, &K, s.nnz);
      if (!rc)
      {
        b_tcd_combine<<<(s.n_dof + 255) / 256, 256, 0, ctx->stream>>>(
            s.n_dof, s.n_active, s.d_row_ptr, s.d_kcol, Mt, a64, a32, d64, d32, -tcd->tau * tcd->th2,
            tcd->tau * tcd->th2 + tcd->tau * tcd->th1, K);
        CD_LAUNCHED(ctx);
        tcd_K = K;
      }
      void *tmp[] = {Mt, a32t, dt, d32t, rt};
      for (void *q : tmp) cudaFreeAsync(q, ctx->stream);
    }
    if (rc) { free_inst(ctx, in); return rc; }
    B.n = s.n_dof;
    B.na = s.n_active;
    B.rp = s.d_row_ptr;
    B.kc = s.d_kcol;
    B.dirst = s.d_dir_start;
    B.color_rows = Lv.d_color_rows;
    B.a32 = a32;
    B.d32 = d32;
    B.a64 = a64;
    if (l > 0)
    {
      // this level is the fine one of the transfer to level l-1
      const Space &c = *h.lev[l - 1].sp;
      B.nc = c.n_dof;
      B.nca = c.n_active;
      B.prp = Lv.d_p_row; B.pkc = Lv.d_p_col; B.pv = Lv.d_p_val32;
      B.rrp = Lv.d_r_row; B.rkc = Lv.d_r_col; B.rv = Lv.d_r_val32;
    }
    if (l == L - 1)
    {
      // FGMRES workspace and the right-hand side
      BCtl c{};
      c.state = ST_RUN;
      c.action = A_START;
      c.n = s.n_dof;
      c.m = m;
      c.rp = s.d_row_ptr;
      c.kc = s.d_kcol;
      c.a64 = a64;
      if ((rc = balloc(ctx, in, &c.V, (size_t)(m + 1) * s.n_dof)) || (rc = balloc(ctx, in, &c.Z, (size_t)(m + 1) * s.n_dof)) ||
          (rc = balloc(ctx, in, &c.w, s.n_dof)) || (rc = balloc(ctx, in, &c.x, s.n_dof)) ||
          (rc = balloc(ctx, in, &c.H, (size_t)(m + 1) * m)))
      {
        free_inst(ctx, in);
        return rc;
      }
      c.b = rhs64;
      c.na = s.n_active;
      if (tcd)
      {
        // idle until the first step; b is the step's right-hand side, f = (f, phi)
        c.state = ST_DONE;
        c.action = 0;
        c.tcd = 1;
        c.c3 = tcd->tau * tcd->th3;
        c.c4 = tcd->tau * tcd->th4;
        c.K = tcd_K;
        c.f = rhs64;
        if ((rc = balloc(ctx, in, &c.b, s.n_dof))) { free_inst(ctx, in); return rc; }
        CD_CUDA(ctx, cudaMemcpyAsync(c.x, h_u0, sizeof(double) * s.n_dof, cudaMemcpyHostToDevice, ctx->stream));
      }
      else
        CD_CUDA(ctx, cudaMemsetAsync(c.x, 0, sizeof(double) * s.n_dof, ctx->stream));
      // initial guess: the Dirichlet values on Dirichlet rows (AssembleMRhs copies them from
      // the right-hand side into the solution, SystemTCD2D.C:120)
      if (s.n_dof > s.n_active)
        CD_CUDA(ctx, cudaMemcpyAsync(c.x + s.n_active, rhs64 + s.n_active, sizeof(double) * (s.n_dof - s.n_active),
                                     cudaMemcpyDeviceToDevice, ctx->stream));
      b_init_ctl<<<1, 1, 0, ctx->stream>>>(b.d_ctl, sl, c);
      CD_LAUNCHED(ctx);
    }
  }
  // exact coarse solve: inverse of the coarsest level's active block
  {
    const Space &c = *h.lev[0].sp;
    BLevel &B = lv[L - 1];
    double *cinv;
    int *piv, *flag;
    const int na = c.n_active;
    if ((rc = balloc(ctx, in, &cinv, (size_t)na * na)) || (rc = balloc(ctx, in, &piv, std::max(na, 1))) ||
        (rc = balloc(ctx, in, &flag, 1)))
    {
      free_inst(ctx, in);
      return rc;
    }
    if (na > 0)
    {
      b_dense_active<<<na, 128, 0, ctx->stream>>>(na, c.d_row_ptr, c.d_kcol, B.a64, cinv);
      CD_LAUNCHED(ctx);
      CD_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream));
      b_coarse_inverse<<<1, 512, 0, ctx->stream>>>(cinv, na, piv, flag);
      CD_LAUNCHED(ctx);
    }
    B.cinv = cinv;
  }
  // pageable host sources: the copy is staged before the call returns.  Assembly errors
  // (a cell coupling missing from the pattern) are collected at the next advance.
  CD_CUDA(ctx, cudaMemcpyAsync(b.d_lev + (size_t)sl * kMaxDepth, lv.data(), sizeof(BLevel) * kMaxDepth,
                               cudaMemcpyHostToDevice, ctx->stream));
  b.check_pending = true;
  in.state = tcd ? ST_DONE : ST_RUN;
  in.tcd = tcd != nullptr;
  b.bytes += in.bytes;
  b.dirty = true;
  *slot = sl;
  return CDGPU_OK;
}
