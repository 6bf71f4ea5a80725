// Assembly kernels of libcdgpu (sm_100a).
//
// The reference assembles cell by cell and adds every local entry into the CSR
// row with a linear search (TMatrix::add -> TStructure::index_of_entry,
// src/FE/Matrix.C:111, src/FE/Structure.C:98; src/System/AssembleMat3D.C:765-787).
// Here the matrix is assembled row by row instead: a group of threads owns one
// CSR row, walks the cells containing the row's DOF in ascending cell order (the
// same order in which the reference's cell loop adds into that row), finds each
// column's slot by binary search in the row's own column list held in shared
// memory, and accumulates in shared memory.  Every entry is written exactly once
// with coalesced stores, there are no atomics and no colouring, and the sum order
// per entry is the reference's.  Local values come from one of two producers:
//   * affine fast path: for parallelogram / parallelepiped cells with constant
//     coefficients the local matrix is sum_t coef[cell][t] * R_t over reference
//     tensors R_t (see reference_tensors in setup.cpp); coef is computed per cell
//     (cell_coef_kernel) and the row kernel evaluates local entries on the fly;
//   * quadrature path: local matrices by Gauss quadrature with the reference's
//     per-point formulas (local_quad_kernel), stored and then gathered.
#include <climits>
#include <cooperative_groups.h>

#include <cmath>

#include "internal.h"

namespace cg = cooperative_groups;

struct Coef
{
  int kind, poly_degree;
  double eps, b1, b2, b3, c, f, delta0;
};

static Coef to_coef(const cdgpu_coeffs &c)
{
  return Coef{c.kind, c.poly_degree > 0 ? c.poly_degree : 1, c.eps, c.b1, c.b2, c.b3,
              c.c, c.f, c.delta0};
}

// SDFEM_TYPE 2 parameter (src/FE/ConvDiff.C:490-582, cases 1/2) with CELL_MEASURE 0
__device__ __forceinline__ double sdfem_delta(double hK, double eps, double b1, double b2,
                                              double b3, double delta0, int polydeg)
{
  if (fabs(eps) < 1e-20) eps = 1e-20;
  double nb = sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  double nu = 1.0 / polydeg, delta = 0.0;
  if (nb > 0)
  {
    double alpha = nu * nb * hK / (2 * eps);
    delta = nu * hK * (1 / tanh(alpha) - 1 / alpha) / (2 * nb);
  }
  return delta * delta0;
}

__device__ __forceinline__ void coef_at(const Coef &co, const double *tab, const double *x,
                                        double *k)
{
  k[0] = co.eps; k[1] = co.b1; k[2] = co.b2; k[3] = co.b3; k[4] = co.c; k[5] = co.f;
  if (co.kind == CDGPU_COEFF_SINE)
  {
    k[1] = k[2] = k[3] = k[4] = 0.0;
    k[5] = 2 * M_PI * M_PI * co.eps * sin(M_PI * x[0]) * sin(M_PI * x[1]);
  }
  else if (co.kind == CDGPU_COEFF_ROTATING)
  {
    k[1] = -x[1] + 0.5;
    k[2] = x[0] - 0.5;
  }
  else if (co.kind == CDGPU_COEFF_TABLE && tab)
  {
    for (int i = 0; i < 6; i++) k[i] = tab[i];
  }
}

__device__ __forceinline__ double d_invert(int dim, const double *J, double *Ji)
{
  if (dim == 2)
  {
    double det = J[0] * J[3] - J[1] * J[2];
    Ji[0] = J[3] / det; Ji[1] = -J[1] / det; Ji[2] = -J[2] / det; Ji[3] = J[0] / det;
    return det;
  }
  double c00 = J[4] * J[8] - J[5] * J[7], c01 = J[5] * J[6] - J[3] * J[8], c02 = J[3] * J[7] - J[4] * J[6];
  double det = J[0] * c00 + J[1] * c01 + J[2] * c02;
  Ji[0] = c00 / det; Ji[1] = (J[2] * J[7] - J[1] * J[8]) / det; Ji[2] = (J[1] * J[5] - J[2] * J[4]) / det;
  Ji[3] = c01 / det; Ji[4] = (J[0] * J[8] - J[2] * J[6]) / det; Ji[5] = (J[2] * J[3] - J[0] * J[5]) / det;
  Ji[6] = c02 / det; Ji[7] = (J[1] * J[6] - J[0] * J[7]) / det; Ji[8] = (J[0] * J[4] - J[1] * J[3]) / det;
  return det;
}

// reference -> physical map of a quadrilateral / hexahedron at xi: x and J[r*dim + b] =
// dx_r/dxi_b; affine cells from three (four) vertices, others multilinear
// (TQuadAffin / TQuadBilinear::GetOrigFromRef, src/FE/QuadAffin.C, src/FE/QuadBilinear.C, and
// their hexahedron counterparts)
__device__ __forceinline__ void d_ref_map(int dim, int nv, bool affine, const double *V, const double *xi,
                                          double *x, double *J)
{
  for (int k = 0; k < 3; k++) x[k] = 0.0;
  for (int k = 0; k < 9; k++) J[k] = 0.0;
  if (affine)
  {
    for (int r = 0; r < dim; r++)
    {
      double c1 = (V[1 * dim + r] - V[r]) * 0.5, c2 = (V[3 * dim + r] - V[r]) * 0.5;
      if (dim == 2)
      {
        x[r] = (V[1 * dim + r] + V[3 * dim + r]) * 0.5 + c1 * xi[0] + c2 * xi[1];
        J[r * 2] = c1; J[r * 2 + 1] = c2;
      }
      else
      {
        double c3 = (V[4 * dim + r] - V[r]) * 0.5;
        x[r] = (V[1 * dim + r] + V[3 * dim + r] + V[4 * dim + r] - V[r]) * 0.5 + c1 * xi[0] +
               c2 * xi[1] + c3 * xi[2];
        J[r * 3] = c1; J[r * 3 + 1] = c2; J[r * 3 + 2] = c3;
      }
    }
  }
  else
  {
    const double r2[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    for (int v = 0; v < nv; v++)
    {
      double rv[3];
      if (dim == 2) { rv[0] = r2[v][0]; rv[1] = r2[v][1]; }
      else { rv[0] = r2[v & 3][0]; rv[1] = r2[v & 3][1]; rv[2] = v < 4 ? -1.0 : 1.0; }
      double f[3], N = 1;
      for (int b = 0; b < dim; b++) { f[b] = 0.5 * (1 + rv[b] * xi[b]); N *= f[b]; }
      for (int b = 0; b < dim; b++)
      {
        double dN = 0.5 * rv[b];
        for (int e = 0; e < dim; e++)
          if (e != b) dN *= f[e];
        for (int r = 0; r < dim; r++) J[r * dim + b] += dN * V[v * dim + r];
      }
      for (int r = 0; r < dim; r++) x[r] += N * V[v * dim + r];
    }
  }
}

__device__ __forceinline__ double d_diameter(int dim, const double *V)
{
  double best = 0;
  if (dim == 2)
  {
    for (int e = 0; e < 2; e++)
    {
      int a = e, b = e + 2;
      double dx = V[2 * a] - V[2 * b], dy = V[2 * a + 1] - V[2 * b + 1];
      best = fmax(best, dx * dx + dy * dy);
    }
  }
  else
  {
    const int p0[4] = {0, 1, 2, 3}, p1[4] = {6, 7, 4, 5};
    for (int e = 0; e < 4; e++)
    {
      double s = 0;
      for (int a = 0; a < 3; a++)
      {
        double d = V[3 * p0[e] + a] - V[3 * p1[e] + a];
        s += d * d;
      }
      best = fmax(best, s);
    }
  }
  return sqrt(best);
}

// ---------------------------------------------------------------------------
// affine fast path: per-cell coefficients of the reference tensors
// ---------------------------------------------------------------------------
struct CellCoefArgs
{
  int dim, nv, n_cells, disctype, T, Tr;
  Coef co;
  const double *coords;
  double *out; // n_cells x (T + Tr)
};

__global__ void cell_coef_kernel(CellCoefArgs a)
{
  CD_PDL_ENTRY();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n_cells) return;
  const int dim = a.dim;
  double V[24];
  for (int k = 0; k < a.nv * dim; k++) V[k] = a.coords[(size_t)c * a.nv * dim + k];
  double J[9], Ji[9];
  for (int r = 0; r < dim; r++)
  {
    J[r * dim + 0] = (V[1 * dim + r] - V[r]) * 0.5;
    J[r * dim + 1] = (V[3 * dim + r] - V[r]) * 0.5;
    if (dim == 3) J[r * dim + 2] = (V[4 * dim + r] - V[r]) * 0.5;
  }
  double w = fabs(d_invert(dim, J, Ji));
  double b[3] = {a.co.b1, a.co.b2, dim == 3 ? a.co.b3 : 0.0};
  double G[9], beta[3];
  for (int p = 0; p < dim; p++)
  {
    double s = 0;
    for (int q = 0; q < dim; q++) s += Ji[p * dim + q] * b[q];
    beta[p] = s;
    for (int r = 0; r < dim; r++)
    {
      double g = 0;
      for (int q = 0; q < dim; q++) g += Ji[p * dim + q] * Ji[r * dim + q];
      G[p * dim + r] = g;
    }
  }
  double eps = a.co.eps, cr = a.co.c, f = a.co.f;
  bool supg = a.disctype == CDGPU_SUPG;
  double delta = supg ? sdfem_delta(d_diameter(dim, V), eps, b[0], b[1], b[2], a.co.delta0,
                                    a.co.poly_degree)
                      : 0.0;
  double K[9];
  for (int p = 0; p < dim * dim; p++) K[p] = eps * G[p];
  if (supg)
    for (int p = 0; p < dim; p++)
      for (int r = 0; r < dim; r++) K[p * dim + r] += delta * beta[p] * beta[r];
  double *o = a.out + (size_t)c * (a.T + a.Tr);
  if (a.disctype == CDGPU_MASS)
  {
    o[0] = w;
    o[1] = w * f;
    return;
  }
  if (dim == 2)
  {
    o[0] = w * K[0]; o[1] = w * K[3]; o[2] = w * K[1];
    o[3] = w * beta[0]; o[4] = w * beta[1]; o[5] = w * cr;
    if (supg)
    {
      o[6] = w * delta * cr * beta[0];
      o[7] = w * delta * cr * beta[1];
      double s = -w * delta * eps;
      o[8] = s * G[0] * beta[0]; o[9] = s * G[0] * beta[1];
      o[10] = s * G[3] * beta[0]; o[11] = s * G[3] * beta[1];
      o[12] = s * G[1] * beta[0]; o[13] = s * G[1] * beta[1];
    }
  }
  else
  {
    o[0] = w * K[0]; o[1] = w * K[4]; o[2] = w * K[8];
    o[3] = w * K[1]; o[4] = w * K[2]; o[5] = w * K[5];
    o[6] = w * beta[0]; o[7] = w * beta[1]; o[8] = w * beta[2]; o[9] = w * cr;
    if (supg)
      for (int p = 0; p < 3; p++) o[10 + p] = w * delta * cr * beta[p];
  }
  double *orr = o + a.T;
  orr[0] = w * f;
  if (supg)
    for (int p = 0; p < dim; p++) orr[1 + p] = w * f * delta * beta[p];
}

// ---------------------------------------------------------------------------
// quadrature path: the reference's per-point local forms (src/FE/ConvDiff2D.C:32-162,
// src/FE/ConvDiff3D.C:61-190) summed over the Gauss points in the reference's order.  Writes
// nbf*nbf matrix entries then nbf rhs entries per cell.
//
// Persistent CTAs.  The reference element's tables (Gauss points and weights, basis values
// and gradients, 2D second derivatives) are staged in shared memory once per CTA by one bulk
// copy (cp.async.bulk, 1D TMA); each cell's geometry (vertex coordinates) and, for tabulated
// coefficients, its per-point coefficient records are staged by bulk copies into one of two
// stages, the next cell's copy in flight while the current cell is computed.  Every wait is
// bounded: on a timeout the CTA sets the assembly's error flag (5), stops, and waits (bounded)
// for its copies still in flight.
// ---------------------------------------------------------------------------
struct LocalArgs
{
  int dim, nv, nbf, nq, n_cells, disctype, affine_all;
  Coef co;
  const double *coords, *tab; // tab: n_cells x nq x 6 (kind TABLE)
  const double *qtab;         // packed qx | qw | phi | dphi | hphi
  int n_qx, n_qw, n_phi, n_dphi, n_stage_tab; // lengths (doubles); staged table = n_stage_tab
  double *out;
  int *err;
};

constexpr long kLqSpin = 1L << 22;

__device__ __forceinline__ uint32_t lq_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool lq_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t done;
  asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
               "selp.b32 %0, 1, 0, P1;\n\t}"
               : "=r"(done)
               : "r"(lq_smem_u32(bar)), "r"(parity)
               : "memory");
  return done != 0;
}

__device__ __forceinline__ bool lq_wait(uint64_t *bar, uint32_t parity)
{
  for (long it = 0; it < kLqSpin; it++)
    if (lq_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void lq_bulk(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   lq_smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(lq_smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void lq_expect(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(lq_smem_u32(bar)), "r"(bytes)
               : "memory");
}

__host__ __device__ inline int lq_even(int n) { return (n + 1) & ~1; } // doubles -> 16-byte multiple

// shared-memory layout (in doubles) of local_quad_kernel
struct LqLayout
{
  int tabs, g, lap, mult, kq, dl, Jis, stage0, stage_len, total;
  __host__ __device__ LqLayout(int dim, int nv, int nbf, int nq, int disctype, int n_stage_tab, bool table)
  {
    tabs = 0;
    g = lq_even(n_stage_tab);
    lap = g + nq * nbf * dim;
    const int nlap = (dim == 2 && disctype == CDGPU_SUPG) ? nq * nbf : 0;
    mult = lap + nlap;
    kq = mult + nq;
    dl = kq + nq * 6;
    Jis = dl + nq;
    stage0 = lq_even(Jis + nq * dim * dim);
    stage_len = lq_even(nv * dim) + (table ? nq * 6 : 0);
    total = stage0 + 2 * stage_len;
  }
};

// Q27: Q2 hexahedra (27 local DOFs) with the register-tiled entry phase; the other elements
// take the one-entry-per-thread loop in an instance of their own, so that its register count
// (and with it the resident CTAs per SM) is not the tiled phase's
template <bool Q27>
__global__ void __launch_bounds__(256) local_quad_kernel(LocalArgs a)
{
  CD_PDL_ENTRY();
  extern __shared__ __align__(16) double sm[];
  __shared__ __align__(8) uint64_t bar[3]; // tables, cell stage 0, cell stage 1
  const int dim = a.dim, nbf = a.nbf, nq = a.nq, nv = a.nv;
  const bool table = a.tab != nullptr;
  const LqLayout lay(dim, nv, nbf, nq, a.disctype, a.n_stage_tab, table);
  const double *qx = sm, *qw = sm + a.n_qx, *phi = qw + a.n_qw, *dphi = phi + a.n_phi, *hphi = dphi + a.n_dphi;
  double *g = sm + lay.g, *lap = sm + lay.lap, *mult = sm + lay.mult, *kq = sm + lay.kq, *dl = sm + lay.dl,
         *Jis = sm + lay.Jis;
  const uint32_t vbytes = (uint32_t)lq_even(nv * dim) * 8u, tbytes = table ? (uint32_t)nq * 48u : 0u;
  // stage the cell's vertex coordinates (nv*dim doubles: 64 or 192 bytes) and coefficient
  // records (nq * 48 bytes); both sizes and both offsets are multiples of 16 bytes
  auto issue = [&](int c, int st) {
    double *dst = sm + lay.stage0 + st * lay.stage_len;
    lq_expect(&bar[1 + st], (uint32_t)(nv * dim * 8) + tbytes);
    lq_bulk(dst, a.coords + (size_t)c * nv * dim, (uint32_t)(nv * dim * 8), &bar[1 + st]);
    if (table) lq_bulk(dst + vbytes / 8, a.tab + (size_t)c * nq * 6, tbytes, &bar[1 + st]);
  };
  int issued0 = 0, issued1 = 0, waited0 = 0, waited1 = 0; // thread 0's copies per stage; waits
  if (threadIdx.x == 0)
  {
    for (int k = 0; k < 3; k++) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(lq_smem_u32(&bar[k])), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint32_t tb = (uint32_t)lq_even(a.n_stage_tab) * 8u;
    lq_expect(&bar[0], tb);
    lq_bulk(sm, a.qtab, tb, &bar[0]);
    if (blockIdx.x < a.n_cells) { issue(blockIdx.x, 0); issued0++; }
    if (blockIdx.x + gridDim.x < a.n_cells) { issue(blockIdx.x + gridDim.x, 1); issued1++; }
  }
  __syncthreads();
  bool ok = __syncthreads_and(lq_wait(&bar[0], 0u)) != 0;
  if (!ok && threadIdx.x == 0) atomicExch(a.err, 5);
  int li = 0;
  for (int c = blockIdx.x; ok && c < a.n_cells; c += gridDim.x, li++)
  {
    const int st = li & 1;
    const bool got = lq_wait(&bar[1 + st], (uint32_t)(li >> 1) & 1u);
    if (!__syncthreads_and(got))
    {
      if (threadIdx.x == 0) atomicExch(a.err, 5);
      ok = false;
      break;
    }
    if (st) waited1++; else waited0++;
    const double *V = sm + lay.stage0 + st * lay.stage_len;
    const double *ctab = V + vbytes / 8;
    for (int q = threadIdx.x; q < nq; q += blockDim.x)
    {
      const double *xi = qx + q * dim;
      double x[3], J[9], Ji[9];
      d_ref_map(dim, nv, a.affine_all, V, xi, x, J);
      double det = d_invert(dim, J, Ji);
      mult[q] = qw[q] * fabs(det);
      for (int k = 0; k < dim * dim; k++) Jis[q * dim * dim + k] = Ji[k];
      double k6[6];
      coef_at(a.co, table ? ctab + q * 6 : nullptr, x, k6);
      for (int k = 0; k < 6; k++) kq[q * 6 + k] = k6[k];
      dl[q] = a.disctype == CDGPU_SUPG
                  ? sdfem_delta(d_diameter(dim, V), k6[0], k6[1], k6[2], dim == 3 ? k6[3] : 0.0,
                                a.co.delta0, a.co.poly_degree)
                  : 0.0;
    }
    __syncthreads();
    // physical gradients, component-major: g[(q * dim + r) * nbf + b]
    for (int t = threadIdx.x; t < nq * nbf; t += blockDim.x)
    {
      int q = t / nbf, b = t % nbf;
      const double *Ji = Jis + q * dim * dim;
      const double *dp = dphi + (size_t)(q * nbf + b) * dim;
      for (int r = 0; r < dim; r++)
      {
        double s = 0;
        for (int e = 0; e < dim; e++) s += Ji[e * dim + r] * dp[e];
        g[(q * dim + r) * nbf + b] = s;
      }
      if (dim == 2 && a.disctype == CDGPU_SUPG)
      {
        // physical second derivatives Ji^T (H - G) Ji: on a bilinear cell
        // x = c0 + c1 xi + c2 eta + c3 xi eta the mixed reference derivative also carries
        // grad(phi) . c3 (the D11 row of the 5x5 system of QuadBilinear::GetOrigValues,
        // src/FE/QuadBilinear.C:531-549); an affine map has c3 = 0
        double l = 0;
        const double *hp = hphi + (size_t)(q * nbf + b) * 4;
        double gm = 0;
        if (!a.affine_all)
          for (int r = 0; r < 2; r++)
            gm += g[(q * dim + r) * nbf + b] * 0.25 * (V[r] - V[2 + r] + V[4 + r] - V[6 + r]);
        for (int r = 0; r < 2; r++)
          for (int e = 0; e < 2; e++)
            for (int f = 0; f < 2; f++) l += Ji[e * 2 + r] * Ji[f * 2 + r] * (hp[e * 2 + f] - (e != f ? gm : 0.0));
        lap[q * nbf + b] = l;
      }
    }
    __syncthreads();
    double *out = a.out + (size_t)c * (nbf * nbf + nbf);
    if constexpr (Q27)
    {
      // Q2 hexahedra: 243 threads = 3 groups x 81; a group takes the Gauss points q = grp mod 3
      // and a thread of it the 3 x 3 entries (ib + 9u, jb + 9v), so every value loaded from
      // shared memory serves three entries; the three groups' partial sums are added in group
      // order afterwards.  Threads 243..255 take the right-hand side.
      const int t = threadIdx.x;
      double acc[3][3];
#pragma unroll
      for (int u = 0; u < 3; u++)
#pragma unroll
        for (int v = 0; v < 3; v++) acc[u][v] = 0.0;
      const int grp = t / 81, tt = t % 81, ib = tt / 9, jb = tt % 9;
      if (t < 243)
      {
        for (int q = grp; q < nq; q += 3)
        {
          const double *k6 = kq + q * 6;
          const double c0 = k6[0], c1 = k6[1], c2 = k6[2], c3 = k6[3], cr = k6[4];
          const double m = mult[q], delta = dl[q];
          const double *g0 = g + (q * 3) * 27, *g1 = g0 + 27, *g2 = g1 + 27, *ph = phi + q * 27;
          double gi[3][3], pi[3], bi[3], gj[3][3], pj[3], bj[3];
#pragma unroll
          for (int u = 0; u < 3; u++)
          {
            const int i = ib + 9 * u, j = jb + 9 * u;
            gi[u][0] = g0[i]; gi[u][1] = g1[i]; gi[u][2] = g2[i]; pi[u] = ph[i];
            gj[u][0] = g0[j]; gj[u][1] = g1[j]; gj[u][2] = g2[j]; pj[u] = ph[j];
            bi[u] = c1 * gi[u][0] + c2 * gi[u][1] + c3 * gi[u][2];
            bj[u] = c1 * gj[u][0] + c2 * gj[u][1] + c3 * gj[u][2];
          }
#pragma unroll
          for (int u = 0; u < 3; u++)
#pragma unroll
            for (int v = 0; v < 3; v++)
            {
              double val;
              if (a.disctype == CDGPU_MASS)
                val = pj[v] * pi[u]; // MatrixMRhsAssemble, ConvDiff2D.C:411
              else
              {
                val = c0 * (gi[u][0] * gj[v][0] + gi[u][1] * gj[v][1] + gi[u][2] * gj[v][2]);
                val += bj[v] * pi[u];
                val += cr * pj[v] * pi[u];
                if (a.disctype == CDGPU_SUPG) val += delta * (bj[v] + cr * pj[v]) * bi[u];
              }
              acc[u][v] += val * m;
            }
        }
      }
      else
      {
        // right-hand side rows i = t - 243 + 13 r
        for (int r = 0; r < 3; r++)
        {
          const int i = t - 243 + 13 * r;
          if (i >= 27) break;
          double sum = 0;
          for (int q = 0; q < nq; q++)
          {
            const double *k6 = kq + q * 6;
            const double *gq = g + (q * 3) * 27;
            const double phi_i = phi[q * 27 + i];
            const double bgradv = k6[1] * gq[i] + k6[2] * gq[27 + i] + k6[3] * gq[54 + i];
            sum += a.disctype == CDGPU_SUPG ? mult[q] * (phi_i + dl[q] * bgradv) * k6[5] : mult[q] * phi_i * k6[5];
          }
          out[729 + i] = sum;
        }
      }
      // the gradients are no longer needed: their space takes groups 1 and 2's partial sums
      __syncthreads();
      if (t >= 81 && t < 243)
#pragma unroll
        for (int u = 0; u < 3; u++)
#pragma unroll
          for (int v = 0; v < 3; v++) g[(grp - 1) * 729 + (ib + 9 * u) * 27 + jb + 9 * v] = acc[u][v];
      __syncthreads();
      if (t < 81)
#pragma unroll
        for (int u = 0; u < 3; u++)
#pragma unroll
          for (int v = 0; v < 3; v++)
          {
            const int e = (ib + 9 * u) * 27 + jb + 9 * v;
            out[e] = (acc[u][v] + g[e]) + g[729 + e];
          }
    }
    else
      for (int t = threadIdx.x; t < nbf * nbf + nbf; t += blockDim.x)
      {
        bool is_rhs = t >= nbf * nbf;
        int i = is_rhs ? t - nbf * nbf : t / nbf, j = is_rhs ? 0 : t % nbf;
        double acc = 0;
        for (int q = 0; q < nq; q++)
        {
          const double *k6 = kq + q * 6;
          double c0 = k6[0], c1 = k6[1], c2 = k6[2], c3 = dim == 3 ? k6[3] : 0.0, cr = k6[4], f = k6[5];
          const double *gq = g + q * dim * nbf;
          const double gi0 = gq[i], gi1 = gq[nbf + i], gi2 = dim == 3 ? gq[2 * nbf + i] : 0.0;
          double phi_i = phi[q * nbf + i];
          double bgradv = c1 * gi0 + c2 * gi1 + (dim == 3 ? c3 * gi2 : 0.0);
          double delta = dl[q];
          if (is_rhs)
          {
            acc += a.disctype == CDGPU_SUPG ? mult[q] * (phi_i + delta * bgradv) * f : mult[q] * phi_i * f;
            continue;
          }
          const double gj0 = gq[j], gj1 = gq[nbf + j], gj2 = dim == 3 ? gq[2 * nbf + j] : 0.0;
          double phi_j = phi[q * nbf + j];
          if (a.disctype == CDGPU_MASS)
          {
            acc += mult[q] * phi_j * phi_i; // MatrixMRhsAssemble, ConvDiff2D.C:411
            continue;
          }
          double val = c0 * (gi0 * gj0 + gi1 * gj1 + (dim == 3 ? gi2 * gj2 : 0.0));
          double bg = c1 * gj0 + c2 * gj1 + (dim == 3 ? c3 * gj2 : 0.0);
          val += bg * phi_i;
          val += cr * phi_j * phi_i;
          if (a.disctype == CDGPU_SUPG)
          {
            if (dim == 2)
              val += delta * (-c0 * lap[q * nbf + j] + bg + cr * phi_j) * bgradv;
            else
              val += delta * (bg + cr * phi_j) * bgradv;
          }
          val *= mult[q];
          acc += val;
        }
        out[t] = acc;
      }
    // every thread is done with this stage (its geometry and coefficients went into the
    // shared arrays above): refill it with the cell after next
    __syncthreads();
    if (threadIdx.x == 0 && c + 2 * gridDim.x < a.n_cells)
    {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(c + 2 * gridDim.x, st);
      if (st) issued1++; else issued0++;
    }
  }
  // copies still in flight (after a timeout, or never consumed): bounded waits before the
  // CTA's shared memory is released
  if (threadIdx.x == 0)
  {
    if (issued0 > waited0) (void)lq_wait(&bar[1], (uint32_t)(issued0 - 1) & 1u);
    if (issued1 > waited1) (void)lq_wait(&bar[2], (uint32_t)(issued1 - 1) & 1u);
  }
}

// local matrices and right-hand sides of affine cells from their reference-tensor
// coefficients: A_c[i][j] = sum_t coef_{c,t} R_t[i][j], F_c[i] = sum_u coef_{c,T+u} r_u[i]
// (a [cells x T] x [T x nbf^2] product).  Each thread owns one entry q of the local layout
// and keeps its tensor column R_q in registers; blocks walk a range of cells whose
// coefficients they first copy into shared memory with coalesced loads, so the loop over the
// cells reads them as shared-memory broadcasts (no global-memory latency per cell) and the
// writes are coalesced.  TM bounds the number of tensors at compile time (the exact count of
// the common forms, so the loop carries no predicate; CD_MAXT for any other).
template <int TM>
__global__ void __launch_bounds__(256) affine_local_kernel(int n_cells, int nbf, int T, int Tr,
                                                           const double *__restrict__ cellcoef,
                                                           const double *__restrict__ R,
                                                           const double *__restrict__ r, double *__restrict__ out,
                                                           int cells_per_block)
{
  extern __shared__ double cf_s[]; // cells_per_block x (T + Tr)
  CD_PDL_ENTRY();
  const int per = nbf * nbf + nbf;
  const int q = blockIdx.y * blockDim.x + threadIdx.x;
  const bool act = q < per;
  double Rq[TM];
  int nt = 0, off = T;
  if (act)
  {
    if (q < nbf * nbf)
    {
      nt = T;
      off = 0;
#pragma unroll
      for (int u = 0; u < TM; u++) Rq[u] = u < T ? R[(size_t)q * T + u] : 0.0;
    }
    else
    {
      nt = Tr;
      const int i = q - nbf * nbf;
#pragma unroll
      for (int u = 0; u < TM; u++) Rq[u] = u < Tr ? r[i * Tr + u] : 0.0;
    }
  }
  const int c0 = blockIdx.x * cells_per_block, c1 = min(n_cells, c0 + cells_per_block);
  const int TT = T + Tr;
  for (int e = threadIdx.x; e < (c1 - c0) * TT; e += blockDim.x) cf_s[e] = __ldg(cellcoef + (size_t)c0 * TT + e);
  __syncthreads();
  if (!act) return;
  for (int c = c0; c < c1; c++)
  {
    const double *cf = cf_s + (c - c0) * TT + off;
    double v = 0.0;
    if (nt == TM)
    {
#pragma unroll
      for (int u = 0; u < TM; u++) v += cf[u] * Rq[u];
    }
    else
    {
#pragma unroll
      for (int u = 0; u < TM; u++)
        if (u < nt) v += cf[u] * Rq[u];
    }
    out[(size_t)c * per + q] = v;
  }
}

// ---------------------------------------------------------------------------
// row gather: one group of GS threads per CSR row
// ---------------------------------------------------------------------------
struct GatherArgs
{
  int n_dof, n_active, nbf;
  const int *row_ptr, *kcol, *inc_ptr, *inc;
  const unsigned char *slot; // slot map (ensure_slot_map)
  const double *local, *dir; // local matrices + rhs per cell (n_cells x (nbf^2 + nbf))
  double *a, *rhs, *diag;
  float *a32, *diag32;
  int *err;
};

template <int GS, int MAXROW>
__global__ void __launch_bounds__(256) row_gather_kernel(GatherArgs p)
{
  CD_PDL_ENTRY();
  extern __shared__ double smem[];
  const int nbf = p.nbf;
  double *accs = smem; // groups x MAXROW
  auto tile = cg::tiled_partition<GS>(cg::this_thread_block());
  const int lane = tile.thread_rank(), grp = threadIdx.x / GS;
  double *acc = accs + grp * MAXROW;
  const int ngroups = gridDim.x * (blockDim.x / GS);
  const size_t per = (size_t)nbf * nbf + nbf;
  constexpr int CH = GS < 4 ? GS : 4; // incidences per chunk (at most one per lane of the tile)
  for (int r = blockIdx.x * (blockDim.x / GS) + grp; r < p.n_dof; r += ngroups)
  {
    const int base = p.row_ptr[r], len = p.row_ptr[r + 1] - base;
    if (r >= p.n_active)
    {
      // Dirichlet row: identity row (Assemble2D.C:512, AssembleMat3D.C:811-816)
      for (int s = lane; s < len; s += GS)
      {
        bool d = p.kcol[base + s] == r;
        p.a[base + s] = d ? 1.0 : 0.0;
        if (p.a32) p.a32[base + s] = d ? 1.0f : 0.0f;
      }
      if (lane == 0)
      {
        p.rhs[r] = p.dir ? p.dir[r - p.n_active] : 0.0;
        p.diag[r] = 1.0;
        if (p.diag32) p.diag32[r] = 1.0f;
      }
      continue;
    }
    if (len > MAXROW)
    {
      if (lane == 0) atomicExch(p.err, 2);
      continue;
    }
    for (int s = lane; s < len; s += GS) acc[s] = 0.0;
    tile.sync();
    double racc = 0.0;
    // local matrices with the slot map: every lane first loads its column's value and slot
    // for up to CH incidences (independent loads in flight), then they are added in
    // ascending cell order (the reference's order).  Trip counts are uniform over the tile
    // (cnt is the row's, the column loop runs in whole tile widths), so every lane reaches
    // every tile.sync.
    const int t0 = p.inc_ptr[r], nt = p.inc_ptr[r + 1] - t0;
    for (int q0 = 0; q0 < nt; q0 += CH)
    {
      const int cnt = min(CH, nt - q0);
      const int e_lane = lane < cnt ? __ldg(p.inc + t0 + q0 + lane) : 0;
      double F_lane = 0.0;
      if (lane < cnt)
      {
        const int K = e_lane / nbf, i = e_lane - K * nbf;
        F_lane = __ldg(p.local + (size_t)K * per + (size_t)nbf * nbf + i);
      }
      int eq[CH];
#pragma unroll
      for (int q = 0; q < CH; q++) eq[q] = tile.shfl(e_lane, q);
      for (int jb = 0; jb < nbf; jb += GS)
      {
        const int j = jb + lane;
        const bool act = j < nbf;
        double v[CH];
        int sl[CH];
#pragma unroll
        for (int q = 0; q < CH; q++)
        {
          v[q] = 0.0;
          sl[q] = 0;
          if (act && q < cnt)
          {
            const int K = eq[q] / nbf, i = eq[q] - K * nbf;
            v[q] = __ldg(p.local + (size_t)K * per + (size_t)i * nbf + j);
            sl[q] = __ldg(p.slot + (size_t)(t0 + q0 + q) * nbf + j);
          }
        }
#pragma unroll
        for (int q = 0; q < CH; q++)
          if (q < cnt)
          {
            if (act)
            {
              if (sl[q] >= len) atomicExch(p.err, 1);
              else acc[sl[q]] += v[q];
            }
            tile.sync();
          }
      }
      // rhs in ascending cell order
      for (int q = 0; q < cnt; q++) racc += tile.shfl(F_lane, q);
      tile.sync();
    }
    for (int s = lane; s < len; s += GS)
    {
      double v = acc[s];
      p.a[base + s] = v;
      if (p.a32) p.a32[base + s] = (float)v;
      if (__ldg(p.kcol + base + s) == r)
      {
        p.diag[r] = v;
        if (p.diag32) p.diag32[r] = (float)v;
      }
    }
    if (lane == 0) p.rhs[r] = racc;
    tile.sync();
  }
}

// Row gather of an element with NBF <= 32 local DOFs (Q2 hexahedra): one warp per row, lane j =
// local column j.  Each warp owns a contiguous range of at most kGatherRows rows; it first
// copies the range's CSR and incidence pointers and its incidence entries (contiguous in the
// incidence array) into shared memory with coalesced loads, so a row costs one level of global
// loads: the local-matrix rows and slot-map rows of all its incidences (up to CH at once),
// then the sum into the shared-memory row in ascending cell order (the order of the plain
// gather: the entries are the same bit for bit) and the write.  The diagonal's position comes
// from the slot map (the row's own local column), so column indices are read only for
// Dirichlet rows.  Incidences beyond the first CH, or beyond the staged ones, are loaded and
// added one by one after them.
constexpr int kGatherRows = 64, kGatherInc = 512;

template <int NBF, int MAXROW>
__global__ void __launch_bounds__(256, 4) row_gather_lean_kernel(GatherArgs p, int rows_per_warp)
{
  CD_PDL_ENTRY();
  static_assert(NBF <= 32, "one lane per local column");
  constexpr int CH = 8, PER = NBF * NBF + NBF, NW = 8;
  __shared__ double acc_s[NW][MAXROW];
  // per staged incidence: its entry (cell * NBF + local row) and the offset of its local-matrix
  // row in the local array (cell * PER + local row * NBF)
  __shared__ int rp_s[NW][kGatherRows + 1], ip_s[NW][kGatherRows + 1], e_s[NW][kGatherInc], o_s[NW][kGatherInc];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *acc = acc_s[w];
  const int r0 = (blockIdx.x * NW + w) * rows_per_warp, nrows = min(p.n_dof - r0, rows_per_warp);
  if (nrows <= 0) return; // warp-uniform
  const bool col = lane < NBF;
  for (int k = lane; k <= nrows; k += 32)
  {
    rp_s[w][k] = __ldg(p.row_ptr + r0 + k);
    ip_s[w][k] = __ldg(p.inc_ptr + r0 + k);
  }
  __syncwarp();
  const int T0 = ip_s[w][0], n_staged = min(ip_s[w][nrows] - T0, kGatherInc);
  for (int t = lane; t < n_staged; t += 32)
  {
    const int e = __ldg(p.inc + T0 + t), K = e / NBF, li = e - K * NBF;
    e_s[w][t] = e;
    o_s[w][t] = K * PER + li * NBF;
  }
  __syncwarp();
  auto entry = [&](int t) { return t - T0 < n_staged ? e_s[w][t - T0] : __ldg(p.inc + t); };
  auto local_row = [&](int t) {
    if (t - T0 < n_staged) return p.local + o_s[w][t - T0];
    const int e = __ldg(p.inc + t), K = e / NBF;
    return p.local + (size_t)K * PER + (e - K * NBF) * NBF;
  };
  for (int k = 0; k < nrows; k++)
  {
    const int r = r0 + k, base = rp_s[w][k], len = rp_s[w][k + 1] - base;
    const int t0 = ip_s[w][k], nt = ip_s[w][k + 1] - t0;
    if (r >= p.n_active)
    {
      // Dirichlet row: identity row (Assemble2D.C:512, AssembleMat3D.C:811-816)
      for (int s = lane; s < len; s += 32)
      {
        const bool d = p.kcol[base + s] == r;
        p.a[base + s] = d ? 1.0 : 0.0;
        if (p.a32) p.a32[base + s] = d ? 1.0f : 0.0f;
      }
      if (lane == 0)
      {
        p.rhs[r] = p.dir ? p.dir[r - p.n_active] : 0.0;
        p.diag[r] = 1.0;
        if (p.diag32) p.diag32[r] = 1.0f;
      }
      continue;
    }
    if (len > MAXROW)
    {
      if (lane == 0) atomicExch(p.err, 2);
      continue;
    }
    const int n1 = min(nt, CH);
    // every load of the row's first CH incidences at once
    double v[CH];
    int sl[CH];
    const unsigned char *srow = p.slot + (size_t)t0 * NBF + lane;
#pragma unroll
    for (int q = 0; q < CH; q++)
    {
      v[q] = 0.0;
      sl[q] = 0;
      if (q < n1 && col)
      {
        v[q] = __ldg(local_row(t0 + q) + lane);
        sl[q] = __ldg(srow + q * NBF);
      }
    }
    double F = 0.0; // lane q: the local right-hand side of incidence q
    int e_lane = 0;
    if (lane < n1)
    {
      e_lane = entry(t0 + lane);
      const int K = e_lane / NBF, li = e_lane - K * NBF;
      F = __ldg(p.local + (size_t)K * PER + NBF * NBF + li);
    }
    for (int s = lane; s < len; s += 32) acc[s] = 0.0;
    __syncwarp();
    double racc = 0.0;
#pragma unroll
    for (int q = 0; q < CH; q++)
      if (q < n1)
      {
        if (col)
        {
          if (sl[q] >= len) atomicExch(p.err, 1);
          else acc[sl[q]] += v[q];
        }
        racc += __shfl_sync(0xffffffffu, F, q);
        __syncwarp();
      }
    for (int t = t0 + CH; t < t0 + nt; t++)
    {
      const int eq = entry(t), K = eq / NBF, li = eq - K * NBF;
      if (col)
      {
        const double vv = __ldg(p.local + (size_t)K * PER + li * NBF + lane);
        const int ss = __ldg(p.slot + (size_t)t * NBF + lane);
        if (ss >= len) atomicExch(p.err, 1);
        else acc[ss] += vv;
      }
      racc += __ldg(p.local + (size_t)K * PER + NBF * NBF + li);
      __syncwarp();
    }
    // the diagonal: the slot of the row's own local column in its first incidence
    const int e0 = __shfl_sync(0xffffffffu, e_lane, 0), li0 = e0 - (e0 / NBF) * NBF;
    const int dslot = __shfl_sync(0xffffffffu, sl[0], li0);
    for (int s = lane; s < len; s += 32)
    {
      const double x = acc[s];
      p.a[base + s] = x;
      if (p.a32) p.a32[base + s] = (float)x;
    }
    if (lane == 0)
    {
      p.rhs[r] = racc;
      if (n1 > 0 && dslot < len)
      {
        p.diag[r] = acc[dslot];
        if (p.diag32) p.diag32[r] = (float)acc[dslot];
      }
    }
    __syncwarp();
  }
}

// slot map: for every incidence t of an active row and local column j, the position of the
// column within the row (binary search, once per pattern); 255 and the error flag when the
// coupling is missing from the pattern
__global__ void slot_map_kernel(int n_active, int nbf, const int *__restrict__ row_ptr, const int *__restrict__ kcol,
                                const int *__restrict__ inc_ptr, const int *__restrict__ inc,
                                const int *__restrict__ gn, unsigned char *__restrict__ slot, int *err)
{
  const int r = blockIdx.x;
  if (r >= n_active) return;
  const int base = row_ptr[r], len = row_ptr[r + 1] - base;
  for (int t = inc_ptr[r]; t < inc_ptr[r + 1]; t++)
  {
    const int e = inc[t], K = e / nbf;
    for (int j = threadIdx.x; j < nbf; j += blockDim.x)
    {
      const int col = gn[(size_t)K * nbf + j];
      int lo = 0, hi = len - 1, pos = -1;
      while (lo <= hi)
      {
        int mid = (lo + hi) >> 1, v = kcol[base + mid];
        if (v == col) { pos = mid; break; }
        if (v < col) lo = mid + 1; else hi = mid - 1;
      }
      if (pos < 0 || pos > 254) atomicExch(err, 1);
      slot[(size_t)t * nbf + j] = (unsigned char)(pos < 0 || pos > 254 ? 255 : pos);
    }
  }
}

static int ensure_slot_map(cdgpu_ctx *ctx, Space &s)
{
  if (s.d_slot && s.slot_pattern == s.nnz) return CDGPU_OK;
  // incidences of all DOFs = cells x nbf; the map is indexed by incidence position
  const size_t n_inc = (size_t)s.n_cells * s.nbf;
  int rc = dev_alloc(ctx, &s.d_slot, n_inc * s.nbf);
  if (rc) return rc;
  if (s.n_active > 0)
  {
    slot_map_kernel<<<s.n_active, 32, 0, ctx->stream>>>(s.n_active, s.nbf, s.d_row_ptr, s.d_kcol, s.d_inc_ptr,
                                                         s.d_inc, s.d_gn, s.d_slot, ctx->d_err);
    CD_LAUNCHED(ctx);
  }
  s.slot_pattern = s.nnz;
  return CDGPU_OK;
}

template <int GS, int MAXROW>
static int launch_gather(cdgpu_ctx *ctx, const GatherArgs &g, int n_dof)
{
  int groups = 256 / GS;
  size_t sm = (size_t)groups * MAXROW * sizeof(double);
  const void *key = (const void *)row_gather_kernel<GS, MAXROW>;
  int blocks_per_sm = 0;
  for (auto &e : ctx->occupancy)
    if (e.first == key) blocks_per_sm = e.second;
  if (!blocks_per_sm)
  {
    CD_CUDA(ctx, cudaFuncSetAttribute(row_gather_kernel<GS, MAXROW>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    CD_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm,
                                                               row_gather_kernel<GS, MAXROW>, 256, sm));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
    ctx->occupancy.push_back({key, blocks_per_sm});
  }
  long need = (n_dof + groups - 1) / groups;
  long grid = std::min<long>(need, (long)ctx->sm_count * blocks_per_sm);
  if (grid < 1) grid = 1;
  (void)cd_launch(row_gather_kernel<GS, MAXROW>, (int)grid, 256, sm, ctx->stream, g);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

template <int NBF, int MAXROW> static int launch_gather_lean(cdgpu_ctx *ctx, const GatherArgs &g, int n_dof)
{
  // about four blocks of 8 warps per SM, every warp a contiguous range of at most kGatherRows rows
  const long warps = (long)ctx->sm_count * 4 * 8;
  const int rows_per_warp = (int)std::min<long>(kGatherRows, std::max<long>(1, (n_dof + warps - 1) / warps));
  const long need = ((long)n_dof + rows_per_warp - 1) / rows_per_warp;
  const int grid = (int)std::max<long>(1, (need + 7) / 8);
  (void)cd_launch(row_gather_lean_kernel<NBF, MAXROW>, grid, 256, 0, ctx->stream, g, rows_per_warp);
  CD_LAUNCHED(ctx);
  return CDGPU_OK;
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
int assemble_check(cdgpu_ctx *ctx)
{
  CD_CUDA(ctx, cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return err_flag_status(ctx);
}

// the status of the error flag already copied to ctx->h_err (the flag is cleared when set)
int err_flag_status(cdgpu_ctx *ctx)
{
  int e = *ctx->h_err;
  if (e)
  {
    *ctx->h_err = 0;
    CD_CUDA(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    if (e == 1) return fail(ctx, CDGPU_ERR_PATTERN, "assemble: a cell coupling is missing from the CSR pattern");
    if (e == 3) return fail(ctx, CDGPU_ERR_CUDA, "multigrid: a tensor-core product did not complete in time");
    if (e == 4) return fail(ctx, CDGPU_ERR_CUDA, "CSR product: a bulk copy of a matrix tile did not complete in time");
    if (e == 5) return fail(ctx, CDGPU_ERR_CUDA, "assemble: a bulk copy of cell data or tables did not complete in time");
    if (e == 7) return fail(ctx, CDGPU_ERR_INVALID, "errors: a DOF number outside the space");
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "assemble: CSR row longer than the kernel's row buffer");
  }
  return CDGPU_OK;
}

// the assembly's quadrature rule and basis tables on the device: qx, qw, phi, dphi, hphi
static int ensure_quadtab(cdgpu_ctx *ctx, Space &s)
{
  if (s.d_quadtab) return CDGPU_OK;
  // the tables are the space's reference element's: build it first (a space whose errors are
  // evaluated before any assembly has none yet)
  if (!s.re_ready)
  {
    make_ref_element(s.dim, s.order, s.re);
    s.re_ready = true;
  }
  const RefElement &re = s.re;
  std::vector<double> packed;
  packed.insert(packed.end(), re.qx.begin(), re.qx.end());
  packed.insert(packed.end(), re.qw.begin(), re.qw.end());
  packed.insert(packed.end(), re.phi.begin(), re.phi.end());
  packed.insert(packed.end(), re.dphi.begin(), re.dphi.end());
  packed.insert(packed.end(), re.hphi.begin(), re.hphi.end());
  // two spare doubles: the bulk copy of the tables rounds its size up to 16 bytes
  packed.resize(packed.size() + 2, 0.0);
  int rc = dev_alloc(ctx, &s.d_quadtab, packed.size());
  if (rc) return rc;
  CD_CUDA(ctx, cudaMemcpy(s.d_quadtab, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice));
  return CDGPU_OK;
}

// ---------------------------------------------------------------------------
// L2 and H1-semi errors of a 2D solution against the SineLaplace solution
// u = sin(pi x) sin(pi y) (Examples/CD_2D/SineLaplace.h:27-30), as TFEFunction2D::GetErrors
// (src/FE/FEFunction2D.C:73) computes them: the assembly's Gauss rule on every cell, the
// squared errors summed per thread over its cells, per block in a fixed tree, and the block
// partials on the host in block order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) errors_sine_kernel(int n_cells, int nbf, int nq, int nv, int affine_all,
                                                          const double *__restrict__ coords,
                                                          const int *__restrict__ gn, const double *__restrict__ qx,
                                                          const double *__restrict__ qw,
                                                          const double *__restrict__ phi,
                                                          const double *__restrict__ dphi,
                                                          const double *__restrict__ u, double *__restrict__ partial,
                                                          int n_dof, int *__restrict__ err)
{
  CD_PDL_ENTRY();
  __shared__ double red[2][8];
  double e0 = 0.0, e1 = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells; c += gridDim.x * blockDim.x)
  {
    double V[8];
    for (int k = 0; k < nv * 2; k++) V[k] = coords[(size_t)c * nv * 2 + k];
    for (int q = 0; q < nq; q++)
    {
      double x[3], J[9], Ji[9];
      d_ref_map(2, nv, affine_all != 0, V, qx + 2 * q, x, J);
      const double det = d_invert(2, J, Ji);
      double uh = 0.0, ux = 0.0, uy = 0.0;
      for (int b = 0; b < nbf; b++)
      {
        const double *gr = dphi + (size_t)(q * nbf + b) * 2;
        const double gx = Ji[0] * gr[0] + Ji[2] * gr[1], gy = Ji[1] * gr[0] + Ji[3] * gr[1];
        const int gb = gn[(size_t)c * nbf + b];
        if ((unsigned)gb >= (unsigned)n_dof)
        {
          // a DOF number outside the space: flagged, not read
          atomicExch(err, 7);
          continue;
        }
        const double ub = u[gb];
        uh += ub * phi[q * nbf + b];
        ux += ub * gx;
        uy += ub * gy;
      }
      const double ex = sin(M_PI * x[0]) * sin(M_PI * x[1]);
      const double exx = M_PI * cos(M_PI * x[0]) * sin(M_PI * x[1]);
      const double exy = M_PI * sin(M_PI * x[0]) * cos(M_PI * x[1]);
      const double w = qw[q] * fabs(det);
      e0 += w * (uh - ex) * (uh - ex);
      e1 += w * ((ux - exx) * (ux - exx) + (uy - exy) * (uy - exy));
    }
  }
  for (int o = 16; o > 0; o >>= 1)
  {
    e0 += __shfl_xor_sync(0xffffffffu, e0, o);
    e1 += __shfl_xor_sync(0xffffffffu, e1, o);
  }
  if (threadIdx.x % 32 == 0)
  {
    red[0][threadIdx.x / 32] = e0;
    red[1][threadIdx.x / 32] = e1;
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < 8; w++) { a += red[0][w]; b += red[1][w]; }
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
  }
}

// The same errors against any exact solution the host tabulates at the assembly's quadrature
// points (TFEFunction2D/3D::GetErrors with L2H1Errors, src/FE/FEFunction2D.C:73,
// src/FE/FEFunction3D.C:57): ex[(c*nq + q)*(1+dim) + k] = u, du/dx, du/dy[, du/dz] at point q
// of cell c (the points of cdgpu_quadrature_points); 2D and 3D, any supported element.
__global__ void __launch_bounds__(256) errors_table_kernel(int dim, int n_cells, int nbf, int nq, int nv,
                                                           int affine_all, const double *__restrict__ coords,
                                                           const int *__restrict__ gn, const double *__restrict__ qx,
                                                           const double *__restrict__ qw,
                                                           const double *__restrict__ phi,
                                                           const double *__restrict__ dphi,
                                                           const double *__restrict__ u,
                                                           const double *__restrict__ ex,
                                                           double *__restrict__ partial, int n_dof,
                                                           int *__restrict__ err)
{
  CD_PDL_ENTRY();
  __shared__ double red[2][8];
  double e0 = 0.0, e1 = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells; c += gridDim.x * blockDim.x)
  {
    double V[24];
    for (int k = 0; k < nv * dim; k++) V[k] = coords[(size_t)c * nv * dim + k];
    for (int q = 0; q < nq; q++)
    {
      double x[3], J[9], Ji[9];
      d_ref_map(dim, nv, affine_all != 0, V, qx + dim * q, x, J);
      const double det = d_invert(dim, J, Ji);
      double uh = 0.0, g[3] = {0.0, 0.0, 0.0};
      for (int b = 0; b < nbf; b++)
      {
        const double *gr = dphi + (size_t)(q * nbf + b) * dim;
        const int gb = gn[(size_t)c * nbf + b];
        if ((unsigned)gb >= (unsigned)n_dof)
        {
          // a DOF number outside the space: flagged, not read
          atomicExch(err, 7);
          continue;
        }
        const double ub = u[gb];
        uh += ub * phi[q * nbf + b];
        for (int r = 0; r < dim; r++)
        {
          double s = 0.0;
          for (int e = 0; e < dim; e++) s += Ji[e * dim + r] * gr[e];
          g[r] += ub * s;
        }
      }
      const double *xq = ex + ((size_t)c * nq + q) * (1 + dim);
      const double w = qw[q] * fabs(det);
      e0 += w * (uh - xq[0]) * (uh - xq[0]);
      double s1 = 0.0;
      for (int r = 0; r < dim; r++) s1 += (g[r] - xq[1 + r]) * (g[r] - xq[1 + r]);
      e1 += w * s1;
    }
  }
  for (int o = 16; o > 0; o >>= 1)
  {
    e0 += __shfl_xor_sync(0xffffffffu, e0, o);
    e1 += __shfl_xor_sync(0xffffffffu, e1, o);
  }
  if (threadIdx.x % 32 == 0)
  {
    red[0][threadIdx.x / 32] = e0;
    red[1][threadIdx.x / 32] = e1;
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < 8; w++) { a += red[0][w]; b += red[1][w]; }
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
  }
}

int space_errors_table(cdgpu_ctx *ctx, Space &s, const double *d_u, const double *d_ex, double *l2, double *h1semi)
{
  int rc;
  if (!s.re_ready)
  {
    make_ref_element(s.dim, s.order, s.re);
    s.re_ready = true;
  }
  if ((rc = ensure_err_flag(ctx))) return rc;
  if ((rc = ensure_quadtab(ctx, s))) return rc;
  const RefElement &re = s.re;
  const double *qx = s.d_quadtab, *qw = qx + re.qx.size(), *phi = qw + re.qw.size(), *dphi = phi + re.phi.size();
  const int grid = std::max(1, std::min((s.n_cells + 255) / 256, ctx->sm_count * 4));
  double *d_partial = nullptr;
  if ((rc = dev_alloc(ctx, &d_partial, (size_t)2 * grid))) return rc;
  (void)cd_launch(errors_table_kernel, grid, 256, 0, ctx->stream, s.dim, s.n_cells, s.nbf, re.nq, s.nv,
                  s.all_affine ? 1 : 0, (const double *)s.d_coords, (const int *)s.d_gn, qx, qw, phi, dphi, d_u,
                  d_ex, d_partial, s.n_dof, ctx->d_err);
  cudaError_t e = cudaGetLastError();
  std::vector<double> part((size_t)2 * grid);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(part.data(), d_partial, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_partial);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "errors_table");
  CD_LAUNCHED(ctx);
  double a = 0.0, b = 0.0;
  for (int i = 0; i < grid; i++) { a += part[2 * i]; b += part[2 * i + 1]; }
  *l2 = std::sqrt(a);
  *h1semi = std::sqrt(b);
  return assemble_check(ctx); // the DOF-number check of the kernel
}

int space_errors_sine(cdgpu_ctx *ctx, Space &s, const double *d_u, double *l2, double *h1semi)
{
  if (s.dim != 2 || !s.co_set || s.co.kind != CDGPU_COEFF_SINE)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "errors: only 2D spaces with the sine coefficients (SineLaplace) have an exact solution");
  int rc;
  if ((rc = ensure_err_flag(ctx))) return rc;
  if ((rc = ensure_quadtab(ctx, s))) return rc;
  const RefElement &re = s.re;
  const double *qx = s.d_quadtab, *qw = qx + re.qx.size(), *phi = qw + re.qw.size(), *dphi = phi + re.phi.size();
  const int grid = std::max(1, std::min((s.n_cells + 255) / 256, ctx->sm_count * 4));
  double *d_partial = nullptr;
  if ((rc = dev_alloc(ctx, &d_partial, (size_t)2 * grid))) return rc;
  (void)cd_launch(errors_sine_kernel, grid, 256, 0, ctx->stream, s.n_cells, s.nbf, re.nq, s.nv,
                  s.all_affine ? 1 : 0, (const double *)s.d_coords, (const int *)s.d_gn, qx, qw, phi, dphi, d_u,
                  d_partial, s.n_dof, ctx->d_err);
  cudaError_t e = cudaGetLastError();
  std::vector<double> part((size_t)2 * grid);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(part.data(), d_partial, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_partial);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "errors");
  CD_LAUNCHED(ctx);
  double a = 0.0, b = 0.0;
  for (int i = 0; i < grid; i++) { a += part[2 * i]; b += part[2 * i + 1]; }
  *l2 = std::sqrt(a);
  *h1semi = std::sqrt(b);
  return assemble_check(ctx); // the DOF-number check of the kernel
}

int assemble_space(cdgpu_ctx *ctx, Space &s, int disctype, const double *h_dir, bool check)
{
  if (s.nnz < 0) return fail(ctx, CDGPU_ERR_INVALID, "assemble: no pattern (call cdgpu_build_pattern)");
  if (!s.co_set) return fail(ctx, CDGPU_ERR_INVALID, "assemble: coefficients not set");
  if (disctype != CDGPU_GALERKIN && disctype != CDGPU_SUPG && disctype != CDGPU_MASS)
    return fail(ctx, CDGPU_ERR_UNSUPPORTED, "assemble: DISCTYPE must be GALERKIN (1), SUPG (2) or MASS (10)");
  int rc;
  if (!ctx->d_err)
  {
    if ((rc = dev_alloc(ctx, &ctx->d_err, 1))) return rc;
    CD_CUDA(ctx, cudaMallocHost((void **)&ctx->h_err, sizeof(int)));
    CD_CUDA(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
  }
  if (!s.d_a)
  {
    if ((rc = dev_alloc(ctx, &s.d_a, s.nnz + kCsrPad)) || (rc = dev_alloc(ctx, &s.d_a32, s.nnz + kCsrPad)) ||
        (rc = dev_alloc(ctx, &s.d_rhs, s.n_dof)) || (rc = dev_alloc(ctx, &s.d_diag, s.n_dof)) ||
        (rc = dev_alloc(ctx, &s.d_diag32, s.n_dof)))
      return rc;
  }
  int n_dir = s.n_dof - s.n_active;
  const double *d_dir = nullptr;
  if (h_dir && n_dir > 0)
  {
    if (!s.d_dir && (rc = dev_alloc(ctx, &s.d_dir, n_dir))) return rc;
    CD_CUDA(ctx, cudaMemcpyAsync(s.d_dir, h_dir, sizeof(double) * n_dir, cudaMemcpyHostToDevice,
                                 ctx->stream));
    d_dir = s.d_dir;
  }
  if (!s.re_ready)
  {
    make_ref_element(s.dim, s.order, s.re);
    s.re_ready = true;
  }
  const RefElement &re = s.re;
  bool fast = s.all_affine && s.co.kind == CDGPU_COEFF_CONSTANT;
  int T = n_tensors(s.dim, disctype), Tr = n_rhs_tensors(s.dim, disctype);
  // the matrix-free operator follows the cell coefficients of an affine assembly only
  s.mf_T = fast ? T : 0;
  Coef co = to_coef(s.co);
  if (fast)
  {
    if (s.ref_disctype != disctype)
    {
      std::vector<double> R, r;
      reference_tensors(re, disctype, R, r);
      std::vector<double> both(R);
      both.insert(both.end(), r.begin(), r.end());
      if ((rc = dev_alloc(ctx, &s.d_ref, both.size()))) return rc;
      CD_CUDA(ctx, cudaMemcpy(s.d_ref, both.data(), both.size() * sizeof(double), cudaMemcpyHostToDevice));
      s.ref_disctype = disctype;
    }
    if (!s.d_cellcoef && (rc = dev_alloc(ctx, &s.d_cellcoef, (size_t)s.n_cells * (CD_MAXT + 4))))
      return rc;
    CellCoefArgs a{s.dim, s.nv, s.n_cells, disctype, T, Tr, co, s.d_coords, s.d_cellcoef};
    (void)cd_launch(cell_coef_kernel, (s.n_cells + 127) / 128, 128, 0, ctx->stream, a);
    CD_LAUNCHED(ctx);
    // local matrices of every cell, then the gather with prefetched loads
    if (!s.d_local && (rc = dev_alloc(ctx, &s.d_local, (size_t)s.n_cells * (s.nbf * s.nbf + s.nbf))))
      return rc;
    const int per = s.nbf * s.nbf + s.nbf;
    const int qblocks = (per + 255) / 256;
    // cells per block: about 8 blocks per SM, at most 256 (their coefficients in shared memory)
    const int cpb = std::max(1, std::min(256, (int)((long)s.n_cells * qblocks / ((long)ctx->sm_count * 8))));
    dim3 grid((s.n_cells + cpb - 1) / cpb, qblocks);
    const size_t cf_bytes = sizeof(double) * (size_t)cpb * (T + Tr);
    auto kern = T == 10 ? affine_local_kernel<10> : T == 13 ? affine_local_kernel<13> : T == 6 ? affine_local_kernel<6>
              : T == 14 ? affine_local_kernel<14> : affine_local_kernel<CD_MAXT>;
    (void)cd_launch(kern, grid, 256, cf_bytes, ctx->stream, s.n_cells, s.nbf, T, Tr, s.d_cellcoef, s.d_ref,
                                                       s.d_ref + (size_t)s.nbf * s.nbf * T, s.d_local, cpb);
    CD_LAUNCHED(ctx);
  }
  else
  {
    if ((rc = ensure_quadtab(ctx, s))) return rc;
    const double *d_tab = nullptr;
    if (s.co.kind == CDGPU_COEFF_TABLE)
    {
      if (!s.d_tab) return fail(ctx, CDGPU_ERR_INVALID, "assemble: coefficient table missing");
      d_tab = s.d_tab;
    }
    if (!s.d_local && (rc = dev_alloc(ctx, &s.d_local, (size_t)s.n_cells * (s.nbf * s.nbf + s.nbf))))
      return rc;
    LocalArgs a;
    a.dim = s.dim; a.nv = s.nv; a.nbf = s.nbf; a.nq = re.nq; a.n_cells = s.n_cells;
    a.disctype = disctype; a.affine_all = s.all_affine; a.co = co; a.coords = s.d_coords; a.tab = d_tab;
    a.qtab = s.d_quadtab;
    a.n_qx = (int)re.qx.size(); a.n_qw = (int)re.qw.size(); a.n_phi = (int)re.phi.size();
    a.n_dphi = (int)re.dphi.size();
    // the staged tables: the second derivatives only where 2D SUPG reads them
    a.n_stage_tab = a.n_qx + a.n_qw + a.n_phi + a.n_dphi +
                    (s.dim == 2 && disctype == CDGPU_SUPG ? (int)re.hphi.size() : 0);
    a.out = s.d_local;
    a.err = ctx->d_err;
    const LqLayout lay(s.dim, s.nv, s.nbf, re.nq, disctype, a.n_stage_tab, d_tab != nullptr);
    const size_t sm = sizeof(double) * (size_t)lay.total;
    if (sm > 227 * 1024) return fail(ctx, CDGPU_ERR_UNSUPPORTED, "assemble: quadrature tables exceed shared memory");
    auto kern = s.nbf == 27 ? local_quad_kernel<true> : local_quad_kernel<false>;
    CD_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    CD_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, sm));
    const int grid = std::max(1, std::min(s.n_cells, ctx->sm_count * std::max(1, per_sm)));
    (void)cd_launch(kern, grid, 256, sm, ctx->stream, a);
    CD_LAUNCHED(ctx);
  }
  if ((rc = ensure_slot_map(ctx, s))) return rc;
  GatherArgs g;
  g.n_dof = s.n_dof; g.n_active = s.n_active; g.nbf = s.nbf;
  g.slot = s.d_slot;
  g.row_ptr = s.d_row_ptr; g.kcol = s.d_kcol; g.inc_ptr = s.d_inc_ptr; g.inc = s.d_inc;
  g.local = s.d_local; g.dir = d_dir;
  g.a = s.d_a; g.rhs = s.d_rhs; g.diag = s.d_diag; g.a32 = s.d_a32; g.diag32 = s.d_diag32; g.err = ctx->d_err;
  if (s.dim == 2 && s.order == 1) rc = launch_gather<4, 16>(ctx, g, s.n_dof);
  else if (s.dim == 2) rc = launch_gather<16, 32>(ctx, g, s.n_dof);
  else if (s.order == 1) rc = launch_gather<8, 32>(ctx, g, s.n_dof);
  // (the lean gather keeps local-matrix offsets as 32-bit integers)
  else if (s.nbf == 27 && (long)s.n_cells * (27 * 27 + 27) < (long)INT_MAX)
    rc = launch_gather_lean<27, CD_MAXROW>(ctx, g, s.n_dof);
  else rc = launch_gather<32, CD_MAXROW>(ctx, g, s.n_dof);
  if (rc) return rc;
  s.assembled = true;
  s.assembly_version++;
  return check ? assemble_check(ctx) : CDGPU_OK;
}

// ---------------------------------------------------------------------------
// Neumann data (Assemble2D.C:797-827): one CTA, edges in order, so every DOF's sum
// runs in the same order on every call.
// ---------------------------------------------------------------------------
__global__ void neumann_kernel(int order, int nbf, int n_edges, const double *coords,
                               const int *gn, int n_active, const int *cell, const int *edge,
                               const double *g, double *rhs)
{
  const double r2[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  int nl = order + 1;
  double z[4], w[4];
  if (nl == 2) { z[0] = -1.0 / sqrt(3.0); z[1] = -z[0]; w[0] = w[1] = 1.0; }
  else { z[0] = -sqrt(0.6); z[1] = 0; z[2] = sqrt(0.6); w[0] = w[2] = 5.0 / 9.0; w[1] = 8.0 / 9.0; }
  for (int e = 0; e < n_edges; e++)
  {
    int c = cell[e], m = edge[e], m1 = (m + 1) % 4;
    const double *V = coords + (size_t)c * 8;
    double hE = sqrt((V[2 * m1] - V[2 * m]) * (V[2 * m1] - V[2 * m]) +
                     (V[2 * m1 + 1] - V[2 * m + 1]) * (V[2 * m1 + 1] - V[2 * m + 1])) / 2;
    int k = threadIdx.x;
    if (k < nbf)
    {
      int kx = k % (order + 1), ky = k / (order + 1);
      double add = 0;
      for (int l = 0; l < nl; l++)
      {
        double s = 0.5 * (z[l] + 1);
        double xi = r2[m][0] + (r2[m1][0] - r2[m][0]) * s, eta = r2[m][1] + (r2[m1][1] - r2[m][1]) * s;
        double vx, vy;
        if (order == 1) { vx = kx ? 0.5 * (1 + xi) : 0.5 * (1 - xi); vy = ky ? 0.5 * (1 + eta) : 0.5 * (1 - eta); }
        else
        {
          vx = kx == 0 ? 0.5 * xi * (xi - 1) : kx == 1 ? 1 - xi * xi : 0.5 * xi * (xi + 1);
          vy = ky == 0 ? 0.5 * eta * (eta - 1) : ky == 1 ? 1 - eta * eta : 0.5 * eta * (eta + 1);
        }
        add += g[e * nl + l] * hE * w[l] * vx * vy;
      }
      int d = gn[(size_t)c * nbf + k];
      if (d < n_active) rhs[d] += add;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Neumann data on hexahedron faces (the NEUMANN / ROBIN branch of TAssembleMat3D::Assemble3D,
// src/System/AssembleMat3D.C:1068-1170): face m of a cell has the vertices kHexFace[m]
// (THexahedron's face-vertex table) and the bilinear map of the face square [-1,1]^2 through
// them; per Gauss point (t_i, s_j) of an (order+1)^2 rule the area element |n| is the norm of
// the cross product of the map's two derivatives, and the basis functions are evaluated at the
// same bilinear combination of the reference cube's face corners.  One CTA, faces in order.
// ---------------------------------------------------------------------------
__constant__ int kHexFace[6][4] = {{0, 1, 2, 3}, {0, 4, 5, 1}, {1, 5, 6, 2}, {2, 6, 7, 3}, {0, 3, 7, 4}, {4, 7, 6, 5}};

__host__ __device__ inline void gauss_1d(int nl, double *z, double *w)
{
  if (nl == 2) { z[0] = -1.0 / sqrt(3.0); z[1] = -z[0]; w[0] = w[1] = 1.0; }
  else { z[0] = -sqrt(0.6); z[1] = 0; z[2] = sqrt(0.6); w[0] = w[2] = 5.0 / 9.0; w[1] = 8.0 / 9.0; }
}

__device__ inline double lagrange_1d(int order, int k, double x)
{
  if (order == 1) return k ? 0.5 * (1 + x) : 0.5 * (1 - x);
  return k == 0 ? 0.5 * x * (x - 1) : k == 1 ? 1 - x * x : 0.5 * x * (x + 1);
}

__global__ void neumann3d_kernel(int order, int nbf, int n_faces, const double *coords, const int *gn, int n_active,
                                 const int *cell, const int *face, const double *g, double *rhs)
{
  const int nl = order + 1, nq = nl * nl, p1 = order + 1;
  double z[3], w[3];
  gauss_1d(nl, z, w);
  for (int e = 0; e < n_faces; e++)
  {
    const int c = cell[e], m = face[e];
    const double *V = coords + (size_t)c * 24;
    double X[4][3], R[4][3];
    for (int k = 0; k < 4; k++)
    {
      const int v = kHexFace[m][k];
      for (int a = 0; a < 3; a++) X[k][a] = V[v * 3 + a];
      R[k][0] = (v == 1 || v == 2 || v == 5 || v == 6) ? 1.0 : -1.0;
      R[k][1] = (v == 2 || v == 3 || v == 6 || v == 7) ? 1.0 : -1.0;
      R[k][2] = v >= 4 ? 1.0 : -1.0;
    }
    double c1[3], c2[3], c3[3];
    for (int a = 0; a < 3; a++)
    {
      c1[a] = (-X[0][a] + X[1][a] + X[2][a] - X[3][a]) * 0.25;
      c2[a] = (-X[0][a] - X[1][a] + X[2][a] + X[3][a]) * 0.25;
      c3[a] = (X[0][a] - X[1][a] + X[2][a] - X[3][a]) * 0.25;
    }
    const int k = threadIdx.x;
    if (k < nbf)
    {
      const int kx = k % p1, ky = (k / p1) % p1, kz = k / (p1 * p1);
      double add = 0;
      for (int q = 0; q < nq; q++)
      {
        const double t = z[q % nl], s = z[q / nl];
        const double t0 = 0.5 * (t + 1), t1 = 0.5 * (s + 1);
        const double L[4] = {(1 - t0) * (1 - t1), t0 * (1 - t1), t0 * t1, (1 - t0) * t1};
        double xi[3] = {0, 0, 0};
        for (int j = 0; j < 4; j++)
          for (int a = 0; a < 3; a++) xi[a] += L[j] * R[j][a];
        double d1[3], d2[3];
        for (int a = 0; a < 3; a++)
        {
          d1[a] = c1[a] + s * c3[a];
          d2[a] = c2[a] + t * c3[a];
        }
        const double nx = d1[1] * d2[2] - d1[2] * d2[1], ny = d1[2] * d2[0] - d1[0] * d2[2],
                     nz = d1[0] * d2[1] - d1[1] * d2[0];
        const double phi = lagrange_1d(order, kx, xi[0]) * lagrange_1d(order, ky, xi[1]) * lagrange_1d(order, kz, xi[2]);
        add += g[(size_t)e * nq + q] * w[q % nl] * w[q / nl] * sqrt(nx * nx + ny * ny + nz * nz) * phi;
      }
      const int d = gn[(size_t)c * nbf + k];
      if (d < n_active) rhs[d] += add;
    }
    __syncthreads();
  }
}

// physical coordinates of the Gauss points of boundary edges (2D) or faces (3D), in the order
// add_neumann expects the data: 2D (order+1) points from vertex m towards m+1; 3D (order+1)^2
// points q = i + (order+1) j at (t_i, s_j) of the face's bilinear map
void boundary_points(const Space &s, int n, const int *cell, const int *local, double *xyz)
{
  const int nl = s.order + 1;
  double z[3], w[3];
  gauss_1d(nl, z, w);
  static const int hf[6][4] = {{0, 1, 2, 3}, {0, 4, 5, 1}, {1, 5, 6, 2}, {2, 6, 7, 3}, {0, 3, 7, 4}, {4, 7, 6, 5}};
  for (int e = 0; e < n; e++)
  {
    const double *V = &s.h_coords[(size_t)cell[e] * s.nv * s.dim];
    const int m = local[e];
    if (s.dim == 2)
    {
      const int m1 = (m + 1) % 4;
      for (int l = 0; l < nl; l++)
      {
        const double t = 0.5 * (z[l] + 1);
        for (int a = 0; a < 2; a++) xyz[((size_t)e * nl + l) * 2 + a] = V[2 * m + a] + (V[2 * m1 + a] - V[2 * m + a]) * t;
      }
    }
    else
      for (int q = 0; q < nl * nl; q++)
      {
        const double t0 = 0.5 * (z[q % nl] + 1), t1 = 0.5 * (z[q / nl] + 1);
        const double L[4] = {(1 - t0) * (1 - t1), t0 * (1 - t1), t0 * t1, (1 - t0) * t1};
        for (int a = 0; a < 3; a++)
        {
          double x = 0;
          for (int j = 0; j < 4; j++) x += L[j] * V[hf[m][j] * 3 + a];
          xyz[((size_t)e * nl * nl + q) * 3 + a] = x;
        }
      }
  }
}

int add_neumann(cdgpu_ctx *ctx, Space &s, int n_edges, const int *cell, const int *edge,
                const double *g)
{
  if (!s.assembled) return fail(ctx, CDGPU_ERR_INVALID, "Neumann data: assemble first");
  if (n_edges <= 0) return CDGPU_OK;
  int nl = s.dim == 2 ? s.order + 1 : (s.order + 1) * (s.order + 1), rc;
  const int max_local = s.dim == 2 ? 3 : 5;
  int *d_cell = nullptr, *d_edge = nullptr;
  double *d_g = nullptr;
  if ((rc = dev_alloc(ctx, &d_cell, n_edges)) || (rc = dev_alloc(ctx, &d_edge, n_edges)) ||
      (rc = dev_alloc(ctx, &d_g, (size_t)n_edges * nl)))
    return rc;
  for (int e = 0; e < n_edges; e++)
    if (cell[e] < 0 || cell[e] >= s.n_cells || edge[e] < 0 || edge[e] > max_local)
    {
      cudaFree(d_cell); cudaFree(d_edge); cudaFree(d_g);
      return fail(ctx, CDGPU_ERR_INVALID, "Neumann data: bad cell or edge/face index");
    }
  CD_CUDA(ctx, cudaMemcpyAsync(d_cell, cell, sizeof(int) * n_edges, cudaMemcpyHostToDevice, ctx->stream));
  CD_CUDA(ctx, cudaMemcpyAsync(d_edge, edge, sizeof(int) * n_edges, cudaMemcpyHostToDevice, ctx->stream));
  CD_CUDA(ctx, cudaMemcpyAsync(d_g, g, sizeof(double) * n_edges * nl, cudaMemcpyHostToDevice, ctx->stream));
  if (s.dim == 2)
    neumann_kernel<<<1, 32, 0, ctx->stream>>>(s.order, s.nbf, n_edges, s.d_coords, s.d_gn, s.n_active,
                                              d_cell, d_edge, d_g, s.d_rhs);
  else
    neumann3d_kernel<<<1, 32, 0, ctx->stream>>>(s.order, s.nbf, n_edges, s.d_coords, s.d_gn, s.n_active,
                                                d_cell, d_edge, d_g, s.d_rhs);
  CD_LAUNCHED(ctx);
  CD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(d_cell); cudaFree(d_edge); cudaFree(d_g);
  return CDGPU_OK;
}
