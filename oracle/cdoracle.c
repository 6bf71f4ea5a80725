/*
 * cdoracle.c -- CPU restatement of ParMooN's scalar convection-diffusion path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the GPU kernels are
 * checked against; the product (libcdgpu) never links, loads or calls it.
 * Its own correctness is pinned by tests/ against arrays dumped by the
 * compiled reference (oracle/_ref, built by oracle/build_ref.py) and against
 * the reference's recorded known answers (ReadIn/cd2d.out).
 *
 * Each routine cites the reference function it restates.  Local DOF order is
 * the reference's tensor-product order (x fastest), cell vertices are in the
 * reference's counter-clockwise order, and the affine/multilinear reference
 * maps follow src/FE/QuadAffin.C:602, src/FE/HexaAffin.C:865 and their
 * bilinear/trilinear counterparts.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXBF 27
#define MAXQ 64
#define MAXV 8

/* ------------------------------------------------------------------------- */
/* quadrature: src/QuadFormulas/QuadFormulaHexa.C:62 (Gauss3), :90 (Gauss4),  */
/* QuadFormulaQuad.C, QuadFormula1D.C; tensor products with x fastest.        */
/* ------------------------------------------------------------------------- */
static void gauss1d(int n, double *x, double *w)
{
  if (n == 1) { x[0] = 0; w[0] = 2; }
  else if (n == 2)
  {
    double a = 1.0 / sqrt(3.0);
    x[0] = -a; x[1] = a; w[0] = w[1] = 1.0;
  }
  else if (n == 3)
  {
    double a = sqrt(3.0 / 5.0);
    x[0] = -a; x[1] = 0; x[2] = a;
    w[0] = w[2] = 5.0 / 9.0; w[1] = 8.0 / 9.0;
  }
  else
  {
    /* point order of QuadFormulaHexa.C:97-101: a, b, -b, -a */
    double a = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
    double b = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
    double wa = (18.0 + sqrt(30.0)) / 36.0, wb = (18.0 - sqrt(30.0)) / 36.0;
    x[0] = a; x[1] = b; x[2] = -b; x[3] = -a;
    w[0] = wa; w[1] = wb; w[2] = wb; w[3] = wa;
  }
}

/* Gauss points per direction used by the assembly for order p: the reference
 * selects the rule of degree 3p (src/FE/FEDatabase2D.C:1841, FEDatabase3D.C:1184,
 * tables at FEDatabase2D.C:1677 and FEDatabase3D.C:1009): Q1 -> Gauss3, Q2 -> Gauss4. */
int cdo_gauss_points(int order) { return order == 1 ? 3 : 4; }

int cdo_nbf(int dim, int order)
{
  int k = order + 1;
  return dim == 2 ? k * k : k * k * k;
}

int cdo_quadrature(int dim, int n1, double *xi, double *w)
{
  double x[4], ww[4];
  gauss1d(n1, x, ww);
  int l = 0;
  if (dim == 2)
  {
    for (int j = 0; j < n1; j++)
      for (int k = 0; k < n1; k++, l++)
      {
        xi[2 * l] = x[k]; xi[2 * l + 1] = x[j]; w[l] = ww[j] * ww[k];
      }
  }
  else
  {
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n1; j++)
        for (int k = 0; k < n1; k++, l++)
        {
          xi[3 * l] = x[k]; xi[3 * l + 1] = x[j]; xi[3 * l + 2] = x[i];
          w[l] = ww[i] * ww[j] * ww[k];
        }
  }
  return l;
}

/* ------------------------------------------------------------------------- */
/* basis functions: include/FE2D/BF_C_Q_Q1_2D.h, BF_C_Q_Q2_2D.h,             */
/* include/FE3D/BF_C_H_Q1_3D.h, BF_C_H_Q2_3D.h -- tensor-product Lagrange     */
/* polynomials on [-1,1] with nodes {-1,1} (Q1) or {-1,0,1} (Q2).            */
/* ------------------------------------------------------------------------- */
static void lag1d(int order, double t, double *v, double *d, double *dd)
{
  if (order == 1)
  {
    v[0] = 0.5 * (1 - t); v[1] = 0.5 * (1 + t);
    d[0] = -0.5; d[1] = 0.5;
    dd[0] = dd[1] = 0;
  }
  else
  {
    v[0] = 0.5 * t * (t - 1); v[1] = 1 - t * t; v[2] = 0.5 * t * (t + 1);
    d[0] = t - 0.5; d[1] = -2 * t; d[2] = t + 0.5;
    dd[0] = 1; dd[1] = -2; dd[2] = 1;
  }
}

/* values, reference gradients and reference Hessians (row-major dim x dim) */
void cdo_basis(int dim, int order, const double *xi, double *val, double *grad, double *hess)
{
  int k = order + 1;
  double v[3][3], d[3][3], dd[3][3];
  for (int a = 0; a < dim; a++) lag1d(order, xi[a], v[a], d[a], dd[a]);
  if (dim == 2)
  {
    for (int iy = 0; iy < k; iy++)
      for (int ix = 0; ix < k; ix++)
      {
        int b = ix + k * iy;
        val[b] = v[0][ix] * v[1][iy];
        if (grad)
        {
          grad[2 * b] = d[0][ix] * v[1][iy];
          grad[2 * b + 1] = v[0][ix] * d[1][iy];
        }
        if (hess)
        {
          hess[4 * b + 0] = dd[0][ix] * v[1][iy];
          hess[4 * b + 1] = d[0][ix] * d[1][iy];
          hess[4 * b + 2] = d[0][ix] * d[1][iy];
          hess[4 * b + 3] = v[0][ix] * dd[1][iy];
        }
      }
  }
  else
  {
    for (int iz = 0; iz < k; iz++)
      for (int iy = 0; iy < k; iy++)
        for (int ix = 0; ix < k; ix++)
        {
          int b = ix + k * iy + k * k * iz;
          val[b] = v[0][ix] * v[1][iy] * v[2][iz];
          if (grad)
          {
            grad[3 * b] = d[0][ix] * v[1][iy] * v[2][iz];
            grad[3 * b + 1] = v[0][ix] * d[1][iy] * v[2][iz];
            grad[3 * b + 2] = v[0][ix] * v[1][iy] * d[2][iz];
          }
          if (hess)
          {
            double *h = hess + 9 * b;
            h[0] = dd[0][ix] * v[1][iy] * v[2][iz];
            h[4] = v[0][ix] * dd[1][iy] * v[2][iz];
            h[8] = v[0][ix] * v[1][iy] * dd[2][iz];
            h[1] = h[3] = d[0][ix] * d[1][iy] * v[2][iz];
            h[2] = h[6] = d[0][ix] * v[1][iy] * d[2][iz];
            h[5] = h[7] = v[0][ix] * d[1][iy] * d[2][iz];
          }
        }
  }
}

/* reference-cell position of local node b (tensor index) */
static void node_pos(int dim, int order, int b, double *xi)
{
  int k = order + 1;
  int ix = b % k, iy = (b / k) % k, iz = b / (k * k);
  double h = 2.0 / order;
  xi[0] = -1 + h * ix;
  xi[1] = -1 + h * iy;
  if (dim == 3) xi[2] = -1 + h * iz;
}

/* ------------------------------------------------------------------------- */
/* geometry: vertex shape functions of the reference maps.  Vertex order is   */
/* counter-clockwise: 2D (-1,-1),(1,-1),(1,1),(-1,1); 3D the same at zeta=-1, */
/* then at zeta=+1 (src/FE/QuadBilinear.C, src/FE/HexaTrilinear.C).          */
/* ------------------------------------------------------------------------- */
static const double RV2[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
static const double RV3[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                 {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

static int nverts(int dim) { return dim == 2 ? 4 : 8; }

/* true when the cell is a parallelogram / parallelepiped, i.e. the reference
 * uses QuadAffin / HexaAffin (constant Jacobian) for it */
static int cell_is_affine(int dim, const double *V)
{
  double scale = 0;
  int nv = nverts(dim);
  for (int i = 0; i < nv * dim; i++) scale = fmax(scale, fabs(V[i]));
  double tol = 1e-12 * (scale > 0 ? scale : 1);
  for (int a = 0; a < dim; a++)
  {
#define X(v) V[(v) * dim + a]
    if (dim == 2)
    {
      if (fabs(X(0) + X(2) - X(1) - X(3)) > tol) return 0;
    }
    else
    {
      if (fabs(X(2) - (X(1) + X(3) - X(0))) > tol) return 0;
      if (fabs(X(5) - (X(1) + X(4) - X(0))) > tol) return 0;
      if (fabs(X(7) - (X(3) + X(4) - X(0))) > tol) return 0;
      if (fabs(X(6) - (X(1) + X(3) + X(4) - 2 * X(0))) > tol) return 0;
    }
#undef X
  }
  return 1;
}

/* map a reference point: x = F(xi), J[a][b] = dx_a / dxi_b */
static void ref_map(int dim, int affine, const double *V, const double *xi, double *x, double *J)
{
  if (affine)
  {
    /* QuadAffin::SetCell (src/FE/QuadAffin.C:624-633), HexaAffin::SetCell (src/FE/HexaAffin.C:877-895) */
    for (int a = 0; a < dim; a++)
    {
      double c1 = (V[1 * dim + a] - V[0 * dim + a]) * 0.5;
      double c2 = (V[3 * dim + a] - V[0 * dim + a]) * 0.5;
      if (dim == 2)
      {
        double c0 = (V[1 * dim + a] + V[3 * dim + a]) * 0.5;
        x[a] = c0 + c1 * xi[0] + c2 * xi[1];
        J[a * 2 + 0] = c1; J[a * 2 + 1] = c2;
      }
      else
      {
        double c3 = (V[4 * dim + a] - V[0 * dim + a]) * 0.5;
        double c0 = (V[1 * dim + a] + V[3 * dim + a] + V[4 * dim + a] - V[0 * dim + a]) * 0.5;
        x[a] = c0 + c1 * xi[0] + c2 * xi[1] + c3 * xi[2];
        J[a * 3 + 0] = c1; J[a * 3 + 1] = c2; J[a * 3 + 2] = c3;
      }
    }
    return;
  }
  int nv = nverts(dim);
  for (int a = 0; a < dim; a++)
  {
    x[a] = 0;
    for (int b = 0; b < dim; b++) J[a * dim + b] = 0;
  }
  for (int v = 0; v < nv; v++)
  {
    double N = 1, dN[3];
    const double *r = dim == 2 ? RV2[v] : RV3[v];
    double f[3];
    for (int b = 0; b < dim; b++) f[b] = 0.5 * (1 + r[b] * xi[b]);
    for (int b = 0; b < dim; b++) N *= f[b];
    for (int b = 0; b < dim; b++)
    {
      dN[b] = 0.5 * r[b];
      for (int c = 0; c < dim; c++)
        if (c != b) dN[b] *= f[c];
    }
    for (int a = 0; a < dim; a++)
    {
      x[a] += N * V[v * dim + a];
      for (int b = 0; b < dim; b++) J[a * dim + b] += dN[b] * V[v * dim + a];
    }
  }
}

/* determinant and inverse (Jinv[b][a] = dxi_b/dx_a) */
static double inv(int dim, const double *J, double *Ji)
{
  if (dim == 2)
  {
    double det = J[0] * J[3] - J[1] * J[2];
    Ji[0] = J[3] / det; Ji[1] = -J[1] / det;
    Ji[2] = -J[2] / det; Ji[3] = J[0] / det;
    return det;
  }
  double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
               J[2] * (J[3] * J[7] - J[4] * J[6]);
  Ji[0] = (J[4] * J[8] - J[5] * J[7]) / det;
  Ji[1] = (J[2] * J[7] - J[1] * J[8]) / det;
  Ji[2] = (J[1] * J[5] - J[2] * J[4]) / det;
  Ji[3] = (J[5] * J[6] - J[3] * J[8]) / det;
  Ji[4] = (J[0] * J[8] - J[2] * J[6]) / det;
  Ji[5] = (J[2] * J[3] - J[0] * J[5]) / det;
  Ji[6] = (J[3] * J[7] - J[4] * J[6]) / det;
  Ji[7] = (J[1] * J[6] - J[0] * J[7]) / det;
  Ji[8] = (J[0] * J[4] - J[1] * J[3]) / det;
  return det;
}

/* cell diameter, CELL_MEASURE 0: src/Geometry/Quadrangle.C:35 (longer diagonal),
 * src/Geometry/Hexahedron.C:78 (longest space diagonal) */
static double cell_diameter(int dim, const double *V)
{
  double best = 0;
  if (dim == 2)
  {
    int p[2][2] = {{0, 2}, {1, 3}};
    for (int i = 0; i < 2; i++)
    {
      double dx = V[2 * p[i][0]] - V[2 * p[i][1]], dy = V[2 * p[i][0] + 1] - V[2 * p[i][1] + 1];
      best = fmax(best, dx * dx + dy * dy);
    }
  }
  else
  {
    int p[4][2] = {{0, 6}, {1, 7}, {2, 4}, {3, 5}};
    for (int i = 0; i < 4; i++)
    {
      double s = 0;
      for (int a = 0; a < 3; a++)
      {
        double d = V[3 * p[i][0] + a] - V[3 * p[i][1] + a];
        s += d * d;
      }
      best = fmax(best, s);
    }
  }
  return sqrt(best);
}

/* ------------------------------------------------------------------------- */
/* coefficients                                                              */
/* ------------------------------------------------------------------------- */
typedef struct
{
  int kind;     /* 0 constant, 1 sine problem (2D), 2 rotating convection (2D), 3 table */
  int order_pd; /* INTERNAL_POLYNOMIAL_DEGREE used by the SUPG parameter (default 1) */
  double eps, b1, b2, b3, c, f;
  double delta0; /* DELTA0 (default 1) */
} cdo_coeffs;

/* coefficient record at a point: eps, b1, b2, b3, c, f */
static void coeff_at(const cdo_coeffs *co, const double *tab, const double *x, double *k)
{
  k[0] = co->eps; k[1] = co->b1; k[2] = co->b2; k[3] = co->b3; k[4] = co->c; k[5] = co->f;
  if (co->kind == 1)
  {
    /* sine problem: f = 2 pi^2 eps sin(pi x) sin(pi y), b = 0, c = 0 */
    k[1] = k[2] = k[3] = k[4] = 0;
    k[5] = 2 * M_PI * M_PI * co->eps * sin(M_PI * x[0]) * sin(M_PI * x[1]);
  }
  else if (co->kind == 2)
  {
    /* rotating convection b = (0.5 - y, x - 0.5) */
    k[1] = -x[1] + 0.5;
    k[2] = x[0] - 0.5;
  }
  else if (co->kind == 3 && tab)
  {
    for (int i = 0; i < 6; i++) k[i] = tab[i];
  }
}

/* SDFEM_TYPE 2 stabilisation parameter: src/FE/ConvDiff.C:490-582 (case 1/2) with
 * CELL_MEASURE 0 (h_K = diameter), nu = 1/INTERNAL_POLYNOMIAL_DEGREE */
static double sdfem_delta(double hK, double eps, double b1, double b2, double b3, double delta0,
                          int polydeg)
{
  if (fabs(eps) < 1e-20) eps = 1e-20;
  double nb = sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  double nu = 1.0 / polydeg;
  double delta;
  if (nb > 0)
  {
    double alpha = nu * nb * hK / (2 * eps);
    delta = nu * hK * (1 / tanh(alpha) - 1 / alpha) / (2 * nb);
  }
  else
    delta = 0;
  return delta * delta0;
}

/* ------------------------------------------------------------------------- */
/* CSR pattern: TSquareStructure2D/3D(TFESpace*) (src/FE/SquareStructure3D.C:32,    */
/* SquareStructure2D.C:46) followed by Sort() (src/FE/SquareStructure.C:65):        */
/* active rows couple to every DOF of every cell containing them, Dirichlet rows    */
/* hold the diagonal only, columns ascending.  Returns nnz; fills row_ptr always   */
/* and kcol when non-NULL.                                                          */
/* ------------------------------------------------------------------------- */
static int cmp_int(const void *a, const void *b)
{
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

long cdo_pattern(int n_cells, const int *gn, const int *bi, int n_dof, int n_active, int *row_ptr,
                 int *kcol)
{
  /* cells per DOF */
  int *cnt = calloc(n_dof + 1, sizeof(int));
  for (int c = 0; c < n_cells; c++)
    for (int j = bi[c]; j < bi[c + 1]; j++) cnt[gn[j] + 1]++;
  for (int i = 0; i < n_dof; i++) cnt[i + 1] += cnt[i];
  int *cells = malloc(sizeof(int) * (cnt[n_dof] + 1));
  int *fill = calloc(n_dof, sizeof(int));
  for (int c = 0; c < n_cells; c++)
    for (int j = bi[c]; j < bi[c + 1]; j++)
    {
      int d = gn[j];
      cells[cnt[d] + fill[d]++] = c;
    }
  int *mark = malloc(sizeof(int) * n_dof);
  for (int i = 0; i < n_dof; i++) mark[i] = -1;
  int *buf = malloc(sizeof(int) * (n_dof + 1));
  long nnz = 0;
  row_ptr[0] = 0;
  for (int r = 0; r < n_dof; r++)
  {
    int m = 0;
    if (r < n_active)
    {
      for (int t = cnt[r]; t < cnt[r + 1]; t++)
      {
        int c = cells[t];
        for (int j = bi[c]; j < bi[c + 1]; j++)
          if (mark[gn[j]] != r) { mark[gn[j]] = r; buf[m++] = gn[j]; }
      }
      qsort(buf, m, sizeof(int), cmp_int);
    }
    else
      buf[m++] = r;
    if (kcol)
      for (int t = 0; t < m; t++) kcol[nnz + t] = buf[t];
    nnz += m;
    row_ptr[r + 1] = (int)nnz;
  }
  free(cnt); free(cells); free(fill); free(mark); free(buf);
  return nnz;
}

static long find_slot(const int *row_ptr, const int *kcol, int r, int c)
{
  int lo = row_ptr[r], hi = row_ptr[r + 1] - 1;
  while (lo <= hi)
  {
    int mid = (lo + hi) >> 1;
    if (kcol[mid] == c) return mid;
    if (kcol[mid] < c) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

/* ------------------------------------------------------------------------- */
/* assembly: TSystemCD2D::Assemble -> Assemble2D (src/FE/Assemble2D.C:247-770) and  */
/* TSystemCD3D::Assemble -> TAssembleMat3D::Assemble3D (src/System/AssembleMat3D.C: */
/* 230-505), local forms BilinearAssembleGalerkin / BilinearAssemble_SD             */
/* (src/FE/ConvDiff2D.C:32,96), BilinearAssemble / BilinearAssemble_SD              */
/* (src/FE/ConvDiff3D.C:61,124).  Entries and rhs are zeroed first (Reset).         */
/* disctype 1 = Galerkin, 2 = SUPG.  dir_vals: values of the Dirichlet DOFs          */
/* [hanging_bound, n_dof) (the reference's BoundValue at the nodal points), may be  */
/* NULL for homogeneous data.  coeff_tab (kind 3): [cell][q][6].                    */
/* Returns 0, or -1 when a cell pair is missing from the pattern.                   */
/* ------------------------------------------------------------------------- */
int cdo_assemble(int dim, int order, int disctype, int n_cells, const double *coords,
                 const int *gn, const int *bi, int n_dof, int n_active, const int *row_ptr,
                 const int *kcol, const cdo_coeffs *co, const double *coeff_tab,
                 const double *dir_vals, double *entries, double *rhs)
{
  int nbf = cdo_nbf(dim, order), n1 = cdo_gauss_points(order);
  double qx[MAXQ * 3], qw[MAXQ];
  int nq = cdo_quadrature(dim, n1, qx, qw);
  static double phi[MAXQ][MAXBF], dphi[MAXQ][MAXBF * 3], hphi[MAXQ][MAXBF * 9];
  for (int q = 0; q < nq; q++) cdo_basis(dim, order, qx + q * dim, phi[q], dphi[q], hphi[q]);
  int nv = nverts(dim);
  long nnz = row_ptr[n_dof];
  memset(entries, 0, sizeof(double) * nnz);
  memset(rhs, 0, sizeof(double) * n_dof);
  double A[MAXBF][MAXBF], F[MAXBF];
  for (int c = 0; c < n_cells; c++)
  {
    const double *V = coords + (size_t)c * nv * dim;
    int affine = cell_is_affine(dim, V);
    double hK = cell_diameter(dim, V);
    memset(A, 0, sizeof(A));
    memset(F, 0, sizeof(F));
    for (int q = 0; q < nq; q++)
    {
      double x[3], J[9], Ji[9], g[MAXBF][3], lap[MAXBF], k[6];
      ref_map(dim, affine, V, qx + q * dim, x, J);
      double det = inv(dim, J, Ji);
      double mult = qw[q] * fabs(det);
      for (int b = 0; b < nbf; b++)
      {
        for (int a = 0; a < dim; a++)
        {
          double s = 0;
          for (int e = 0; e < dim; e++) s += Ji[e * dim + a] * dphi[q][b * dim + e];
          g[b][a] = s;
        }
        lap[b] = 0;
        if (dim == 2 && disctype == 2)
        {
          /* physical second derivatives D2 = Ji^T (H - G) Ji.  G is zero for an affine map; for
             the bilinear map x = c0 + c1 xi + c2 eta + c3 xi eta its off-diagonal entries are
             grad(phi) . c3, the term the D11 row of the reference's 5x5 system carries
             (xc3, yc3 in src/FE/QuadBilinear.C:531-549) */
          double gm = 0;
          if (!affine)
            for (int a = 0; a < 2; a++)
              gm += g[b][a] * 0.25 * (V[0 * 2 + a] - V[1 * 2 + a] + V[2 * 2 + a] - V[3 * 2 + a]);
          for (int a = 0; a < 2; a++)
            for (int e = 0; e < 2; e++)
              for (int f = 0; f < 2; f++)
                lap[b] += Ji[e * 2 + a] * Ji[f * 2 + a] * (hphi[q][b * 4 + e * 2 + f] - (e != f ? gm : 0.0));
        }
      }
      coeff_at(co, coeff_tab ? coeff_tab + ((size_t)c * nq + q) * 6 : NULL, x, k);
      double eps = k[0], b1 = k[1], b2 = k[2], b3 = dim == 3 ? k[3] : 0, cr = k[4], f = k[5];
      if (disctype == 2)
      {
        double delta = sdfem_delta(hK, eps, b1, b2, b3, co->delta0, co->order_pd > 0 ? co->order_pd : 1);
        for (int i = 0; i < nbf; i++)
        {
          double bgradv = b1 * g[i][0] + b2 * g[i][1] + (dim == 3 ? b3 * g[i][2] : 0);
          F[i] += mult * (phi[q][i] + delta * bgradv) * f;
          for (int j = 0; j < nbf; j++)
          {
            double gg = g[i][0] * g[j][0] + g[i][1] * g[j][1] + (dim == 3 ? g[i][2] * g[j][2] : 0);
            double bg = b1 * g[j][0] + b2 * g[j][1] + (dim == 3 ? b3 * g[j][2] : 0);
            double val = eps * gg + bg * phi[q][i] + cr * phi[q][j] * phi[q][i];
            if (dim == 2)
              val += delta * (-eps * lap[j] + bg + cr * phi[q][j]) * bgradv;
            else
              val += delta * (bg + cr * phi[q][j]) * bgradv;
            A[i][j] += mult * val;
          }
        }
      }
      else if (disctype == 10)
      {
        /* mass form, MatrixMRhsAssemble (src/FE/ConvDiff2D.C:411-445) */
        for (int i = 0; i < nbf; i++)
        {
          F[i] += mult * phi[q][i] * f;
          for (int j = 0; j < nbf; j++) A[i][j] += mult * phi[q][j] * phi[q][i];
        }
      }
      else
      {
        for (int i = 0; i < nbf; i++)
        {
          F[i] += mult * phi[q][i] * f;
          for (int j = 0; j < nbf; j++)
          {
            double gg = g[i][0] * g[j][0] + g[i][1] * g[j][1] + (dim == 3 ? g[i][2] * g[j][2] : 0);
            double bg = b1 * g[j][0] + b2 * g[j][1] + (dim == 3 ? b3 * g[j][2] : 0);
            A[i][j] += mult * (eps * gg + bg * phi[q][i] + cr * phi[q][j] * phi[q][i]);
          }
        }
      }
    }
    /* scatter: Assemble2D.C:456-520 / AssembleMat3D.C:721-827, rhs Assemble2D.C:603-680 */
    const int *dof = gn + bi[c];
    for (int m = 0; m < nbf; m++)
    {
      int l = dof[m];
      if (l < n_active)
      {
        for (int kk = 0; kk < nbf; kk++)
        {
          long s = find_slot(row_ptr, kcol, l, dof[kk]);
          if (s < 0) return -1;
          entries[s] += A[m][kk];
        }
        rhs[l] += F[m];
      }
      else
      {
        long s = find_slot(row_ptr, kcol, l, l);
        if (s < 0) return -1;
        entries[s] = 1.0;
        rhs[l] = dir_vals ? dir_vals[l - n_active] : 0.0;
      }
    }
  }
  return 0;
}

/* Neumann data of the sine problem (boundary component 1 = {x = 1}, value
 * -eps*pi*sin(pi*y)), added like the NEUMANN branch of Assemble2D
 * (src/FE/Assemble2D.C:797-827): line Gauss rule of degree 2p
 * (FEDatabase2D.C:1729-1735), half edge length times weight times value times
 * the basis value, into active rows only. */
void cdo_neumann_sine(int order, int n_cells, const double *coords, const int *gn, const int *bi,
                      int n_active, double eps, double *rhs)
{
  int nbf = cdo_nbf(2, order);
  int nl = order == 1 ? 2 : 3;
  double z[4], w[4];
  gauss1d(nl, z, w);
  for (int c = 0; c < n_cells; c++)
  {
    const double *V = coords + (size_t)c * 8;
    const int *dof = gn + bi[c];
    for (int m = 0; m < 4; m++)
    {
      int m1 = (m + 1) % 4;
      if (!(fabs(V[2 * m] - 1.0) < 1e-12 && fabs(V[2 * m1] - 1.0) < 1e-12)) continue;
      double x0 = V[2 * m], y0 = V[2 * m + 1], x1 = V[2 * m1], y1 = V[2 * m1 + 1];
      double hE = sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0)) / 2;
      for (int l = 0; l < nl; l++)
      {
        double s = 0.5 * (z[l] + 1);
        /* reference point on edge m, running from reference vertex m to m+1 */
        double xi[2];
        xi[0] = RV2[m][0] + (RV2[m1][0] - RV2[m][0]) * s;
        xi[1] = RV2[m][1] + (RV2[m1][1] - RV2[m][1]) * s;
        double t = y0 + (y1 - y0) * s;
        double g = -eps * M_PI * sin(M_PI * t);
        double val[MAXBF];
        cdo_basis(2, order, xi, val, NULL, NULL);
        double sc = g * hE * w[l];
        for (int k = 0; k < nbf; k++)
          if (dof[k] < n_active) rhs[dof[k]] += sc * val[k];
      }
    }
  }
}

/* L2 and H1-semi errors of the sine problem, TFEFunction2D::GetErrors +
 * L2H1Errors (src/FE/FEFunction2D.C:229, src/General/MainUtilities.C:606): the
 * quadrature comes from TFEDatabase2D::GetOrig, i.e. the assembly rule (degree 3p). */
void cdo_errors_sine(int order, int n_cells, const double *coords, const int *gn, const int *bi,
                     const double *u, double *err2)
{
  int nbf = cdo_nbf(2, order);
  double qx[2 * MAXQ], qw[MAXQ];
  int nq = cdo_quadrature(2, cdo_gauss_points(order), qx, qw);
  double e0 = 0, e1 = 0;
  for (int c = 0; c < n_cells; c++)
  {
    const double *V = coords + (size_t)c * 8;
    int affine = cell_is_affine(2, V);
    const int *dof = gn + bi[c];
    for (int q = 0; q < nq; q++)
    {
      double x[2], J[4], Ji[4], val[MAXBF], gr[MAXBF * 2];
      ref_map(2, affine, V, qx + 2 * q, x, J);
      double det = inv(2, J, Ji);
      cdo_basis(2, order, qx + 2 * q, val, gr, NULL);
      double uh = 0, ux = 0, uy = 0;
      for (int b = 0; b < nbf; b++)
      {
        double gx = Ji[0] * gr[2 * b] + Ji[2] * gr[2 * b + 1];
        double gy = Ji[1] * gr[2 * b] + Ji[3] * gr[2 * b + 1];
        uh += u[dof[b]] * val[b];
        ux += u[dof[b]] * gx;
        uy += u[dof[b]] * gy;
      }
      double ex = sin(M_PI * x[0]) * sin(M_PI * x[1]);
      double exx = M_PI * cos(M_PI * x[0]) * sin(M_PI * x[1]);
      double exy = M_PI * sin(M_PI * x[0]) * cos(M_PI * x[1]);
      double w = qw[q] * fabs(det);
      e0 += w * (uh - ex) * (uh - ex);
      e1 += w * ((ux - exx) * (ux - exx) + (uy - exy) * (uy - exy));
    }
  }
  err2[0] = sqrt(e0);
  err2[1] = sqrt(e1);
}

/* L2 and H1-semi errors against u = amp sin(k pi x) sin(k pi y) (2D): the TCD2D example exp.h
 * (Examples/TCD_2D/exp.h:31-41, amp = exp(t), k = 2) through TFEFunction2D::GetErrors
 * (src/FE/FEFunction2D.C:73) with the assembly's Gauss rule, as cdo_errors_sine */
void cdo_errors_sinsin(int order, int n_cells, const double *coords, const int *gn, const int *bi,
                       const double *u, double k, double amp, double *err2)
{
  int nbf = cdo_nbf(2, order);
  double qx[2 * MAXQ], qw[MAXQ];
  int nq = cdo_quadrature(2, cdo_gauss_points(order), qx, qw);
  double e0 = 0, e1 = 0;
  for (int c = 0; c < n_cells; c++)
  {
    const double *V = coords + (size_t)c * 8;
    int affine = cell_is_affine(2, V);
    const int *dof = gn + bi[c];
    for (int q = 0; q < nq; q++)
    {
      double x[2], J[4], Ji[4], val[MAXBF], gr[MAXBF * 2];
      ref_map(2, affine, V, qx + 2 * q, x, J);
      double det = inv(2, J, Ji);
      cdo_basis(2, order, qx + 2 * q, val, gr, NULL);
      double uh = 0, ux = 0, uy = 0;
      for (int b = 0; b < nbf; b++)
      {
        double gx = Ji[0] * gr[2 * b] + Ji[2] * gr[2 * b + 1];
        double gy = Ji[1] * gr[2 * b] + Ji[3] * gr[2 * b + 1];
        uh += u[dof[b]] * val[b];
        ux += u[dof[b]] * gx;
        uy += u[dof[b]] * gy;
      }
      double sx = sin(k * M_PI * x[0]), sy = sin(k * M_PI * x[1]);
      double ex = amp * sx * sy;
      double exx = amp * k * M_PI * cos(k * M_PI * x[0]) * sy;
      double exy = amp * k * M_PI * sx * cos(k * M_PI * x[1]);
      double w = qw[q] * fabs(det);
      e0 += w * (uh - ex) * (uh - ex);
      e1 += w * ((ux - exx) * (ux - exx) + (uy - exy) * (uy - exy));
    }
  }
  err2[0] = sqrt(e0);
  err2[1] = sqrt(e1);
}

/* L2 and H1-semi errors against an exact solution tabulated at the quadrature points of
 * cdo_quad_points: exact[(c * nq + q) * (1 + dim) + k] = u, du/dx, du/dy[, du/dz].  Any space
 * of the path: TFEFunction2D::GetErrors (src/FE/FEFunction2D.C:73) and
 * TFEFunction3D::GetErrors (src/FE/FEFunction3D.C:57) with L2H1Errors
 * (src/General/MainUtilities.C:606), on the assembly's Gauss rule (degree 3p). */
void cdo_errors_table(int dim, int order, int n_cells, const double *coords, const int *gn, const int *bi,
                      const double *u, const double *exact, double *err2)
{
  int nbf = cdo_nbf(dim, order), nv = nverts(dim);
  double qx[3 * MAXQ], qw[MAXQ];
  int nq = cdo_quadrature(dim, cdo_gauss_points(order), qx, qw);
  double e0 = 0, e1 = 0;
  for (int c = 0; c < n_cells; c++)
  {
    const double *V = coords + (size_t)c * nv * dim;
    int affine = cell_is_affine(dim, V);
    const int *dof = gn + bi[c];
    for (int q = 0; q < nq; q++)
    {
      double x[3], J[9], Ji[9], val[MAXBF], gr[MAXBF * 3];
      ref_map(dim, affine, V, qx + dim * q, x, J);
      double det = inv(dim, J, Ji);
      cdo_basis(dim, order, qx + dim * q, val, gr, NULL);
      double uh = 0, g[3] = {0, 0, 0};
      for (int b = 0; b < nbf; b++)
      {
        uh += u[dof[b]] * val[b];
        for (int a = 0; a < dim; a++)
        {
          double t = 0;
          for (int k = 0; k < dim; k++) t += Ji[k * dim + a] * gr[dim * b + k];
          g[a] += u[dof[b]] * t;
        }
      }
      const double *ex = exact + ((size_t)c * nq + q) * (1 + dim);
      double w = qw[q] * fabs(det);
      e0 += w * (uh - ex[0]) * (uh - ex[0]);
      double s1 = 0;
      for (int a = 0; a < dim; a++) s1 += (g[a] - ex[1 + a]) * (g[a] - ex[1 + a]);
      e1 += w * s1;
    }
  }
  err2[0] = sqrt(e0);
  err2[1] = sqrt(e1);
}

/* physical quadrature points of every cell (n_cells x n_quad x dim), in the order the
 * assembly reads a CDGPU_COEFF_TABLE (kind 3) */
void cdo_quad_points(int dim, int order, int n_cells, const double *coords, double *xyz)
{
  double qx[3 * MAXQ], qw[MAXQ];
  int nq = cdo_quadrature(dim, cdo_gauss_points(order), qx, qw), nv = nverts(dim);
  for (int c = 0; c < n_cells; c++)
  {
    const double *V = coords + (size_t)c * nv * dim;
    int affine = cell_is_affine(dim, V);
    for (int q = 0; q < nq; q++)
    {
      double x[3], J[9];
      ref_map(dim, affine, V, qx + dim * q, x, J);
      for (int a = 0; a < dim; a++) xyz[((size_t)c * nq + q) * dim + a] = x[a];
    }
  }
}

/* physical coordinates of every DOF (any cell containing it gives the same point) */
void cdo_dof_coords(int dim, int order, int n_cells, const double *coords, const int *gn,
                    const int *bi, int n_dof, double *xyz)
{
  int nbf = cdo_nbf(dim, order), nv = nverts(dim);
  for (int c = 0; c < n_cells; c++)
  {
    const double *V = coords + (size_t)c * nv * dim;
    int affine = cell_is_affine(dim, V);
    for (int b = 0; b < nbf; b++)
    {
      double xi[3], x[3], J[9];
      node_pos(dim, order, b, xi);
      ref_map(dim, affine, V, xi, x, J);
      for (int a = 0; a < dim; a++) xyz[(size_t)gn[bi[c] + b] * dim + a] = x[a];
    }
  }
}

/* ------------------------------------------------------------------------- */
/* prolongation (src/FE/MGComponents3D.C:182-462, MGComponents2D.C:118): the     */
/* reference applies, per fine cell, the coarse basis evaluated at the fine     */
/* cell's nodes in the parent's reference coordinates (GetProlongationMatrix3D, */
/* src/FE/FEDatabase3D.C:1630) and averages by DOF multiplicity.  For conforming */
/* Lagrange elements every cell gives the same value, so P[i][j] is the coarse  */
/* basis function j at fine node i.  Fine nodes of a nested refinement sit at   */
/* dyadic reference points of the parent, where the values are exact multiples */
/* of 2^-12; they are snapped to that grid.  Returns nnz; two-phase like         */
/* cdo_pattern (pass NULL col/val to count).  Rows are fine DOFs, columns       */
/* ascending.                                                                   */
/* ------------------------------------------------------------------------- */
static void invert_map(int dim, int affine, const double *V, const double *x, double *xi)
{
  for (int a = 0; a < dim; a++) xi[a] = 0;
  for (int it = 0; it < (affine ? 2 : 30); it++)
  {
    double y[3], J[9], Ji[9];
    ref_map(dim, affine, V, xi, y, J);
    inv(dim, J, Ji);
    double r[3], dmax = 0;
    for (int a = 0; a < dim; a++) r[a] = x[a] - y[a];
    for (int b = 0; b < dim; b++)
    {
      double d = 0;
      for (int a = 0; a < dim; a++) d += Ji[b * dim + a] * r[a];
      xi[b] += d;
      dmax = fmax(dmax, fabs(d));
    }
    if (dmax < 1e-15) break;
  }
}

static double snap(double v)
{
  double s = ldexp(1.0, 12);
  double r = nearbyint(v * s) / s;
  return fabs(r - v) < 1e-10 ? r : v;
}

long cdo_prolongation(int dim, int order, int nc_cells, const double *c_coords, const int *c_gn,
                      const int *c_bi, int n_c, int nf_cells, const double *f_coords,
                      const int *f_gn, const int *f_bi, int n_f, const int *parent, int *row_ptr,
                      int *col, double *val)
{
  int nbf = cdo_nbf(dim, order), nv = nverts(dim);
  /* first fine cell of every fine DOF */
  int *owner = malloc(sizeof(int) * n_f), *lb = malloc(sizeof(int) * n_f);
  for (int i = 0; i < n_f; i++) owner[i] = -1;
  for (int c = 0; c < nf_cells; c++)
    for (int b = 0; b < nbf; b++)
    {
      int d = f_gn[f_bi[c] + b];
      if (owner[d] < 0) { owner[d] = c; lb[d] = b; }
    }
  long nnz = 0;
  row_ptr[0] = 0;
  int cols[MAXBF];
  double vals[MAXBF];
  for (int i = 0; i < n_f; i++)
  {
    int c = owner[i], p = parent[c];
    const double *Vf = f_coords + (size_t)c * nv * dim;
    const double *Vc = c_coords + (size_t)p * nv * dim;
    double xi[3], x[3], J[9], eta[3], phi[MAXBF];
    node_pos(dim, order, lb[i], xi);
    ref_map(dim, cell_is_affine(dim, Vf), Vf, xi, x, J);
    invert_map(dim, cell_is_affine(dim, Vc), Vc, x, eta);
    cdo_basis(dim, order, eta, phi, NULL, NULL);
    int m = 0;
    for (int b = 0; b < nbf; b++)
    {
      double v = snap(phi[b]);
      if (v != 0.0) { cols[m] = c_gn[c_bi[p] + b]; vals[m] = v; m++; }
    }
    /* sort by column (insertion sort, m <= 27) */
    for (int a = 1; a < m; a++)
    {
      int cc = cols[a]; double vv = vals[a]; int k = a - 1;
      while (k >= 0 && cols[k] > cc) { cols[k + 1] = cols[k]; vals[k + 1] = vals[k]; k--; }
      cols[k + 1] = cc; vals[k + 1] = vv;
    }
    if (col)
      for (int a = 0; a < m; a++) { col[nnz + a] = cols[a]; val[nnz + a] = vals[a]; }
    nnz += m;
    row_ptr[i + 1] = (int)nnz;
  }
  free(owner); free(lb);
  return nnz;
}

/* ------------------------------------------------------------------------- */
/* linear algebra: ScalarDefect / MatVect (src/FE/Blas2.C:11-87)                */
/* ------------------------------------------------------------------------- */
typedef struct
{
  int n, n_active, hanging_bound, n_dirichlet;
  const int *row_ptr, *kcol;
  const double *a;
} csr;

static void matvec(const csr *A, const double *x, double *y)
{
  for (int i = 0; i < A->n; i++)
  {
    double s = 0;
    for (int j = A->row_ptr[i]; j < A->row_ptr[i + 1]; j++) s += A->a[j] * x[A->kcol[j]];
    y[i] = s;
  }
}

static double defect(const csr *A, const double *x, const double *f, double *d)
{
  double r = 0;
  for (int i = 0; i < A->n; i++)
  {
    double s = f[i];
    for (int j = A->row_ptr[i]; j < A->row_ptr[i + 1]; j++) s -= A->a[j] * x[A->kcol[j]];
    d[i] = s;
    r += s * s;
  }
  return sqrt(r);
}

void cdo_spmv(int n, const int *row_ptr, const int *kcol, const double *a, const double *x, double *y)
{
  csr A = {n, n, n, 0, row_ptr, kcol, a};
  matvec(&A, x, y);
}

static double dot(int n, const double *x, const double *y)
{
  double s = 0;
  for (int i = 0; i < n; i++) s += x[i] * y[i];
  return s;
}

/* ------------------------------------------------------------------------- */
/* multigrid: TMultiGrid3D::Cycle / Smooth (src/FE/MultiGrid3D.C:91-669),        */
/* TMGLevel3D::Jacobi/SOR/SSOR/Update/CorrectNodes/CorrectDefect                 */
/* (src/FE/MGLevel3D.C:254-615), TMultiGridScaIte::Iterate (MultiGridScaIte.C:63) */
/* ------------------------------------------------------------------------- */
typedef struct
{
  int solver;          /* SC_SOLVER_SCALAR: 16 FGMRES, 11 fixed point */
  int restart;         /* SC_GMRES_RESTART */
  int maxit;           /* SC_LIN_MAXIT_SCALAR */
  int minit;           /* SC_MINIT */
  int smoother;        /* SC_SMOOTHER_SCALAR: 1 Jacobi, 2 SOR, 3 SSOR */
  int coarse_smoother; /* SC_COARSE_SMOOTHER_SCALAR: 1, 2, 3, 17 (exact) */
  int pre, post;       /* SC_PRE_SMOOTH_SCALAR, SC_POST_SMOOTH_SCALAR */
  int coarse_maxit;    /* SC_COARSE_MAXIT_SCALAR */
  int cycle;           /* SC_MG_CYCLE_SCALAR: 1 V, 2 W, 0 F */
  int slc;             /* SC_STEP_LENGTH_CONTROL_ALL_SCALAR */
  int slc_fine;        /* SC_STEP_LENGTH_CONTROL_FINE_SCALAR */
  double red_factor;   /* SC_LIN_RED_FACTOR_SCALAR */
  double res_norm_min; /* SC_LIN_RES_NORM_MIN_SCALAR */
  double div_factor;   /* SC_DIV_FACTOR */
  double omega;        /* SC_SMOOTH_DAMP_FACTOR_SCALAR (Parameters[0]) */
  double coarse_red;   /* SC_COARSE_RED_FACTOR_SCALAR */
  double gmg_damp;     /* SC_GMG_DAMP_FACTOR_SCALAR */
} cdo_solver_params;

typedef struct
{
  csr A;
  double *sol, *rhs, *aux[4];
  /* prolongation from the next coarser level (rows = this level's DOFs) */
  const int *p_row, *p_col;
  const double *p_val;
  int *r_row, *r_col; /* restriction = transposed prolongation */
  double *r_val;
  double *lu;         /* dense LU of the coarsest level (coarse_smoother 17) */
  int *piv;
} mglevel;

typedef struct
{
  int L;
  mglevel *lev;
  const cdo_solver_params *p;
  int rec[64];
} mg;

static void jacobi(mglevel *lv, double omega)
{
  /* MGLevel3D.C:443-537 */
  const csr *A = &lv->A;
  double *sol = lv->sol, *f = lv->rhs, *aux = lv->aux[1];
  memcpy(aux, sol, sizeof(double) * A->n);
  for (int i = A->hanging_bound; i < A->hanging_bound + A->n_dirichlet; i++) sol[i] = f[i];
  for (int i = 0; i < A->n_active; i++)
  {
    double s = f[i], diag = 1;
    for (int j = A->row_ptr[i]; j < A->row_ptr[i + 1]; j++)
    {
      int c = A->kcol[j];
      if (c == i) diag = A->a[j]; else s -= A->a[j] * aux[c];
    }
    sol[i] = (1 - omega) * aux[i] + omega * s / diag;
  }
}

static void sor_sweep(mglevel *lv, double omega, int backward)
{
  const csr *A = &lv->A;
  double *sol = lv->sol, *f = lv->rhs;
  for (int ii = 0; ii < A->n_active; ii++)
  {
    int i = backward ? A->n_active - 1 - ii : ii;
    double s = f[i], diag = 1;
    if (!backward)
    {
      for (int j = A->row_ptr[i]; j < A->row_ptr[i + 1]; j++)
      {
        int c = A->kcol[j];
        if (c == i) diag = A->a[j]; else s -= A->a[j] * sol[c];
      }
    }
    else
    {
      for (int j = A->row_ptr[i + 1] - 1; j >= A->row_ptr[i]; j--)
      {
        int c = A->kcol[j];
        if (c == i) diag = A->a[j]; else s -= A->a[j] * sol[c];
      }
    }
    double t = sol[i];
    sol[i] = omega * (s / diag - t) + t;
  }
}

static void sor(mglevel *lv, double omega)
{
  /* MGLevel3D.C:254-333 */
  const csr *A = &lv->A;
  for (int i = A->hanging_bound; i < A->hanging_bound + A->n_dirichlet; i++) lv->sol[i] = lv->rhs[i];
  sor_sweep(lv, omega, 0);
}

static void ssor(mglevel *lv, double omega)
{
  /* MGLevel3D.C:337-440 */
  const csr *A = &lv->A;
  for (int i = A->hanging_bound; i < A->hanging_bound + A->n_dirichlet; i++) lv->sol[i] = lv->rhs[i];
  sor_sweep(lv, omega, 0);
  sor_sweep(lv, omega, 1);
}

static void exact_solve(mglevel *lv)
{
  /* MGLevel3D.C:839-880 (dense solve of the full coarse system) */
  int n = lv->A.n;
  if (!lv->lu)
  {
    lv->lu = calloc((size_t)n * n, sizeof(double));
    lv->piv = malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++)
      for (int j = lv->A.row_ptr[i]; j < lv->A.row_ptr[i + 1]; j++)
        lv->lu[(size_t)i * n + lv->A.kcol[j]] = lv->A.a[j];
    double *M = lv->lu;
    for (int k = 0; k < n; k++)
    {
      int p = k;
      for (int i = k + 1; i < n; i++)
        if (fabs(M[(size_t)i * n + k]) > fabs(M[(size_t)p * n + k])) p = i;
      lv->piv[k] = p;
      if (p != k)
        for (int j = 0; j < n; j++)
        {
          double t = M[(size_t)k * n + j]; M[(size_t)k * n + j] = M[(size_t)p * n + j]; M[(size_t)p * n + j] = t;
        }
      for (int i = k + 1; i < n; i++)
      {
        double l = M[(size_t)i * n + k] / M[(size_t)k * n + k];
        M[(size_t)i * n + k] = l;
        for (int j = k + 1; j < n; j++) M[(size_t)i * n + j] -= l * M[(size_t)k * n + j];
      }
    }
  }
  double *x = lv->sol, *M = lv->lu;
  memcpy(x, lv->rhs, sizeof(double) * n);
  for (int k = 0; k < n; k++)
  {
    int p = lv->piv[k];
    if (p != k) { double t = x[k]; x[k] = x[p]; x[p] = t; }
    for (int i = k + 1; i < n; i++) x[i] -= M[(size_t)i * n + k] * x[k];
  }
  for (int k = n - 1; k >= 0; k--)
  {
    double s = x[k];
    for (int j = k + 1; j < n; j++) s -= M[(size_t)k * n + j] * x[j];
    x[k] = s / M[(size_t)k * n + k];
  }
}

static void smooth(mg *m, int lvl, int kind, int count)
{
  mglevel *lv = &m->lev[lvl];
  for (int it = 0; it < count; it++)
  {
    if (kind == 1) jacobi(lv, m->p->omega);
    else if (kind == 2) sor(lv, m->p->omega);
    else ssor(lv, m->p->omega);
  }
}

static void prolongate(const mglevel *fine, const double *coarse, double *out)
{
  for (int i = 0; i < fine->A.n; i++)
  {
    double s = 0;
    for (int j = fine->p_row[i]; j < fine->p_row[i + 1]; j++) s += fine->p_val[j] * coarse[fine->p_col[j]];
    out[i] = s;
  }
}

static void restrict_(const mglevel *fine, int n_c, const double *f, double *out)
{
  for (int i = 0; i < n_c; i++)
  {
    double s = 0;
    for (int j = fine->r_row[i]; j < fine->r_row[i + 1]; j++) s += fine->r_val[j] * f[fine->r_col[j]];
    out[i] = s;
  }
}

static double step_length(mglevel *lv, const double *old, const double *olddef, double omega0)
{
  /* MGLevel3D.C:882-932 */
  int n = lv->A.n;
  double *x = malloc(sizeof(double) * 2 * n), *y = x + n;
  for (int i = 0; i < n; i++) x[i] = lv->sol[i] - old[i];
  matvec(&lv->A, x, y);
  double num = dot(n, olddef, y), den = dot(n, y, y), om;
  om = den > 0 ? num / den : omega0;
  if (fabs(om) < 0.1) om = omega0;
  free(x);
  return om;
}

static void cycle(mg *m, int i, double *res)
{
  const cdo_solver_params *p = m->p;
  mglevel *cur = &m->lev[i];
  int n = cur->A.n;
  double *D = cur->aux[0];
  if (i == 0)
  {
    /* coarse grid: MultiGrid3D.C:199-311 */
    double r = defect(&cur->A, cur->sol, cur->rhs, D);
    double red = p->coarse_red * r;
    int it = 0;
    while (r > red && it < p->coarse_maxit)
    {
      if (p->coarse_smoother == 17) exact_solve(cur);
      else smooth(m, 0, p->coarse_smoother, 1);
      r = defect(&cur->A, cur->sol, cur->rhs, D);
      it++;
    }
    *res = r;
    return;
  }
  int slc = p->slc || (p->slc_fine && i == m->L - 1);
  mglevel *crs = &m->lev[i - 1];
  double oldres = defect(&cur->A, cur->sol, cur->rhs, D);
  if (slc)
  {
    memcpy(cur->aux[2], cur->sol, sizeof(double) * n);
    memcpy(cur->aux[3], D, sizeof(double) * n);
  }
  smooth(m, i, p->smoother, p->pre);
  oldres = defect(&cur->A, cur->sol, cur->rhs, D);
  restrict_(cur, crs->A.n, D, crs->rhs);
  memset(crs->rhs + crs->A.n_active, 0, sizeof(double) * (crs->A.n - crs->A.n_active));
  memset(crs->sol, 0, sizeof(double) * crs->A.n);
  for (int j = 0; j < m->rec[i]; j++) cycle(m, i - 1, res);
  if (p->cycle < 1) m->rec[i] = 1;
  prolongate(cur, crs->sol, D);
  memset(D + cur->A.hanging_bound, 0, sizeof(double) * cur->A.n_dirichlet);
  for (int k = 0; k < n; k++) cur->sol[k] += p->gmg_damp * D[k];
  smooth(m, i, p->smoother, p->post);
  if (slc)
  {
    double alpha = step_length(cur, cur->aux[2], cur->aux[3], p->omega);
    for (int k = 0; k < n; k++) cur->sol[k] = cur->aux[2][k] + alpha * (cur->sol[k] - cur->aux[2][k]);
  }
  *res = defect(&cur->A, cur->sol, cur->rhs, D);
  (void)oldres;
}

static void mg_prec(mg *m, const double *rhs, double *sol)
{
  /* TMultiGridScaIte::Iterate with zero start */
  mglevel *f = &m->lev[m->L - 1];
  int n = f->A.n;
  memset(f->sol, 0, sizeof(double) * n);
  memcpy(f->rhs, rhs, sizeof(double) * n);
  memcpy(f->sol + f->A.hanging_bound, f->rhs + f->A.hanging_bound, sizeof(double) * f->A.n_dirichlet);
  /* SetRecursion(levels = L-1): MultiGrid3D.C:691-703 */
  int gam = m->p->cycle;
  m->rec[1] = 1;
  for (int k = 2; k <= m->L - 1; k++) m->rec[k] = gam > 0 ? gam : 2;
  double res;
  cycle(m, m->L - 1, &res);
  memcpy(sol, f->sol, sizeof(double) * n);
}

/* ------------------------------------------------------------------------- */
/* Krylov drivers: TFgmresIte::Iterate flexible branch (src/FE/FgmresIte.C:219-582) */
/* and TFixedPointIte::Iterate (src/FE/FixedPointIte.C:150-303).                    */
/* ------------------------------------------------------------------------- */
static void gen_rot(double dx, double dy, double *cs, double *sn)
{
  if (dy == 0.0) { *cs = 1.0; *sn = 0.0; }
  else if (fabs(dy) > fabs(dx))
  {
    double t = dx / dy;
    *sn = 1.0 / sqrt(1.0 + t * t);
    *cs = t * *sn;
  }
  else
  {
    double t = dy / dx;
    *cs = 1.0 / sqrt(1.0 + t * t);
    *sn = t * *cs;
  }
}

static void app_rot(double *dx, double *dy, double cs, double sn)
{
  double t = cs * *dx + sn * *dy;
  *dy = -sn * *dx + cs * *dy;
  *dx = t;
}

static void update_iterate(double *x, int n, int k, double *H, int ldh, double *s, double **z)
{
  for (int i = k; i >= 0; i--)
  {
    s[i] /= H[i * ldh + i];
    for (int j = i - 1; j >= 0; j--) s[j] -= H[j * ldh + i] * s[i];
  }
  for (int j = 0; j <= k; j++)
    for (int i = 0; i < n; i++) x[i] += z[j][i] * s[j];
}

/* returns the iteration count (like the reference), or -1 on divergence
 * (the reference calls exit(4711) there); res_hist receives |s_{i+1}| per
 * iteration when non-NULL (capacity maxit+1). */
static int fgmres(mg *m, const csr *A, double *sol, const double *rhs, double *res_hist,
                  double *final_res)
{
  const cdo_solver_params *p = m->p;
  int n = A->n, mr = p->restart < p->maxit ? p->restart : p->maxit;
  if (mr <= 0) mr = 10;
  double **v = malloc(sizeof(double *) * (mr + 1)), **z = malloc(sizeof(double *) * (mr + 1));
  for (int i = 0; i <= mr; i++)
  {
    v[i] = calloc(n, sizeof(double));
    z[i] = calloc(n, sizeof(double));
  }
  double *H = calloc((size_t)(mr + 1) * mr, sizeof(double));
  double *s = calloc(mr + 1, sizeof(double)), *cs = calloc(mr + 1, sizeof(double)),
         *sn = calloc(mr + 1, sizeof(double)), *w = calloc(n, sizeof(double));
  int ret = 0, maxite = p->maxit;
  double res = defect(A, sol, rhs, v[0]);
  double res0 = res, beta = res;
  if (res_hist) res_hist[0] = res;
  if (beta <= p->res_norm_min)
  {
    if (p->minit == 0 || beta < 1e-20) { ret = 0; goto done; }
    maxite = p->minit;
  }
  int j = 1;
  while (j <= maxite)
  {
    for (int k = 0; k < n; k++) v[0][k] *= 1.0 / beta;
    memset(s, 0, sizeof(double) * (mr + 1));
    s[0] = beta;
    int i;
    for (i = 0; i < mr && j <= maxite; i++, j++)
    {
      memset(z[i], 0, sizeof(double) * n);
      mg_prec(m, v[i], z[i]);
      matvec(A, z[i], w);
      for (int k = 0; k <= i; k++)
      {
        H[k * mr + i] = dot(n, w, v[k]);
        double h = H[k * mr + i];
        for (int t = 0; t < n; t++) w[t] -= h * v[k][t];
      }
      H[(i + 1) * mr + i] = sqrt(dot(n, w, w));
      memcpy(v[i + 1], w, sizeof(double) * n);
      if (H[(i + 1) * mr + i] != 0)
        for (int t = 0; t < n; t++) v[i + 1][t] *= 1 / H[(i + 1) * mr + i];
      for (int k = 0; k < i; k++) app_rot(&H[k * mr + i], &H[(k + 1) * mr + i], cs[k], sn[k]);
      gen_rot(H[i * mr + i], H[(i + 1) * mr + i], &cs[i], &sn[i]);
      app_rot(&H[i * mr + i], &H[(i + 1) * mr + i], cs[i], sn[i]);
      app_rot(&s[i], &s[i + 1], cs[i], sn[i]);
      res = fabs(s[i + 1]);
      if (res_hist) res_hist[j] = res;
      if (j >= p->minit && (res < p->res_norm_min || res < p->red_factor * res0))
      {
        memset(w, 0, sizeof(double) * n);
        update_iterate(w, n, i, H, mr, s, z);
        for (int t = 0; t < n; t++) sol[t] += w[t];
        ret = j;
        goto done;
      }
      if (res > p->div_factor * res0) { ret = -1; goto done; }
    }
    memset(v[0], 0, sizeof(double) * n);
    update_iterate(v[0], n, mr - 1, H, mr, s, z);
    for (int t = 0; t < n; t++) sol[t] += v[0][t];
    res = defect(A, sol, rhs, v[0]);
    res0 = beta = res;
  }
  ret = j > maxite ? maxite : j;
done:
  if (final_res) *final_res = res;
  for (int i = 0; i <= mr; i++) { free(v[i]); free(z[i]); }
  free(v); free(z); free(H); free(s); free(cs); free(sn); free(w);
  return ret;
}

static int fixed_point(mg *m, const csr *A, double *sol, const double *rhs, double *res_hist,
                       double *final_res)
{
  const cdo_solver_params *p = m->p;
  int n = A->n, maxite = p->maxit, i;
  double *d = malloc(sizeof(double) * n);
  double res = defect(A, sol, rhs, d), res0 = res;
  if (res_hist) res_hist[0] = res;
  if (res <= p->res_norm_min) maxite = p->minit;
  for (i = 1; i <= maxite; i++)
  {
    mg_prec(m, d, d);
    for (int t = 0; t < n; t++) sol[t] += d[t];
    res = defect(A, sol, rhs, d);
    if (res_hist) res_hist[i] = res;
    if (i < p->minit) continue;
    if (res <= res0 * p->red_factor) break;
    if (res <= p->res_norm_min) break;
    if (res > p->div_factor * res0) { i = -1; break; }
  }
  if (final_res) *final_res = res;
  free(d);
  return i;
}

/* Solve A_fine x = rhs with the reference's multigrid-preconditioned Krylov method.
 * Per level l (0 = coarsest): n[l], n_active[l], row_ptr/kcol/entries[l]; for l > 0
 * the prolongation from level l-1 as CSR over level-l rows.  sol holds the initial
 * guess (Dirichlet values included) and receives the result.  Returns the
 * reference's iteration count or -1 on divergence. */
int cdo_solve(int L, const int *n, const int *n_active, const int *const *row_ptr,
              const int *const *kcol, const double *const *entries, const int *const *p_row,
              const int *const *p_col, const double *const *p_val, const cdo_solver_params *prm,
              const double *rhs, double *sol, double *res_hist, double *final_res)
{
  mg m;
  m.L = L;
  m.p = prm;
  m.lev = calloc(L, sizeof(mglevel));
  for (int l = 0; l < L; l++)
  {
    mglevel *lv = &m.lev[l];
    lv->A.n = n[l];
    lv->A.n_active = n_active[l];
    lv->A.hanging_bound = n_active[l];
    lv->A.n_dirichlet = n[l] - n_active[l];
    lv->A.row_ptr = row_ptr[l];
    lv->A.kcol = kcol[l];
    lv->A.a = entries[l];
    lv->sol = calloc(n[l], sizeof(double));
    lv->rhs = calloc(n[l], sizeof(double));
    for (int k = 0; k < 4; k++) lv->aux[k] = calloc(n[l], sizeof(double));
    if (l > 0)
    {
      lv->p_row = p_row[l]; lv->p_col = p_col[l]; lv->p_val = p_val[l];
      int nc = n[l - 1], nnz = p_row[l][n[l]];
      lv->r_row = calloc(nc + 1, sizeof(int));
      lv->r_col = malloc(sizeof(int) * (nnz + 1));
      lv->r_val = malloc(sizeof(double) * (nnz + 1));
      for (int t = 0; t < nnz; t++) lv->r_row[p_col[l][t] + 1]++;
      for (int t = 0; t < nc; t++) lv->r_row[t + 1] += lv->r_row[t];
      int *fill = calloc(nc, sizeof(int));
      for (int i = 0; i < n[l]; i++)
        for (int t = p_row[l][i]; t < p_row[l][i + 1]; t++)
        {
          int c = p_col[l][t];
          int pos = lv->r_row[c] + fill[c]++;
          lv->r_col[pos] = i;
          lv->r_val[pos] = p_val[l][t];
        }
      free(fill);
    }
  }
  int its;
  const csr *A = &m.lev[L - 1].A;
  if (prm->solver == 11) its = fixed_point(&m, A, sol, rhs, res_hist, final_res);
  else its = fgmres(&m, A, sol, rhs, res_hist, final_res);
  for (int l = 0; l < L; l++)
  {
    mglevel *lv = &m.lev[l];
    free(lv->sol); free(lv->rhs);
    for (int k = 0; k < 4; k++) free(lv->aux[k]);
    free(lv->r_row); free(lv->r_col); free(lv->r_val); free(lv->lu); free(lv->piv);
  }
  free(m.lev);
  return its;
}
