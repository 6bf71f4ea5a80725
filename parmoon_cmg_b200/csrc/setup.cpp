// Host-side set-up of libcdgpu: reference element tables, the CSR pattern, the
// DOF->cell incidence used by the row-gather assembly, transfer operators and the
// dense coarse inverse.  All of it runs once per mesh (the reference's
// "construction" phase), not per assembly or solve.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

// ---------------------------------------------------------------------------
// Gauss rules.  The reference picks the rule of degree 3p (src/FE/FEDatabase2D.C:1841,
// src/FE/FEDatabase3D.C:1184): Gauss3 for Q1, Gauss4 for Q2, as tensor products with
// x fastest (src/QuadFormulas/QuadFormulaHexa.C:62-119).
// ---------------------------------------------------------------------------
static void gauss1d(int n, double *x, double *w)
{
  if (n == 2)
  {
    double a = 1.0 / std::sqrt(3.0);
    x[0] = -a; x[1] = a; w[0] = w[1] = 1.0;
  }
  else if (n == 3)
  {
    double a = std::sqrt(3.0 / 5.0);
    x[0] = -a; x[1] = 0; x[2] = a;
    w[0] = w[2] = 5.0 / 9.0; w[1] = 8.0 / 9.0;
  }
  else
  {
    double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    double b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    double wa = (18.0 + std::sqrt(30.0)) / 36.0, wb = (18.0 - std::sqrt(30.0)) / 36.0;
    x[0] = a; x[1] = b; x[2] = -b; x[3] = -a;
    w[0] = wa; w[1] = wb; w[2] = wb; w[3] = wa;
  }
}

// 1D Lagrange polynomials on [-1,1] with nodes {-1,1} or {-1,0,1}
static void lag1d(int order, double t, double *v, double *d, double *dd)
{
  if (order == 1)
  {
    v[0] = 0.5 * (1 - t); v[1] = 0.5 * (1 + t);
    d[0] = -0.5; d[1] = 0.5; dd[0] = dd[1] = 0;
  }
  else
  {
    v[0] = 0.5 * t * (t - 1); v[1] = 1 - t * t; v[2] = 0.5 * t * (t + 1);
    d[0] = t - 0.5; d[1] = -2 * t; d[2] = t + 0.5;
    dd[0] = 1; dd[1] = -2; dd[2] = 1;
  }
}

// tensor-product basis in the reference's local order (x fastest), as in
// include/FE2D/BF_C_Q_Q{1,2}_2D.h and include/FE3D/BF_C_H_Q{1,2}_3D.h
static void basis_full(int dim, int order, const double *xi, double *val, double *grad,
                       double *hess)
{
  int k = order + 1;
  double v[3][3], d[3][3], dd[3][3];
  for (int a = 0; a < dim; a++) lag1d(order, xi[a], v[a], d[a], dd[a]);
  int nbf = dim == 2 ? k * k : k * k * k;
  for (int b = 0; b < nbf; b++)
  {
    int ix = b % k, iy = (b / k) % k, iz = dim == 3 ? b / (k * k) : 0;
    int id[3] = {ix, iy, iz};
    double pv = 1;
    for (int a = 0; a < dim; a++) pv *= v[a][id[a]];
    val[b] = pv;
    for (int a = 0; a < dim; a++)
    {
      double g = 1;
      for (int c = 0; c < dim; c++) g *= (c == a ? d[c][id[c]] : v[c][id[c]]);
      if (grad) grad[b * dim + a] = g;
      for (int e = 0; e < dim; e++)
      {
        double h = 1;
        for (int c = 0; c < dim; c++)
        {
          int cnt = (c == a) + (c == e);
          h *= cnt == 0 ? v[c][id[c]] : cnt == 1 ? d[c][id[c]] : dd[c][id[c]];
        }
        if (hess) hess[(b * dim + a) * dim + e] = h;
      }
    }
  }
}

void basis_eval(int dim, int order, const double *xi, double *val, double *grad)
{
  basis_full(dim, order, xi, val, grad, nullptr);
}

void make_ref_element(int dim, int order, RefElement &re)
{
  re.dim = dim;
  re.order = order;
  int k = order + 1;
  re.nbf = dim == 2 ? k * k : k * k * k;
  re.nv = dim == 2 ? 4 : 8;
  int n1 = order == 1 ? 3 : 4;
  double x[4], w[4];
  gauss1d(n1, x, w);
  re.nq = dim == 2 ? n1 * n1 : n1 * n1 * n1;
  re.qx.assign(re.nq * dim, 0);
  re.qw.assign(re.nq, 0);
  int l = 0;
  for (int i = 0; i < (dim == 3 ? n1 : 1); i++)
    for (int j = 0; j < n1; j++)
      for (int kk = 0; kk < n1; kk++, l++)
      {
        re.qx[l * dim + 0] = x[kk];
        re.qx[l * dim + 1] = x[j];
        if (dim == 3) re.qx[l * dim + 2] = x[i];
        re.qw[l] = w[j] * w[kk] * (dim == 3 ? w[i] : 1.0);
      }
  re.phi.assign(re.nq * re.nbf, 0);
  re.dphi.assign(re.nq * re.nbf * dim, 0);
  re.hphi.assign(re.nq * re.nbf * dim * dim, 0);
  for (int q = 0; q < re.nq; q++)
    basis_full(dim, order, &re.qx[q * dim], &re.phi[q * re.nbf], &re.dphi[q * re.nbf * dim],
               &re.hphi[q * re.nbf * dim * dim]);
}

// ---------------------------------------------------------------------------
// Reference tensors of the affine fast path.  On a parallelogram/parallelepiped with
// constant coefficients every term of the local forms (src/FE/ConvDiff2D.C:32-162,
// src/FE/ConvDiff3D.C:61-190) is a per-cell scalar times an integral over the
// reference cell, so the local matrix is sum_t coef[cell][t] * R_t:
//   2D: I00, I11, I01+I10, C0, C1, M  [+ SUPG: D0, D1, E(00)0, E(00)1, E(11)0, E(11)1,
//       E(01)0, E(01)1]
//   3D: I00, I11, I22, I01+I10, I02+I20, I12+I21, C0, C1, C2, M  [+ SUPG: D0, D1, D2]
// with Iab_ij = int d_a phi_i d_b phi_j, Cb_ij = int phi_i d_b phi_j,
// Da_ij = int d_a phi_i phi_j, M_ij = int phi_i phi_j,
// E(cd)e_ij = int d_cd phi_j d_e phi_i (both orders summed for c != d); right-hand side
// vectors m_i = int phi_i [+ SUPG: g_a,i = int d_a phi_i].  Integrals use the assembly's
// own Gauss rule, so they are exact for these polynomial integrands.
// ---------------------------------------------------------------------------
int n_tensors(int dim, int disctype)
{
  if (disctype == CDGPU_MASS) return 1;
  if (dim == 2) return disctype == CDGPU_SUPG ? 14 : 6;
  return disctype == CDGPU_SUPG ? 13 : 10;
}

int n_rhs_tensors(int dim, int disctype) { return disctype == CDGPU_SUPG ? 1 + dim : 1; }

void reference_tensors(const RefElement &re, int disctype, std::vector<double> &R,
                       std::vector<double> &r)
{
  int dim = re.dim, nbf = re.nbf, T = n_tensors(dim, disctype), Tr = n_rhs_tensors(dim, disctype);
  R.assign((size_t)nbf * nbf * T, 0.0);
  r.assign((size_t)nbf * Tr, 0.0);
  for (int q = 0; q < re.nq; q++)
  {
    double w = re.qw[q];
    const double *ph = &re.phi[q * nbf];
    const double *dp = &re.dphi[q * nbf * dim];
    const double *hp = &re.hphi[q * nbf * dim * dim];
    for (int i = 0; i < nbf; i++)
    {
      r[i * Tr + 0] += w * ph[i];
      if (disctype == CDGPU_SUPG)
        for (int a = 0; a < dim; a++) r[i * Tr + 1 + a] += w * dp[i * dim + a];
      for (int j = 0; j < nbf; j++)
      {
        double *o = &R[((size_t)i * nbf + j) * T];
        auto I = [&](int a, int b) { return dp[i * dim + a] * dp[j * dim + b]; };
        auto Cb = [&](int b) { return ph[i] * dp[j * dim + b]; };
        auto Da = [&](int a) { return dp[i * dim + a] * ph[j]; };
        auto E = [&](int c, int d, int e) { return hp[(j * dim + c) * dim + d] * dp[i * dim + e]; };
        if (disctype == CDGPU_MASS)
          o[0] += w * ph[i] * ph[j];
        else if (dim == 2)
        {
          o[0] += w * I(0, 0);
          o[1] += w * I(1, 1);
          o[2] += w * (I(0, 1) + I(1, 0));
          o[3] += w * Cb(0);
          o[4] += w * Cb(1);
          o[5] += w * ph[i] * ph[j];
          if (disctype == CDGPU_SUPG)
          {
            o[6] += w * Da(0);
            o[7] += w * Da(1);
            o[8] += w * E(0, 0, 0);
            o[9] += w * E(0, 0, 1);
            o[10] += w * E(1, 1, 0);
            o[11] += w * E(1, 1, 1);
            o[12] += w * (E(0, 1, 0) + E(1, 0, 0));
            o[13] += w * (E(0, 1, 1) + E(1, 0, 1));
          }
        }
        else
        {
          o[0] += w * I(0, 0);
          o[1] += w * I(1, 1);
          o[2] += w * I(2, 2);
          o[3] += w * (I(0, 1) + I(1, 0));
          o[4] += w * (I(0, 2) + I(2, 0));
          o[5] += w * (I(1, 2) + I(2, 1));
          o[6] += w * Cb(0);
          o[7] += w * Cb(1);
          o[8] += w * Cb(2);
          o[9] += w * ph[i] * ph[j];
          if (disctype == CDGPU_SUPG)
          {
            o[10] += w * Da(0);
            o[11] += w * Da(1);
            o[12] += w * Da(2);
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// geometry: the reference maps QuadAffin/HexaAffin (src/FE/QuadAffin.C:602,
// src/FE/HexaAffin.C:865) for parallelograms/parallelepipeds and the bilinear /
// trilinear maps otherwise; vertices counter-clockwise, top face after bottom face.
// ---------------------------------------------------------------------------
static const double RV2[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
static const double RV3[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                 {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

bool cell_is_affine(int dim, const double *V)
{
  int nv = dim == 2 ? 4 : 8;
  double scale = 0;
  for (int i = 0; i < nv * dim; i++) scale = std::max(scale, std::fabs(V[i]));
  double tol = 1e-12 * (scale > 0 ? scale : 1);
  for (int a = 0; a < dim; a++)
  {
    auto X = [&](int v) { return V[v * dim + a]; };
    if (dim == 2)
    {
      if (std::fabs(X(0) + X(2) - X(1) - X(3)) > tol) return false;
    }
    else
    {
      if (std::fabs(X(2) - (X(1) + X(3) - X(0))) > tol) return false;
      if (std::fabs(X(5) - (X(1) + X(4) - X(0))) > tol) return false;
      if (std::fabs(X(7) - (X(3) + X(4) - X(0))) > tol) return false;
      if (std::fabs(X(6) - (X(1) + X(3) + X(4) - 2 * X(0))) > tol) return false;
    }
  }
  return true;
}

void ref_map(int dim, bool affine, const double *V, const double *xi, double *x, double *J)
{
  if (affine)
  {
    for (int a = 0; a < dim; a++)
    {
      double c1 = (V[1 * dim + a] - V[a]) * 0.5, c2 = (V[3 * dim + a] - V[a]) * 0.5;
      if (dim == 2)
      {
        double c0 = (V[1 * dim + a] + V[3 * dim + a]) * 0.5;
        x[a] = c0 + c1 * xi[0] + c2 * xi[1];
        J[a * 2] = c1; J[a * 2 + 1] = c2;
      }
      else
      {
        double c3 = (V[4 * dim + a] - V[a]) * 0.5;
        double c0 = (V[1 * dim + a] + V[3 * dim + a] + V[4 * dim + a] - V[a]) * 0.5;
        x[a] = c0 + c1 * xi[0] + c2 * xi[1] + c3 * xi[2];
        J[a * 3] = c1; J[a * 3 + 1] = c2; J[a * 3 + 2] = c3;
      }
    }
    return;
  }
  int nv = dim == 2 ? 4 : 8;
  for (int a = 0; a < dim; a++)
  {
    x[a] = 0;
    for (int b = 0; b < dim; b++) J[a * dim + b] = 0;
  }
  for (int v = 0; v < nv; v++)
  {
    const double *rv = dim == 2 ? RV2[v] : RV3[v];
    double f[3], N = 1;
    for (int b = 0; b < dim; b++) { f[b] = 0.5 * (1 + rv[b] * xi[b]); N *= f[b]; }
    for (int b = 0; b < dim; b++)
    {
      double dN = 0.5 * rv[b];
      for (int c = 0; c < dim; c++)
        if (c != b) dN *= f[c];
      for (int a = 0; a < dim; a++) J[a * dim + b] += dN * V[v * dim + a];
    }
    for (int a = 0; a < dim; a++) x[a] += N * V[v * dim + a];
  }
}

double invert(int dim, const double *J, double *Ji)
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

// CELL_MEASURE 0: src/Geometry/Quadrangle.C:35 (longer diagonal) and
// src/Geometry/Hexahedron.C:78 (longest space diagonal)
double cell_diameter(int dim, const double *V)
{
  double best = 0;
  if (dim == 2)
  {
    const int p[2][2] = {{0, 2}, {1, 3}};
    for (auto &e : p)
    {
      double dx = V[2 * e[0]] - V[2 * e[1]], dy = V[2 * e[0] + 1] - V[2 * e[1] + 1];
      best = std::max(best, dx * dx + dy * dy);
    }
  }
  else
  {
    const int p[4][2] = {{0, 6}, {1, 7}, {2, 4}, {3, 5}};
    for (auto &e : p)
    {
      double s = 0;
      for (int a = 0; a < 3; a++)
      {
        double d = V[3 * e[0] + a] - V[3 * e[1] + a];
        s += d * d;
      }
      best = std::max(best, s);
    }
  }
  return std::sqrt(best);
}

// ---------------------------------------------------------------------------
// CSR pattern, the structure of TSquareStructure2D/3D(TFESpace*) followed by Sort()
// (src/FE/SquareStructure3D.C:32-200, src/FE/SquareStructure.C:65): an active row
// holds every DOF of every cell containing it, a Dirichlet row only its diagonal,
// columns ascending.  Because the column set of a row is a set and the order is
// ascending, the result is bit-identical to the reference's for the same DOF map.
// ---------------------------------------------------------------------------
void build_incidence(const Space &s, std::vector<int> &ptr, std::vector<int> &inc)
{
  ptr.assign(s.n_dof + 1, 0);
  for (int c = 0; c < s.n_cells; c++)
    for (int i = 0; i < s.nbf; i++) ptr[s.h_gn[(size_t)c * s.nbf + i] + 1]++;
  for (int d = 0; d < s.n_dof; d++) ptr[d + 1] += ptr[d];
  inc.assign(ptr[s.n_dof], 0);
  std::vector<int> fill(s.n_dof, 0);
  for (int c = 0; c < s.n_cells; c++) // ascending cells per DOF by construction
    for (int i = 0; i < s.nbf; i++)
    {
      int d = s.h_gn[(size_t)c * s.nbf + i];
      inc[ptr[d] + fill[d]++] = c * s.nbf + i;
    }
}

void build_pattern(const Space &s, std::vector<int> &row_ptr, std::vector<int> &kcol)
{
  std::vector<int> ptr, inc;
  build_incidence(s, ptr, inc);
  row_ptr.assign(s.n_dof + 1, 0);
  kcol.clear();
  kcol.reserve((size_t)s.n_dof * (s.dim == 3 ? (s.order == 2 ? 60 : 27) : (s.order == 2 ? 20 : 9)));
  std::vector<int> mark(s.n_dof, -1), buf;
  for (int r = 0; r < s.n_dof; r++)
  {
    buf.clear();
    if (r < s.n_active)
    {
      for (int t = ptr[r]; t < ptr[r + 1]; t++)
      {
        int c = inc[t] / s.nbf;
        for (int j = 0; j < s.nbf; j++)
        {
          int d = s.h_gn[(size_t)c * s.nbf + j];
          if (mark[d] != r) { mark[d] = r; buf.push_back(d); }
        }
      }
      std::sort(buf.begin(), buf.end());
    }
    else
      buf.push_back(r);
    kcol.insert(kcol.end(), buf.begin(), buf.end());
    row_ptr[r + 1] = (int)kcol.size();
  }
}

// ---------------------------------------------------------------------------
// Prolongation as a sparse matrix.  The reference's Prolongate (src/FE/MGComponents3D.C:
// 182-462, MGComponents2D.C:118) applies per fine cell the coarse basis evaluated at the
// fine nodes in the parent's reference coordinates (GetProlongationMatrix3D,
// src/FE/FEDatabase3D.C:1630) and divides by the DOF multiplicity.  For conforming
// Lagrange elements all cells sharing a fine node agree, so P[i][j] = phi_j(x_i).
// The fine nodes of a nested refinement lie at dyadic reference points of the parent,
// where these values are exact multiples of 2^-12; they are snapped to that grid.
// DefectRestriction (MGComponents3D.C:706-988) is the transpose of the same map.
// ---------------------------------------------------------------------------
static void node_pos(int dim, int order, int b, double *xi)
{
  int k = order + 1;
  double h = 2.0 / order;
  xi[0] = -1 + h * (b % k);
  xi[1] = -1 + h * ((b / k) % k);
  if (dim == 3) xi[2] = -1 + h * (b / (k * k));
}

static void invert_map(int dim, bool affine, const double *V, const double *x, double *xi)
{
  for (int a = 0; a < dim; a++) xi[a] = 0;
  for (int it = 0; it < (affine ? 2 : 30); it++)
  {
    double y[3], J[9], Ji[9];
    ref_map(dim, affine, V, xi, y, J);
    invert(dim, J, Ji);
    double dmax = 0;
    double r[3];
    for (int a = 0; a < dim; a++) r[a] = x[a] - y[a];
    for (int b = 0; b < dim; b++)
    {
      double d = 0;
      for (int a = 0; a < dim; a++) d += Ji[b * dim + a] * r[a];
      xi[b] += d;
      dmax = std::max(dmax, std::fabs(d));
    }
    if (dmax < 1e-15) break;
  }
}

void build_prolongation(const Space &coarse, const Space &fine, const int *parent,
                        std::vector<int> &row, std::vector<int> &col, std::vector<double> &val)
{
  int dim = fine.dim, order = fine.order, nbf = fine.nbf, nv = fine.nv;
  std::vector<int> owner(fine.n_dof, -1), lb(fine.n_dof, 0);
  for (int c = 0; c < fine.n_cells; c++)
    for (int b = 0; b < nbf; b++)
    {
      int d = fine.h_gn[(size_t)c * nbf + b];
      if (owner[d] < 0) { owner[d] = c; lb[d] = b; }
    }
  row.assign(fine.n_dof + 1, 0);
  col.clear();
  val.clear();
  const double grid = std::ldexp(1.0, 12);
  for (int i = 0; i < fine.n_dof; i++)
  {
    int c = owner[i], p = parent[c];
    const double *Vf = &fine.h_coords[(size_t)c * nv * dim];
    const double *Vc = &coarse.h_coords[(size_t)p * nv * dim];
    double xi[3], x[3], J[9], eta[3], phi[CD_MAXBF];
    node_pos(dim, order, lb[i], xi);
    ref_map(dim, cell_is_affine(dim, Vf), Vf, xi, x, J);
    invert_map(dim, cell_is_affine(dim, Vc), Vc, x, eta);
    basis_eval(dim, order, eta, phi, nullptr);
    std::vector<std::pair<int, double>> e;
    for (int b = 0; b < nbf; b++)
    {
      double v = phi[b], s = std::nearbyint(v * grid) / grid;
      if (std::fabs(s - v) < 1e-10) v = s;
      if (v != 0.0) e.push_back({coarse.h_gn[(size_t)p * nbf + b], v});
    }
    std::sort(e.begin(), e.end());
    for (auto &kv : e) { col.push_back(kv.first); val.push_back(kv.second); }
    row[i + 1] = (int)col.size();
  }
}

// explicit inverse by Gauss-Jordan elimination with partial pivoting (row-major, in place)
bool dense_inverse(int n, std::vector<double> &a)
{
  std::vector<double> inv((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = 1.0;
  for (int k = 0; k < n; k++)
  {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(a[(size_t)i * n + k]) > std::fabs(a[(size_t)p * n + k])) p = i;
    if (a[(size_t)p * n + k] == 0.0) return false;
    if (p != k)
      for (int j = 0; j < n; j++)
      {
        std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
        std::swap(inv[(size_t)k * n + j], inv[(size_t)p * n + j]);
      }
    double d = a[(size_t)k * n + k];
    for (int j = 0; j < n; j++) { a[(size_t)k * n + j] /= d; inv[(size_t)k * n + j] /= d; }
    for (int i = 0; i < n; i++)
    {
      if (i == k) continue;
      double l = a[(size_t)i * n + k];
      if (l == 0.0) continue;
      for (int j = 0; j < n; j++)
      {
        a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
        inv[(size_t)i * n + j] -= l * inv[(size_t)k * n + j];
      }
    }
  }
  a.swap(inv);
  return true;
}

// threads per row of the CSR kernels: 1, 2 or 4 threads (8 loads each in flight) when that
// covers the longest row, 8 threads (16 loads each) up to 128 entries, else 32
CsrShape csr_shape(const int *rp, int n)
{
  int longest = 0;
  for (int r = 0; r < n; r++) longest = std::max(longest, rp[r + 1] - rp[r]);
  CsrShape sh;
  sh.gs = longest <= 8 ? 1 : longest <= 16 ? 2 : longest <= 32 ? 4 : longest <= 128 ? 8 : 32;
  return sh;
}
