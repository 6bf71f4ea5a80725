// TSystemCD2D on libcdgpu: the reference-side binding that lets ParMooN's own
// 2DPrograms/CD2D_ParMooN.C run unchanged with assembly and a multigrid solve on a B200.
//
// This file replaces src/System/SystemCD2D.C in a ParMooN build (same class, same header
// include/System/SystemCD2D.h).  The reference's TSystemCD2D holds one FE space and solves
// directly (UMFPACK; its GMG branch prints "not yet implemented", SystemCD2D.C:191-193).
// Here the solve is the library's multigrid-preconditioned FGMRES on a hierarchy that the
// binding builds from the mesh's refinement tree:
//
//   Init      coarser levels: the parents of the finest cells (TBaseCell::GetParent) form the
//             next coarser collection, and so on while every cell has a parent; each gets a
//             TFESpace2D of the same order and boundary conditions (the reference's own DOF
//             numbering); coarsest levels without active DOFs are dropped.  Every level is
//             uploaded (cell vertices, DOF map), its pattern built (bit-identical to
//             TSquareStructure2D + Sort), the hierarchy made from the parent maps, and the
//             example's BilinearCoeffs evaluated at the library's quadrature points of every
//             cell (a field that is the same everywhere becomes one constant record).
//   Assemble  every level assembled on the device; on the finest level the Dirichlet values
//             by the reference's nodal functionals on every Dirichlet edge and the Neumann
//             edges' boundary integral of BoundValue (the two branches of Assemble2D,
//             src/FE/Assemble2D.C:700-800), rhs copied into the caller's array, its
//             Dirichlet part into sol (SystemCD2D.C:125-179)
//   Solve     SOLVER_TYPE GMG: FGMRES / fixed point with the SC_* keys; any other solver type
//             (the main asks for DIRECT) is served by FGMRES(30) with one V(2,2) damped-Jacobi
//             cycle (omega 0.8) and the exact coarse solve, to ||r|| <= 1e-13 ||r0||.
//
// DISCTYPE GALERKIN (1) and SUPG (2) are accepted, others print a message and exit(4711), as
// do errors of the library.  CDGPU_PRECISION=1 selects the mixed form, CDGPU_DEVICE the GPU,
// CDGPU_DUMP_SOLUTION=<file> writes the solution for an external check.
#include <Database.h>
#include <FEDatabase2D.h>
#include <FESpace2D.h>
#include <NodalFunctional2D.h>
#include <BoundEdge.h>
#include <BoundComp2D.h>
#include <Joint.h>
#include <Collection.h>
#include <SystemCD2D.h>
#include <MooNMD_Io.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/cdgpu.h"

namespace
{
struct Shim2D
{
  cdgpu_ctx *ctx = nullptr;
  std::vector<TFESpace2D *> spaces; // coarsest first; the last is the main's own space
  std::vector<TCollection *> colls; // collections made here (coarse levels)
  std::vector<int> sids;
  int mg = -1;
  std::vector<double> rhs_scratch;
};

std::map<const TSystemCD2D *, Shim2D> g_state2d;

void check(cdgpu_ctx *ctx, int rc, const char *what)
{
  if (rc == CDGPU_OK) return;
  OutPut("libcdgpu: " << what << ": " << cdgpu_status_string(rc) << " (" << cdgpu_last_error(ctx) << ")" << endl);
  exit(4711);
}

int env_int(const char *name, int dflt)
{
  const char *v = getenv(name);
  return v ? atoi(v) : dflt;
}

// boundary edges of a space with the condition valid along them (Assemble2D tests both ends)
struct BdEdge
{
  int cell, m, comp;
  double t0, t1;
  BoundCond cond;
};

void boundary_edges(TFESpace2D *space, BoundCondFunct2D *bc, std::vector<BdEdge> &out)
{
  out.clear();
  TCollection *coll = space->GetCollection();
  const double eps = 1e-8;
  for (int c = 0; c < coll->GetN_Cells(); c++)
  {
    TBaseCell *cell = coll->GetCell(c);
    for (int m = 0; m < cell->GetN_Edges(); m++)
    {
      TJoint *joint = cell->GetJoint(m);
      if (joint->GetType() != BoundaryEdge) continue;
      TBoundEdge *be = (TBoundEdge *)joint;
      double t0, t1;
      be->GetParameters(t0, t1);
      const int comp = be->GetBoundComp()->GetID();
      BoundCond c0, c1;
      bc(comp, t0 < t1 ? t0 + eps : t0 - eps, c0);
      bc(comp, t0 < t1 ? t1 - eps : t1 + eps, c1);
      if (c0 != c1) continue; // the reference skips such edges too
      out.push_back(BdEdge{c, m, comp, t0, t1, c0});
    }
  }
}
} // namespace

TSystemCD2D::TSystemCD2D(TFESpace2D *fespace, int disctype, int solver)
{
  FeSpace = fespace;
  N_DOF = FeSpace->GetN_DegreesOfFreedom();
  N_Active = FeSpace->GetActiveBound();
  Disctype = disctype;
  SOLVER = solver;
  N_Matrices = 1;
  sqstructure = nullptr;
  sqmatrixA = nullptr;
  Shim2D &st = g_state2d[this];
  int rc = cdgpu_create(&st.ctx, env_int("CDGPU_DEVICE", 0));
  if (rc != CDGPU_OK)
  {
    OutPut("libcdgpu: no context: " << cdgpu_status_string(rc) << endl);
    exit(4711);
  }
}

TSystemCD2D::~TSystemCD2D()
{
  auto it = g_state2d.find(this);
  if (it == g_state2d.end()) return;
  cdgpu_destroy(it->second.ctx);
  for (size_t l = 0; l + 1 < it->second.spaces.size(); l++) delete it->second.spaces[l];
  for (TCollection *c : it->second.colls) delete c;
  g_state2d.erase(it);
}

void TSystemCD2D::Init(CoeffFct2D *BilinearCoeffs, BoundCondFunct2D *BoundCond, BoundValueFunct2D *BoundValue)
{
  if (Disctype != GALERKIN && Disctype != SUPG)
  {
    OutPut("Unknown DISCTYPE" << endl);
    exit(4711);
  }
  BoundaryConditions[0] = BoundCond;
  BoundaryValues[0] = BoundValue;
  Shim2D &st = g_state2d[this];
  const int *bi = FeSpace->GetBeginIndex();
  const int nbf = bi[1] - bi[0];
  const int order = nbf == 4 ? 1 : nbf == 9 ? 2 : 0;
  if (!order)
  {
    OutPut("libcdgpu: only Q1 and Q2 quadrilaterals are supported" << endl);
    exit(4711);
  }
  // the hierarchy from the refinement tree, finest first while building
  std::vector<TFESpace2D *> fine_first{FeSpace};
  std::vector<std::vector<int>> parent_maps; // parent_maps[k]: parents of level k's cells (finest first)
  char name[] = "cdgpu coarse level", desc[] = "coarse level of the libcdgpu multigrid";
  for (;;)
  {
    TCollection *coll = fine_first.back()->GetCollection();
    const int nc = coll->GetN_Cells();
    std::vector<TBaseCell *> parents;
    std::map<TBaseCell *, int> index;
    std::vector<int> pmap(nc);
    bool all = nc > 1;
    for (int c = 0; c < nc && all; c++)
    {
      TBaseCell *p = coll->GetCell(c)->GetParent();
      if (!p) { all = false; break; }
      auto it = index.find(p);
      if (it == index.end())
      {
        it = index.emplace(p, (int)parents.size()).first;
        parents.push_back(p);
      }
      pmap[c] = it->second;
    }
    if (!all) break;
    TBaseCell **cells = new TBaseCell *[parents.size()];
    for (size_t i = 0; i < parents.size(); i++) cells[i] = parents[i];
    TCollection *cc = new TCollection((int)parents.size(), cells);
    TFESpace2D *cs = new TFESpace2D(cc, name, desc, BoundCond, order, nullptr);
    if (cs->GetActiveBound() == 0)
    {
      delete cs;
      delete cc;
      break;
    }
    st.colls.push_back(cc);
    parent_maps.push_back(pmap);
    fine_first.push_back(cs);
  }
  const int L = (int)fine_first.size();
  st.spaces.assign(fine_first.rbegin(), fine_first.rend());
  std::vector<const int *> pp(L, nullptr);
  for (int l = 1; l < L; l++) pp[l] = parent_maps[L - 1 - l].data();
  for (int l = 0; l < L; l++)
  {
    TFESpace2D *sp = st.spaces[l];
    TCollection *coll = sp->GetCollection();
    const int nc = coll->GetN_Cells();
    std::vector<double> xy((size_t)nc * 8);
    for (int c = 0; c < nc; c++)
      for (int v = 0; v < 4; v++)
        coll->GetCell(c)->GetVertex(v)->GetCoords(xy[(size_t)c * 8 + v * 2], xy[(size_t)c * 8 + v * 2 + 1]);
    int sid, nnz;
    check(st.ctx, cdgpu_upload_space(st.ctx, 2, order, nc, xy.data(), sp->GetGlobalNumbers(), sp->GetBeginIndex(),
                                     sp->GetN_DegreesOfFreedom(), sp->GetActiveBound(), sp->GetHangingBound(), &sid),
          "upload_space");
    check(st.ctx, cdgpu_build_pattern(st.ctx, sid, &nnz), "build_pattern");
    st.sids.push_back(sid);
    // coefficients at the library's quadrature points (2D layout: eps, b1, b2, c, f)
    int nq = 0;
    check(st.ctx, cdgpu_quadrature_points(st.ctx, sid, nullptr, &nq), "quadrature_points");
    std::vector<double> q((size_t)nc * nq * 2), tab((size_t)nc * nq * 6);
    check(st.ctx, cdgpu_quadrature_points(st.ctx, sid, q.data(), &nq), "quadrature_points");
    std::vector<double> X(nq), Y(nq), cbuf((size_t)nq * 20), pbuf((size_t)nq * 20, 0.0);
    std::vector<double *> cptr(nq), pptr(nq);
    for (int k = 0; k < nq; k++)
    {
      cptr[k] = &cbuf[(size_t)k * 20];
      pptr[k] = &pbuf[(size_t)k * 20];
    }
    bool constant = true;
    for (int c = 0; c < nc; c++)
    {
      for (int k = 0; k < nq; k++)
      {
        X[k] = q[((size_t)c * nq + k) * 2];
        Y[k] = q[((size_t)c * nq + k) * 2 + 1];
      }
      std::fill(cbuf.begin(), cbuf.end(), 0.0);
      BilinearCoeffs(nq, X.data(), Y.data(), pptr.data(), cptr.data());
      for (int k = 0; k < nq; k++)
      {
        const double rec[6] = {cptr[k][0], cptr[k][1], cptr[k][2], 0.0, cptr[k][3], cptr[k][4]};
        for (int i = 0; i < 6; i++)
        {
          tab[((size_t)c * nq + k) * 6 + i] = rec[i];
          constant = constant && rec[i] == tab[i];
        }
      }
    }
    cdgpu_coeffs co;
    std::memset(&co, 0, sizeof(co));
    co.poly_degree = TDatabase::ParamDB->INTERNAL_POLYNOMIAL_DEGREE > 0 ? TDatabase::ParamDB->INTERNAL_POLYNOMIAL_DEGREE : 1;
    co.delta0 = TDatabase::ParamDB->DELTA0;
    co.eps = tab[0];
    co.b1 = tab[1];
    co.b2 = tab[2];
    co.c = tab[4];
    co.f = tab[5];
    co.kind = constant ? CDGPU_COEFF_CONSTANT : CDGPU_COEFF_TABLE;
    check(st.ctx, cdgpu_set_coeffs(st.ctx, sid, &co, constant ? nullptr : tab.data()), "set_coeffs");
  }
  check(st.ctx, cdgpu_hierarchy(st.ctx, L, st.sids.data(), pp.data(), &st.mg), "hierarchy");
  OutPut("libcdgpu: " << L << " multigrid levels from the refinement tree" << endl);
}

void TSystemCD2D::Assemble(TAuxParam2D *aux, double *sol, double *rhs)
{
  (void)aux;
  Shim2D &st = g_state2d[this];
  const int L = (int)st.spaces.size();
  for (int l = 0; l + 1 < L; l++) // coarse levels: matrices only (Dirichlet rows are identities)
  {
    check(st.ctx, cdgpu_assemble(st.ctx, st.sids[l], Disctype, nullptr, nullptr, nullptr), "assemble");
  }
  TCollection *coll = FeSpace->GetCollection();
  std::vector<BdEdge> edges;
  boundary_edges(FeSpace, BoundaryConditions[0], edges);
  // Dirichlet values by the nodal functionals of every Dirichlet edge (Assemble2D.C:737-752)
  std::vector<double> dir(N_DOF - N_Active, 0.0);
  int *gn = FeSpace->GetGlobalNumbers(), *bi = FeSpace->GetBeginIndex();
  double pv[MaxN_PointsForNodal2D], fv[MaxN_BaseFunctions2D];
  for (const BdEdge &e : edges)
  {
    if (e.cond != DIRICHLET) continue;
    TBaseCell *cell = coll->GetCell(e.cell);
    TFE2D *ele = TFEDatabase2D::GetFE2D(FeSpace->GetFE2D(e.cell, cell));
    TNodalFunctional2D *nf = ele->GetNodalFunctional2D();
    TFEDesc2D *desc = ele->GetFEDesc2D();
    int np;
    double *pts;
    nf->GetPointsForEdge(np, pts);
    for (int l = 0; l < np; l++) BoundaryValues[0](e.comp, 0.5 * (e.t0 * (1 - pts[l]) + e.t1 * (1 + pts[l])), pv[l]);
    nf->GetEdgeFunctionals(coll, cell, e.m, pv, fv);
    const int *jd = desc->GetJointDOF(e.m);
    const int *dof = gn + bi[e.cell];
    for (int l = 0; l < desc->GetN_JointDOF(); l++)
      if (dof[jd[l]] >= N_Active) dir[dof[jd[l]] - N_Active] = fv[l];
  }
  check(st.ctx, cdgpu_assemble(st.ctx, st.sids[L - 1], Disctype, dir.empty() ? nullptr : dir.data(), nullptr, rhs),
        "assemble");
  // Neumann edges: BoundValue at the library's Gauss points of the edge, parameter
  // t = t0 + (t1 - t0) s from vertex m (Assemble2D.C:753-786)
  std::vector<int> cells, locals;
  std::vector<double> g;
  const int nl = (bi[1] - bi[0]) == 9 ? 3 : 2;
  const double z3[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)}, z2[2] = {-1.0 / std::sqrt(3.0), 1.0 / std::sqrt(3.0)};
  for (const BdEdge &e : edges)
  {
    if (e.cond != NEUMANN && e.cond != ROBIN) continue;
    cells.push_back(e.cell);
    locals.push_back(e.m);
    for (int l = 0; l < nl; l++)
    {
      const double s = 0.5 * ((nl == 3 ? z3[l] : z2[l]) + 1);
      double v;
      BoundaryValues[0](e.comp, e.t0 + (e.t1 - e.t0) * s, v);
      g.push_back(v);
    }
  }
  if (!cells.empty())
    check(st.ctx, cdgpu_add_neumann(st.ctx, st.sids[L - 1], (int)cells.size(), cells.data(), locals.data(), g.data(), rhs),
          "add_neumann");
  std::memcpy(sol + N_Active, rhs + N_Active, (size_t)(N_DOF - N_Active) * sizeof(double));
}

void TSystemCD2D::Solve(double *sol, double *rhs)
{
  Shim2D &st = g_state2d[this];
  TParamDB *db = TDatabase::ParamDB;
  cdgpu_solver_params p;
  std::memset(&p, 0, sizeof(p));
  if (SOLVER == GMG)
  {
    p.solver = db->SC_SOLVER_SCALAR;
    p.restart = db->SC_GMRES_RESTART;
    p.maxit = db->SC_LIN_MAXIT_SCALAR;
    p.minit = db->SC_MINIT;
    p.smoother = db->SC_SMOOTHER_SCALAR;
    p.coarse_smoother = db->SC_COARSE_SMOOTHER_SCALAR;
    p.pre = db->SC_PRE_SMOOTH_SCALAR;
    p.post = db->SC_POST_SMOOTH_SCALAR;
    p.coarse_maxit = db->SC_COARSE_MAXIT_SCALAR;
    p.cycle = db->SC_MG_CYCLE_SCALAR;
    p.slc = db->SC_STEP_LENGTH_CONTROL_ALL_SCALAR || db->SC_STEP_LENGTH_CONTROL_FINE_SCALAR;
    p.stop_rule = 0;
    p.red_factor = db->SC_LIN_RED_FACTOR_SCALAR;
    p.res_norm_min = db->SC_LIN_RES_NORM_MIN_SCALAR;
    p.div_factor = db->SC_DIV_FACTOR;
    p.omega = db->SC_SMOOTH_DAMP_FACTOR_SCALAR;
    p.coarse_red = db->SC_COARSE_RED_FACTOR_SCALAR;
    p.gmg_damp = db->SC_GMG_DAMP_FACTOR_SCALAR;
  }
  else
  {
    // the direct solve the main asks for, served by the multigrid FGMRES to 1e-13
    p.solver = 16;
    p.restart = 30;
    p.maxit = 1000;
    p.smoother = 1;
    p.coarse_smoother = 17;
    p.pre = p.post = 2;
    p.coarse_maxit = 10;
    p.cycle = 1;
    p.stop_rule = 1;
    p.red_factor = 1e-13;
    p.div_factor = 1e10;
    p.omega = 0.8;
    p.coarse_red = 0.1;
    p.gmg_damp = 1.0;
  }
  p.precision = env_int("CDGPU_PRECISION", 0);
  cdgpu_solve_info info;
  check(st.ctx, cdgpu_solve(st.ctx, st.mg, &p, rhs, sol, &info), "solve");
  OutPut("libcdgpu " << (p.solver == 11 ? "FIXED POINT" : "FGMRES") << " ITE: " << info.iterations
                     << " res: " << info.final_residual << " initial: " << info.initial_residual << endl);
  if (info.status == CDGPU_ERR_DIVERGED)
  {
    OutPut("libcdgpu: solver diverged" << endl);
    exit(4711);
  }
  if (info.status == CDGPU_ERR_NOT_CONVERGED) OutPut("libcdgpu: solver not converged" << endl);
  if (const char *path = getenv("CDGPU_DUMP_SOLUTION"))
  {
    if (FILE *f = fopen(path, "wb"))
    {
      fwrite(sol, sizeof(double), N_DOF, f);
      fclose(f);
    }
  }
}
