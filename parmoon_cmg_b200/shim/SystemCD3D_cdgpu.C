// TSystemCD3D on libcdgpu: the reference-side binding that lets ParMooN's own
// 3DPrograms/CD3D_ParMooN.C run unchanged with assembly and multigrid solve on a B200.
//
// This file replaces src/System/SystemCD3D.C in a ParMooN build (same class, same header
// include/System/SystemCD3D.h, same call surface: constructor, Init, Assemble, Solve,
// destructor) and links libcdgpu.so.  It is compiled against the reference's headers; the
// rest of ParMooN (mesh, FE spaces, output, error evaluation) is unchanged.
//
//   constructor  uploads every multigrid level's cell vertices and DOF map
//                (TFESpace3D::GetGlobalNumbers / GetBeginIndex / GetActiveBound), builds
//                the CSR pattern on the library side (bit-identical to TSquareStructure3D +
//                Sort) and the hierarchy from the cells' parents (TBaseCell::GetParent)
//   Init         evaluates the example's BilinearCoeffs at the library's quadrature points
//                of every cell (a constant field becomes one coefficient record); keeps
//                BoundCondition / BoundValue for the Dirichlet data
//   Assemble     per level: Dirichlet values by the reference's nodal functionals on every
//                Dirichlet face (the loop of TAssembleMat3D::Assemble3D,
//                src/System/AssembleMat3D.C:969-1066), cdgpu_assemble into RhsArray[i]
//                (entries stay on the device), the Neumann / Robin faces' boundary integral
//                of the example's BoundValue (AssembleMat3D.C:1068-1170) by
//                cdgpu_add_neumann, Dirichlet part of rhs copied into SolArray[i]
//                (src/System/SystemCD3D.C:314-339)
//   Solve        cdgpu_solve with the ParamDB keys of TSystemCD3D::Solve's GMG branch
//                (FGMRES 16 / fixed point 11, multigrid preconditioner 5)
//
// Like the reference, only DISCTYPE GALERKIN and SOLVER_TYPE GMG are accepted; other values
// print a message and exit(4711).  The multigrid runs in FP64 (the drop-in) unless the
// environment variable CDGPU_PRECISION=1 selects the mixed form; CDGPU_DEVICE picks the GPU.
// Errors of the library are reported as the reference reports its own: a message and
// exit(4711).
#include <Database.h>
#include <FEDatabase3D.h>
#include <FESpace3D.h>
#include <NodalFunctional3D.h>
#include <BoundFace.h>
#include <BoundComp3D.h>
#include <Joint.h>
#include <SystemCD3D.h>
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
struct ShimState
{
  cdgpu_ctx *ctx = nullptr;
  std::vector<int> sids;
  int mg = -1;
  CoeffFct3D *coeffs = nullptr;
};

std::map<const TSystemCD3D *, ShimState> g_state;

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

// Dirichlet values of one level's DOFs [ActiveBound, N_DOF): the nodal functionals of every
// boundary face whose centre has a DIRICHLET condition, as TAssembleMat3D::Assemble3D sets
// RHS[DOF] on such faces (non-isoparametric branch)
void dirichlet_values(TFESpace3D *space, BoundCondFunct3D *bc, BoundValueFunct3D *bv, std::vector<double> &dir)
{
  TCollection *coll = space->GetCollection();
  const int n = space->GetN_DegreesOfFreedom(), na = space->GetActiveBound();
  dir.assign(n - na, 0.0);
  int *gn = space->GetGlobalNumbers(), *bi = space->GetBeginIndex();
  double *xi, *eta, *zeta; // the nodal functional's own face points
  double X[MaxN_PointsForNodal3D], Y[MaxN_PointsForNodal3D], Z[MaxN_PointsForNodal3D];
  double absdet[MaxN_PointsForNodal3D], pv[MaxN_PointsForNodal3D], fv[MaxN_PointsForNodal3D];
  for (int c = 0; c < coll->GetN_Cells(); c++)
  {
    TBaseCell *cell = coll->GetCell(c);
    FE3D fe = space->GetFE3D(c, cell);
    TFE3D *ele = TFEDatabase3D::GetFE3D(fe);
    TNodalFunctional3D *nf = ele->GetNodalFunctional3D();
    TFEDesc3D *desc = ele->GetFEDesc3D();
    const RefTrans3D rt = ele->GetRefTransID();
    const int *dof = gn + bi[c];
    const int *fv_idx, *flen;
    int maxlen;
    cell->GetShapeDesc()->GetFaceVertex(fv_idx, flen, maxlen);
    bool map_set = false;
    for (int m = 0; m < cell->GetN_Faces(); m++)
    {
      TJoint *joint = cell->GetJoint(m);
      if (joint->GetType() != BoundaryFace && joint->GetType() != IsoBoundFace) continue;
      double xf = 0, yf = 0, zf = 0;
      for (int l = 0; l < flen[m]; l++)
      {
        double x, y, z;
        cell->GetVertex(fv_idx[m * maxlen + l])->GetCoords(x, y, z);
        xf += x / flen[m];
        yf += y / flen[m];
        zf += z / flen[m];
      }
      const int id = ((TBoundFace *)joint)->GetBoundComp()->GetID();
      BoundCond cond;
      bc(id, xf, yf, zf, cond); // the face takes the condition valid at its centre
      if (cond != DIRICHLET) continue;
      if (!map_set)
      {
        TFEDatabase3D::SetCellForRefTrans(cell, rt);
        map_set = true;
      }
      int np;
      nf->GetPointsForFace(m, np, xi, eta, zeta);
      TFEDatabase3D::GetOrigFromRef(rt, np, xi, eta, zeta, X, Y, Z, absdet);
      for (int l = 0; l < np; l++) bv(id, X[l], Y[l], Z[l], pv[l]);
      nf->GetFaceFunctionals(coll, cell, m, pv, fv);
      const int *jd = desc->GetJointDOF(m);
      for (int l = 0; l < desc->GetN_JointDOF(); l++)
        if (dof[jd[l]] >= na) dir[dof[jd[l]] - na] = fv[l];
    }
  }
}
// boundary faces whose centre has a NEUMANN or ROBIN condition (their rhs part, as
// TAssembleMat3D::Assemble3D adds it; the Robin matrix part belongs to the main program)
void neumann_faces(TFESpace3D *space, BoundCondFunct3D *bc, std::vector<int> &cells, std::vector<int> &faces,
                   std::vector<int> &ids)
{
  TCollection *coll = space->GetCollection();
  cells.clear();
  faces.clear();
  ids.clear();
  for (int c = 0; c < coll->GetN_Cells(); c++)
  {
    TBaseCell *cell = coll->GetCell(c);
    const int *fv_idx, *flen;
    int maxlen;
    cell->GetShapeDesc()->GetFaceVertex(fv_idx, flen, maxlen);
    for (int m = 0; m < cell->GetN_Faces(); m++)
    {
      TJoint *joint = cell->GetJoint(m);
      if (joint->GetType() != BoundaryFace && joint->GetType() != IsoBoundFace) continue;
      double xf = 0, yf = 0, zf = 0;
      for (int l = 0; l < flen[m]; l++)
      {
        double x, y, z;
        cell->GetVertex(fv_idx[m * maxlen + l])->GetCoords(x, y, z);
        xf += x / flen[m];
        yf += y / flen[m];
        zf += z / flen[m];
      }
      const int id = ((TBoundFace *)joint)->GetBoundComp()->GetID();
      BoundCond cond;
      bc(id, xf, yf, zf, cond);
      if (cond != NEUMANN && cond != ROBIN) continue;
      cells.push_back(c);
      faces.push_back(m);
      ids.push_back(id);
    }
  }
}
} // namespace

TSystemCD3D::TSystemCD3D(int N_levels, TFESpace3D **fespaces, double **sol, double **rhs, int disctype, int solver)
{
  N_Levels = N_levels;
  FeSpaces = fespaces;
  SolArray = sol;
  RhsArray = rhs;
  Disctype = disctype;
  SOLVER = solver;
  N_DOF = FeSpaces[N_Levels - 1]->GetN_DegreesOfFreedom();
  Start_Level = 0;
  sqstructure = nullptr;
  sqmatrixA = nullptr;
  AMatRhsAssemble = nullptr;
  Itmethod = prec = nullptr;
  MG = nullptr;
  if (SOLVER != GMG)
  {
    OutPut("libcdgpu: only SOLVER_TYPE GMG (" << GMG << ") runs on the GPU" << endl);
    exit(4711);
  }
  ShimState &st = g_state[this];
  int rc = cdgpu_create(&st.ctx, env_int("CDGPU_DEVICE", 0));
  if (rc != CDGPU_OK)
  {
    OutPut("libcdgpu: no context: " << cdgpu_status_string(rc) << endl);
    exit(4711);
  }
  std::vector<std::vector<int>> parents(N_Levels);
  for (int l = 0; l < N_Levels; l++)
  {
    TFESpace3D *sp = FeSpaces[l];
    TCollection *coll = sp->GetCollection();
    const int nc = coll->GetN_Cells();
    std::vector<double> xyz((size_t)nc * 24);
    for (int c = 0; c < nc; c++)
      for (int v = 0; v < 8; v++)
        coll->GetCell(c)->GetVertex(v)->GetCoords(xyz[(size_t)c * 24 + v * 3], xyz[(size_t)c * 24 + v * 3 + 1],
                                                  xyz[(size_t)c * 24 + v * 3 + 2]);
    const int *bi = sp->GetBeginIndex();
    const int nbf = bi[1] - bi[0];
    const int order = nbf == 8 ? 1 : nbf == 27 ? 2 : 0;
    if (!order)
    {
      OutPut("libcdgpu: only Q1 and Q2 hexahedra are supported" << endl);
      exit(4711);
    }
    int sid;
    check(st.ctx, cdgpu_upload_space(st.ctx, 3, order, nc, xyz.data(), sp->GetGlobalNumbers(), bi,
                                     sp->GetN_DegreesOfFreedom(), sp->GetActiveBound(), sp->GetHangingBound(), &sid),
          "upload_space");
    int nnz;
    check(st.ctx, cdgpu_build_pattern(st.ctx, sid, &nnz), "build_pattern");
    st.sids.push_back(sid);
    if (l > 0)
    {
      TCollection *cc = FeSpaces[l - 1]->GetCollection();
      for (int c = 0; c < cc->GetN_Cells(); c++) cc->GetCell(c)->SetClipBoard(c);
      parents[l].resize(nc);
      for (int c = 0; c < nc; c++) parents[l][c] = coll->GetCell(c)->GetParent()->GetClipBoard();
    }
  }
  std::vector<const int *> pp(N_Levels, nullptr);
  for (int l = 1; l < N_Levels; l++) pp[l] = parents[l].data();
  check(st.ctx, cdgpu_hierarchy(st.ctx, N_Levels, st.sids.data(), pp.data(), &st.mg), "hierarchy");
}

TSystemCD3D::~TSystemCD3D()
{
  auto it = g_state.find(this);
  if (it == g_state.end()) return;
  cdgpu_destroy(it->second.ctx);
  g_state.erase(it);
}

void TSystemCD3D::Init(CoeffFct3D *BilinearCoeffs, BoundCondFunct3D *BoundCond, BoundValueFunct3D *BoundValue,
                       TAuxParam3D *aux)
{
  (void)aux; // no FE-function parameters on this path (TAuxParam3D with N_Parameters 0)
  if (Disctype != GALERKIN)
  {
    OutPut("Unknown DISCTYPE" << endl);
    exit(4711);
  }
  BoundaryConditions[0] = BoundCond;
  BoundaryValues[0] = BoundValue;
  ShimState &st = g_state[this];
  st.coeffs = BilinearCoeffs;
  // the coefficients at the library's quadrature points of every cell; a field that is the
  // same everywhere is handed over as one constant record (the affine fast path)
  for (int l = 0; l < N_Levels; l++)
  {
    const int sid = st.sids[l];
    const int nc = FeSpaces[l]->GetCollection()->GetN_Cells();
    int nq = 0;
    check(st.ctx, cdgpu_quadrature_points(st.ctx, sid, nullptr, &nq), "quadrature_points");
    std::vector<double> q((size_t)nc * nq * 3), tab((size_t)nc * nq * 6);
    check(st.ctx, cdgpu_quadrature_points(st.ctx, sid, q.data(), &nq), "quadrature_points");
    std::vector<double> X(nq), Y(nq), Z(nq), cbuf((size_t)nq * 20), pbuf((size_t)nq * 20, 0.0);
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
        X[k] = q[((size_t)c * nq + k) * 3];
        Y[k] = q[((size_t)c * nq + k) * 3 + 1];
        Z[k] = q[((size_t)c * nq + k) * 3 + 2];
      }
      std::fill(cbuf.begin(), cbuf.end(), 0.0);
      BilinearCoeffs(nq, X.data(), Y.data(), Z.data(), pptr.data(), cptr.data());
      for (int k = 0; k < nq; k++)
        for (int i = 0; i < 6; i++)
        {
          double v = cptr[k][i];
          tab[((size_t)c * nq + k) * 6 + i] = v;
          constant = constant && v == tab[i];
        }
    }
    cdgpu_coeffs co;
    std::memset(&co, 0, sizeof(co));
    co.poly_degree = TDatabase::ParamDB->INTERNAL_POLYNOMIAL_DEGREE > 0 ? TDatabase::ParamDB->INTERNAL_POLYNOMIAL_DEGREE : 1;
    co.delta0 = TDatabase::ParamDB->DELTA0;
    co.eps = tab[0];
    co.b1 = tab[1];
    co.b2 = tab[2];
    co.b3 = tab[3];
    co.c = tab[4];
    co.f = tab[5];
    co.kind = constant ? CDGPU_COEFF_CONSTANT : CDGPU_COEFF_TABLE;
    check(st.ctx, cdgpu_set_coeffs(st.ctx, sid, &co, constant ? nullptr : tab.data()), "set_coeffs");
  }
}

void TSystemCD3D::Assemble()
{
  ShimState &st = g_state[this];
  std::vector<double> dir;
  for (int i = 0; i < N_Levels; i++)
  {
    TFESpace3D *sp = FeSpaces[i];
    const int n = sp->GetN_DegreesOfFreedom(), na = sp->GetActiveBound();
    dirichlet_values(sp, BoundaryConditions[0], BoundaryValues[0], dir);
    check(st.ctx, cdgpu_assemble(st.ctx, st.sids[i], Disctype, dir.empty() ? nullptr : dir.data(), nullptr, RhsArray[i]),
          "assemble");
    // Neumann data: the example's BoundValue at the library's Gauss points of every such face
    std::vector<int> cells, faces, ids;
    neumann_faces(sp, BoundaryConditions[0], cells, faces, ids);
    if (!cells.empty())
    {
      const int order = sp->GetBeginIndex()[1] - sp->GetBeginIndex()[0] == 27 ? 2 : 1, nq = (order + 1) * (order + 1);
      std::vector<double> xyz(cells.size() * nq * 3), g(cells.size() * nq);
      check(st.ctx, cdgpu_boundary_points(st.ctx, st.sids[i], (int)cells.size(), cells.data(), faces.data(), xyz.data()),
            "boundary_points");
      for (size_t e = 0; e < cells.size(); e++)
        for (int q = 0; q < nq; q++)
        {
          const double *x = &xyz[(e * nq + q) * 3];
          BoundaryValues[0](ids[e], x[0], x[1], x[2], g[e * nq + q]);
        }
      check(st.ctx, cdgpu_add_neumann(st.ctx, st.sids[i], (int)cells.size(), cells.data(), faces.data(), g.data(),
                                      RhsArray[i]),
            "add_neumann");
    }
    std::memcpy(SolArray[i] + na, RhsArray[i] + na, (size_t)(n - na) * sizeof(double));
  }
}

void TSystemCD3D::Solve(double *sol, double *rhs)
{
  ShimState &st = g_state[this];
  TParamDB *db = TDatabase::ParamDB;
  if (db->SC_PRECONDITIONER_SCALAR != 5)
  {
    OutPut("libcdgpu: SC_PRECONDITIONER_SCALAR must be 5 (multigrid)" << endl);
    exit(4711);
  }
  cdgpu_solver_params p;
  std::memset(&p, 0, sizeof(p));
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
  p.precision = env_int("CDGPU_PRECISION", 0);
  p.stop_rule = 0; // the reference's own rule (FgmresIte.C:430-431, 557)
  p.red_factor = db->SC_LIN_RED_FACTOR_SCALAR;
  p.res_norm_min = db->SC_LIN_RES_NORM_MIN_SCALAR;
  p.div_factor = db->SC_DIV_FACTOR;
  p.omega = db->SC_SMOOTH_DAMP_FACTOR_SCALAR;
  p.coarse_red = db->SC_COARSE_RED_FACTOR_SCALAR;
  p.gmg_damp = db->SC_GMG_DAMP_FACTOR_SCALAR;
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
  // optional copy of the solution and of the DOF positions (TFESpace3D::GetDOFPosition) for an
  // external check (no counterpart in the reference)
  if (const char *path = getenv("CDGPU_DUMP_SOLUTION"))
  {
    if (FILE *f = fopen(path, "wb"))
    {
      fwrite(sol, sizeof(double), N_DOF, f);
      fclose(f);
    }
    std::vector<double> x(N_DOF), y(N_DOF), z(N_DOF), xyz(3 * (size_t)N_DOF);
    FeSpaces[N_Levels - 1]->GetDOFPosition(x.data(), y.data(), z.data());
    for (int i = 0; i < N_DOF; i++)
    {
      xyz[3 * (size_t)i] = x[i];
      xyz[3 * (size_t)i + 1] = y[i];
      xyz[3 * (size_t)i + 2] = z[i];
    }
    std::string p2 = std::string(path) + ".xyz";
    if (FILE *f = fopen(p2.c_str(), "wb"))
    {
      fwrite(xyz.data(), sizeof(double), xyz.size(), f);
      fclose(f);
    }
  }
}
