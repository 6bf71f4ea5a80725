// Project-written driver for the compiled reference, 3D (test infrastructure only).
//
// Runs ParMooN's own stationary CD3D path -- TDomain refinement, TFESpace3D,
// TSystemCD3D(Init, Assemble, Solve) with TMultiGridScaIte + TFgmresIte -- the
// same call sequence as 3DPrograms/CD3D_ParMooN.C:388-441, on a mesh given by
// the .dat file, with constant coefficients from the command line:
//
//   cd3d_dump <file.dat> <outdir|-> eps b1 b2 b3 c f [prolong_max_ndof]
//
// and writes every array the GPU path consumes or produces (cell vertices, DOF
// maps, CSR pattern, matrix entries, right-hand sides, parent maps, the dense
// prolongation on small levels, the solution) plus wall-clock timings of
// Assemble() and Solve() measured with std::chrono::steady_clock (the
// reference's own GetTime() is CPU user time, src/General/MainUtilities.C:54).
// With outdir "-" nothing is written and only the timing line is printed.
#include <Domain.h>
#include <Database.h>
#include <FEDatabase3D.h>
#include <LinAlg.h>
#include <FESpace3D.h>
#include <SystemCD3D.h>
#include <MainUtilities.h>
#include <LinAlg.h>
#include <ItMethod.h>
#include <FgmresIte.h>
#include <FixedPointIte.h>

#include <string.h>
#include <math.h>
#include <vector>

#include "dump_common.h"

double bound = 0;
double timeC = 0;

static double C_eps = 1, C_b1 = 0, C_b2 = 0, C_b3 = 0, C_c = 0, C_f = 1;

void ExampleFile() { OutPut("Example: constant-coefficient CD3D dump driver" << endl); }

void Exact(double x, double y, double z, double *values)
{
  for (int i = 0; i < 5; i++) values[i] = 0;
}

void BoundCondition(int BdID, double x, double y, double z, BoundCond &cond) { cond = DIRICHLET; }

void BoundValue(int BdID, double x, double y, double z, double &value) { value = 0; }

void BilinearCoeffs(int n_points, double *x, double *y, double *z,
                    double **parameters, double **coeffs)
{
  for (int i = 0; i < n_points; i++)
  {
    double *c = coeffs[i];
    c[0] = C_eps; c[1] = C_b1; c[2] = C_b2; c[3] = C_b3; c[4] = C_c; c[5] = C_f;
  }
}

// exposes the protected members of the reference facade without changing it
class DumpSystemCD3D : public TSystemCD3D
{
 public:
  DumpSystemCD3D(int n, TFESpace3D **s, double **sol, double **rhs, int disc, int solver)
      : TSystemCD3D(n, s, sol, rhs, disc, solver) {}
  TSquareMatrix3D *A(int i) { return sqmatrixA[i]; }
  // same steps as TSystemCD3D::Solve GMG branch (src/System/SystemCD3D.C:348-368), returning
  // the iteration count that the facade discards
  int SolveCount(double *sol, double *rhs)
  {
    if (TDatabase::ParamDB->SC_PRECONDITIONER_SCALAR == 5)
    {
      memcpy(Itmethod_sol, sol, N_DOF * SizeOfDouble);
      memcpy(Itmethod_rhs, rhs, N_DOF * SizeOfDouble);
    }
    else { Itmethod_sol = sol; Itmethod_rhs = rhs; }
    int its = Itmethod->Iterate(sqmatrices, NULL, Itmethod_sol, Itmethod_rhs);
    if (TDatabase::ParamDB->SC_PRECONDITIONER_SCALAR == 5)
    {
      memcpy(sol, Itmethod_sol, N_DOF * SizeOfDouble);
      memcpy(rhs, Itmethod_rhs, N_DOF * SizeOfDouble);
    }
    return its;
  }
  // one application of the multigrid preconditioner (TMultiGridScaIte::Iterate)
  void ApplyPrec(double *z, double *r) { prec->Iterate(sqmatrices, NULL, z, r); }
  // re-create the Krylov method after ParamDB changes, with the constructor calls of
  // src/System/SystemCD3D.C:180-199 (the method reads its tolerances when constructed)
  void RebuildKrylov()
  {
    delete Itmethod;
    if (TDatabase::ParamDB->SC_SOLVER_SCALAR == 11)
      Itmethod = new TFixedPointIte(MatVect_Scalar, Defect_Scalar, prec, 0, N_DOF, 1);
    else
      Itmethod = new TFgmresIte(MatVect_Scalar, Defect_Scalar, prec, 0, N_DOF, 1);
  }
};

int main(int argc, char *argv[])
{
  if (argc < 9)
  {
    fprintf(stderr, "usage: %s file.dat outdir|- eps b1 b2 b3 c f [prolong_max_ndof [rtol_initial]]\n",
            argv[0]);
    return 2;
  }
  TDatabase *Database = new TDatabase();
  TFEDatabase3D *FEDatabase = new TFEDatabase3D();
  TDomain *Domain = new TDomain(argv[1]);
  const char *outdir = strcmp(argv[2], "-") ? argv[2] : nullptr;
  C_eps = atof(argv[3]); C_b1 = atof(argv[4]); C_b2 = atof(argv[5]); C_b3 = atof(argv[6]);
  C_c = atof(argv[7]); C_f = atof(argv[8]);
  long prolong_max = argc > 9 ? atol(argv[9]) : 0;
  double rtol_initial = argc > 10 ? atof(argv[10]) : 0.0; // > 0: stop relative to the initial residual
  dump_open(outdir);

  if (TDatabase::ParamDB->PROBLEM_TYPE == 0) TDatabase::ParamDB->PROBLEM_TYPE = 1;
  OpenFiles();

  double t0 = wall_now();
  Domain->Init(TDatabase::ParamDB->BNDFILE, TDatabase::ParamDB->GEOFILE);
  int LEVELS = TDatabase::ParamDB->LEVELS;
  for (int i = 0; i < TDatabase::ParamDB->UNIFORM_STEPS; i++) Domain->RegRefineAll();

  int ORDER = TDatabase::ParamDB->ANSATZ_ORDER;
  std::vector<TCollection *> colls(LEVELS);
  TFESpace3D **spaces = new TFESpace3D *[LEVELS + 1];
  double **Sol = new double *[LEVELS + 1];
  double **Rhs = new double *[LEVELS + 1];
  char Name[] = "name", Desc[] = "description";
  for (int i = 0; i < LEVELS; i++)
  {
    if (i) Domain->RegRefineAll();
    colls[i] = Domain->GetCollection(It_Finest, 0);
    spaces[i] = new TFESpace3D(colls[i], Name, Desc, BoundCondition, ORDER);
    int n = spaces[i]->GetN_DegreesOfFreedom();
    Sol[i] = new double[n];
    Rhs[i] = new double[n];
    memset(Sol[i], 0, n * sizeof(double));
    memset(Rhs[i], 0, n * sizeof(double));
  }
  double t_mesh = wall_now() - t0;

  t0 = wall_now();
  DumpSystemCD3D *S = new DumpSystemCD3D(LEVELS, spaces, Sol, Rhs,
                                         TDatabase::ParamDB->DISCTYPE,
                                         TDatabase::ParamDB->SOLVER_TYPE);
  S->Init(BilinearCoeffs, BoundCondition, BoundValue, NULL);
  double t_construct = wall_now() - t0;

  t0 = wall_now();
  S->Assemble();
  double t_assemble = wall_now() - t0;

  meta_i("levels", LEVELS);
  meta_i("order", ORDER);
  for (int l = 0; l < LEVELS; l++)
  {
    TFESpace3D *sp = spaces[l];
    TCollection *coll = colls[l];
    int n_cells = coll->GetN_Cells();
    int n = sp->GetN_DegreesOfFreedom();
    int *bi = sp->GetBeginIndex();
    int nbf = bi[1] - bi[0];
    TSquareMatrix3D *A = S->A(l);
    int nnz = A->GetRowPtr()[n];
    meta_i(lvl(l, "n_dof"), n);
    meta_i(lvl(l, "n_active"), sp->GetN_ActiveDegrees());
    meta_i(lvl(l, "hanging_bound"), sp->GetHangingBound());
    meta_i(lvl(l, "n_dirichlet"), sp->GetN_Dirichlet());
    meta_i(lvl(l, "n_cells"), n_cells);
    meta_i(lvl(l, "n_bf"), nbf);
    meta_i(lvl(l, "nnz"), nnz);
    if (!outdir) continue;
    std::vector<double> xyz((size_t)n_cells * 8 * 3);
    for (int c = 0; c < n_cells; c++)
    {
      TBaseCell *cell = coll->GetCell(c);
      for (int v = 0; v < 8; v++)
      {
        double x, y, z;
        cell->GetVertex(v)->GetCoords(x, y, z);
        xyz[(size_t)c * 24 + v * 3 + 0] = x;
        xyz[(size_t)c * 24 + v * 3 + 1] = y;
        xyz[(size_t)c * 24 + v * 3 + 2] = z;
      }
    }
    dump_f64(lvl(l, "coords"), xyz.data(), (long)xyz.size());
    dump_i32(lvl(l, "begin_index"), bi, n_cells + 1);
    dump_i32(lvl(l, "global_numbers"), sp->GetGlobalNumbers(), bi[n_cells]);
    dump_i32(lvl(l, "row_ptr"), A->GetRowPtr(), n + 1);
    dump_i32(lvl(l, "kcol"), A->GetKCol(), nnz);
    dump_f64(lvl(l, "entries"), A->GetEntries(), nnz);
    dump_f64(lvl(l, "rhs"), Rhs[l], n);
    if (l > 0)
    {
      TCollection *cc = colls[l - 1];
      for (int c = 0; c < cc->GetN_Cells(); c++) cc->GetCell(c)->SetClipBoard(c);
      std::vector<int> parent(n_cells), child(n_cells);
      for (int c = 0; c < n_cells; c++)
      {
        TBaseCell *cell = coll->GetCell(c);
        TBaseCell *p = cell->GetParent();
        parent[c] = p->GetClipBoard();
        child[c] = p->GetChildNumber(cell);
      }
      dump_i32(lvl(l, "parent"), parent.data(), n_cells);
      dump_i32(lvl(l, "child"), child.data(), n_cells);
      int nc = spaces[l - 1]->GetN_DegreesOfFreedom();
      if ((long)n * nc <= prolong_max)
      {
        // the reference's cell-wise prolongation (src/FE/MGComponents3D.C:182) applied to unit vectors
        std::vector<double> P((size_t)n * nc), e(nc), out(n), aux(n);
        for (int j = 0; j < nc; j++)
        {
          std::fill(e.begin(), e.end(), 0.0);
          e[j] = 1.0;
          Prolongate(spaces[l - 1], sp, e.data(), out.data(), aux.data());
          for (int i = 0; i < n; i++) P[(size_t)i * nc + j] = out[i];
        }
        dump_f64(lvl(l, "prolong_dense"), P.data(), (long)P.size());
      }
    }
  }

  int its = -1;
  double t_solve = 0;
  int nf = spaces[LEVELS - 1]->GetN_DegreesOfFreedom();
  if (TDatabase::ParamDB->SOLVER_TYPE == 1 && outdir)
  {
    // the preconditioner applied once to the assembled right-hand side; it works in the
    // finest level's own sol/rhs arrays, so those are saved and restored around it
    std::vector<double> s0(Sol[LEVELS - 1], Sol[LEVELS - 1] + nf), r0(Rhs[LEVELS - 1], Rhs[LEVELS - 1] + nf);
    std::vector<double> z(nf, 0.0), r(r0);
    S->ApplyPrec(z.data(), r.data());
    dump_f64("prec_rhs", z.data(), nf);
    memcpy(Sol[LEVELS - 1], s0.data(), nf * sizeof(double));
    memcpy(Rhs[LEVELS - 1], r0.data(), nf * sizeof(double));
  }
  if (TDatabase::ParamDB->SOLVER_TYPE == 1)
  {
    t0 = wall_now();
    if (rtol_initial > 0)
    {
      // stop at ||r|| <= rtol * ||r0||: the absolute SC_LIN_RES_NORM_MIN_SCALAR set from the
      // initial residual (ScalarDefect, src/FE/Blas2.C:11), relative test switched off
      std::vector<double> d(nf);
      double r0 = 0;
      ScalarDefect(S->A(LEVELS - 1), Sol[LEVELS - 1], Rhs[LEVELS - 1], d.data(), r0);
      TDatabase::ParamDB->SC_LIN_RES_NORM_MIN_SCALAR = rtol_initial * r0;
      TDatabase::ParamDB->SC_LIN_RED_FACTOR_SCALAR = 0.0;
      S->RebuildKrylov();
      meta_d("initial_residual", r0);
    }
    its = S->SolveCount(Sol[LEVELS - 1], Rhs[LEVELS - 1]);
    t_solve = wall_now() - t0;
    dump_f64("solution", Sol[LEVELS - 1], nf);
  }
  meta_i("iterations", its);
  meta_d("t_mesh", t_mesh);
  meta_d("t_construct", t_construct);
  meta_d("t_assemble", t_assemble);
  meta_d("t_solve", t_solve);
  printf("{\"n_dof\": %d, \"n_cells\": %d, \"iterations\": %d, \"t_mesh\": %.6f, "
         "\"t_construct\": %.6f, \"t_assemble\": %.6f, \"t_solve\": %.6f}\n",
         nf, colls[LEVELS - 1]->GetN_Cells(), its, t_mesh, t_construct, t_assemble, t_solve);
  if (g_meta) fclose(g_meta);
  CloseFiles();
  return 0;
}
