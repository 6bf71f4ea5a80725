// Project-written driver for the compiled reference, 2D (test infrastructure only).
//
// Runs ParMooN's own stationary CD2D assembly -- TDomain refinement, TFESpace2D,
// TSystemCD2D(Init, Assemble) per level (src/System/SystemCD2D.C:39-179) -- and,
// because TSystemCD2D::Solve has no multigrid branch (src/System/SystemCD2D.C:191-193),
// wires the reference's own 2D multigrid classes (TMultiGrid2D, TMGLevel2D,
// TMultiGridScaIte, TFgmresIte / TFixedPointIte) the same way TSystemCD3D does in
// 3D (src/System/SystemCD3D.C:147-199, 285-308, 342-368):
//
//   cd2d_dump <file.dat> <outdir|-> example eps b1 b2 c f [prolong_max_ndof]
//
// example 0: constant coefficients from the command line, Dirichlet 0 on the whole boundary.
// example 1: the sine problem of Examples/CD_2D/SineLaplace.h (eps = 1/PE_NR, Neumann on
//            boundary component 1, Dirichlet 0 elsewhere); L2 and H1-semi errors are computed
//            with the reference's TFEFunction2D::GetErrors + L2H1Errors.
#include <Domain.h>
#include <Database.h>
#include <FEDatabase2D.h>
#include <LinAlg.h>
#include <FESpace2D.h>
#include <FEFunction2D.h>
#include <SystemCD2D.h>
#include <MainUtilities.h>
#include <LinAlg.h>
#include <MultiGrid2D.h>
#include <MGLevel2D.h>
#include <ItMethod.h>
#include <FgmresIte.h>
#include <FixedPointIte.h>
#include <MultiGridScaIte.h>
#include <AuxParam2D.h>

#include <string.h>
#include <math.h>
#include <vector>

#include "dump_common.h"

double bound = 0;
double timeC = 0;
// timing accumulators that the 3D multigrid files define and TFixedPointIte references
double tSmoother = 0, tS = 0, tD = 0, tP = 0, tR = 0;

static int Example = 0;
static double C_eps = 1, C_b1 = 0, C_b2 = 0, C_c = 0, C_f = 1;

void ExampleFile() { OutPut("Example: CD2D dump driver, example " << Example << endl); }

void Exact(double x, double y, double *values)
{
  if (Example == 1)
  {
    values[0] = sin(Pi * x) * sin(Pi * y);
    values[1] = Pi * cos(Pi * x) * sin(Pi * y);
    values[2] = Pi * sin(Pi * x) * cos(Pi * y);
    values[3] = -2 * Pi * Pi * sin(Pi * x) * sin(Pi * y);
  }
  else
    values[0] = values[1] = values[2] = values[3] = 0;
}

void BoundCondition(int BdComp, double t, BoundCond &cond)
{
  cond = (Example == 1 && BdComp == 1) ? NEUMANN : DIRICHLET;
}

void BoundValue(int BdComp, double Param, double &value)
{
  if (Example == 1 && BdComp == 1)
    value = -C_eps * Pi * sin(Pi * Param);
  else
    value = 0;
}

void BilinearCoeffs(int n_points, double *x, double *y, double **parameters, double **coeffs)
{
  for (int i = 0; i < n_points; i++)
  {
    double *c = coeffs[i];
    if (Example == 1)
    {
      c[0] = C_eps; c[1] = 0; c[2] = 0; c[3] = 0;
      c[4] = (2 * Pi * Pi * C_eps) * sin(Pi * x[i]) * sin(Pi * y[i]);
    }
    else
    {
      c[0] = C_eps; c[1] = C_b1; c[2] = C_b2; c[3] = C_c; c[4] = C_f;
    }
  }
}

class DumpSystemCD2D : public TSystemCD2D
{
 public:
  DumpSystemCD2D(TFESpace2D *s, int disc, int solver) : TSystemCD2D(s, disc, solver) {}
  TSquareMatrix2D *A() { return sqmatrixA; }
};

int main(int argc, char *argv[])
{
  if (argc < 9)
  {
    fprintf(stderr, "usage: %s file.dat outdir|- example eps b1 b2 c f [prolong_max_ndof]\n", argv[0]);
    return 2;
  }
  TDatabase *Database = new TDatabase();
  TFEDatabase2D *FEDatabase = new TFEDatabase2D();
  TDomain *Domain = new TDomain(argv[1]);
  const char *outdir = strcmp(argv[2], "-") ? argv[2] : nullptr;
  Example = atoi(argv[3]);
  C_eps = atof(argv[4]); C_b1 = atof(argv[5]); C_b2 = atof(argv[6]);
  C_c = atof(argv[7]); C_f = atof(argv[8]);
  if (Example == 1) C_eps = 1.0 / TDatabase::ParamDB->PE_NR;
  long prolong_max = argc > 9 ? atol(argv[9]) : 0;
  dump_open(outdir);

  if (TDatabase::ParamDB->PROBLEM_TYPE == 0) TDatabase::ParamDB->PROBLEM_TYPE = 1;
  OpenFiles();

  double t0 = wall_now();
  Domain->Init(TDatabase::ParamDB->BNDFILE, TDatabase::ParamDB->GEOFILE);
  int LEVELS = TDatabase::ParamDB->LEVELS;
  int solver = TDatabase::ParamDB->SOLVER_TYPE;  // 1 = GMG, 2 = a single level, assembly only
  if (solver != 1) LEVELS = 1;
  for (int i = 0; i < TDatabase::ParamDB->UNIFORM_STEPS; i++) Domain->RegRefineAll();

  int ORDER = TDatabase::ParamDB->ANSATZ_ORDER;
  std::vector<TCollection *> colls(LEVELS);
  std::vector<TFESpace2D *> spaces(LEVELS);
  std::vector<double *> Sol(LEVELS), Rhs(LEVELS);
  char Name[] = "name", Desc[] = "description";
  for (int i = 0; i < LEVELS; i++)
  {
    if (i) Domain->RegRefineAll();
    colls[i] = Domain->GetCollection(It_Finest, 0);
    spaces[i] = new TFESpace2D(colls[i], Name, Desc, BoundCondition, ORDER, NULL);
    int n = spaces[i]->GetN_DegreesOfFreedom();
    Sol[i] = new double[n];
    Rhs[i] = new double[n];
    memset(Sol[i], 0, n * sizeof(double));
    memset(Rhs[i], 0, n * sizeof(double));
  }
  double t_mesh = wall_now() - t0;

  t0 = wall_now();
  std::vector<DumpSystemCD2D *> S(LEVELS);
  for (int i = 0; i < LEVELS; i++)
  {
    S[i] = new DumpSystemCD2D(spaces[i], TDatabase::ParamDB->DISCTYPE, 2);
    S[i]->Init(BilinearCoeffs, BoundCondition, BoundValue);
  }
  double t_construct = wall_now() - t0;

  t0 = wall_now();
  for (int i = 0; i < LEVELS; i++) S[i]->Assemble(NULL, Sol[i], Rhs[i]);
  double t_assemble = wall_now() - t0;

  meta_i("levels", LEVELS);
  meta_i("order", ORDER);
  for (int l = 0; l < LEVELS; l++)
  {
    TFESpace2D *sp = spaces[l];
    TCollection *coll = colls[l];
    int n_cells = coll->GetN_Cells();
    int n = sp->GetN_DegreesOfFreedom();
    int *bi = sp->GetBeginIndex();
    int nbf = bi[1] - bi[0];
    TSquareMatrix2D *A = S[l]->A();
    int nnz = A->GetRowPtr()[n];
    meta_i(lvl(l, "n_dof"), n);
    meta_i(lvl(l, "n_active"), sp->GetN_ActiveDegrees());
    meta_i(lvl(l, "hanging_bound"), sp->GetHangingBound());
    meta_i(lvl(l, "n_dirichlet"), sp->GetN_Dirichlet());
    meta_i(lvl(l, "n_cells"), n_cells);
    meta_i(lvl(l, "n_bf"), nbf);
    meta_i(lvl(l, "nnz"), nnz);
    if (!outdir) continue;
    std::vector<double> xy((size_t)n_cells * 4 * 2);
    for (int c = 0; c < n_cells; c++)
    {
      TBaseCell *cell = coll->GetCell(c);
      for (int v = 0; v < 4; v++)
      {
        double x, y;
        cell->GetVertex(v)->GetCoords(x, y);
        xy[(size_t)c * 8 + v * 2 + 0] = x;
        xy[(size_t)c * 8 + v * 2 + 1] = y;
      }
    }
    dump_f64(lvl(l, "coords"), xy.data(), (long)xy.size());
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
        // the reference's cell-wise prolongation (src/FE/MGComponents2D.C:118) applied to unit vectors
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
  int L = LEVELS - 1;
  int nf = spaces[L]->GetN_DegreesOfFreedom();
  if (solver == 1)
  {
    // multigrid wiring in the order of src/System/SystemCD3D.C:147-199 and 285-308
    double Parameters[2];
    Parameters[0] = TDatabase::ParamDB->SC_SMOOTH_DAMP_FACTOR_SCALAR;
    Parameters[1] = TDatabase::ParamDB->SC_SMOOTH_DAMP_FACTOR_FINE_SCALAR;
    TMultiGrid2D *MG = new TMultiGrid2D(1, 2, Parameters);
    int N_aux = (TDatabase::ParamDB->SC_STEP_LENGTH_CONTROL_ALL_SCALAR ||
                 TDatabase::ParamDB->SC_STEP_LENGTH_CONTROL_FINE_SCALAR) ? 4 : 2;
    for (int i = 0; i < LEVELS; i++)
      MG->AddLevel(new TMGLevel2D(i, S[i]->A(), Rhs[i], Sol[i], N_aux, NULL));
    TItMethod *prec = new TMultiGridScaIte(MatVect_Scalar, Defect_Scalar, NULL, 0, nf, MG, 1);
    TItMethod *it;
    if (TDatabase::ParamDB->SC_SOLVER_SCALAR == 11)
      it = new TFixedPointIte(MatVect_Scalar, Defect_Scalar, prec, 0, nf, 1);
    else
      it = new TFgmresIte(MatVect_Scalar, Defect_Scalar, prec, 0, nf, 1);
    std::vector<double> isol(nf), irhs(nf);
    TSquareMatrix *sq[1] = {S[L]->A()};
    t0 = wall_now();
    memcpy(isol.data(), Sol[L], nf * sizeof(double));
    memcpy(irhs.data(), Rhs[L], nf * sizeof(double));
    its = it->Iterate(sq, NULL, isol.data(), irhs.data());
    memcpy(Sol[L], isol.data(), nf * sizeof(double));
    t_solve = wall_now() - t0;
    dump_f64("solution", Sol[L], nf);
  }
  meta_i("iterations", its);
  meta_d("t_mesh", t_mesh);
  meta_d("t_construct", t_construct);
  meta_d("t_assemble", t_assemble);
  meta_d("t_solve", t_solve);

  if (Example == 1 && solver == 1)
  {
    TFEFunction2D *u = new TFEFunction2D(spaces[L], (char *)"u", (char *)"u", Sol[L], nf);
    TFESpace2D *fesp[1] = {spaces[L]};
    TAuxParam2D *aux = new TAuxParam2D(1, 0, 0, 0, fesp, NULL, NULL, NULL, NULL, 0, NULL);
    MultiIndex2D AllDerivatives[3] = {D00, D10, D01};
    double errors[4] = {0, 0, 0, 0};
    u->GetErrors(Exact, 3, AllDerivatives, 2, L2H1Errors, BilinearCoeffs, aux, 1, fesp, errors);
    meta_d("err_l2", errors[0]);
    meta_d("err_h1", errors[1]);
    printf("L2: %.6e H1-semi: %.6e\n", errors[0], errors[1]);
  }
  printf("{\"n_dof\": %d, \"n_cells\": %d, \"iterations\": %d, \"t_mesh\": %.6f, "
         "\"t_construct\": %.6f, \"t_assemble\": %.6f, \"t_solve\": %.6f}\n",
         nf, colls[L]->GetN_Cells(), its, t_mesh, t_construct, t_assemble, t_solve);
  if (g_meta) fclose(g_meta);
  CloseFiles();
  return 0;
}
