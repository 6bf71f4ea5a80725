// Abort-stubs for symbols of libraries that the convection-diffusion path never calls
// (LAPACK, PARDISO, UMFPACK direct solver, tecplot, tetgen, triangle).  The
// reference links prebuilt binaries for them; the oracle build links none, so
// any call reaching one of these aborts loudly instead of computing anything.
#include <cstdio>
#include <cstdlib>

#define CDGPU_STUB(name)                                                        \
  extern "C" void name()                                                        \
  {                                                                             \
    fprintf(stderr, "oracle build: off-path external '%s' was called\n", #name); \
    abort();                                                                    \
  }

CDGPU_STUB(dgetrf_)
CDGPU_STUB(dgetrs_)
CDGPU_STUB(dgemm_)
CDGPU_STUB(dgetri_)
CDGPU_STUB(dsptrd_)
CDGPU_STUB(dopgtr_)
CDGPU_STUB(dsteqr_)
CDGPU_STUB(dgesv_)
CDGPU_STUB(dgemv_)
CDGPU_STUB(pardiso_)
CDGPU_STUB(pardisoinit_)
CDGPU_STUB(triangulate)
// tecplot writer (TOutput2D/3D::WriteTecplot); the header comes from EXT_LIB, the library does not
CDGPU_STUB(tecini112)
CDGPU_STUB(teczne112)
CDGPU_STUB(tecdat112)
CDGPU_STUB(tecnod112)
CDGPU_STUB(tecend112)
CDGPU_STUB(tecend)
CDGPU_STUB(tetrahedralize)

// UMFPACK-backed direct solver (src/FE/DirectSolver.C needs PARDISO/cblas headers and is
// not built); only the DIRECT solver type reaches it.
class TSquareMatrix;
void DirectSolver(TSquareMatrix *, double *, double *)
{
  fprintf(stderr, "oracle build: DirectSolver (UMFPACK) is not available\n");
  abort();
}
