"""Direct tests of the operator forms the mixed solve applies: the FP32 forms of its multigrid
cycle and the matrix-free FP64 form of its FGMRES product.

One product y = A x of each form through the C ABI (cdgpu_apply_fp32, cdgpu_apply_fp64), against the FP64 CSR
product of the same assembled level (itself pinned to the reference by the golden and
headline tests):
  form 0  the FP32 copy of the CSR entries,
  form 1  the matrix-free per-cell products A_c x_c = sum_t coef_t R_t x_c on CUDA cores,
  form 2  the same products on the tensor cores (tcgen05.mma kind::tf32, TMEM accumulator).
The bound is normwise against |A| |x| (the size of the terms summed): 1e-5 for the FP32 forms,
4e-3 for the TF32 form (its inputs keep 10 mantissa bits).  A wrong tile edge, lane mapping or
cell order would give errors of order one in the rows it touches.  Sizes: 5^3 cells (one
partial 128-cell tile), 27^3 (154 tiles: more tiles than SMs, so CTAs take a second tile, and
a partial last tile) and 32^3 (the benchmark's finest level, 256 full tiles).
"""
import numpy as np
import pytest
import scipy.sparse as sps

from parmoon_cmg_b200 import _lib, mesh
from parmoon_cmg_b200.system import GALERKIN, SUPG, Context, coeffs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from parmoon_cmg_b200 import _build
    _build.build()
    c = Context(0)
    yield c
    c.close()


def assembled(ctx, n, disc):
    sp = mesh.structured_space(3, 2, n)
    sid = ctx.upload_space(sp)
    nnz = ctx.build_pattern(sid)
    ctx.set_coeffs(sid, coeffs(0, eps=1e-2, b=(0.57735026918962573,) * 3, c=0.1, f=1.0, delta0=1.0 / 3.0))
    ent, _ = ctx.assemble(sid, disc, sp["n_dof"], nnz)
    rp, kc = ctx.get_pattern(sid, sp["n_dof"], nnz)
    A = sps.csr_matrix((ent, kc, rp), shape=(sp["n_dof"],) * 2)
    return sp, sid, A


@pytest.mark.parametrize("n", [5, 27, 32])
@pytest.mark.parametrize("disc", [GALERKIN, SUPG])
def test_fp32_operator_forms(ctx, n, disc):
    sp, sid, A = assembled(ctx, n, disc)
    x = np.random.default_rng(n + 10 * disc).uniform(-1, 1, sp["n_dof"]).astype(np.float32)
    x64 = x.astype(np.float64)
    y64 = A @ x64
    scale = np.abs(abs(A) @ np.abs(x64)).max()
    y = {f: ctx.apply_fp32(sid, x, f).astype(np.float64) for f in (0, 1, 2)}
    na = sp["n_active"]
    for f in (0, 1, 2):
        assert np.array_equal(y[f][na:], x64[na:]), f"form {f}: Dirichlet rows are identity rows"
    err = {f: np.abs(y[f] - y64).max() / scale for f in (0, 1, 2)}
    print(f"n={n} disc={disc}: normwise errors {err}")
    assert err[0] <= 1e-5
    assert err[1] <= 1e-5
    assert err[2] <= 4e-3
    assert np.abs(y[2] - y[1]).max() / scale <= 4e-3
    # every cell contributes: a tile that was skipped or written to the wrong cells would leave
    # rows far off, so also the row with the worst error stays within the bound
    worst = int(np.argmax(np.abs(y[2] - y64)))
    assert abs(y[2][worst] - y64[worst]) <= 4e-3 * scale


@pytest.mark.parametrize("n", [5, 27, 32])
@pytest.mark.parametrize("disc", [GALERKIN, SUPG])
def test_fp64_matrix_free_form(ctx, n, disc):
    """The mixed solve's FGMRES product: the sum-factorised FP64 per-cell products (values and
    gradients at the 3 x 3 x 3 Gauss points by one-dimensional passes) against the FP64 CSR
    product of the same assembly (library and scipy), normwise 1e-14: the same matrix up to
    rounding.  5^3 cells leave a partial 32-cell group; 27^3 and 32^3 give more groups than
    the persistent grid has blocks."""
    sp, sid, A = assembled(ctx, n, disc)
    x = np.random.default_rng(7 * n + disc).uniform(-1, 1, sp["n_dof"])
    y_csr = ctx.apply_fp64(sid, x, 0)
    y_mf = ctx.apply_fp64(sid, x, 1)
    y_ref = A @ x
    scale = np.abs(abs(A) @ np.abs(x)).max()
    na = sp["n_active"]
    assert np.array_equal(y_mf[na:], x[na:]), "Dirichlet rows are identity rows"
    err_csr = np.abs(y_mf - y_csr).max() / scale
    err_ref = np.abs(y_mf - y_ref).max() / scale
    print(f"n={n} disc={disc}: matrix-free vs CSR {err_csr:.2e}, vs scipy {err_ref:.2e}")
    assert err_csr <= 1e-14 and err_ref <= 1e-14
    # deterministic: the rows sum their cells in a fixed order
    assert np.array_equal(ctx.apply_fp64(sid, x, 1), y_mf)
    # the device-vector entry point enqueues the same product
    import torch
    dx = torch.from_numpy(x).cuda()
    dy = torch.zeros_like(dx)
    ctx.check(ctx.lib.cdgpu_apply_fp64_device(ctx.h, sid, 1, dx.data_ptr(), dy.data_ptr()))
    torch.cuda.synchronize()
    assert np.array_equal(dy.cpu().numpy(), y_mf)


def test_fp32_operator_forms_unsupported(ctx):
    """The matrix-free forms exist for Q2 hexahedra only; the CSR form for every space."""
    sp = mesh.structured_space(2, 1, 8)
    sid = ctx.upload_space(sp)
    nnz = ctx.build_pattern(sid)
    ctx.set_coeffs(sid, coeffs(0, eps=1.0))
    ctx.assemble(sid, GALERKIN, sp["n_dof"], nnz)
    x = np.ones(sp["n_dof"], np.float32)
    y = ctx.apply_fp32(sid, x, 0)
    assert np.isfinite(y).all()
    with pytest.raises(_lib.CdgpuError) as e:
        ctx.apply_fp32(sid, x, 2)
    assert e.value.status == _lib.ERR_UNSUPPORTED
    with pytest.raises(_lib.CdgpuError) as e:
        ctx.apply_fp64(sid, x.astype(np.float64), 1)
    assert e.value.status == _lib.ERR_UNSUPPORTED


def test_mixed_solve_with_matrix_free_supg_product(ctx):
    """A 32^3 Q2 SUPG finest level (32,768 cells, 13 reference tensors): the mixed solve applies
    its FGMRES product and defect matrix-free in FP64 (the SUPG tensors in the point-wise
    fluxes) and must land within 1e-8 of the FP64 form's solution, with the same iteration count
    up to one."""
    from parmoon_cmg_b200.system import TSystemCD3D, solver_params
    spaces, parents = mesh.structured_hierarchy(3, 2, 2, 5)
    S = TSystemCD3D(spaces, parents, disctype=SUPG, ctx=ctx, coarse_disctype=SUPG)
    S.Init(coeffs(0, eps=1e-2, b=(0.57735026918962573,) * 3, c=0.1, f=1.0, delta0=1.0 / 3.0))
    rhs = np.zeros(S.N_DOF)
    sol0 = np.zeros(S.N_DOF)
    S.Assemble(sol0, rhs)
    common = dict(coarse_smoother=17, stop_rule=1, red_factor=1e-12, res_norm_min=0.0)
    x64 = sol0.copy()
    i64 = S.Solve(x64, rhs, solver_params(precision=0, **common))
    xm = sol0.copy()
    im = S.Solve(xm, rhs, solver_params(precision=1, **common))
    assert i64.status == 0 and im.status == 0
    err = np.abs(xm - x64).max() / np.abs(x64).max()
    print(f"SUPG 32^3: FP64 {i64.iterations} its, mixed {im.iterations} its, rel. diff {err:.2e}")
    assert err <= 1e-8
    assert abs(im.iterations - i64.iterations) <= 1
