"""TSystemTCD3D against the reference's time-dependent 3D known answer (example amc.h).

The time loop of 3DPrograms/TCD3D_ParMooN.C:540-720 -- AssembleMRhs, then per step the old
solution and right-hand side kept, CURRENTTIME += tau, AssembleARhs (f and the Dirichlet
data at the new time), AssembleSystMat (the 3D order of the matrix updates,
src/System/SystemTCD3D.C:228-294), Solve, RestoreMassMat, GetErrors -- over 19
Crank-Nicolson steps of 16^3 Q1 hexahedra.  The oracle's restatement (CPU) and the library
(GPU, FP64 and mixed form, errors evaluated on the device) must print the compiled
reference's L2 and H1-semi errors (tests/golden/tcd3d_amc_16.json) after every step to all
printed digits, and the L2 column recorded in ReadIn/tcd3d_GMG.out:398-515.
"""
import numpy as np
import pytest

import tcd3d_amc as amc
from parmoon_cmg_b200 import _lib, mesh

MASS = 10


def _fine_rows(space):
    return len(space["begin_index"]) - 1


def test_known_answer_fixture_matches_recorded_log():
    """The compiled reference reproduces the recorded L2 column; its times are the loop's."""
    rows = amc.fixture()
    assert [r[1] for r in rows] == amc.LOG_L2
    assert [r[0] for r in rows[1:]] == [f"{t:.6e}" for t in amc.times()]


def test_oracle_tcd3d_known_answer(oracle_lib):
    """The oracle's 3D theta steps (tcd_step with the 3D update order) print the compiled
    reference's errors after every step."""
    spaces, parents = mesh.structured_hierarchy(3, 1, 2, 4)  # 2^3 .. 16^3 Q1
    fin = spaces[-1]
    nc = _fine_rows(fin)
    levels = []
    for l, sp in enumerate(spaces):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(3, 1, spaces[l - 1], dict(sp),
                                                                            parents[l])
        levels.append(lv)
    co = oracle_lib.coeffs(3)  # CDGPU_COEFF_TABLE: the table carries every coefficient
    xq = oracle_lib.quad_points(3, 1, fin["coords"], nc)
    xyz = oracle_lib.dof_coords(3, 1, fin["coords"], fin["global_numbers"], fin["begin_index"], fin["n_dof"])
    na = int(fin["n_active"])

    def forms(disctype, t):
        M, rhs = [], None
        for sp, lv in zip(spaces, levels):
            n = _fine_rows(sp)
            q = oracle_lib.quad_points(3, 1, sp["coords"], n)
            fine = sp is fin
            dv = amc.values(xyz, t)[na:] if fine else None
            e, rhs = oracle_lib.assemble(3, 1, disctype, sp["coords"], sp["global_numbers"], sp["begin_index"],
                                         sp["n_dof"], sp["n_active"], lv["row_ptr"], lv["kcol"], co,
                                         coeff_tab=amc.coeff_table(q, t, with_f=fine), dir_vals=dv)
            M.append(e)
        return M, rhs

    def errors(u, t):
        e = oracle_lib.errors_table(3, 1, fin["coords"], fin["global_numbers"], fin["begin_index"], u,
                                    amc.exact_table(xq, t))
        return amc.fmt(e)

    rows = amc.fixture()
    u = amc.values(xyz, 0.0)
    assert errors(u, 0.0) == tuple(rows[0][1:])
    M, f = forms(MASS, 0.0)
    prm = oracle_lib.solver_params(coarse_smoother=3, red_factor=0.0, res_norm_min=1e-13, maxit=300)
    for k, t in enumerate(amc.times(), start=1):
        f_old = f
        A, f = forms(1, t)
        u, its = oracle_lib.tcd_step(levels, M, A, f_old, f, u, amc.TAU, *amc.THETA, prm, fine_only_theta2=True)
        assert its > 0
        assert errors(u, t) == tuple(rows[k][1:]), (k, t)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_tcd3d_known_answer_gpu(oracle_lib, precision):
    """TSystemTCD3D on the GPU: amc.h's coefficients at the library's quadrature points
    (CDGPU_COEFF_TABLE, f on the finest level), its Dirichlet data at the new time
    (cdgpu_tcd_set_dirichlet) and errors on the device (cdgpu_errors_table) print the
    compiled reference's L2 and H1-semi errors after each of 19 steps, FP64 and mixed."""
    from parmoon_cmg_b200 import _build
    from parmoon_cmg_b200.system import Context, TSystemTCD3D, coeffs, solver_params
    _build.build()
    spaces, parents = mesh.structured_hierarchy(3, 1, 2, 4)
    fin = spaces[-1]
    nc = _fine_rows(fin)
    na = int(fin["n_active"])
    xyz = oracle_lib.dof_coords(3, 1, fin["coords"], fin["global_numbers"], fin["begin_index"], fin["n_dof"])
    rows = amc.fixture()
    ctx = Context(0)
    try:
        S = TSystemTCD3D(spaces, parents, ctx=ctx)
        fine_sid = S.sids[-1]
        # the coarse levels carry only the operator (eps = 1); the finest level's table has f
        for sid in S.sids[:-1]:
            ctx.set_coeffs(sid, coeffs(0, eps=1.0, b=(0.0, 0.0, 0.0), c=0.0, f=0.0))
        xq = ctx.quadrature_points(fine_sid, nc, 3)

        def set_time(t):
            ctx.set_coeffs(fine_sid, coeffs(_lib.COEFF_TABLE), amc.coeff_table(xq, t))
            S.SetDirichlet(amc.values(xyz, t)[na:])

        sol = amc.values(xyz, 0.0)
        assert amc.fmt(ctx.errors_table(fine_sid, sol, amc.exact_table(xq, 0.0))) == tuple(rows[0][1:])
        set_time(0.0)
        S.AssembleMRhs()
        prm = solver_params(precision=precision, coarse_smoother=3, red_factor=0.0, res_norm_min=1e-13,
                            maxit=300)
        for k, t in enumerate(amc.times(), start=1):
            set_time(t)
            S.AssembleARhs()
            info = S.Step(sol, amc.TAU, *amc.THETA, params=prm)
            assert info.status == 0
            e = ctx.errors_table(fine_sid, sol, amc.exact_table(xq, t))
            assert amc.fmt(e) == tuple(rows[k][1:]), (k, t, e)
            assert amc.fmt(e)[0] == amc.LOG_L2[k]
    finally:
        ctx.close()
