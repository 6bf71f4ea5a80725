"""Theta-scheme time stepping (TSystemTCD2D) on the GPU against the oracle.

The time loop of 2DPrograms/TCD2D_ParMooN.C:241-290 -- save the old right-hand side,
AssembleARhs, AssembleSystMat, Solve, RestoreMassMat -- runs through the C ABI and
through the oracle's restatement (oracle.tcd_step) on the same hierarchy; every
step's solution agrees within the FP64 solution bar.
"""
import numpy as np
import pytest

from parmoon_cmg_b200 import _lib, mesh
from parmoon_cmg_b200.system import Context, TSystemTCD2D, TSystemTCD3D, coeffs, solver_params

TOL_SOL = 1e-10
MASS = 10


def oracle_levels(oracle_lib, spaces, parents, dim, order):
    levels = []
    for l, sp in enumerate(spaces):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(
                dim, order, spaces[l - 1], dict(sp), parents[l])
        levels.append(lv)
    return levels


def oracle_forms(oracle_lib, spaces, levels, dim, order, disctype, co):
    ent, rhs = [], None
    for sp, lv in zip(spaces, levels):
        e, rhs = oracle_lib.assemble(dim, order, disctype, sp["coords"], sp["global_numbers"],
                                     sp["begin_index"], sp["n_dof"], sp["n_active"], lv["row_ptr"],
                                     lv["kcol"], co)
        ent.append(e)
    return ent, rhs


def test_oracle_backward_euler_reaches_steady_state(oracle_lib):
    """Property of the oracle's restatement: implicit Euler with long steps converges to
    the stationary solution A u = f of the same problem."""
    spaces, parents = mesh.structured_hierarchy(2, 1, 4, 2)
    levels = oracle_levels(oracle_lib, spaces, parents, 2, 1)
    co = oracle_lib.coeffs(0, eps=0.1, b=(1.0, 0.5), f=1.0)
    M, fm = oracle_forms(oracle_lib, spaces, levels, 2, 1, MASS, co)
    A, f = oracle_forms(oracle_lib, spaces, levels, 2, 1, 1, co)
    prm = oracle_lib.solver_params(red_factor=1e-13, restart=32, maxit=200)
    M0 = [m.copy() for m in M]
    u = np.zeros(spaces[-1]["n_dof"])
    for _ in range(12):
        u, its = oracle_lib.tcd_step(levels, M, A, f, f, u, 1e3, 1.0, 0.0, 0.0, 1.0, prm)
        assert its >= 0
    steady = [dict(lv, entries=a) for lv, a in zip(levels, A)]
    us, _, _, _ = oracle_lib.solve(steady, prm, f, np.zeros_like(f))
    assert np.abs(u - us).max() <= 1e-8 * np.abs(us).max()
    # RestoreMassMat brings M back up to rounding
    for m, m0 in zip(M, M0):
        assert np.abs(m - m0).max() <= 1e-12 * np.abs(m0).max()


def test_oracle_backward_euler_reaches_steady_state_3d(oracle_lib):
    """The 3D order of the updates (fine_only_theta2, SystemTCD3D.C:257-278) keeps the
    property: implicit Euler with long steps converges to the stationary solution, and
    RestoreMassMat brings every level's M back up to rounding."""
    spaces, parents = mesh.structured_hierarchy(3, 1, 2, 2)
    levels = oracle_levels(oracle_lib, spaces, parents, 3, 1)
    co = oracle_lib.coeffs(0, eps=0.1, b=(1.0, 0.5, 0.25), f=1.0)
    M, fm = oracle_forms(oracle_lib, spaces, levels, 3, 1, MASS, co)
    A, f = oracle_forms(oracle_lib, spaces, levels, 3, 1, 1, co)
    prm = oracle_lib.solver_params(red_factor=1e-13, restart=32, maxit=200)
    M0 = [m.copy() for m in M]
    u = np.zeros(spaces[-1]["n_dof"])
    for _ in range(12):
        u, its = oracle_lib.tcd_step(levels, M, A, f, f, u, 1e3, 1.0, 0.0, 0.0, 1.0, prm, fine_only_theta2=True)
        assert its >= 0
    steady = [dict(lv, entries=a) for lv, a in zip(levels, A)]
    us, _, _, _ = oracle_lib.solve(steady, prm, f, np.zeros_like(f))
    assert np.abs(u - us).max() <= 1e-8 * np.abs(us).max()
    for m, m0 in zip(M, M0):
        assert np.abs(m - m0).max() <= 1e-12 * np.abs(m0).max()


@pytest.mark.gpu
@pytest.mark.parametrize("order,scheme", [(1, "crank_nicolson"), (2, "backward_euler")])
def test_tcd_steps_vs_oracle(oracle_lib, order, scheme):
    from parmoon_cmg_b200 import _build
    _build.build()
    th = dict(crank_nicolson=(0.5, 0.5, 0.5, 0.5), backward_euler=(1.0, 0.0, 0.0, 1.0))[scheme]
    tau = 0.05
    spaces, parents = mesh.structured_hierarchy(2, order, 4, 3)
    ctx = Context(0)
    try:
        S = TSystemTCD2D(spaces, parents, ctx=ctx)
        co_steps = [coeffs(0, eps=0.05, b=(1.0, 0.5), c=0.1, f=1.0 + 0.5 * k) for k in range(4)]
        S.Init(co_steps[0])
        n = spaces[-1]["n_dof"]
        sol = np.zeros(n)
        S.AssembleMRhs(sol)
        levels = oracle_levels(oracle_lib, spaces, parents, 2, order)

        def oco(c):
            return oracle_lib.coeffs(0, eps=c.eps, b=(c.b1, c.b2), c=c.c, f=c.f)

        M, f = oracle_forms(oracle_lib, spaces, levels, 2, order, MASS, oco(co_steps[0]))
        assert np.abs(S.rhs() - f).max() <= 1e-12 * np.abs(f).max()
        u = sol.copy()
        prm_o = oracle_lib.solver_params(red_factor=1e-13, restart=32, maxit=200)
        prm = solver_params(coarse_smoother=3, red_factor=1e-13, restart=32, maxit=200)
        for k in range(1, 4):
            # the right-hand side changes in time (UpdateRhs in the reference's loop)
            for sid in S.sids:
                ctx.set_coeffs(sid, co_steps[k])
            f_old = f
            S.AssembleARhs()
            A, f = oracle_forms(oracle_lib, spaces, levels, 2, order, 1, oco(co_steps[k]))
            info = S.Step(sol, tau, *th, params=prm)
            assert info.status == 0
            u, its = oracle_lib.tcd_step(levels, M, A, f_old, f, u, tau, *th, prm_o)
            assert its >= 0
            assert np.abs(sol - u).max() <= TOL_SOL * np.abs(u).max()
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2])
def test_tcd3d_steps_vs_oracle(oracle_lib, order):
    """TSystemTCD3D: Crank-Nicolson steps on a 3D hierarchy with the 3D reference's order of
    the matrix updates (the oracle's tcd_step with fine_only_theta2) agree with the oracle
    within the FP64 solution bar."""
    from parmoon_cmg_b200 import _build
    _build.build()
    th, tau = (0.5, 0.5, 0.5, 0.5), 0.05
    spaces, parents = mesh.structured_hierarchy(3, order, 2, 2)
    ctx = Context(0)
    try:
        S = TSystemTCD3D(spaces, parents, ctx=ctx)
        b = (0.57735026918962573,) * 3
        co_steps = [coeffs(0, eps=0.05, b=b, c=0.1, f=1.0 + 0.5 * k) for k in range(4)]
        S.Init(co_steps[0])
        sol = np.zeros(spaces[-1]["n_dof"])
        S.AssembleMRhs(sol)
        levels = oracle_levels(oracle_lib, spaces, parents, 3, order)

        def oco(c):
            return oracle_lib.coeffs(0, eps=c.eps, b=(c.b1, c.b2, c.b3), c=c.c, f=c.f)

        M, f = oracle_forms(oracle_lib, spaces, levels, 3, order, MASS, oco(co_steps[0]))
        assert np.abs(S.rhs() - f).max() <= 1e-12 * np.abs(f).max()
        nnz = [len(lv["kcol"]) for lv in levels]
        u = sol.copy()
        # the reference's relative stopping rule, so that the iteration counts are comparable
        prm_o = oracle_lib.solver_params(coarse_smoother=3, red_factor=1e-10, restart=32, maxit=200)
        prm = solver_params(coarse_smoother=3, red_factor=1e-10, restart=32, maxit=200)
        for k in range(1, 4):
            for sid in S.sids:
                ctx.set_coeffs(sid, co_steps[k])
            f_old = f
            S.AssembleARhs()
            A, f = oracle_forms(oracle_lib, spaces, levels, 3, order, 1, oco(co_steps[k]))
            if k == 1:
                M0 = [S.matrices(l, nnz[l])[0] for l in range(len(levels))]
                for l in range(len(levels)):
                    assert np.abs(M0[l] - M[l]).max() <= 1e-12 * np.abs(M[l]).max()
            info = S.Step(sol, tau, *th, params=prm)
            assert info.status == 0
            u, its = oracle_lib.tcd_step(levels, M, A, f_old, f, u, tau, *th, prm_o, fine_only_theta2=True)
            assert abs(info.iterations - its) <= 1, (k, info.iterations, its)
            assert np.abs(sol - u).max() <= 1e-8 * np.abs(u).max()
            for l in range(len(levels)):
                Ml, Al, Sl = S.matrices(l, nnz[l])
                # RestoreMassMat leaves every level's mass matrix where it was before the step
                # (to rounding), and in the oracle's in-place sequence
                assert np.abs(Ml - M0[l]).max() <= 1e-13 * np.abs(M0[l]).max()
                assert np.abs(Ml - M[l]).max() <= 1e-13 * np.abs(M[l]).max()
                # the system matrix of every level is M + tau*theta1*A on the active rows and
                # an identity row on the Dirichlet rows
                ka = int(levels[l]["row_ptr"][levels[l]["n_active"]])
                expect = M0[l][:ka] + tau * th[0] * Al[:ka]
                assert np.abs(Sl[:ka] - expect).max() <= 1e-13 * np.abs(expect).max()
                assert np.abs(Al - A[l]).max() <= 1e-12 * np.abs(A[l]).max()
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_tcd2d_known_answer_gpu(oracle_lib, precision):
    """ReadIn/tcd2d.out:485-543 on the GPU: TSystemTCD2D with the exp.h coefficients evaluated
    at the library's quadrature points every step (CDGPU_COEFF_TABLE), 32x32 Q1,
    Crank-Nicolson, tau 0.05: the reference's printed L2 and H1-semi errors after each of 10
    steps, in the FP64 and in the mixed form."""
    import tcd_exp
    from parmoon_cmg_b200 import _build
    _build.build()
    spaces, parents = mesh.structured_hierarchy(2, 1, 4, 4)
    fin = spaces[-1]
    ctx = Context(0)
    try:
        S = TSystemTCD2D(spaces, parents, ctx=ctx)

        def set_time(t):
            for sid, sp in zip(S.sids, spaces):
                xq = ctx.quadrature_points(sid, len(sp["begin_index"]) - 1, 2)
                ctx.set_coeffs(sid, coeffs(_lib.COEFF_TABLE), tcd_exp.coeff_table(xq, t))

        xyz = oracle_lib.dof_coords(2, 1, fin["coords"], fin["global_numbers"], fin["begin_index"], fin["n_dof"])
        sol = tcd_exp.initial(xyz)
        set_time(0.0)
        S.AssembleMRhs(sol)
        prm = solver_params(precision=precision, coarse_smoother=3, red_factor=0.0, res_norm_min=1e-13,
                            maxit=300)
        for k in range(1, len(tcd_exp.KNOWN)):
            t = tcd_exp.KNOWN[k][0]
            set_time(t)
            S.AssembleARhs()
            info = S.Step(sol, tcd_exp.TAU, *tcd_exp.THETA, params=prm)
            assert info.status == 0
            e = oracle_lib.errors_sinsin(1, fin["coords"], fin["global_numbers"], fin["begin_index"], sol,
                                         2.0, np.exp(t))
            assert tcd_exp.fmt(e) == tcd_exp.KNOWN[k][1:], t
    finally:
        ctx.close()


@pytest.mark.gpu
def test_tcd_rejects_bad_use():
    from parmoon_cmg_b200 import _build
    _build.build()
    spaces, parents = mesh.structured_hierarchy(2, 1, 4, 2)
    ctx = Context(0)
    try:
        S = TSystemTCD2D(spaces, parents, ctx=ctx)
        S.Init(coeffs(0, eps=1.0, f=1.0))
        with pytest.raises(_lib.CdgpuError):
            S.Step(np.zeros(spaces[-1]["n_dof"]), 0.1, 1.0, 0.0, 0.0, 1.0)
        with pytest.raises(_lib.CdgpuError):
            import ctypes as C
            ctx.check(ctx.lib.cdgpu_tcd_create(ctx.h, S.mg, _lib.SUPG, C.byref(C.c_int())))
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("smoother", [1, 3])
def test_batched_tcd_steps_vs_oracle(oracle_lib, smoother):
    """Time-dependent instances in a batch (one graph per step) follow the oracle's
    theta-scheme steps: Crank-Nicolson, rotating convection, Gaussian initial bump."""
    from parmoon_cmg_b200 import _build
    from parmoon_cmg_b200.system import Batch
    _build.build()
    tau, th = 1e-3, (0.5, 0.5, 0.5, 0.5)
    ctx = Context(0)
    try:
        B = Batch(solver_params(smoother=smoother, omega=0.8 if smoother == 1 else 1.0, stop_rule=1,
                                red_factor=1e-13, restart=30, maxit=200), ctx)
        cases = []
        for order, n0, L, eps in [(2, 2, 3, 1e-3), (1, 2, 4, 1e-4)]:
            spaces, parents = mesh.structured_hierarchy(2, order, n0, L)
            sid = B.add_structure(spaces, parents)
            xy = mesh.dof_coords(spaces[-1])
            u0 = np.exp(-((xy[:, 0] - 0.3) ** 2 + (xy[:, 1] - 0.3) ** 2) / (2 * 0.05 ** 2))
            co = coeffs(_lib.COEFF_ROTATING, eps=eps, f=0.0)
            slot = B.submit_tcd(sid, co, tau, *th, u0)
            levels = oracle_levels(oracle_lib, spaces, parents, 2, order)
            oco = oracle_lib.coeffs(_lib.COEFF_ROTATING, eps=eps, f=0.0)
            M, f = oracle_forms(oracle_lib, spaces, levels, 2, order, MASS, oco)
            A, f = oracle_forms(oracle_lib, spaces, levels, 2, order, 1, oco)
            u = u0.copy()
            u[spaces[-1]["n_active"]:] = f[spaces[-1]["n_active"]:]
            cases.append(dict(slot=slot, levels=levels, M=M, A=A, f=f, u=u, n=spaces[-1]["n_dof"]))
        prm_o = oracle_lib.solver_params(red_factor=1e-13, restart=32, maxit=200)
        for step in range(4):
            B.tcd_step(4)
            for c in cases:
                c["u"], its = oracle_lib.tcd_step(c["levels"], c["M"], c["A"], c["f"], c["f"], c["u"], tau, *th,
                                                  prm_o)
                x, info = B.fetch(c["slot"], c["n"])
                assert info.status == 0
                assert np.abs(x - c["u"]).max() <= 1e-9 * np.abs(c["u"]).max(), step
    finally:
        ctx.close()
