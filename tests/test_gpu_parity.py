"""GPU parity: libcdgpu against the compiled reference's golden fixtures and the oracle.

Bars (from the FP64 drop-in contract): CSR pattern and DOF numbering bit-exact;
matrix entries and right-hand sides within 1e-12 relative; converged solution
within 1e-10 relative; the mixed form within 1e-8 relative of the FP64 solution.
All calls go through the C ABI (parmoon_cmg_b200.system.Context wraps ctypes).
"""
import numpy as np
import pytest

from conftest import golden, golden_names

import refdump

from parmoon_cmg_b200 import _lib, mesh
from parmoon_cmg_b200.system import Context, TSystemCD2D, TSystemCD3D, coeffs, solver_params

pytestmark = pytest.mark.gpu

TOL_ENTRIES = 1e-12
TOL_SOL = 1e-10
TOL_MIXED = 1e-8


@pytest.fixture(scope="module")
def ctx():
    from parmoon_cmg_b200 import _build
    _build.build()
    c = Context(0)
    yield c
    c.close()


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def golden_coeffs(d):
    b = tuple(np.atleast_1d(d["b"])) + (0.0,) * 3
    if int(d["example"]) == 1:
        return coeffs(_lib.COEFF_SINE, eps=float(d["eps"]))
    return coeffs(_lib.COEFF_CONSTANT, eps=float(d["eps"]), b=b[:3], c=float(d["c"]), f=float(d["f"]))


def sine_neumann_edges(L, order, eps):
    """Edges on boundary component 1 (x = 1) with the flux of the sine problem at the
    edge's Gauss points, running from local vertex m to m+1."""
    V = L["coords"].reshape(-1, 4, 2)
    nl = order + 1
    z = np.array([-1 / np.sqrt(3), 1 / np.sqrt(3)]) if nl == 2 else np.array([-np.sqrt(0.6), 0, np.sqrt(0.6)])
    cells, edges, g = [], [], []
    for c in range(V.shape[0]):
        for m in range(4):
            m1 = (m + 1) % 4
            if abs(V[c, m, 0] - 1) < 1e-12 and abs(V[c, m1, 0] - 1) < 1e-12:
                s = 0.5 * (z + 1)
                y = V[c, m, 1] + (V[c, m1, 1] - V[c, m, 1]) * s
                cells.append(c)
                edges.append(m)
                g.append(-eps * np.pi * np.sin(np.pi * y))
    return np.array(cells), np.array(edges), np.array(g).reshape(-1)


def setup_golden(ctx, d):
    dim, order, disc = int(d["dim"]), int(d["order"]), int(d["disctype"])
    lv = [refdump.level(d, l) for l in range(int(d["levels"]))]
    sids = []
    for L in lv:
        sp = dict(dim=dim, order=order, coords=L["coords"], global_numbers=L["global_numbers"],
                  begin_index=L["begin_index"], n_dof=L["n_dof"], n_active=L["n_active"])
        sid = ctx.upload_space(sp)
        ctx.build_pattern(sid)
        ctx.set_coeffs(sid, golden_coeffs(d))
        sids.append(sid)
    return dim, order, disc, lv, sids


@pytest.mark.parametrize("name", golden_names())
def test_golden_assembly(ctx, name):
    d = golden(name)
    dim, order, disc, lv, sids = setup_golden(ctx, d)
    for L, sid in zip(lv, sids):
        rp, kc = ctx.get_pattern(sid, L["n_dof"], len(L["kcol"]))
        assert np.array_equal(rp, L["row_ptr"]) and np.array_equal(kc, L["kcol"])
        ent, rhs = ctx.assemble(sid, disc, L["n_dof"], len(kc))
        if int(d["example"]) == 1:
            cells, edges, g = sine_neumann_edges(L, order, float(d["eps"]))
            rhs = ctx.add_neumann(sid, cells, edges, g, n_dof=L["n_dof"])
        assert rel(ent, L["entries"]) <= TOL_ENTRIES
        assert rel(rhs, L["rhs"]) <= TOL_ENTRIES


# the solve needs a multigrid hierarchy: a single-level fixture would make its whole problem
# the coarsest level, whose exact solve is a dense inverse in one thread block and whose
# smoother loop is sequential; its entries and rhs are checked above, and the benchmark
# coefficients it carries are solved at 32^3 against the oracle and the compiled reference
# (test_gpu_headline.py)
@pytest.mark.parametrize("name", [n for n in golden_names() if int(golden(n)["levels"]) > 1])
def test_golden_solve(ctx, name):
    d = golden(name)
    dim, order, disc, lv, sids = setup_golden(ctx, d)
    parents = [None] + [L["parent"] for L in lv[1:]]
    mg = ctx.hierarchy(sids, parents)
    for L, sid in zip(lv, sids):
        ctx.assemble(sid, disc, L["n_dof"], len(L["kcol"]), want_entries=False)
    fin = lv[-1]
    if int(d["example"]) == 1:
        cells, edges, g = sine_neumann_edges(fin, order, float(d["eps"]))
        ctx.add_neumann(sids[-1], cells, edges, g)
    rhs = fin["rhs"]  # the reference's right-hand side (checked bit-close above)
    sol0 = np.zeros(fin["n_dof"])
    sol0[fin["n_active"]:] = rhs[fin["n_active"]:]
    for cs in (17, 3, 1):
        prm = solver_params(red_factor=0.0, res_norm_min=1e-14 * np.linalg.norm(rhs), maxit=2000,
                            coarse_smoother=cs)
        sol, info = ctx.solve(mg, prm, rhs, sol0)
        assert info.status == 0, info.status
        assert rel(sol, d["solution"]) <= TOL_SOL, (cs, rel(sol, d["solution"]))


def test_sine_known_answer_gpu(ctx, oracle_lib):
    d = golden("cd2d_q1_sine_32")
    dim, order, disc, lv, sids = setup_golden(ctx, d)
    mg = ctx.hierarchy(sids, [None] + [L["parent"] for L in lv[1:]])
    for L, sid in zip(lv, sids):
        ctx.assemble(sid, disc, L["n_dof"], len(L["kcol"]), want_entries=False)
    fin = lv[-1]
    cells, edges, g = sine_neumann_edges(fin, order, float(d["eps"]))
    rhs = ctx.add_neumann(sids[-1], cells, edges, g, n_dof=fin["n_dof"])
    sol0 = np.zeros(fin["n_dof"])
    prm = solver_params(red_factor=1e-13)
    sol, info = ctx.solve(mg, prm, rhs, sol0)
    e = oracle_lib.errors_sine(1, fin["coords"], fin["global_numbers"], fin["begin_index"], sol)
    assert f"{e[0]:.6e}" == "4.751079e-04" and f"{e[1]:.6e}" == "6.295197e-02"
    # the same errors evaluated on the device (GetErrors)
    g = ctx.errors(sids[-1], sol)
    assert f"{g[0]:.6e}" == "4.751079e-04" and f"{g[1]:.6e}" == "6.295197e-02"
    assert abs(g[0] - e[0]) <= 1e-12 * e[0] and abs(g[1] - e[1]) <= 1e-12 * e[1]
    # no exact solution for other coefficient kinds
    sp3 = mesh.structured_space(3, 1, 2)
    sid3 = ctx.upload_space(sp3)
    ctx.build_pattern(sid3)
    ctx.set_coeffs(sid3, coeffs(0, eps=1.0))
    with pytest.raises(_lib.CdgpuError) as err:
        ctx.errors(sid3, np.zeros(sp3["n_dof"]))
    assert err.value.status == _lib.ERR_UNSUPPORTED


def structured_case(ctx, dim, order, n_coarse, n_levels, co, disc):
    spaces, parents = mesh.structured_hierarchy(dim, order, n_coarse, n_levels)
    sids = []
    for sp in spaces:
        sid = ctx.upload_space(sp)
        ctx.build_pattern(sid)
        ctx.set_coeffs(sid, co)
        sids.append(sid)
    mg = ctx.hierarchy(sids, parents)
    return spaces, parents, sids, mg


def oracle_coeffs(oracle_lib, co):
    return oracle_lib.coeffs(co.kind, eps=co.eps, b=(co.b1, co.b2, co.b3), c=co.c, f=co.f,
                             delta0=co.delta0, order_pd=co.poly_degree)


@pytest.mark.parametrize("dim,order,disc,kind", [
    (2, 1, 2, 0), (2, 2, 2, 0), (2, 2, 1, 2), (2, 1, 2, 2), (3, 1, 1, 0), (3, 2, 1, 0),
    (3, 2, 2, 0), (3, 1, 2, 0)])
def test_structured_assembly_vs_oracle(ctx, oracle_lib, dim, order, disc, kind):
    n = 8 if dim == 2 else 4
    co = coeffs(kind, eps=1e-3, b=(0.8, -0.6, 0.3)[:dim] if kind == 0 else (0, 0, 0), c=0.25, f=1.5)
    spaces, parents, sids, mg = structured_case(ctx, dim, order, n, 1, co, disc)
    sp, sid = spaces[0], sids[0]
    rp_o, kc_o = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
    nnz = len(kc_o)
    rp, kc = ctx.get_pattern(sid, sp["n_dof"], nnz)
    assert np.array_equal(rp, rp_o) and np.array_equal(kc, kc_o)
    dirv = np.linspace(0.0, 1.0, sp["n_dof"] - sp["n_active"])
    ent, rhs = ctx.assemble(sid, disc, sp["n_dof"], nnz, dirichlet=dirv)
    ent_o, rhs_o = oracle_lib.assemble(dim, order, disc, sp["coords"], sp["global_numbers"],
                                       sp["begin_index"], sp["n_dof"], sp["n_active"], rp_o, kc_o,
                                       oracle_coeffs(oracle_lib, co), dir_vals=dirv)
    assert rel(ent, ent_o) <= TOL_ENTRIES
    assert rel(rhs, rhs_o) <= TOL_ENTRIES


@pytest.mark.parametrize("dim,order", [(2, 2), (3, 2), (3, 1)])
def test_quadrature_path_equals_tensor_path(ctx, dim, order):
    """The general quadrature path (table coefficients) and the affine fast path agree."""
    n = 4
    co = coeffs(0, eps=0.01, b=(0.3, 0.4, 0.5)[:dim], c=0.1, f=2.0)
    spaces, parents, sids, mg = structured_case(ctx, dim, order, n, 1, co, 1)
    sp, sid = spaces[0], sids[0]
    nnz = ctx.build_pattern(sid)
    e1, r1 = ctx.assemble(sid, 1, sp["n_dof"], nnz)
    q = ctx.quadrature_points(sid, sp["n_cells"], dim)
    tab = np.zeros(q.shape[:2] + (6,))
    tab[..., 0], tab[..., 1], tab[..., 2] = 0.01, 0.3, 0.4
    tab[..., 3] = 0.5 if dim == 3 else 0.0
    tab[..., 4], tab[..., 5] = 0.1, 2.0
    ctx.set_coeffs(sid, coeffs(_lib.COEFF_TABLE), tab)
    e2, r2 = ctx.assemble(sid, 1, sp["n_dof"], nnz)
    assert rel(e2, e1) <= TOL_ENTRIES and rel(r2, r1) <= TOL_ENTRIES


def test_assembly_deterministic(ctx):
    co = coeffs(0, eps=1e-2, b=(0.57735, 0.57735, 0.57735))
    spaces, parents, sids, mg = structured_case(ctx, 3, 2, 4, 1, co, 1)
    sp, sid = spaces[0], sids[0]
    nnz = ctx.build_pattern(sid)
    a1, b1 = ctx.assemble(sid, 1, sp["n_dof"], nnz)
    a2, b2 = ctx.assemble(sid, 1, sp["n_dof"], nnz)
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)


@pytest.mark.parametrize("dim,order,n0,L,disc,eps", [
    (2, 1, 4, 5, 2, 1e-3),    # config 1 (64x64 Q1 SUPG, 5 levels)
    (3, 2, 2, 3, 1, 1e-1),    # 8^3 Q2 Galerkin, 3 levels
    (3, 1, 2, 4, 1, 1e-1),    # 16^3 Q1 Galerkin, 4 levels
])
def test_structured_solve_vs_oracle(ctx, oracle_lib, dim, order, n0, L, disc, eps):
    b = (1.0, 0.5) if dim == 2 else (0.57735026918962573,) * 3
    co = coeffs(0, eps=eps, b=b, f=1.0)
    spaces, parents, sids, mg = structured_case(ctx, dim, order, n0, L, co, disc)
    levels = []
    for l, (sp, sid) in enumerate(zip(spaces, sids)):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        ent, rhs = oracle_lib.assemble(dim, order, disc, sp["coords"], sp["global_numbers"],
                                       sp["begin_index"], sp["n_dof"], sp["n_active"], rp, kc,
                                       oracle_coeffs(oracle_lib, co))
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc, entries=ent)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(
                dim, order, spaces[l - 1], dict(sp), parents[l])
        levels.append(lv)
        ctx.assemble(sid, disc, sp["n_dof"], len(kc), want_entries=False)
    sol0 = np.zeros(spaces[-1]["n_dof"])
    tight = dict(red_factor=0.0, res_norm_min=1e-14 * np.linalg.norm(rhs), maxit=3000)
    x_o, its_o, _, _ = oracle_lib.solve(levels, oracle_lib.solver_params(**tight), rhs, sol0)
    x, info = ctx.solve(mg, solver_params(coarse_smoother=3, **tight), rhs, sol0)
    assert info.status == 0
    assert rel(x, x_o) <= TOL_SOL
    # the mixed form (FP32 multigrid inside FP64 FGMRES) reaches the same solution
    xm, infom = ctx.solve(mg, solver_params(precision=1, **tight), rhs, sol0)
    assert infom.status == 0
    assert rel(xm, x_o) <= TOL_MIXED
    # and at the configs' own stopping rule (relative residual 1e-10) the iteration
    # counts of the faithful FP64 form track the oracle's
    x1, i1 = ctx.solve(mg, solver_params(coarse_smoother=3), rhs, sol0)
    _, its1, _, _ = oracle_lib.solve(levels, oracle_lib.solver_params(), rhs, sol0)
    assert abs(i1.iterations - its1) <= 2


@pytest.mark.parametrize("dim,order,n0,L", [
    (3, 2, 4, 2),    # 4^3 Q2 coarsest level: 343 active DOFs
    (2, 1, 16, 2),   # 16^2 Q1 coarsest level: 225 active DOFs
])
def test_exact_coarse_solve_large_block_vs_oracle(ctx, oracle_lib, dim, order, n0, L):
    """Exact coarse solve (SolveExact, MGLevel3D.C:839) on a coarsest level whose active block
    is too large for the Gauss-Jordan inversion in shared memory (more than 160 rows): the
    inversion runs in the global buffer; FP64 and mixed solutions against the oracle's, and
    the iteration counts at the configs' stopping rule."""
    b = (1.0, 0.5) if dim == 2 else (0.57735026918962573,) * 3
    co = coeffs(0, eps=1e-1, b=b, f=1.0)
    spaces, parents, sids, mg = structured_case(ctx, dim, order, n0, L, co, 1)
    assert spaces[0]["n_active"] > 160
    levels = []
    for l, (sp, sid) in enumerate(zip(spaces, sids)):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        ent, rhs = oracle_lib.assemble(dim, order, 1, sp["coords"], sp["global_numbers"],
                                       sp["begin_index"], sp["n_dof"], sp["n_active"], rp, kc,
                                       oracle_coeffs(oracle_lib, co))
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc, entries=ent)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(
                dim, order, spaces[l - 1], dict(sp), parents[l])
        levels.append(lv)
        ctx.assemble(sid, 1, sp["n_dof"], len(kc), want_entries=False)
    sol0 = np.zeros(spaces[-1]["n_dof"])
    tight = dict(coarse_smoother=17, red_factor=0.0, res_norm_min=1e-14 * np.linalg.norm(rhs), maxit=3000)
    x_o, its_o, _, _ = oracle_lib.solve(levels, oracle_lib.solver_params(**tight), rhs, sol0)
    assert its_o > 0
    x, info = ctx.solve(mg, solver_params(**tight), rhs, sol0)
    assert info.status == 0
    assert rel(x, x_o) <= TOL_SOL, rel(x, x_o)
    xm, infom = ctx.solve(mg, solver_params(precision=1, **tight), rhs, sol0)
    assert infom.status == 0
    assert rel(xm, x_o) <= TOL_MIXED, rel(xm, x_o)
    _, its1, _, _ = oracle_lib.solve(levels, oracle_lib.solver_params(coarse_smoother=17), rhs, sol0)
    _, i1 = ctx.solve(mg, solver_params(coarse_smoother=17), rhs, sol0)
    assert abs(i1.iterations - its1) <= 1, (i1.iterations, its1)


@pytest.mark.parametrize("restart,minit", [(4, 0), (5, 9)])
def test_fgmres_restart_cycles_vs_oracle(ctx, oracle_lib, restart, minit):
    """FGMRES over several restart cycles (FgmresIte.C:536-560) and with a minimum iteration
    count: the device-side Arnoldi vectors, the iterations enqueued ahead of the host's Givens
    step and the restart update give the oracle's iterates, in FP64 and in the mixed form."""
    co = coeffs(0, eps=1e-3, b=(1.0, 0.5), f=1.0)
    dim, order, disc = 2, 1, 2
    spaces, parents, sids, mg = structured_case(ctx, dim, order, 4, 4, co, disc)
    levels = []
    for l, (sp, sid) in enumerate(zip(spaces, sids)):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        ent, rhs = oracle_lib.assemble(dim, order, disc, sp["coords"], sp["global_numbers"],
                                       sp["begin_index"], sp["n_dof"], sp["n_active"], rp, kc,
                                       oracle_coeffs(oracle_lib, co))
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc, entries=ent)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(
                dim, order, spaces[l - 1], dict(sp), parents[l])
        levels.append(lv)
        ctx.assemble(sid, disc, sp["n_dof"], len(kc), want_entries=False)
    sol0 = np.zeros(spaces[-1]["n_dof"])
    tight = dict(red_factor=0.0, res_norm_min=1e-12 * np.linalg.norm(rhs), maxit=400, restart=restart,
                 minit=minit)
    x_o, its_o, _, _ = oracle_lib.solve(levels, oracle_lib.solver_params(**tight), rhs, sol0)
    assert its_o > restart  # several restart cycles
    x, info = ctx.solve(mg, solver_params(coarse_smoother=3, **tight), rhs, sol0)
    assert info.status == 0
    assert abs(info.iterations - its_o) <= 2
    assert rel(x, x_o) <= TOL_SOL
    xm, infom = ctx.solve(mg, solver_params(precision=1, **tight), rhs, sol0)
    assert infom.status == 0
    assert rel(xm, x_o) <= TOL_MIXED


@pytest.mark.parametrize("dim", [2, 3])
def test_facade_assemble_and_solve(ctx, dim):
    """The TSystemCD3D / TSystemCD2D mirror: Assemble over the whole hierarchy in one call
    (rhs copied straight into the caller's array) gives the per-level assembly's rhs, and
    Solve in place into the caller's array gives the same solution as the copying path."""
    order, n0, L = (1, 4, 3) if dim == 2 else (2, 2, 2)
    spaces, parents = mesh.structured_hierarchy(dim, order, n0, L)
    b = (1.0, 0.5) if dim == 2 else (0.57735026918962573,) * 3
    cls = TSystemCD2D if dim == 2 else TSystemCD3D
    S = cls(spaces, parents, ctx=ctx)
    S.Init(coeffs(0, eps=1e-1, b=b, f=1.0))
    n = S.N_DOF
    sol, rhs = np.zeros(n), np.zeros(n)
    _, r = S.Assemble(sol, rhs)
    assert r is rhs
    ent2, r2 = S.Assemble(entries=True)          # per-level path with a copy of the entries
    assert np.array_equal(rhs, r2) and ent2 is not None
    prm = solver_params(precision=1, red_factor=1e-10)
    sol_a = np.zeros(n)
    sol_a[S.N_Active:] = rhs[S.N_Active:]
    sol_b = np.zeros(2 * n)[::2]                 # not contiguous: the copying path
    sol_b[S.N_Active:] = rhs[S.N_Active:]
    ia = S.Solve(sol_a, rhs, prm)
    ib = S.Solve(sol_b, rhs, prm)
    assert ia.status == 0 and ib.status == 0 and ia.iterations == ib.iterations
    assert np.array_equal(sol_a, sol_b)


def test_spmv_and_defect_vs_oracle(ctx, oracle_lib):
    co = coeffs(0, eps=1e-2, b=(0.2, 0.3, 0.4))
    spaces, parents, sids, mg = structured_case(ctx, 3, 2, 6, 1, co, 1)
    sp, sid = spaces[0], sids[0]
    nnz = ctx.build_pattern(sid)
    ent, rhs = ctx.assemble(sid, 1, sp["n_dof"], nnz)
    rp, kc = ctx.get_pattern(sid, sp["n_dof"], nnz)
    x = np.random.default_rng(1).standard_normal(sp["n_dof"])
    y = ctx.spmv(sid, x)
    y_o = oracle_lib.spmv(rp, kc, ent, x)
    assert rel(y, y_o) <= 1e-13
    dd, res = ctx.defect(sid, x, rhs)
    assert rel(dd, rhs - y_o) <= 1e-12
    assert abs(res - np.linalg.norm(rhs - y_o)) <= 1e-12 * np.linalg.norm(rhs - y_o)


def test_errors_are_reported(ctx):
    sp = mesh.structured_space(2, 1, 4)
    sid = ctx.upload_space(sp)
    # a pattern without the cell couplings
    rp = np.arange(sp["n_dof"] + 1, dtype=np.int32)
    kc = np.arange(sp["n_dof"], dtype=np.int32)
    ctx.upload_pattern(sid, rp, kc)
    ctx.set_coeffs(sid, coeffs(0, eps=1.0))
    with pytest.raises(_lib.CdgpuError) as e:
        ctx.assemble(sid, 1, sp["n_dof"], len(kc))
    assert e.value.status == _lib.ERR_PATTERN
    with pytest.raises(_lib.CdgpuError) as e:
        ctx.set_coeffs(sid, coeffs(0, eps=float("nan")))
    assert e.value.status == _lib.ERR_INVALID
    bad = dict(sp)
    bad["global_numbers"] = sp["global_numbers"].copy()
    bad["global_numbers"][0] = sp["n_dof"] + 5
    with pytest.raises(_lib.CdgpuError):
        ctx.upload_space(bad)


def test_matrix_free_cycle_q2_hex(ctx):
    """The mixed form's FP32 cycle applies the Q2-hexahedron operator matrix-free on levels of
    at least 16,384 cells (per-cell products from the assembly's reference tensors); its
    solution equals the FP64 form's (CSR throughout) within the mixed bar, with about the same
    number of FGMRES iterations."""
    co = coeffs(0, eps=1e-2, b=(0.57735026918962573,) * 3, f=1.0, delta0=1.0 / 3.0)
    spaces, parents, sids, mg = structured_case(ctx, 3, 2, 2, 5, co, 1)
    ctx.assemble_hierarchy(mg, 1, 2)
    nd = spaces[-1]["n_dof"]
    rhs = ctx.assemble(sids[-1], 1, nd, 1, want_entries=False)[1]
    sol0 = np.zeros(nd)
    prm = dict(stop_rule=1, red_factor=1e-12, maxit=200)
    x64, i64 = ctx.solve(mg, solver_params(precision=0, **prm), rhs, sol0)
    xm, im = ctx.solve(mg, solver_params(precision=1, **prm), rhs, sol0)
    assert i64.status == 0 and im.status == 0
    assert rel(xm, x64) <= TOL_MIXED
    assert abs(im.iterations - i64.iterations) <= 2


@pytest.mark.parametrize("solver,cycle", [(11, 1), (11, 2), (16, 2), (16, 0)])
def test_solver_variants_vs_oracle(ctx, oracle_lib, solver, cycle):
    """The fixed-point iteration (TFixedPointIte::Iterate, FixedPointIte.C:150-303) and the W-
    and F-cycles (SetRecursion, MultiGrid3D.C:691-703) against the oracle's restatement: the
    converged solution within 1e-10, the iteration count at the reference's stopping rule
    within one (fixed point) or two (FGMRES) of the oracle's, FP64 and mixed."""
    co = coeffs(0, eps=0.05, b=(1.0, 0.5), f=1.0)
    dim, order, disc = 2, 2, 1
    spaces, parents, sids, mg = structured_case(ctx, dim, order, 2, 4, co, disc)
    levels = []
    for l, (sp, sid) in enumerate(zip(spaces, sids)):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        ent, rhs = oracle_lib.assemble(dim, order, disc, sp["coords"], sp["global_numbers"],
                                       sp["begin_index"], sp["n_dof"], sp["n_active"], rp, kc,
                                       oracle_coeffs(oracle_lib, co))
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc, entries=ent)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(
                dim, order, spaces[l - 1], dict(sp), parents[l])
        levels.append(lv)
        ctx.assemble(sid, disc, sp["n_dof"], len(kc), want_entries=False)
    sol0 = np.zeros(spaces[-1]["n_dof"])
    common = dict(solver=solver, cycle=cycle, coarse_smoother=17, maxit=500)
    tight = dict(red_factor=0.0, res_norm_min=1e-13 * np.linalg.norm(rhs), **common)
    x_o, its_o, _, _ = oracle_lib.solve(levels, oracle_lib.solver_params(**tight), rhs, sol0)
    assert its_o > 0
    x, info = ctx.solve(mg, solver_params(**tight), rhs, sol0)
    assert info.status == 0
    assert rel(x, x_o) <= TOL_SOL, rel(x, x_o)
    xm, im = ctx.solve(mg, solver_params(precision=1, **tight), rhs, sol0)
    assert im.status == 0
    assert rel(xm, x_o) <= TOL_MIXED
    # the reference's own rule: residual reduced by 1e-10
    _, its1, _, _ = oracle_lib.solve(levels, oracle_lib.solver_params(red_factor=1e-10, **common), rhs, sol0)
    _, i1 = ctx.solve(mg, solver_params(red_factor=1e-10, **common), rhs, sol0)
    assert abs(i1.iterations - its1) <= (1 if solver == 11 else 2), (i1.iterations, its1)


@pytest.mark.parametrize("n", [27, 32])
def test_large_spmv_and_defect_vs_oracle(ctx, oracle_lib, n):
    """Matrices too large for L2 (27^3 and 32^3 Q2: 9.6M and 15.8M nonzeros) take the product
    whose matrix tiles are streamed into shared memory by bulk copies; product and defect
    against the oracle's CSR product, and the defect norm."""
    co = coeffs(0, eps=1e-2, b=(0.57735026918962573,) * 3, c=0.3, f=1.0)
    sp = mesh.structured_space(3, 2, n)
    sid = ctx.upload_space(sp)
    nnz = ctx.build_pattern(sid)
    ctx.set_coeffs(sid, co)
    ent, rhs = ctx.assemble(sid, 1, sp["n_dof"], nnz)
    rp, kc = ctx.get_pattern(sid, sp["n_dof"], nnz)
    rng = np.random.default_rng(n)
    for _ in range(2):
        x = rng.standard_normal(sp["n_dof"])
        y_o = oracle_lib.spmv(rp, kc, ent, x)
        y = ctx.spmv(sid, x)
        assert rel(y, y_o) <= 1e-13
        dd, res = ctx.defect(sid, x, rhs)
        assert rel(dd, rhs - y_o) <= 1e-12
        assert abs(res - np.linalg.norm(rhs - y_o)) <= 1e-12 * np.linalg.norm(rhs - y_o)


def test_errors_table_equals_sine_errors(ctx):
    """The tabulated-exact-solution error evaluation agrees with the SineLaplace one (the
    reference's recorded known answer) on the same solution."""
    d = golden("cd2d_q1_sine_32")
    dim, order, disc, lv, sids = setup_golden(ctx, d)
    fin = lv[-1]
    x = d["solution"]
    l2s, h1s = ctx.errors(sids[-1], x)
    nc = len(fin["begin_index"]) - 1
    q = ctx.quadrature_points(sids[-1], nc, 2)
    s, c = np.sin(np.pi * q), np.cos(np.pi * q)
    ex = np.stack([s[..., 0] * s[..., 1], np.pi * c[..., 0] * s[..., 1], np.pi * s[..., 0] * c[..., 1]], -1)
    l2, h1 = ctx.errors_table(sids[-1], x, ex)
    # both on a space that was never assembled (the reference element is built on demand), and
    # both the errors the reference printed for its own solution on this fixture
    l2_ref, h1_ref = float(d["err_l2"]), float(d["err_h1"])
    assert abs(l2s - l2_ref) <= 1e-9 * l2_ref and abs(h1s - h1_ref) <= 1e-9 * h1_ref, (l2s, h1s)
    assert abs(l2 - l2s) <= 1e-12 * l2s and abs(h1 - h1s) <= 1e-12 * h1s


@pytest.mark.parametrize("name", golden_names())
def test_device_pattern_equals_reference(ctx, name):
    """The CSR pattern built on the device (cdgpu_build_pattern_device) is the reference's
    TSquareStructure + Sort, bit for bit, on every level of every fixture (the non-affine meshes
    and the reference's own DOF numbering included)."""
    d = golden(name)
    dim, order = int(d["dim"]), int(d["order"])
    for l in range(int(d["levels"])):
        L = refdump.level(d, l)
        sid = ctx.upload_space(dict(dim=dim, order=order, coords=L["coords"], global_numbers=L["global_numbers"],
                                    begin_index=L["begin_index"], n_dof=L["n_dof"], n_active=L["n_active"]))
        nnz = ctx.build_pattern_device(sid)
        assert nnz == len(L["kcol"])
        rp, kc = ctx.get_pattern(sid, L["n_dof"], nnz)
        assert np.array_equal(rp, L["row_ptr"]) and np.array_equal(kc, L["kcol"])


@pytest.mark.parametrize("dim,order,n", [(3, 2, 32), (3, 1, 48), (2, 2, 256), (2, 1, 300)])
def test_device_pattern_equals_host_build(ctx, dim, order, n):
    """Large structured meshes: device build == host build, and the device build's matrix
    assembles and multiplies like the host build's."""
    import time
    sp = mesh.structured_space(dim, order, n)
    a = ctx.upload_space(sp)
    b = ctx.upload_space(sp)
    t0 = time.perf_counter()
    nnz_h = ctx.build_pattern(a)
    t1 = time.perf_counter()
    nnz_d = ctx.build_pattern_device(b)
    t2 = time.perf_counter()
    print(f"{dim}D Q{order} n={n}: host build {1e3 * (t1 - t0):.1f} ms, device build {1e3 * (t2 - t1):.1f} ms")
    assert nnz_h == nnz_d
    ra, ka = ctx.get_pattern(a, sp["n_dof"], nnz_h)
    rb, kb = ctx.get_pattern(b, sp["n_dof"], nnz_d)
    assert np.array_equal(ra, rb) and np.array_equal(ka, kb)
    co = coeffs(0, eps=1e-2, b=(0.3, 0.2, 0.1)[:dim], f=1.0)
    ctx.set_coeffs(a, co)
    ctx.set_coeffs(b, co)
    ea, _ = ctx.assemble(a, 1, sp["n_dof"], nnz_h)
    eb, _ = ctx.assemble(b, 1, sp["n_dof"], nnz_d)
    assert np.array_equal(ea, eb)
