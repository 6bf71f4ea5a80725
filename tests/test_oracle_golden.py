"""Pin the CPU oracle (oracle/cdoracle.c) to the compiled reference.

The fixtures in tests/golden/ were written by the reference's own code path
(tests/golden/make_golden.py runs TSystemCD3D / TSystemCD2D + the reference's
multigrid and FGMRES from oracle/_ref).  The oracle must reproduce them:
CSR pattern bit-exact, matrix entries and right-hand sides within 1e-12
relative, prolongation exactly, converged solution within 1e-10 relative, and
the sine problem's recorded errors (ReadIn/cd2d.out:434-435).
"""
import numpy as np
import pytest

from conftest import golden, golden_names

import refdump


def levels_of(d):
    return [refdump.level(d, l) for l in range(int(d["levels"]))]


def oracle_level(oracle, d, L):
    dim, order, disc = int(d["dim"]), int(d["order"]), int(d["disctype"])
    rp, kc = oracle.pattern(L["global_numbers"], L["begin_index"], L["n_dof"], L["n_active"])
    b = tuple(np.atleast_1d(d["b"])) + (0.0,) * 3
    if int(d["example"]) == 1:
        co = oracle.coeffs(1, eps=float(d["eps"]))
    else:
        co = oracle.coeffs(0, eps=float(d["eps"]), b=b[:3], c=float(d["c"]), f=float(d["f"]))
    ent, rhs = oracle.assemble(dim, order, disc, L["coords"], L["global_numbers"], L["begin_index"],
                               L["n_dof"], L["n_active"], rp, kc, co)
    if int(d["example"]) == 1:
        oracle.neumann_sine(order, L["coords"], L["global_numbers"], L["begin_index"],
                            L["n_active"], float(d["eps"]), rhs)
    return rp, kc, ent, rhs


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", golden_names())
def test_pattern_entries_rhs(oracle_lib, name):
    d = golden(name)
    for L in levels_of(d):
        rp, kc, ent, rhs = oracle_level(oracle_lib, d, L)
        assert np.array_equal(rp, L["row_ptr"]) and np.array_equal(kc, L["kcol"]), "pattern"
        assert rel(ent, L["entries"]) <= 1e-12
        assert rel(rhs, L["rhs"]) <= 1e-12


@pytest.mark.parametrize("name", golden_names())
def test_prolongation_exact(oracle_lib, name):
    d = golden(name)
    lv = levels_of(d)
    dim, order = int(d["dim"]), int(d["order"])
    for l in range(1, len(lv)):
        C, F = lv[l - 1], lv[l]
        if "prolong_dense" not in F:
            continue
        rp, col, val = oracle_lib.prolongation(dim, order, C, F, F["parent"])
        P = np.zeros((F["n_dof"], C["n_dof"]))
        for i in range(F["n_dof"]):
            P[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
        assert np.array_equal(P, F["prolong_dense"].reshape(F["n_dof"], C["n_dof"]))


def oracle_solve(oracle, d, tight=True):
    lv = levels_of(d)
    dim, order = int(d["dim"]), int(d["order"])
    levels = []
    for l, L in enumerate(lv):
        rp, kc, ent, rhs = oracle_level(oracle, d, L)
        e = dict(n_dof=L["n_dof"], n_active=L["n_active"], row_ptr=rp, kcol=kc, entries=ent)
        if l > 0:
            e["p_row"], e["p_col"], e["p_val"] = oracle.prolongation(dim, order, lv[l - 1], L,
                                                                     L["parent"])
        levels.append(e)
    sol0 = np.zeros(lv[-1]["n_dof"])
    sol0[lv[-1]["n_active"]:] = rhs[lv[-1]["n_active"]:]
    if tight:
        prm = oracle.solver_params(red_factor=0.0, res_norm_min=1e-14 * np.linalg.norm(rhs),
                                   maxit=2000)
    else:
        prm = oracle.solver_params()
    return oracle.solve(levels, prm, rhs, sol0), lv


@pytest.mark.parametrize("name", golden_names())
def test_solution(oracle_lib, name):
    d = golden(name)
    (sol, its, hist, fres), lv = oracle_solve(oracle_lib, d)
    assert its > 0
    assert rel(sol, d["solution"]) <= 1e-10


def test_sine_known_answer(oracle_lib):
    """ReadIn/cd2d.out:434-435: SineLaplace, 32x32 Q1 Galerkin, PE_NR 10 ->
    L2 4.751079e-04, H1-semi 6.295197e-02 (printed to 7 digits)."""
    d = golden("cd2d_q1_sine_32")
    (sol, its, _, _), lv = oracle_solve(oracle_lib, d)
    L = lv[-1]
    e = oracle_lib.errors_sine(1, L["coords"], L["global_numbers"], L["begin_index"], sol)
    assert f"{e[0]:.6e}" == "4.751079e-04"
    assert f"{e[1]:.6e}" == "6.295197e-02"
    # the reference run behind the fixture printed the same numbers
    assert f"{float(d['err_l2']):.6e}" == "4.751079e-04"
    assert f"{float(d['err_h1']):.6e}" == "6.295197e-02"


def test_tcd2d_known_answer(oracle_lib):
    """ReadIn/tcd2d.out:485-543: the oracle's theta-scheme step (oracle.tcd_step, the
    restatement of SystemTCD2D.C:154-210) on exp.h, 32x32 Q1, Crank-Nicolson, tau 0.05, gives
    the reference's printed L2 and H1-semi errors at t = 0 and after each of 10 steps."""
    import tcd_exp
    from parmoon_cmg_b200 import mesh
    spaces, parents = mesh.structured_hierarchy(2, 1, 4, 4)
    fin = spaces[-1]
    assert (fin["n_dof"], fin["n_active"]) == (1089, 961)
    levels = []
    for l, sp in enumerate(spaces):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(2, 1, spaces[l - 1], dict(sp), parents[l])
        levels.append(lv)
    co = oracle_lib.coeffs(3)

    def forms(disc, t):
        out, r = [], None
        for sp, lv in zip(spaces, levels):
            xq = oracle_lib.quad_points(2, 1, sp["coords"], len(sp["begin_index"]) - 1)
            e, r = oracle_lib.assemble(2, 1, disc, sp["coords"], sp["global_numbers"], sp["begin_index"],
                                       sp["n_dof"], sp["n_active"], lv["row_ptr"], lv["kcol"], co,
                                       coeff_tab=tcd_exp.coeff_table(xq, t))
            out.append(e)
        return out, r

    def errors(u, t):
        return tcd_exp.fmt(oracle_lib.errors_sinsin(1, fin["coords"], fin["global_numbers"],
                                                    fin["begin_index"], u, 2.0, np.exp(t)))

    M, f = forms(10, 0.0)
    xyz = oracle_lib.dof_coords(2, 1, fin["coords"], fin["global_numbers"], fin["begin_index"], fin["n_dof"])
    u = tcd_exp.initial(xyz)
    assert errors(u, 0.0) == tcd_exp.KNOWN[0][1:]
    prm = oracle_lib.solver_params(red_factor=0.0, res_norm_min=1e-13, maxit=300)
    for k in range(1, len(tcd_exp.KNOWN)):
        t = tcd_exp.KNOWN[k][0]
        A, fnew = forms(1, t)
        u, its = oracle_lib.tcd_step(levels, M, A, f, fnew, u, tcd_exp.TAU, *tcd_exp.THETA, prm)
        assert its > 0
        f = fnew
        assert errors(u, t) == tcd_exp.KNOWN[k][1:], t


def test_mg_preconditioner_matches_reference(oracle_lib):
    """One multigrid application equals the reference's (cd3d dump 'prec_rhs')."""
    d = golden("cd3d_q1_gal_4")
    lv = levels_of(d)
    levels = []
    for l, L in enumerate(lv):
        e = dict(n_dof=L["n_dof"], n_active=L["n_active"], row_ptr=L["row_ptr"], kcol=L["kcol"],
                 entries=L["entries"])
        if l > 0:
            e["p_row"], e["p_col"], e["p_val"] = oracle_lib.prolongation(3, 1, lv[l - 1], L, L["parent"])
        levels.append(e)
    prm = oracle_lib.solver_params(solver=11, maxit=1, red_factor=0.0)
    z, _, _, _ = oracle_lib.solve(levels, prm, lv[-1]["rhs"], np.zeros(lv[-1]["n_dof"]))
    assert rel(z, d["prec_rhs"]) <= 1e-13
