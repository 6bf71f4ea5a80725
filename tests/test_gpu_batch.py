"""Batched solves (cdgpu_batch_*): many instances per launch, device-side FGMRES control.

Every instance of a batch -- mixed 2D/3D, Q1/Q2, sizes, coefficients -- reaches the oracle's
FP64 solution of its own system within 1e-8 relative (the batched configs' bar), with the
Jacobi smoother and with the multicolour SSOR smoother.  An instance's result does not
depend on the other instances: solved alone or submitted into a running mix, its solution
and iteration count are bit-identical.
"""
import math

import numpy as np
import pytest

from parmoon_cmg_b200 import _lib, mesh
from parmoon_cmg_b200.system import SUPG, Batch, Context, coeffs, solver_params

pytestmark = pytest.mark.gpu

TOL = 1e-8

CASES = [  # dim, order, n0, levels, eps, angle
    (2, 1, 4, 3, 1e-2, 0.3),
    (2, 2, 4, 2, 1e-3, 2.0),
    (2, 1, 5, 3, 1e-5, 4.1),
    (2, 2, 3, 3, 1e-1, 5.5),
    (3, 1, 2, 3, 1e-1, 0.0),
]


def case_coeffs(dim, eps, ang):
    b = (math.cos(ang), math.sin(ang)) if dim == 2 else (0.57735026918962573,) * 3
    return b, eps


def oracle_solution(oracle_lib, dim, order, spaces, parents, eps, b, disc):
    co = oracle_lib.coeffs(0, eps=eps, b=b, f=1.0, order_pd=order)
    levels = []
    for l, sp in enumerate(spaces):
        rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
        ent, rhs = oracle_lib.assemble(dim, order, disc, sp["coords"], sp["global_numbers"], sp["begin_index"],
                                       sp["n_dof"], sp["n_active"], rp, kc, co)
        lv = dict(n_dof=sp["n_dof"], n_active=sp["n_active"], row_ptr=rp, kcol=kc, entries=ent)
        if l > 0:
            lv["p_row"], lv["p_col"], lv["p_val"] = oracle_lib.prolongation(dim, order, spaces[l - 1], dict(sp),
                                                                            parents[l])
        levels.append(lv)
    # the oracle's own multigrid may stall on the convection-dominated cases: use a direct
    # solve of the finest system (scipy, FP64) as the reference solution
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    f = levels[-1]
    A = sps.csr_matrix((f["entries"], f["kcol"], f["row_ptr"]), shape=(f["n_dof"],) * 2)
    return spl.spsolve(A.tocsc(), rhs)


@pytest.fixture(scope="module")
def ctx():
    from parmoon_cmg_b200 import _build
    _build.build()
    c = Context(0)
    yield c
    c.close()


def batch_params(smoother):
    return solver_params(smoother=smoother, omega=0.8 if smoother == 1 else 1.0, stop_rule=1, red_factor=1e-12,
                         maxit=600, restart=30)


@pytest.mark.parametrize("smoother", [1, 3])
def test_batch_matches_fp64_solutions(ctx, oracle_lib, smoother):
    B = Batch(batch_params(smoother), ctx)
    meta = []
    for dim, order, n0, L, eps, ang in CASES:
        spaces, parents = mesh.structured_hierarchy(dim, order, n0, L)
        sid = B.add_structure(spaces, parents)
        b, eps = case_coeffs(dim, eps, ang)
        slot = B.submit(sid, coeffs(0, eps=eps, b=b, f=1.0, poly_degree=order), SUPG)
        meta.append((slot, spaces, parents, dim, order, eps, b))
    done = B.run(4)
    assert sorted(done) == sorted(m[0] for m in meta)
    # the iterations ran in the device-side loop: one conditional graph launch per advance
    mode, graph_launches, host_iterations = B.loop_info()
    assert mode in (1, 2) and graph_launches > 0 and host_iterations == 0, B.loop_info()
    for slot, spaces, parents, dim, order, eps, b in meta:
        x, info = B.fetch(slot, spaces[-1]["n_dof"])
        ref = oracle_solution(oracle_lib, dim, order, spaces, parents, eps, b, SUPG)
        assert info.status == 0, (dim, order, eps, info.iterations)
        err = np.abs(x - ref).max() / np.abs(ref).max()
        assert err <= TOL, (dim, order, eps, err, info.iterations)


def test_batch_instance_independent_of_the_mix(ctx):
    prm = batch_params(1)
    spaces, parents = mesh.structured_hierarchy(2, 2, 4, 3)
    co = coeffs(0, eps=1e-3, b=(0.6, 0.8), f=1.0, poly_degree=2)
    # alone
    A = Batch(prm, ctx)
    s0 = A.add_structure(spaces, parents)
    a = A.submit(s0, co, SUPG)
    A.run(3)
    x_alone, i_alone = A.fetch(a, spaces[-1]["n_dof"])
    # in a mix: other instances first, ours submitted while they are running
    M = Batch(prm, ctx)
    s1 = M.add_structure(spaces, parents)
    sp2, pa2 = mesh.structured_hierarchy(2, 1, 4, 4)
    s2 = M.add_structure(sp2, pa2)
    others = [M.submit(s2, coeffs(0, eps=10.0 ** -k, b=(1.0, 0.0), f=1.0), SUPG) for k in range(1, 4)]
    others.append(M.submit(s1, coeffs(0, eps=1e-1, b=(0.0, 1.0), f=1.0, poly_degree=2), SUPG))
    M.advance(5)
    mine = M.submit(s1, co, SUPG)
    M.advance(2)
    M.release(others[0])  # one leaves mid-run
    M.run(3)
    x_mix, i_mix = M.fetch(mine, spaces[-1]["n_dof"])
    assert i_mix.iterations == i_alone.iterations
    assert np.array_equal(x_mix, x_alone)


def test_batch_release_reuses_slots_and_memory(ctx):
    B = Batch(batch_params(1), ctx)
    spaces, parents = mesh.structured_hierarchy(2, 1, 4, 2)
    s = B.add_structure(spaces, parents)
    per = B.instance_bytes(s)
    slots = [B.submit(s, coeffs(0, eps=1e-2, b=(1.0, 0.0), f=1.0), SUPG) for _ in range(3)]
    assert B.memory() >= 3 * per * 0.5
    B.run(4)
    for sl in slots:
        B.release(sl)
    assert B.memory() == 0
    again = B.submit(s, coeffs(0, eps=1e-2, b=(1.0, 0.0), f=1.0), SUPG)
    assert again in slots
    B.run(4)
    x, info = B.fetch(again, spaces[-1]["n_dof"])
    assert info.status == 0 and np.isfinite(x).all()


def test_batch_rejects_bad_parameters(ctx):
    with pytest.raises(_lib.CdgpuError):
        Batch(solver_params(coarse_smoother=3), ctx)
    with pytest.raises(_lib.CdgpuError):
        Batch(solver_params(smoother=4), ctx)
