"""The drop-in boundary, compiled: ParMooN's own 3DPrograms/CD3D_ParMooN.C, unchanged.

oracle/build_ref.py links the reference's main program twice from its unchanged source:
  cd3d_main      with the reference's own TSystemCD3D (src/System/SystemCD3D.C, CPU),
  cd3d_main_gpu  with parmoon_cmg_b200/shim/SystemCD3D_cdgpu.C, the TSystemCD3D that runs
                 assembly and the multigrid FGMRES solve in libcdgpu on the GPU.
Both read the same .dat (unit cube, Q2, 3 multigrid levels 2^3..8^3, Examples/CD_3D/Laplace.h:
-Laplace u = 3 pi^2 sin(pi x) sin(pi y) sin(pi z), its exact solution as Dirichlet data,
MEASURE_ERRORS on).  The GPU program must print the CPU program's L2 and H1-semi errors digit
for digit, in the FP64 and in the mixed form, and its solution must match the oracle's tight
FP64 solution of the same discrete problem (the reference's own mesh, dumped by
oracle/_ref/cd3d_dump, matched by DOF position) within 1e-10 (FP64) and 1e-8 (mixed).
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

DAT = """VERSION: 1
LOGFILE: logfile
OUTFILE: {out}
BNDFILE: {mesh}/unit_cube.PRM
GEOFILE: {mesh}/unit_cube.GEO
MESH_TYPE: 0
UNIFORM_STEPS: 1
LEVELS: 3
ANSATZ_ORDER: 2
DISCTYPE: 1
RE_NR: 1
SOLVER_TYPE: 1
SC_SOLVER_SCALAR: 16
SC_PRECONDITIONER_SCALAR: 5
SC_SMOOTHER_SCALAR: 1
SC_COARSE_SMOOTHER_SCALAR: 3
SC_SMOOTH_DAMP_FACTOR_SCALAR: 0.8
SC_SMOOTH_DAMP_FACTOR_FINE_SCALAR: 0.8
SC_PRE_SMOOTH_SCALAR: 2
SC_POST_SMOOTH_SCALAR: 2
SC_MG_CYCLE_SCALAR: 1
SC_STEP_LENGTH_CONTROL_ALL_SCALAR: 0
SC_STEP_LENGTH_CONTROL_FINE_SCALAR: 0
SC_GMRES_RESTART: 30
SC_LIN_RED_FACTOR_SCALAR: 1e-13
SC_LIN_RES_NORM_MIN_SCALAR: 0
SC_LIN_MAXIT_SCALAR: 30
SC_VERBOSE: 0
MEASURE_ERRORS: 1
WRITE_VTK: 0
"""


def run_main(exe, tmp, env_extra=None):
    dat = os.path.join(tmp, "cd3d.dat")
    with open(dat, "w") as f:
        f.write(DAT.format(out=os.path.join(tmp, "cd3d.out"), mesh=os.path.join(ROOT, "oracle", "meshes")))
    env = dict(os.environ)
    env.update(env_extra or {})
    p = subprocess.run([exe, dat], cwd=tmp, capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    l2 = re.findall(r"^L2: (\S+)", p.stdout, re.M)
    h1 = re.findall(r"^H1-semi: (\S+)", p.stdout, re.M)
    assert l2 and h1, p.stdout[-2000:]
    return l2[-1], h1[-1], p.stdout


@pytest.fixture(scope="module")
def cpu_errors():
    exe = os.path.join(REF, "cd3d_main")
    assert os.path.exists(exe), "oracle/_ref/cd3d_main is missing (oracle/build_ref.py)"
    with tempfile.TemporaryDirectory() as tmp:
        l2, h1, _ = run_main(exe, tmp)
    return l2, h1


@pytest.mark.parametrize("precision", [0, 1])
def test_unchanged_cd3d_main_on_gpu(cpu_errors, oracle_lib, precision):
    from parmoon_cmg_b200 import _build
    _build.build()
    exe = os.path.join(REF, "cd3d_main_gpu")
    assert os.path.exists(exe), "oracle/_ref/cd3d_main_gpu is missing (oracle/build_ref.py)"
    with tempfile.TemporaryDirectory() as tmp:
        sol_path = os.path.join(tmp, "sol.f64")
        l2, h1, out = run_main(exe, tmp, {"CDGPU_PRECISION": str(precision), "CDGPU_DUMP_SOLUTION": sol_path})
        assert "libcdgpu FGMRES ITE:" in out
        sol = np.fromfile(sol_path, dtype=np.float64)
        xyz = np.fromfile(sol_path + ".xyz", dtype=np.float64).reshape(-1, 3)
    # the reference's own output, digit for digit
    assert (l2, h1) == cpu_errors, ((l2, h1), cpu_errors)
    # the oracle's solution on cd3d_dump's numbering, matched to the main's DOFs by position
    x_o, xyz_o = laplace_oracle_solution(oracle_lib)
    key = lambda X: np.rint(X * 16).astype(np.int64) @ np.array([1, 17, 289])
    order_o = np.argsort(key(xyz_o))
    order_m = np.argsort(key(xyz))
    assert np.array_equal(key(xyz_o)[order_o], key(xyz)[order_m])
    x_m = np.empty_like(sol)
    x_m[order_m] = x_o[order_o]
    err = np.abs(sol - x_m).max() / np.abs(x_m).max()
    assert err <= (1e-10 if precision == 0 else 1e-8), err


def laplace_oracle_solution(oracle):
    """The oracle's FP64 solution of the same discrete problem on the reference's own mesh and
    DOF numbering (cd3d_dump with the same .dat): coefficients of Laplace.h at the oracle's
    quadrature points, its exact solution at the Dirichlet nodes, solved to 1e-14."""
    import refdump
    with tempfile.TemporaryDirectory() as tmp:
        dat = os.path.join(tmp, "d.dat")
        with open(dat, "w") as f:
            f.write(DAT.format(out=os.path.join(tmp, "d.out"), mesh=os.path.join(ROOT, "oracle", "meshes")))
        out = os.path.join(tmp, "dump")
        os.makedirs(out)
        subprocess.run([os.path.join(REF, "cd3d_dump"), dat, out, "1", "0", "0", "0", "0", "0", "0"], cwd=tmp,
                       check=True, capture_output=True)
        d = refdump.load_dir(out)
    L = int(d["levels"])
    lv = [refdump.level(d, l) for l in range(L)]
    levels, rhs = [], None
    for l, S in enumerate(lv):
        nc = len(S["begin_index"]) - 1
        q = oracle.quad_points(3, 2, S["coords"], nc)
        tab = np.zeros(q.shape[:2] + (6,))
        tab[..., 0] = 1.0
        tab[..., 5] = 3 * np.pi ** 2 * np.sin(np.pi * q[..., 0]) * np.sin(np.pi * q[..., 1]) * np.sin(np.pi * q[..., 2])
        xyz = oracle.dof_coords(3, 2, S["coords"], S["global_numbers"], S["begin_index"], S["n_dof"])
        na = S["n_active"]
        g = np.sin(np.pi * xyz[na:, 0]) * np.sin(np.pi * xyz[na:, 1]) * np.sin(np.pi * xyz[na:, 2])
        rp, kc = oracle.pattern(S["global_numbers"], S["begin_index"], S["n_dof"], na)
        ent, rhs = oracle.assemble(3, 2, 1, S["coords"], S["global_numbers"], S["begin_index"], S["n_dof"], na,
                                   rp, kc, oracle.coeffs(3), coeff_tab=tab, dir_vals=g)
        e = dict(n_dof=S["n_dof"], n_active=na, row_ptr=rp, kcol=kc, entries=ent)
        if l > 0:
            e["p_row"], e["p_col"], e["p_val"] = oracle.prolongation(3, 2, lv[l - 1], S, S["parent"])
        levels.append(e)
    fin = lv[-1]
    sol0 = np.zeros(fin["n_dof"])
    sol0[fin["n_active"]:] = rhs[fin["n_active"]:]
    prm = oracle.solver_params(red_factor=0.0, res_norm_min=1e-14 * np.linalg.norm(rhs), maxit=300)
    x, _, _, _ = oracle.solve(levels, prm, rhs, sol0)
    return x, oracle.dof_coords(3, 2, fin["coords"], fin["global_numbers"], fin["begin_index"], fin["n_dof"])


@pytest.fixture(scope="module")
def laplace_gpu():
    """The Laplace example solved through the C ABI on the reference's own mesh and DOF
    numbering (cd3d_dump with the same .dat), coefficients tabulated at the library's
    quadrature points, the exact solution as Dirichlet data."""
    import oracle
    import refdump
    from parmoon_cmg_b200 import _build, _lib
    from parmoon_cmg_b200.system import Context, coeffs, solver_params
    _build.build()
    with tempfile.TemporaryDirectory() as tmp:
        dat = os.path.join(tmp, "d.dat")
        with open(dat, "w") as f:
            f.write(DAT.format(out=os.path.join(tmp, "d.out"), mesh=os.path.join(ROOT, "oracle", "meshes")))
        out = os.path.join(tmp, "dump")
        os.makedirs(out)
        subprocess.run([os.path.join(REF, "cd3d_dump"), dat, out, "1", "0", "0", "0", "0", "0", "0"], cwd=tmp,
                       check=True, capture_output=True)
        d = refdump.load_dir(out)
    lv = [refdump.level(d, l) for l in range(int(d["levels"]))]
    ctx = Context(0)
    sids = []
    for S in lv:
        sid = ctx.upload_space(dict(dim=3, order=2, coords=S["coords"], global_numbers=S["global_numbers"],
                                    begin_index=S["begin_index"], n_dof=S["n_dof"], n_active=S["n_active"]))
        ctx.build_pattern(sid)
        nc = len(S["begin_index"]) - 1
        q = ctx.quadrature_points(sid, nc, 3)
        tab = np.zeros(q.shape[:2] + (6,))
        tab[..., 0] = 1.0
        tab[..., 5] = 3 * np.pi ** 2 * np.prod(np.sin(np.pi * q), axis=-1)
        ctx.set_coeffs(sid, coeffs(_lib.COEFF_TABLE), tab)
        sids.append(sid)
    mg = ctx.hierarchy(sids, [None] + [S["parent"] for S in lv[1:]])
    rhs = None
    for S, sid in zip(lv, sids):
        xyz = oracle.dof_coords(3, 2, S["coords"], S["global_numbers"], S["begin_index"], S["n_dof"])
        g = np.prod(np.sin(np.pi * xyz[S["n_active"]:]), axis=-1)
        _, rhs = ctx.assemble(sid, 1, S["n_dof"], 1, dirichlet=g, want_entries=False)
    fin = lv[-1]
    sol0 = np.zeros(fin["n_dof"])
    sol0[fin["n_active"]:] = rhs[fin["n_active"]:]
    x, info = ctx.solve(mg, solver_params(coarse_smoother=3, red_factor=1e-13, maxit=30), rhs, sol0)
    assert info.status == 0
    yield dict(ctx=ctx, sids=sids, lv=lv, x=x)
    ctx.close()


def test_errors_table_reproduces_reference_output(cpu_errors, laplace_gpu):
    """GetErrors on the device for any exact solution (cdgpu_errors_table): the L2 and H1-semi
    errors that the reference's CD3D main prints, digit for digit."""
    ctx, sids, fin, x = laplace_gpu["ctx"], laplace_gpu["sids"], laplace_gpu["lv"][-1], laplace_gpu["x"]
    nc = len(fin["begin_index"]) - 1
    q = ctx.quadrature_points(sids[-1], nc, 3)
    s, c = np.sin(np.pi * q), np.cos(np.pi * q)
    ex = np.stack([s[..., 0] * s[..., 1] * s[..., 2], np.pi * c[..., 0] * s[..., 1] * s[..., 2],
                   np.pi * s[..., 0] * c[..., 1] * s[..., 2], np.pi * s[..., 0] * s[..., 1] * c[..., 2]], -1)
    l2, h1 = ctx.errors_table(sids[-1], x, ex)
    assert (f"{l2:g}", f"{h1:g}") == cpu_errors, ((l2, h1), cpu_errors)


def read_vtk(path):
    """POINTS, CELLS (connectivity rows) and the first POINT_DATA scalar field of a legacy VTK file."""
    tok = open(path).read().split()
    i = tok.index("POINTS")
    n = int(tok[i + 1])
    pts = np.array(tok[i + 3:i + 3 + 3 * n], float).reshape(n, 3)
    i = tok.index("CELLS")
    nc = int(tok[i + 1])
    cells, j = [], i + 3
    for _ in range(nc):
        k = int(tok[j])
        cells.append([int(t) for t in tok[j + 1:j + 1 + k]])
        j += k + 1
    i = tok.index("POINT_DATA")
    j = tok.index("LOOKUP_TABLE", i) + 2
    vals = np.array(tok[j:j + n], float)
    return pts, cells, vals


def test_vtk_from_device_buffer_matches_reference_output(laplace_gpu):
    """cdgpu_write_vtk from a solution held on the device writes the points, hexahedra and
    vertex values that the reference's own TOutput3D::WriteVtk writes for the same problem
    (its CD3D main with WRITE_VTK), up to the order of the points and the printed digits."""
    import torch
    ctx, sid, x = laplace_gpu["ctx"], laplace_gpu["sids"][-1], laplace_gpu["x"]
    with tempfile.TemporaryDirectory() as tmp:
        dat = os.path.join(tmp, "v.dat")
        with open(dat, "w") as f:
            f.write(DAT.format(out=os.path.join(tmp, "v.out"), mesh=os.path.join(ROOT, "oracle", "meshes"))
                    .replace("WRITE_VTK: 0", "WRITE_VTK: 1\nVTKBASENAME: ref"))
        subprocess.run([os.path.join(REF, "cd3d_main"), dat], cwd=tmp, check=True, capture_output=True, timeout=600)
        vtks = sorted(f for f in os.listdir(os.path.join(tmp, "VTK")) if f.endswith(".vtk"))
        assert vtks, "the reference wrote no VTK file"
        p_ref, c_ref, v_ref = read_vtk(os.path.join(tmp, "VTK", vtks[-1]))
        d_x = torch.tensor(x, device="cuda:0")
        torch.cuda.synchronize()
        ours = os.path.join(tmp, "ours.vtk")
        ctx.write_vtk(sid, d_x.data_ptr(), ours, on_device=True)
        p, cells, v = read_vtk(ours)
    assert len(p) == len(p_ref) and len(cells) == len(c_ref)
    key = lambda P: np.rint(P * 8).astype(np.int64) @ np.array([1, 9, 81])
    o, o_ref = np.argsort(key(p)), np.argsort(key(p_ref))
    assert np.array_equal(key(p)[o], key(p_ref)[o_ref])
    assert np.abs(v[o] - v_ref[o_ref]).max() <= 1e-5 * np.abs(v_ref).max()
    # the same cells, as sets of vertex positions
    cell_key = lambda P, C: sorted(tuple(sorted(key(P[c]).tolist())) for c in C)
    assert cell_key(p, cells) == cell_key(p_ref, c_ref)
