"""The drop-in boundary, compiled: ParMooN's own 3DPrograms/CD3D_ParMooN.C, unchanged.

oracle/build_ref.py links the reference's main program twice from its unchanged source:
  cd3d_main      with the reference's own TSystemCD3D (src/System/SystemCD3D.C, CPU),
  cd3d_main_gpu  with parmoon_cmg_b200/shim/SystemCD3D_cdgpu.C, the TSystemCD3D that runs
                 assembly and the multigrid FGMRES solve in libcdgpu on the GPU.
Both read the same .dat: unit cube, Q2, 3 multigrid levels 2^3..8^3, the main's own example
Examples/CD_3D/Laplace.h (eps = 1/RE_NR, no source term, Dirichlet data BoundValue on the
faces whose boundary component is not 0 and Neumann data 1 on component 0), VTK output and
MEASURE_ERRORS on.  The main writes the solution to VTK (TOutput3D::WriteVtk), then replaces
it by the interpolant of Exact() and prints that interpolant's L2 / H1-semi errors.

Checked: the GPU program's VTK has the CPU program's points, cells and values (6 printed
digits), in the FP64 and in the mixed form (the two forms' solutions within 1e-8 of each
other); the printed errors match digit for digit; cdgpu_errors_table gives those printed
errors for the same interpolant; cdgpu_write_vtk from a device buffer writes the CPU
program's VTK content.
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
WRITE_VTK: 1
VTKBASENAME: cd3d
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


def last_vtk(tmp):
    vtks = sorted(f for f in os.listdir(os.path.join(tmp, "VTK")) if f.endswith(".vtk"))
    assert vtks, "no VTK file written"
    return read_vtk(os.path.join(tmp, "VTK", vtks[-1]))


def pkey(P):
    return np.rint(P * 16).astype(np.int64) @ np.array([1, 17, 289])


def run_main(exe, env_extra=None):
    """Run a main program on the .dat; returns its printed L2 / H1-semi errors, its VTK output
    and, for the GPU program, the solution it solved (with the DOF positions)."""
    with tempfile.TemporaryDirectory() as tmp:
        dat = os.path.join(tmp, "cd3d.dat")
        with open(dat, "w") as f:
            f.write(DAT.format(out=os.path.join(tmp, "cd3d.out"), mesh=os.path.join(ROOT, "oracle", "meshes")))
        env = dict(os.environ)
        env.update(env_extra or {})
        sol_path = os.path.join(tmp, "sol.f64")
        env["CDGPU_DUMP_SOLUTION"] = sol_path
        p = subprocess.run([exe, dat], cwd=tmp, capture_output=True, text=True, env=env, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        l2 = re.findall(r"^L2: (\S+)", p.stdout, re.M)
        h1 = re.findall(r"^H1-semi: (\S+)", p.stdout, re.M)
        assert l2 and h1, p.stdout[-2000:]
        out = dict(errors=(l2[-1], h1[-1]), vtk=last_vtk(tmp), stdout=p.stdout)
        if os.path.exists(sol_path):
            out["sol"] = np.fromfile(sol_path, dtype=np.float64)
            out["xyz"] = np.fromfile(sol_path + ".xyz", dtype=np.float64).reshape(-1, 3)
    return out


@pytest.fixture(scope="module")
def cpu_run():
    exe = os.path.join(REF, "cd3d_main")
    assert os.path.exists(exe), "oracle/_ref/cd3d_main is missing (oracle/build_ref.py)"
    return run_main(exe)


@pytest.fixture(scope="module")
def gpu_runs():
    from parmoon_cmg_b200 import _build
    _build.build()
    exe = os.path.join(REF, "cd3d_main_gpu")
    assert os.path.exists(exe), "oracle/_ref/cd3d_main_gpu is missing (oracle/build_ref.py)"
    return {prec: run_main(exe, {"CDGPU_PRECISION": str(prec)}) for prec in (0, 1)}


def same_vtk(a, b, tol):
    """Same points (by position), same cells (as sets of positions), values within tol of the
    largest value."""
    (p, c, v), (p_r, c_r, v_r) = a, b
    assert len(p) == len(p_r) and len(c) == len(c_r)
    o, o_r = np.argsort(pkey(p)), np.argsort(pkey(p_r))
    assert np.array_equal(pkey(p)[o], pkey(p_r)[o_r])
    cell_key = lambda P, C: sorted(tuple(sorted(pkey(P[cc]).tolist())) for cc in C)
    assert cell_key(p, c) == cell_key(p_r, c_r)
    err = np.abs(v[o] - v_r[o_r]).max() / np.abs(v_r).max()
    assert err <= tol, err


@pytest.mark.parametrize("precision", [0, 1])
def test_unchanged_cd3d_main_on_gpu(cpu_run, gpu_runs, precision):
    g = gpu_runs[precision]
    assert "libcdgpu FGMRES ITE:" in g["stdout"]
    # the solution as the reference's own VTK writer prints it (6 significant digits)
    same_vtk(g["vtk"], cpu_run["vtk"], 2e-6)
    assert g["errors"] == cpu_run["errors"]
    if precision == 1:
        x64, xm = gpu_runs[0]["sol"], g["sol"]
        assert np.abs(xm - x64).max() <= 1e-8 * np.abs(x64).max()


@pytest.fixture(scope="module")
def ref_mesh():
    """The finest level of the same mesh as the reference builds it (cd3d_dump, same .dat)."""
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
    return refdump.level(d, int(d["levels"]) - 1)


def test_errors_table_reproduces_reference_output(cpu_run, ref_mesh, oracle_lib):
    """GetErrors on the device for any exact solution (cdgpu_errors_table): for the interpolant
    of Laplace.h's Exact() the L2 and H1-semi errors that the reference's CD3D main prints for
    the same interpolant, digit for digit."""
    from parmoon_cmg_b200.system import Context
    L = ref_mesh
    ctx = Context(0)
    try:
        sid = ctx.upload_space(dict(dim=3, order=2, coords=L["coords"], global_numbers=L["global_numbers"],
                                    begin_index=L["begin_index"], n_dof=L["n_dof"], n_active=L["n_active"]))
        xyz = oracle_lib.dof_coords(3, 2, L["coords"], L["global_numbers"], L["begin_index"], L["n_dof"])
        u_int = np.prod(np.sin(np.pi * xyz), axis=-1)
        nc = len(L["begin_index"]) - 1
        q = ctx.quadrature_points(sid, nc, 3)
        s, c = np.sin(np.pi * q), np.cos(np.pi * q)
        ex = np.stack([s[..., 0] * s[..., 1] * s[..., 2], np.pi * c[..., 0] * s[..., 1] * s[..., 2],
                       np.pi * s[..., 0] * c[..., 1] * s[..., 2], np.pi * s[..., 0] * s[..., 1] * c[..., 2]], -1)
        l2, h1 = ctx.errors_table(sid, u_int, ex)
    finally:
        ctx.close()
    assert (f"{l2:g}", f"{h1:g}") == cpu_run["errors"], ((l2, h1), cpu_run["errors"])


def test_vtk_from_device_buffer_matches_reference_output(cpu_run, gpu_runs, ref_mesh, oracle_lib):
    """cdgpu_write_vtk, from the GPU program's solution held in device memory, writes the points,
    hexahedra and vertex values that the reference's own TOutput3D::WriteVtk wrote."""
    import torch
    from parmoon_cmg_b200.system import Context
    L, g = ref_mesh, gpu_runs[0]
    xyz = oracle_lib.dof_coords(3, 2, L["coords"], L["global_numbers"], L["begin_index"], L["n_dof"])
    # the GPU program's solution in cd3d_dump's numbering (matched by DOF position)
    o, o_g = np.argsort(pkey(xyz)), np.argsort(pkey(g["xyz"]))
    assert np.array_equal(pkey(xyz)[o], pkey(g["xyz"])[o_g])
    x = np.empty(L["n_dof"])
    x[o] = g["sol"][o_g]
    ctx = Context(0)
    try:
        sid = ctx.upload_space(dict(dim=3, order=2, coords=L["coords"], global_numbers=L["global_numbers"],
                                    begin_index=L["begin_index"], n_dof=L["n_dof"], n_active=L["n_active"]))
        d_x = torch.tensor(x, device="cuda:0")
        torch.cuda.synchronize()
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "ours.vtk")
            ctx.write_vtk(sid, d_x.data_ptr(), path, name="C", on_device=True)
            ours = read_vtk(path)
    finally:
        ctx.close()
    same_vtk(ours, cpu_run["vtk"], 2e-6)
