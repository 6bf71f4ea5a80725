"""The 2D drop-in, compiled: ParMooN's own 2DPrograms/CD2D_ParMooN.C, unchanged, built with its
own test switch (_TEST: the SineLaplace example, CD2D_ParMooN.C:21-26) and linked with
parmoon_cmg_b200/shim/SystemCD2D_cdgpu.C (the TSystemCD2D whose solve is the library's
multigrid FGMRES on a hierarchy built from the mesh's refinement tree).

On the unit square refined to 32 x 32 Q1 cells (eps = 1/PE_NR = 0.1, Neumann data on boundary
component 1) the program must print the reference's recorded known answer,
ReadIn/cd2d.out:434-435: "L2: 4.751079e-04" and "H1-semi: 6.295197e-02", and its solution must
match the compiled reference's solution of the same problem (tests/golden/cd2d_q1_sine_32.npz,
written by oracle/_ref/cd2d_dump) within 1e-9.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

DAT = """VERSION: 1
LOGFILE: logfile
OUTFILE: {out}
BNDFILE: {mesh}/unit_square.PRM
GEOFILE: {mesh}/unit_square.GEO
MESH_TYPE: 0
UNIFORM_STEPS: 5
ANSATZ_ORDER: 1
DISCTYPE: 1
PE_NR: 10
MEASURE_ERRORS: 1
WRITE_VTK: 0
WRITE_PS: 0
SC_VERBOSE: 0
"""


@pytest.mark.parametrize("precision", [0, 1])
def test_unchanged_cd2d_main_known_answer(precision):
    from parmoon_cmg_b200 import _build
    _build.build()
    exe = os.path.join(REF, "cd2d_main_gpu")
    assert os.path.exists(exe), "oracle/_ref/cd2d_main_gpu is missing (oracle/build_ref.py)"
    with tempfile.TemporaryDirectory() as tmp:
        dat = os.path.join(tmp, "cd2d.dat")
        out = os.path.join(tmp, "cd2d.out")
        with open(dat, "w") as f:
            f.write(DAT.format(out=out, mesh=os.path.join(ROOT, "oracle", "meshes")))
        env = dict(os.environ, CDGPU_PRECISION=str(precision), CDGPU_DUMP_SOLUTION=os.path.join(tmp, "sol.f64"))
        p = subprocess.run([exe, dat], cwd=tmp, capture_output=True, text=True, env=env, timeout=600)
        assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-2000:]
        assert "libcdgpu FGMRES ITE:" in p.stdout
        log = open(out).read()
        sol = np.fromfile(os.path.join(tmp, "sol.f64"), dtype=np.float64)
    # the reference's recorded output (ReadIn/cd2d.out:434-435), as the unchanged main writes it
    assert re.search(r"^L2: 4\.751079e-04$", log, re.M), re.findall(r"^L2: .*$", log, re.M)
    assert re.search(r"^H1-semi: 6\.295197e-02$", log, re.M), re.findall(r"^H1-semi: .*$", log, re.M)
    d = golden("cd2d_q1_sine_32")
    ref = d["solution"]
    assert len(sol) == len(ref)
    assert np.abs(sol - ref).max() <= 1e-9 * np.abs(ref).max()
