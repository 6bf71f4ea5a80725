#!/usr/bin/env python3
"""Regenerate the golden fixtures in tests/golden/ from the compiled reference.

Runs the reference dump drivers (oracle/_ref/cd2d_dump, cd3d_dump, built by
oracle/build_ref.py from the reference's own sources) on small unit-square /
unit-cube problems and stores everything they dump -- cell vertices, DOF maps,
CSR patterns, matrix entries, right-hand sides, parent maps, dense
prolongations, solutions, iteration counts and (sine problem) the L2 / H1-semi
errors -- as compressed .npz files, and the errors that the reference's unchanged
TCD3D program prints over a Crank-Nicolson run (tcd3d_amc_16.json).  Needs the
reference build; the tests only read the fixtures.

Usage: python tests/golden/make_golden.py [case names; default all]
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refdump  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
MESH = os.path.join(ROOT, "oracle", "meshes")

SOLVER_KEYS = """SOLVER_TYPE: 1
SC_SOLVER_SCALAR: 16
SC_PRECONDITIONER_SCALAR: 5
SC_SMOOTHER_SCALAR: 1
SC_SMOOTH_DAMP_FACTOR_SCALAR: 0.8
SC_SMOOTH_DAMP_FACTOR_FINE_SCALAR: 0.8
SC_PRE_SMOOTH_SCALAR: 2
SC_POST_SMOOTH_SCALAR: 2
SC_MG_CYCLE_SCALAR: 1
SC_STEP_LENGTH_CONTROL_ALL_SCALAR: 0
SC_STEP_LENGTH_CONTROL_FINE_SCALAR: 0
SC_GMRES_RESTART: 30
SC_LIN_RED_FACTOR_SCALAR: {red}
SC_LIN_RES_NORM_MIN_SCALAR: 0
SC_LIN_MAXIT_SCALAR: {maxit}
SC_VERBOSE: 0
"""

B3 = (0.5773502691896258,) * 3  # (1,1,1)/sqrt(3)

# name, dim, order, disctype, uniform steps, levels, example, eps, b, c, f, extra keys, mesh
# (mesh None: the unit square / unit cube).  skew_quad is one quadrilateral that is not a
# parallelogram and frustum one hexahedron that is not a parallelepiped, so every cell of
# their refinements takes the reference's bilinear / trilinear map (QuadBilinear,
# HexaTrilinear) instead of the affine one.
CASES = [
    ("cd3d_q1_gal_4", 3, 1, 1, 1, 2, 0, 1e-2, B3, 0.0, 1.0, "", None),
    ("cd3d_q2_gal_4", 3, 2, 1, 1, 2, 0, 1e-1, (0.2886751345948129,) * 3, 0.0, 1.0, "", None),
    ("cd3d_q1_gal_8", 3, 1, 1, 1, 3, 0, 1e-1, (1.0, 0.3, -0.2), 0.5, 1.0, "", None),
    ("cd2d_q1_sine_32", 2, 1, 1, 1, 5, 1, 0.0, (0.0, 0.0), 0.0, 0.0, "PE_NR: 10\n", None),
    ("cd2d_q1_supg_16", 2, 1, 2, 2, 3, 0, 1e-3, (1.0, 0.5), 0.0, 1.0, "", None),
    ("cd2d_q2_supg_8", 2, 2, 2, 1, 3, 0, 1e-3, (1.0, 0.5), 0.0, 1.0, "", None),
    ("cd2d_q2_gal_8", 2, 2, 1, 1, 3, 0, 1e-1, (-0.6, 0.8), 1.0, 1.0, "", None),
    # the coefficients of the CD3D Q2 32^3 benchmark (eps 1e-2, b = (1,1,1)/sqrt(3), f = 1)
    # on the 8^3 mesh with the same element; one level, because the reference's Galerkin
    # multigrid does not converge at this Peclet number (its FGMRES stalls at rate 1 with 2 or
    # 3 levels), while FGMRES preconditioned by its SSOR coarse-level loop alone converges
    ("cd3d_q2_gal_8_bench", 3, 2, 1, 3, 1, 0, 1e-2, B3, 0.0, 1.0, "", None),
    # non-affine cells
    ("cd2d_q1_skew_supg_16", 2, 1, 2, 2, 3, 0, 1e-3, (1.0, 0.5), 0.0, 1.0, "", "skew_quad"),
    ("cd2d_q2_skew_supg_8", 2, 2, 2, 1, 3, 0, 1e-2, (0.6, -0.8), 0.5, 1.0, "", "skew_quad"),
    ("cd2d_q2_skew_gal_8", 2, 2, 1, 1, 3, 0, 1e-1, (-0.6, 0.8), 1.0, 1.0, "", "skew_quad"),
    ("cd3d_q1_frustum_gal_8", 3, 1, 1, 1, 3, 0, 1e-1, (1.0, 0.3, -0.2), 0.5, 1.0, "", "frustum"),
    ("cd3d_q2_frustum_gal_4", 3, 2, 1, 1, 2, 0, 1e-1, (0.3, 0.2, -0.4), 0.5, 1.0, "", "frustum"),
]


def run_case(name, dim, order, disc, steps, levels, example, eps, b, c, f, extra, mesh, tmp):
    geo = mesh or ("unit_cube" if dim == 3 else "unit_square")
    dat = os.path.join(tmp, name + ".dat")
    with open(dat, "w") as fh:
        fh.write(f"VERSION: 1\nLOGFILE: logfile\nOUTFILE: {os.path.join(tmp, name + '.out')}\n"
                 f"BNDFILE: {MESH}/{geo}.PRM\nGEOFILE: {MESH}/{geo}.GEO\nMESH_TYPE: 0\n"
                 f"UNIFORM_STEPS: {steps}\nLEVELS: {levels}\nANSATZ_ORDER: {order}\n"
                 f"DISCTYPE: {disc}\n" + extra + SOLVER_KEYS.format(red=1e-12, maxit=30))
    out = os.path.join(tmp, name)
    os.makedirs(out, exist_ok=True)
    if dim == 3:
        cmd = [os.path.join(REF, "cd3d_dump"), dat, out, repr(eps), *map(repr, b), repr(c), repr(f),
               "2000000"]
    else:
        cmd = [os.path.join(REF, "cd2d_dump"), dat, out, str(example), repr(eps), *map(repr, b),
               repr(c), repr(f), "2000000"]
    subprocess.run(cmd, check=True, cwd=tmp, capture_output=True)
    d = refdump.load_dir(out)
    d.update(dim=dim, order=order, disctype=disc, example=example,
             eps=(0.1 if example == 1 else eps), b=np.array(b, float), c=c, f=f)
    for k in [k for k in d if k.startswith("t_")]:
        del d[k]
    # quality gate: the stored solution must be converged (the reference's FGMRES
    # measures its stopping test against the residual at the last restart, so a
    # run that restarts can chase an unreachable target; maxit = restart avoids it)
    L = refdump.level(d, levels - 1)
    import oracle
    r = L["rhs"] - oracle.spmv(L["row_ptr"], L["kcol"], L["entries"], d["solution"])
    d["solution_rel_residual"] = np.linalg.norm(r) / np.linalg.norm(L["rhs"])
    assert d["solution_rel_residual"] < 1e-10, (name, d["solution_rel_residual"])
    np.savez_compressed(os.path.join(HERE, name + ".npz"),
                        **{k: np.asarray(v) for k, v in d.items()})
    print(f"{name}: levels={d['levels']} n_dof={d[f'L{levels - 1}_n_dof']} its={d['iterations']}")


# The reference's own time-dependent program, unchanged: 3DPrograms/TCD3D_ParMooN.C with its
# example Examples/TCD_3D/amc.h, in the setting of ReadIn/tcd3d_GMG.out (Q1 on the unit cube
# refined 4 times, Crank-Nicolson, tau 0.1082532, end time 2, multigrid fixed point).
TCD3D_DAT = """VERSION: 1
LOGFILE: logfile
OUTFILE: {out}
BNDFILE: {mesh}/unit_cube.PRM
GEOFILE: {mesh}/unit_cube.GEO
MESH_TYPE: 0
ANSATZ_ORDER: 1
LEVELS: 1
UNIFORM_STEPS: 4
DISCTYPE: 1
SOLVER_TYPE: 1
SC_MG_TYPE_SCALAR: 1
SC_SOLVER_SCALAR: 11
SC_PRECONDITIONER_SCALAR: 5
SC_LIN_RED_FACTOR_SCALAR: 0.0
SC_LIN_RES_NORM_MIN_SCALAR: 1e-11
SC_LIN_MAXIT_SCALAR: 100
SC_MG_CYCLE_SCALAR: 1
SC_SMOOTHER_SCALAR: 2
SC_PRE_SMOOTH_SCALAR: 2
SC_POST_SMOOTH_SCALAR: 2
SC_COARSE_SMOOTHER_SCALAR: 3
SC_COARSE_MAXIT_SCALAR: 10
SC_COARSE_RED_FACTOR_SCALAR: 0.1
SC_STEP_LENGTH_CONTROL_FINE_SCALAR: 0
SC_STEP_LENGTH_CONTROL_ALL_SCALAR: 0
MEASURE_ERRORS: 1
WRITE_VTK: 0
WRITE_PS: 0
SC_VERBOSE: 0
TIME_DISC: 2
STARTTIME: 0
ENDTIME: 2
TIMESTEPLENGTH: 0.1082532
PE_NR: 1
RE_NR: 1
"""


def run_tcd3d_amc(tmp):
    """Run oracle/_ref/tcd3d_main (the reference's TCD3D main, unchanged) and keep what it
    prints after the initial interpolation and after every step: time, L2, H1-semi."""
    import json
    import re
    out = os.path.join(tmp, "tcd3d.out")
    dat = os.path.join(tmp, "tcd3d.dat")
    with open(dat, "w") as fh:
        fh.write(TCD3D_DAT.format(out=out, mesh=MESH))
    subprocess.run([os.path.join(REF, "tcd3d_main"), dat], check=True, cwd=tmp, capture_output=True)
    text = open(out).read()
    rows = re.findall(r"^time: (\S+)\nL2: (\S+)\nH1-semi: (\S+)$", text, re.M)
    its = [int(v) for v in re.findall(r"^ FP ITE:\s+(\d+)", text, re.M)]
    assert len(rows) == 20 and len(its) == 19, (len(rows), len(its))
    with open(os.path.join(HERE, "tcd3d_amc_16.json"), "w") as fh:
        json.dump({"program": "3DPrograms/TCD3D_ParMooN.C (Examples/TCD_3D/amc.h)",
                   "dat": TCD3D_DAT.format(out="tcd3d.out", mesh="oracle/meshes"),
                   "rows": [list(r) for r in rows], "fp_iterations": its}, fh, indent=1)
    print(f"tcd3d_amc_16: {len(rows)} error lines, last {rows[-1]}")


def main():
    only = set(sys.argv[1:])
    with tempfile.TemporaryDirectory() as tmp:
        for case in CASES:
            if not only or case[0] in only:
                run_case(*case, tmp)
        if not only or "tcd3d_amc_16" in only:
            run_tcd3d_amc(tmp)


if __name__ == "__main__":
    main()
