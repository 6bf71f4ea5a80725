#!/usr/bin/env python3
"""Regenerate the golden fixtures in tests/golden/ from the compiled reference.

Runs the reference dump drivers (oracle/_ref/cd2d_dump, cd3d_dump, built by
oracle/build_ref.py from the reference's own sources) on small unit-square /
unit-cube problems and stores everything they dump -- cell vertices, DOF maps,
CSR patterns, matrix entries, right-hand sides, parent maps, dense
prolongations, solutions, iteration counts and (sine problem) the L2 / H1-semi
errors -- as compressed .npz files.  Needs the reference build; the tests only
read the .npz files.

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


def main():
    only = set(sys.argv[1:])
    with tempfile.TemporaryDirectory() as tmp:
        for case in CASES:
            if not only or case[0] in only:
                run_case(*case, tmp)


if __name__ == "__main__":
    main()
