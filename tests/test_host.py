"""CPU-side checks: the C ABI library loads and exports what include/cdgpu.h declares,
the ctypes structures match the C layout, and the host-side mesh / DOF-map
generation produces the reference's data layout."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

from parmoon_cmg_b200 import _build, _lib, mesh


@pytest.fixture(scope="module")
def lib():
    _build.build()
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    names = _lib.declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.SIGNATURES), "binding and header disagree"


def test_status_strings(lib):
    assert lib.cdgpu_status_string(0) == b"ok"
    assert lib.cdgpu_status_string(5) == b"solver diverged"


def test_struct_layout_matches_c():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "cdgpu.h"
int main(void) {
  printf("%zu %zu %zu\n", sizeof(cdgpu_coeffs), offsetof(cdgpu_coeffs, eps), offsetof(cdgpu_coeffs, delta0));
  printf("%zu %zu %zu\n", sizeof(cdgpu_solver_params), offsetof(cdgpu_solver_params, red_factor),
         offsetof(cdgpu_solver_params, gmg_damp));
  printf("%zu %zu\n", sizeof(cdgpu_solve_info), offsetof(cdgpu_solve_info, final_residual));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as t:
        c = os.path.join(t, "l.c")
        open(c, "w").write(src)
        exe = os.path.join(t, "l")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    a = list(map(int, out[0].split()))
    assert a == [C.sizeof(_lib.Coeffs), _lib.Coeffs.eps.offset, _lib.Coeffs.delta0.offset]
    b = list(map(int, out[1].split()))
    assert b == [C.sizeof(_lib.SolverParams), _lib.SolverParams.red_factor.offset,
                 _lib.SolverParams.gmg_damp.offset]
    c = list(map(int, out[2].split()))
    assert c == [C.sizeof(_lib.SolveInfo), _lib.SolveInfo.final_residual.offset]


def test_create_without_device_reports_no_device(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    assert lib.cdgpu_create(C.byref(h), 0) == _lib.ERR_NO_DEVICE


@pytest.mark.parametrize("dim,order,n", [(2, 1, 4), (2, 2, 4), (3, 1, 2), (3, 2, 2)])
def test_structured_space_layout(dim, order, n):
    sp = mesh.structured_space(dim, order, n)
    m = order * n + 1
    nbf = (order + 1) ** dim
    assert sp["n_dof"] == m ** dim
    assert sp["n_active"] == (m - 2) ** dim
    gn = sp["global_numbers"].reshape(-1, nbf)
    assert gn.shape[0] == n ** dim
    assert set(np.unique(gn)) == set(range(sp["n_dof"]))
    x = mesh.dof_coords(sp)
    bnd = np.any((x < 1e-12) | (x > 1 - 1e-12), axis=1)
    # [inner | Dirichlet] ordering with the whole boundary Dirichlet
    assert not bnd[:sp["n_active"]].any() and bnd[sp["n_active"]:].all()
    # counter-clockwise vertices: the local basis function 1 sits at vertex 1, function
    # (p+1) at vertex 3 (tensor order x fastest)
    v = sp["coords"].reshape(-1, 2 ** dim, dim)
    assert np.allclose(x[gn[:, order]], v[:, 1])
    assert np.allclose(x[gn[:, order * (order + 1)]], v[:, 3])


def test_parent_map_nests():
    for dim in (2, 3):
        c = mesh.structured_space(dim, 1, 2)
        f = mesh.structured_space(dim, 1, 4)
        par = mesh.parent_map(dim, 4)
        vc = c["coords"].reshape(-1, 2 ** dim, dim)
        vf = f["coords"].reshape(-1, 2 ** dim, dim)
        cen_f = vf.mean(1)
        lo, hi = vc.min(1), vc.max(1)
        assert np.all((cen_f > lo[par]) & (cen_f < hi[par]))


def test_oracle_pattern_on_structured_mesh(oracle_lib):
    sp = mesh.structured_space(3, 2, 2)
    rp, kc = oracle_lib.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
    lens = np.diff(rp)
    assert lens[:sp["n_active"]].max() == 125 and (lens[sp["n_active"]:] == 1).all()
    for r in range(sp["n_dof"]):
        assert np.all(np.diff(kc[rp[r]:rp[r + 1]]) > 0)
