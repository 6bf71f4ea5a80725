"""cdgpu_defect_noalloc: the allocation-free defect, for callers that cannot call cudaMalloc.

Such callers (code running while another allocator already holds the device memory, or
code that must not trigger the device synchronisation of cudaFree) get the defect
d = f - A x and its norm without any device allocation: the partial sums live in a fixed
array inside the library.  This test calls the entry point through the C ABI twice in a
row and checks both calls against cdgpu_defect, the allocating entry point, within the
tolerance of the other defect tests.  It lives in a file of its own that pytest collects
last and also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

from parmoon_cmg_b200 import mesh
from parmoon_cmg_b200.system import Context, coeffs

pytestmark = pytest.mark.gpu

TOL = 1e-12


# 3D Q2 takes the 32-thread row groups; 2D Q1 and 3D Q1 the 16-thread ones, on more than 2048
# rows so that several blocks write partial sums
@pytest.mark.parametrize("dim,order,n", [(3, 2, 6), (2, 1, 64), (3, 1, 16)])
def test_defect_noalloc_matches_defect(dim, order, n):
    import torch
    from parmoon_cmg_b200 import _build
    _build.build()
    ctx = Context(0)
    try:
        sp = mesh.structured_space(dim, order, n)
        sid = ctx.upload_space(sp)
        nnz = ctx.build_pattern(sid)
        ctx.set_coeffs(sid, coeffs(0, eps=1e-2, b=(0.3, 0.2, 0.1)[:dim], c=0.5))
        ctx.assemble(sid, 1, sp["n_dof"], nnz, want_entries=False)
        rng = np.random.default_rng(7)
        for call in range(2):
            x = rng.standard_normal(sp["n_dof"])
            f = rng.standard_normal(sp["n_dof"])
            d_ref, res_ref = ctx.defect(sid, x, f)
            dx = torch.tensor(x, device="cuda:0")
            df = torch.tensor(f, device="cuda:0")
            dd = torch.full_like(dx, float("nan"))
            torch.cuda.synchronize()
            res = C.c_double(-1.0)
            st = ctx.lib.cdgpu_defect_noalloc(ctx.h, sid, dx.data_ptr(), df.data_ptr(), dd.data_ptr(),
                                              C.byref(res))
            ctx.check(st)
            torch.cuda.synchronize()
            d = dd.cpu().numpy()
            assert np.abs(d - d_ref).max() <= TOL * np.abs(d_ref).max(), call
            assert abs(res.value - res_ref) <= TOL * res_ref, call
    finally:
        ctx.close()
