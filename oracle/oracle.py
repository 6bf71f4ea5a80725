"""Python front of the CPU oracle (test infrastructure only).

Loads ``oracle/_build/libcdoracle.so`` (built from ``oracle/cdoracle.c`` by
:func:`build`) and exposes numpy-friendly wrappers.  Only the tests,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` use
this module, and only as the checker; the product library never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libcdoracle.so")

_lib = None


def build(force=False):
    """Compile the C restatement (gcc, -O2, no fast-math so the arithmetic stays IEEE)."""
    src = os.path.join(HERE, "cdoracle.c")
    os.makedirs(BUILD, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-D_GNU_SOURCE", src, "-o",
                    LIB, "-lm"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _declare(_lib)
    return _lib


class Coeffs(C.Structure):
    """Mirror of ``cdo_coeffs``: kind 0 constant, 1 sine problem, 2 rotating convection, 3 table."""
    _fields_ = [("kind", C.c_int), ("order_pd", C.c_int), ("eps", C.c_double),
                ("b1", C.c_double), ("b2", C.c_double), ("b3", C.c_double),
                ("c", C.c_double), ("f", C.c_double), ("delta0", C.c_double)]


class SolverParams(C.Structure):
    """Mirror of ``cdo_solver_params`` (names follow the reference's ParamDB keys)."""
    _fields_ = [("solver", C.c_int), ("restart", C.c_int), ("maxit", C.c_int),
                ("minit", C.c_int), ("smoother", C.c_int), ("coarse_smoother", C.c_int),
                ("pre", C.c_int), ("post", C.c_int), ("coarse_maxit", C.c_int),
                ("cycle", C.c_int), ("slc", C.c_int), ("slc_fine", C.c_int),
                ("red_factor", C.c_double), ("res_norm_min", C.c_double),
                ("div_factor", C.c_double), ("omega", C.c_double), ("coarse_red", C.c_double),
                ("gmg_damp", C.c_double)]


def solver_params(**kw):
    """Defaults = the configuration used by the multigrid configs (FGMRES(30), V(2,2) damped
    Jacobi omega 0.8, SSOR coarse smoother as ParMooN's default, no step-length control)."""
    d = dict(solver=16, restart=30, maxit=1000, minit=0, smoother=1, coarse_smoother=3, pre=2,
             post=2, coarse_maxit=10, cycle=1, slc=0, slc_fine=0, red_factor=1e-10,
             res_norm_min=0.0, div_factor=1e10, omega=0.8, coarse_red=0.1, gmg_damp=1.0)
    d.update(kw)
    return SolverParams(**d)


def coeffs(kind=0, eps=1.0, b=(0.0, 0.0, 0.0), c=0.0, f=1.0, delta0=1.0, order_pd=1):
    b = tuple(b) + (0.0,) * (3 - len(b))
    return Coeffs(kind=kind, order_pd=order_pd, eps=eps, b1=b[0], b2=b[1], b3=b[2], c=c, f=f,
                  delta0=delta0)


_P = C.c_void_p


def _declare(L):
    L.cdo_nbf.restype = C.c_int
    L.cdo_gauss_points.restype = C.c_int
    L.cdo_quadrature.restype = C.c_int
    L.cdo_pattern.restype = C.c_long
    L.cdo_pattern.argtypes = [C.c_int, _P, _P, C.c_int, C.c_int, _P, _P]
    L.cdo_assemble.restype = C.c_int
    L.cdo_assemble.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, C.c_int, C.c_int,
                               _P, _P, C.POINTER(Coeffs), _P, _P, _P, _P]
    L.cdo_neumann_sine.argtypes = [C.c_int, C.c_int, _P, _P, _P, C.c_int, C.c_double, _P]
    L.cdo_errors_sine.argtypes = [C.c_int, C.c_int, _P, _P, _P, _P, _P]
    L.cdo_errors_sinsin.argtypes = [C.c_int, C.c_int, _P, _P, _P, _P, C.c_double, C.c_double, _P]
    L.cdo_errors_table.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P]
    L.cdo_quad_points.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P]
    L.cdo_dof_coords.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, _P, C.c_int, _P]
    L.cdo_prolongation.restype = C.c_long
    L.cdo_prolongation.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, _P, C.c_int, C.c_int, _P,
                                   _P, _P, C.c_int, _P, _P, _P, _P]
    L.cdo_spmv.argtypes = [C.c_int, _P, _P, _P, _P, _P]
    L.cdo_solve.restype = C.c_int
    L.cdo_solve.argtypes = [C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, C.POINTER(SolverParams),
                            _P, _P, _P, _P]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def pattern(gn, bi, n_dof, n_active):
    gn, bi = _i32(gn), _i32(bi)
    n_cells = len(bi) - 1
    rp = np.zeros(n_dof + 1, np.int32)
    nnz = lib().cdo_pattern(n_cells, _p(gn), _p(bi), n_dof, n_active, _p(rp), None)
    kc = np.zeros(nnz, np.int32)
    lib().cdo_pattern(n_cells, _p(gn), _p(bi), n_dof, n_active, _p(rp), _p(kc))
    return rp, kc


def assemble(dim, order, disctype, coords, gn, bi, n_dof, n_active, row_ptr, kcol, co,
             coeff_tab=None, dir_vals=None):
    coords, gn, bi = _f64(coords), _i32(gn), _i32(bi)
    row_ptr, kcol = _i32(row_ptr), _i32(kcol)
    ent = np.zeros(int(row_ptr[-1]), np.float64)
    rhs = np.zeros(n_dof, np.float64)
    tab = _f64(coeff_tab) if coeff_tab is not None else None
    dv = _f64(dir_vals) if dir_vals is not None else None
    rc = lib().cdo_assemble(dim, order, disctype, len(bi) - 1, _p(coords), _p(gn), _p(bi), n_dof,
                            n_active, _p(row_ptr), _p(kcol), C.byref(co), _p(tab), _p(dv),
                            _p(ent), _p(rhs))
    if rc != 0:
        raise RuntimeError("oracle assembly: cell coupling missing from the pattern")
    return ent, rhs


def neumann_sine(order, coords, gn, bi, n_active, eps, rhs):
    coords, gn, bi = _f64(coords), _i32(gn), _i32(bi)
    lib().cdo_neumann_sine(order, len(bi) - 1, _p(coords), _p(gn), _p(bi), n_active, eps, _p(rhs))


def errors_sine(order, coords, gn, bi, u):
    coords, gn, bi, u = _f64(coords), _i32(gn), _i32(bi), _f64(u)
    out = np.zeros(2)
    lib().cdo_errors_sine(order, len(bi) - 1, _p(coords), _p(gn), _p(bi), _p(u), _p(out))
    return out


def errors_sinsin(order, coords, gn, bi, u, k, amp):
    """L2 and H1-semi errors of a 2D solution against amp*sin(k pi x)*sin(k pi y)."""
    coords, gn, bi, u = _f64(coords), _i32(gn), _i32(bi), _f64(u)
    out = np.zeros(2)
    lib().cdo_errors_sinsin(order, len(bi) - 1, _p(coords), _p(gn), _p(bi), _p(u), k, amp, _p(out))
    return out


def errors_table(dim, order, coords, gn, bi, u, exact):
    """L2 and H1-semi errors against an exact solution tabulated at the quadrature points
    (n_cells x n_quad x (1 + dim): value, gradient), TFEFunction3D::GetErrors."""
    coords, gn, bi, u, exact = _f64(coords), _i32(gn), _i32(bi), _f64(u), _f64(exact)
    out = np.zeros(2)
    lib().cdo_errors_table(dim, order, len(bi) - 1, _p(coords), _p(gn), _p(bi), _p(u), _p(exact), _p(out))
    return out


def quad_points(dim, order, coords, n_cells):
    """Physical quadrature points (n_cells x n_quad x dim) in the oracle's table order."""
    coords = _f64(coords)
    nq = cdo_nq(dim, order)
    out = np.zeros((n_cells, nq, dim))
    lib().cdo_quad_points(dim, order, n_cells, _p(coords), _p(out))
    return out


def cdo_nq(dim, order):
    n1 = 3 if order == 1 else 4
    return n1 ** dim


def dof_coords(dim, order, coords, gn, bi, n_dof):
    coords, gn, bi = _f64(coords), _i32(gn), _i32(bi)
    out = np.zeros((n_dof, dim))
    lib().cdo_dof_coords(dim, order, len(bi) - 1, _p(coords), _p(gn), _p(bi), n_dof, _p(out))
    return out


def prolongation(dim, order, coarse, fine, parent):
    """coarse/fine: dicts with coords, global_numbers, begin_index, n_dof."""
    cc, cg, cb = _f64(coarse["coords"]), _i32(coarse["global_numbers"]), _i32(coarse["begin_index"])
    fc, fg, fb = _f64(fine["coords"]), _i32(fine["global_numbers"]), _i32(fine["begin_index"])
    parent = _i32(parent)
    nf = int(fine["n_dof"])
    rp = np.zeros(nf + 1, np.int32)
    args = [dim, order, len(cb) - 1, _p(cc), _p(cg), _p(cb), int(coarse["n_dof"]), len(fb) - 1,
            _p(fc), _p(fg), _p(fb), nf, _p(parent), _p(rp)]
    nnz = lib().cdo_prolongation(*args, None, None)
    col = np.zeros(nnz, np.int32)
    val = np.zeros(nnz, np.float64)
    lib().cdo_prolongation(*args, _p(col), _p(val))
    return rp, col, val


def spmv(row_ptr, kcol, a, x):
    row_ptr, kcol, a, x = _i32(row_ptr), _i32(kcol), _f64(a), _f64(x)
    y = np.zeros(len(row_ptr) - 1)
    lib().cdo_spmv(len(row_ptr) - 1, _p(row_ptr), _p(kcol), _p(a), _p(x), _p(y))
    return y


def solve(levels, prm, rhs, sol0):
    """levels: list (coarsest first) of dicts with n_dof, n_active, row_ptr, kcol, entries and,
    for all but the first, p_row/p_col/p_val.  Returns (sol, iterations, residual history,
    final residual)."""
    L = len(levels)
    keep = []

    def arr(vals, ctype):
        a = (ctype * L)(*vals)
        keep.append(a)
        return C.cast(a, C.c_void_p)

    ptrs = {}
    for key, conv in [("row_ptr", _i32), ("kcol", _i32), ("entries", _f64), ("p_row", _i32),
                      ("p_col", _i32), ("p_val", _f64)]:
        vals = []
        for lv in levels:
            if key in lv and lv[key] is not None:
                a = conv(lv[key])
                keep.append(a)
                vals.append(a.ctypes.data)
            else:
                vals.append(None)
        ptrs[key] = arr(vals, C.c_void_p)
    n = np.array([lv["n_dof"] for lv in levels], np.int32)
    na = np.array([lv["n_active"] for lv in levels], np.int32)
    sol = _f64(sol0).copy()
    rhs = _f64(rhs)
    hist = np.zeros(prm.maxit + 2)
    fres = C.c_double(0)
    its = lib().cdo_solve(L, _p(n), _p(na), ptrs["row_ptr"], ptrs["kcol"], ptrs["entries"],
                          ptrs["p_row"], ptrs["p_col"], ptrs["p_val"], C.byref(prm), _p(rhs),
                          _p(sol), _p(hist), C.byref(fres))
    return sol, its, hist[:max(its, 0) + 1], fres.value


def tcd_step(levels, M, A, f_old, f, sol, tau, th1, th2, th3, th4, prm, fine_only_theta2=False):
    """One theta-scheme step of TSystemTCD2D on the oracle's CSR levels.

    levels: as for :func:`solve` (their ``entries`` are replaced by the system matrices);
    M, A: per-level mass and stiffness entries (M is updated in place like the
    reference's sqmatrixM and restored at the end).  Follows
    src/System/SystemTCD2D.C:231-277 (AssembleSystMat), 323-330 (Solve with GMG) and
    279-305 (RestoreMassMat): MatAdd acts on the active rows only (Blas2.C MatAdd),
    B = tau*th3*f_old + tau*th4*f + M_active u_old, Dirichlet entries of B and u from f.
    fine_only_theta2: the order of TSystemTCD3D (src/System/SystemTCD3D.C:257-278), where
    M - tau*th2*A is formed on the finest level only and the coarser levels' system matrices
    are M + tau*th1*A.  Returns (new solution, iterations)."""
    fine = levels[-1]
    na = int(fine["n_active"])
    L = len(levels)
    for l, (lv, m, a) in enumerate(zip(levels, M, A)):
        if fine_only_theta2 and l < L - 1:
            continue
        k = int(lv["row_ptr"][lv["n_active"]])
        m[:k] += (-tau * th2) * a[:k]
    B = np.zeros(len(f))
    B[:na] += tau * th3 * f_old[:na]
    B[:na] += tau * th4 * f[:na]
    Mu = spmv(fine["row_ptr"], fine["kcol"], M[-1], sol)
    B[:na] += Mu[:na]
    B[na:] = f[na:]
    u = _f64(sol).copy()
    u[na:] = f[na:]
    gamma = -tau * th2
    sys_levels = []
    for l, (lv, m, a) in enumerate(zip(levels, M, A)):
        k = int(lv["row_ptr"][lv["n_active"]])
        m[:k] += (tau * th1 if fine_only_theta2 and l < L - 1 else -gamma + tau * th1) * a[:k]
        d = dict(lv)
        d["entries"] = m.copy()
        sys_levels.append(d)
    u, its, _, _ = solve(sys_levels, prm, B, u)
    for lv, m, a in zip(levels, M, A):
        k = int(lv["row_ptr"][lv["n_active"]])
        m[:k] += (-tau * th1) * a[:k]
    return u, its
