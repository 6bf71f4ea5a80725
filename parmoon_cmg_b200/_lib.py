"""ctypes binding of libcdgpu.so (the C ABI declared in include/cdgpu.h).

The shared library is built in-tree by :mod:`parmoon_cmg_b200._build`; importing
this module never falls back to anything else: if the library is missing or a
call fails, an exception says so.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcdgpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "cdgpu.h")

GALERKIN, SUPG = 1, 2
COEFF_CONSTANT, COEFF_SINE, COEFF_ROTATING, COEFF_TABLE = 0, 1, 2, 3
OK, ERR_INVALID, ERR_OOM, ERR_CUDA, ERR_NOT_CONVERGED, ERR_DIVERGED, ERR_UNSUPPORTED, \
    ERR_PATTERN, ERR_NO_DEVICE = range(9)


class CdgpuError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"cdgpu status {status}: {msg}")
        self.status = status


class Coeffs(C.Structure):
    _fields_ = [("kind", C.c_int), ("poly_degree", C.c_int), ("eps", C.c_double),
                ("b1", C.c_double), ("b2", C.c_double), ("b3", C.c_double), ("c", C.c_double),
                ("f", C.c_double), ("delta0", C.c_double)]


class SolverParams(C.Structure):
    _fields_ = [("solver", C.c_int), ("restart", C.c_int), ("maxit", C.c_int),
                ("minit", C.c_int), ("smoother", C.c_int), ("coarse_smoother", C.c_int),
                ("pre", C.c_int), ("post", C.c_int), ("coarse_maxit", C.c_int),
                ("cycle", C.c_int), ("slc", C.c_int), ("precision", C.c_int),
                ("stop_rule", C.c_int), ("pad_", C.c_int), ("red_factor", C.c_double), ("res_norm_min", C.c_double),
                ("div_factor", C.c_double), ("omega", C.c_double), ("coarse_red", C.c_double),
                ("gmg_damp", C.c_double)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int),
                ("initial_residual", C.c_double), ("final_residual", C.c_double)]


_P = C.c_void_p
_I = C.c_int
# name -> (restype, argtypes); every function declared in include/cdgpu.h
SIGNATURES = {
    "cdgpu_create": (_I, [C.POINTER(C.c_void_p), _I]),
    "cdgpu_destroy": (None, [_P]),
    "cdgpu_status_string": (C.c_char_p, [_I]),
    "cdgpu_last_error": (C.c_char_p, [_P]),
    "cdgpu_stream": (C.c_ulonglong, [_P]),
    "cdgpu_kernel_launches": (C.c_longlong, [_P]),
    "cdgpu_upload_space": (_I, [_P, _I, _I, _I, _P, _P, _P, _I, _I, _I, C.POINTER(_I)]),
    "cdgpu_build_pattern": (_I, [_P, _I, C.POINTER(_I)]),
    "cdgpu_upload_pattern": (_I, [_P, _I, _P, _P, _I]),
    "cdgpu_build_pattern_device": (_I, [_P, _I, C.POINTER(_I)]),
    "cdgpu_get_pattern": (_I, [_P, _I, _P, _P]),
    "cdgpu_set_coeffs": (_I, [_P, _I, C.POINTER(Coeffs), _P]),
    "cdgpu_quadrature_points": (_I, [_P, _I, _P, C.POINTER(_I)]),
    "cdgpu_assemble": (_I, [_P, _I, _I, _P, _P, _P]),
    "cdgpu_add_neumann": (_I, [_P, _I, _I, _P, _P, _P, _P]),
    "cdgpu_boundary_points": (_I, [_P, _I, _I, _P, _P, _P]),
    "cdgpu_spmv": (_I, [_P, _I, _P, _P]),
    "cdgpu_defect": (_I, [_P, _I, _P, _P, _P, C.POINTER(C.c_double)]),
    "cdgpu_errors": (_I, [_P, _I, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "cdgpu_errors_table": (_I, [_P, _I, _P, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "cdgpu_write_vtk": (_I, [_P, _I, _P, _I, C.c_char_p, C.c_char_p]),
    "cdgpu_spmv_device": (_I, [_P, _I, _P, _P]),
    "cdgpu_apply_fp32": (_I, [_P, _I, _I, _P, _P]),
    "cdgpu_apply_fp64": (_I, [_P, _I, _I, _P, _P]),
    "cdgpu_apply_fp64_device": (_I, [_P, _I, _I, _P, _P]),
    "cdgpu_product_tuning": (_I, [_P, _I, C.c_char_p, _I]),
    "cdgpu_defect_noalloc": (_I, [_P, _I, _P, _P, _P, C.POINTER(C.c_double)]),
    "cdgpu_hierarchy": (_I, [_P, _I, _P, _P, C.POINTER(_I)]),
    "cdgpu_solve": (_I, [_P, _I, C.POINTER(SolverParams), _P, _P, C.POINTER(SolveInfo)]),
    "cdgpu_solve_device": (_I, [_P, _I, C.POINTER(SolverParams), _P, _P, C.POINTER(SolveInfo)]),
    "cdgpu_assemble_hierarchy": (_I, [_P, _I, _I, _I]),
    "cdgpu_get_rhs": (_I, [_P, _I, _P]),
    "cdgpu_rhs_device": (_I, [_P, _I, C.POINTER(C.c_void_p)]),
    "cdgpu_tcd_create": (_I, [_P, _I, _I, C.POINTER(_I)]),
    "cdgpu_tcd_assemble_mass": (_I, [_P, _I]),
    "cdgpu_tcd_assemble_stiffness": (_I, [_P, _I]),
    "cdgpu_tcd_step": (_I, [_P, _I, C.POINTER(SolverParams), C.c_double, C.c_double, C.c_double,
                            C.c_double, C.c_double, _P, C.POINTER(SolveInfo)]),
    "cdgpu_tcd_step_device": (_I, [_P, _I, C.POINTER(SolverParams), C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, _P, C.POINTER(SolveInfo)]),
    "cdgpu_tcd_rhs": (_I, [_P, _I, _P]),
    "cdgpu_tcd_set_dirichlet": (_I, [_P, _I, _P]),
    "cdgpu_tcd_matrices": (_I, [_P, _I, _I, _P, _P, _P]),
    "cdgpu_batch_create": (_I, [_P, C.POINTER(SolverParams), C.POINTER(_I)]),
    "cdgpu_batch_submit": (_I, [_P, _I, _I, C.POINTER(Coeffs), _I, _I, C.POINTER(_I)]),
    "cdgpu_batch_advance": (_I, [_P, _I, _I, C.POINTER(_I)]),
    "cdgpu_batch_submit_tcd": (_I, [_P, _I, _I, C.POINTER(Coeffs), _I, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, _P, C.POINTER(_I)]),
    "cdgpu_batch_tcd_step": (_I, [_P, _I, _I, C.POINTER(_I)]),
    "cdgpu_batch_tcd_solution": (_I, [_P, _I, _I, _P, C.POINTER(SolveInfo)]),
    "cdgpu_batch_poll": (_I, [_P, _I, _P, _I, C.POINTER(_I)]),
    "cdgpu_batch_fetch": (_I, [_P, _I, _I, _P, C.POINTER(SolveInfo)]),
    "cdgpu_batch_release": (_I, [_P, _I, _I]),
    "cdgpu_batch_memory": (_I, [_P, _I, C.POINTER(C.c_ulonglong)]),
    "cdgpu_batch_loop_info": (_I, [_P, _I, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "cdgpu_batch_instance_bytes": (_I, [_P, _I, _I, C.POINTER(C.c_ulonglong)]),
}

_lib = None


def load():
    """Load libcdgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with parmoon_cmg_b200._build.build()")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def declared_symbols():
    """Function names declared in include/cdgpu.h."""
    import re
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(cdgpu_\w+)\s*\(", txt)))
