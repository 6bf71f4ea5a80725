"""Host-side mirror of ParMooN's convection-diffusion facade over libcdgpu.

``TSystemCD3D`` and ``TSystemCD2D`` keep the reference's call surface
(src/System/SystemCD3D.C:36-396, src/System/SystemCD2D.C:39-205):
construct with the FE spaces of all multigrid levels, ``Init`` with the
coefficients and boundary data, ``Assemble``, ``Solve(sol, rhs)``.  All work
runs in libcdgpu through its C ABI; this module only marshals numpy arrays.
Errors raise :class:`CdgpuError` where the reference prints a message and
calls ``exit(4711)``.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import CdgpuError, Coeffs, SolveInfo, SolverParams

GALERKIN, SUPG = _lib.GALERKIN, _lib.SUPG
GMG = 1  # SOLVER_TYPE, 3DPrograms/CD3D_ParMooN.C:33


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _is_f64_out(a, n):
    """a can receive n float64 values in place (a writable C-contiguous float64 ndarray)"""
    return (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and
            a.flags.writeable and a.size == n)


class Context:
    """One libcdgpu context (device + CUDA stream)."""

    def __init__(self, device=0):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.cdgpu_create(C.byref(h), device)
        if st != 0:
            raise CdgpuError(st, self.lib.cdgpu_status_string(st).decode())
        self.h = h

    def check(self, st):
        if st != 0:
            msg = self.lib.cdgpu_last_error(self.h).decode()
            raise CdgpuError(st, f"{self.lib.cdgpu_status_string(st).decode()}: {msg}")

    @property
    def stream(self):
        return int(self.lib.cdgpu_stream(self.h))

    @property
    def kernel_launches(self):
        return int(self.lib.cdgpu_kernel_launches(self.h))

    def close(self):
        if self.h:
            self.lib.cdgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- thin wrappers of the C ABI -------------------------------------
    def upload_space(self, sp):
        sid = C.c_int()
        coords, gn, bi = _f64(sp["coords"]), _i32(sp["global_numbers"]), _i32(sp["begin_index"])
        self.check(self.lib.cdgpu_upload_space(
            self.h, sp["dim"], sp["order"], len(bi) - 1, _p(coords), _p(gn), _p(bi),
            int(sp["n_dof"]), int(sp["n_active"]), int(sp.get("hanging_bound", sp["n_active"])),
            C.byref(sid)))
        return sid.value

    def build_pattern(self, sid):
        nnz = C.c_int()
        self.check(self.lib.cdgpu_build_pattern(self.h, sid, C.byref(nnz)))
        return nnz.value

    def build_pattern_device(self, sid):
        """The CSR pattern built on the device (bit-identical to build_pattern)."""
        nnz = C.c_int()
        self.check(self.lib.cdgpu_build_pattern_device(self.h, sid, C.byref(nnz)))
        return nnz.value

    def upload_pattern(self, sid, row_ptr, kcol):
        row_ptr, kcol = _i32(row_ptr), _i32(kcol)
        self.check(self.lib.cdgpu_upload_pattern(self.h, sid, _p(row_ptr), _p(kcol), len(kcol)))

    def get_pattern(self, sid, n_dof, nnz):
        rp = np.zeros(n_dof + 1, np.int32)
        kc = np.zeros(nnz, np.int32)
        self.check(self.lib.cdgpu_get_pattern(self.h, sid, _p(rp), _p(kc)))
        return rp, kc

    def set_coeffs(self, sid, coeffs, table=None):
        tab = _f64(table) if table is not None else None
        self.check(self.lib.cdgpu_set_coeffs(self.h, sid, C.byref(coeffs), _p(tab)))

    def quadrature_points(self, sid, n_cells, dim):
        nq = C.c_int()
        self.check(self.lib.cdgpu_quadrature_points(self.h, sid, None, C.byref(nq)))
        out = np.zeros((n_cells, nq.value, dim))
        self.check(self.lib.cdgpu_quadrature_points(self.h, sid, _p(out), C.byref(nq)))
        return out

    def assemble(self, sid, disctype, n_dof, nnz, dirichlet=None, want_entries=True, want_rhs=True):
        ent = np.zeros(nnz) if want_entries else None
        rhs = np.zeros(n_dof) if want_rhs else None
        d = _f64(dirichlet) if dirichlet is not None else None
        self.check(self.lib.cdgpu_assemble(self.h, sid, disctype, _p(d), _p(ent), _p(rhs)))
        return ent, rhs

    def errors(self, sid, sol):
        """(L2, H1-semi) errors of ``sol`` against the SineLaplace solution, on the device."""
        l2, h1 = C.c_double(), C.c_double()
        self.check(self.lib.cdgpu_errors(self.h, sid, _p(_f64(sol)), C.byref(l2), C.byref(h1)))
        return l2.value, h1.value

    def errors_table(self, sid, sol, exact):
        """(L2, H1-semi) errors of ``sol`` against an exact solution tabulated at the
        quadrature points: exact[cell, q] = (u, du/dx, du/dy[, du/dz]), on the device."""
        l2, h1 = C.c_double(), C.c_double()
        self.check(self.lib.cdgpu_errors_table(self.h, sid, _p(_f64(sol)), _p(_f64(exact)), C.byref(l2),
                                               C.byref(h1)))
        return l2.value, h1.value

    def write_vtk(self, sid, sol, path, name="u", on_device=False):
        """Legacy VTK file of a solution (host array, or a device pointer with on_device)."""
        ptr = C.c_void_p(sol) if on_device else _p(_f64(sol))
        self.check(self.lib.cdgpu_write_vtk(self.h, sid, ptr, 1 if on_device else 0, path.encode(), name.encode()))

    def add_neumann(self, sid, cells, edges, g, n_dof=None):
        """Add Neumann data; returns the updated right-hand side when n_dof is given."""
        cells, edges, g = _i32(cells), _i32(edges), _f64(g)
        rhs = np.zeros(n_dof) if n_dof is not None else None
        self.check(self.lib.cdgpu_add_neumann(self.h, sid, len(cells), _p(cells), _p(edges), _p(g),
                                              _p(rhs)))
        return rhs

    def spmv(self, sid, x):
        x = _f64(x)
        y = np.zeros_like(x)
        self.check(self.lib.cdgpu_spmv(self.h, sid, _p(x), _p(y)))
        return y

    def product_tuning(self, sid):
        """The tile-shape choice of the FP64 product of a space's matrix, as text."""
        buf = C.create_string_buffer(1024)
        self.check(self.lib.cdgpu_product_tuning(self.h, sid, buf, 1024))
        return buf.value.decode()

    def apply_fp32(self, sid, x, form):
        """y = A x with an FP32 form of the operator: 0 CSR copy, 1 matrix-free on CUDA cores,
        2 matrix-free on the tensor cores."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros_like(x)
        self.check(self.lib.cdgpu_apply_fp32(self.h, sid, form, _p(x), _p(y)))
        return y

    def apply_fp64(self, sid, x, form):
        """y = A x with an FP64 form of the operator: 0 the CSR entries, 1 matrix-free (sum
        factorisation, the mixed solve's FGMRES product)."""
        x = _f64(x)
        y = np.zeros_like(x)
        self.check(self.lib.cdgpu_apply_fp64(self.h, sid, form, _p(x), _p(y)))
        return y

    def defect(self, sid, x, f):
        x, f = _f64(x), _f64(f)
        d = np.zeros_like(x)
        res = C.c_double()
        self.check(self.lib.cdgpu_defect(self.h, sid, _p(x), _p(f), _p(d), C.byref(res)))
        return d, res.value

    def hierarchy(self, sids, parents):
        L = len(sids)
        ids = (C.c_int * L)(*sids)
        keep = [_i32(p) if p is not None else None for p in parents]
        ptrs = (C.c_void_p * L)(*[(a.ctypes.data if a is not None else None) for a in keep])
        mg = C.c_int()
        self.check(self.lib.cdgpu_hierarchy(self.h, L, C.cast(ids, C.c_void_p),
                                            C.cast(ptrs, C.c_void_p), C.byref(mg)))
        return mg.value

    def assemble_hierarchy(self, mg, disctype, coarse_disctype=None):
        cd = disctype if coarse_disctype is None else coarse_disctype
        self.check(self.lib.cdgpu_assemble_hierarchy(self.h, mg, disctype, cd))

    def solve(self, mg, params, rhs, sol):
        rhs = _f64(rhs)
        sol = _f64(sol).copy()
        info = SolveInfo()
        self.check(self.lib.cdgpu_solve(self.h, mg, C.byref(params), _p(rhs), _p(sol), C.byref(info)))
        return sol, info

    def solve_device(self, mg, params, d_rhs, d_sol):
        info = SolveInfo()
        self.check(self.lib.cdgpu_solve_device(self.h, mg, C.byref(params), C.c_void_p(d_rhs),
                                               C.c_void_p(d_sol), C.byref(info)))
        return info

    def rhs_device(self, sid):
        p = C.c_void_p()
        self.check(self.lib.cdgpu_rhs_device(self.h, sid, C.byref(p)))
        return p.value


def coeffs(kind=_lib.COEFF_CONSTANT, eps=1.0, b=(0.0, 0.0, 0.0), c=0.0, f=1.0, delta0=1.0,
           poly_degree=1):
    b = tuple(b) + (0.0,) * (3 - len(b))
    return Coeffs(kind=kind, poly_degree=poly_degree, eps=eps, b1=b[0], b2=b[1], b3=b[2], c=c,
                  f=f, delta0=delta0)


def solver_params(**kw):
    """ParamDB-style solver settings; defaults are the multigrid configs' (FGMRES(30),
    V(2,2) damped Jacobi with omega 0.8, relative residual 1e-10, FP64 everywhere) with the
    exact FP64 coarse solve."""
    d = dict(solver=16, restart=30, maxit=1000, minit=0, smoother=1, coarse_smoother=17, pre=2,
             post=2, coarse_maxit=10, cycle=1, slc=0, precision=0, stop_rule=0, red_factor=1e-10,
             res_norm_min=0.0, div_factor=1e10, omega=0.8, coarse_red=0.1, gmg_damp=1.0)
    d.update(kw)
    return SolverParams(**d)


class TSystemCD3D:
    """Mirror of TSystemCD3D (include/System/SystemCD3D.h:97-110) on the GPU.

    fespaces: spaces of all multigrid levels, coarsest first (dicts as produced by
    :func:`parmoon_cmg_b200.mesh.structured_space` or by the reference's TFESpace3D);
    parents[l]: parent cell map of level l (index 0 unused)."""

    dim = 3

    def __init__(self, fespaces, parents, disctype=GALERKIN, solver=GMG, ctx=None, pattern=None,
                 coarse_disctype=None):
        if solver != GMG:
            raise CdgpuError(_lib.ERR_UNSUPPORTED, "only the GMG solver type runs on the GPU")
        self.ctx = ctx or Context()
        self.spaces = fespaces
        self.disctype = disctype
        # discretisation of the coarse multigrid levels (the reference uses disctype everywhere)
        self.coarse_disctype = disctype if coarse_disctype is None else coarse_disctype
        self.sids = [self.ctx.upload_space(s) for s in fespaces]
        self.nnz = []
        for i, sid in enumerate(self.sids):
            if pattern is not None and pattern[i] is not None:
                self.ctx.upload_pattern(sid, *pattern[i])
                self.nnz.append(len(pattern[i][1]))
            else:
                self.nnz.append(self.ctx.build_pattern(sid))
        self.mg = self.ctx.hierarchy(self.sids, parents)
        self.N_DOF = int(fespaces[-1]["n_dof"])
        self.N_Active = int(fespaces[-1]["n_active"])

    def Init(self, coeff, table=None):
        for i, sid in enumerate(self.sids):
            self.ctx.set_coeffs(sid, coeff, table[i] if table is not None else None)

    def Assemble(self, sol=None, rhs=None, dirichlet=None, entries=False):
        """Assemble all levels (SystemCD3D.C:314-339); returns the finest (entries, rhs) and
        copies the Dirichlet part of rhs into sol like SystemCD3D.C:330."""
        if dirichlet is None and not entries:
            # every level in one call; the finest rhs is copied straight into ``rhs`` when it
            # is a contiguous float64 array
            self.ctx.assemble_hierarchy(self.mg, self.disctype, self.coarse_disctype)
            r = rhs if _is_f64_out(rhs, self.N_DOF) else np.zeros(self.N_DOF)
            self.ctx.check(self.ctx.lib.cdgpu_get_rhs(self.ctx.h, self.sids[-1], _p(r)))
            if rhs is not None and r is not rhs:
                rhs[:] = r
            if sol is not None:
                sol[self.N_Active:] = r[self.N_Active:]
            return None, r
        out = None
        for i, sid in enumerate(self.sids):
            sp = self.spaces[i]
            last = i == len(self.sids) - 1
            d = dirichlet if last else None
            disc = self.disctype if last else self.coarse_disctype
            ent, r = self.ctx.assemble(sid, disc, int(sp["n_dof"]), self.nnz[i], d,
                                       want_entries=entries and last, want_rhs=last)
            if last:
                out = (ent, r)
        if rhs is not None:
            rhs[:] = out[1]
        if sol is not None:
            sol[self.N_Active:] = out[1][self.N_Active:]
        return out

    def Solve(self, sol, rhs, params=None):
        """FGMRES / fixed point with one multigrid cycle as preconditioner (SystemCD3D.C:342-368)."""
        params = params or solver_params()
        if _is_f64_out(sol, self.N_DOF):
            # the library reads the initial guess from and writes the solution into ``sol``
            info = SolveInfo()
            self.ctx.check(self.ctx.lib.cdgpu_solve(self.ctx.h, self.mg, C.byref(params), _p(_f64(rhs)),
                                                    _p(sol), C.byref(info)))
        else:
            x, info = self.ctx.solve(self.mg, params, rhs, sol)
            sol[:] = x
        if info.status == _lib.ERR_DIVERGED:
            raise CdgpuError(info.status, "fgmres iteration diverges")
        return info


class TSystemTCD2D:
    """Mirror of TSystemTCD2D (src/System/SystemTCD2D.C) for theta schemes on the GPU.

    The time loop of 2DPrograms/TCD2D_ParMooN.C:241-290 becomes::

        S = TSystemTCD2D(spaces, parents); S.Init(coeffs(...))
        S.AssembleMRhs(sol)                   # mass matrices, initial rhs
        for step: S.AssembleARhs()            # stiffness + rhs at the new time (saves the old rhs)
                  S.Step(sol, tau, theta...)  # AssembleSystMat + Solve + RestoreMassMat
    """

    def __init__(self, fespaces, parents, disctype=GALERKIN, ctx=None):
        self.ctx = ctx or Context()
        self.spaces = fespaces
        self.sids = [self.ctx.upload_space(s) for s in fespaces]
        for sid in self.sids:
            self.ctx.build_pattern(sid)
        self.mg = self.ctx.hierarchy(self.sids, parents)
        tid = C.c_int()
        self.ctx.check(self.ctx.lib.cdgpu_tcd_create(self.ctx.h, self.mg, disctype, C.byref(tid)))
        self.tcd = tid.value
        self.N_DOF = int(fespaces[-1]["n_dof"])
        self.N_Active = int(fespaces[-1]["n_active"])

    def Init(self, coeff):
        for sid in self.sids:
            self.ctx.set_coeffs(sid, coeff)

    def rhs(self):
        r = np.zeros(self.N_DOF)
        self.ctx.check(self.ctx.lib.cdgpu_tcd_rhs(self.ctx.h, self.tcd, _p(r)))
        return r

    def matrices(self, level, nnz):
        """(M, A, S) of a level (0 = coarsest): the mass matrix as updated in place, the
        stiffness matrix and the system matrix of the last step."""
        out = [np.zeros(nnz) for _ in range(3)]
        self.ctx.check(self.ctx.lib.cdgpu_tcd_matrices(self.ctx.h, self.tcd, level, *[_p(a) for a in out]))
        return tuple(out)

    def SetDirichlet(self, values=None):
        """BoundValue at the finest level's Dirichlet DOFs (N_DOF - N_Active values) for the
        next assemblies, at the time they are assembled for; None = zero values."""
        if values is None:
            self.ctx.check(self.ctx.lib.cdgpu_tcd_set_dirichlet(self.ctx.h, self.tcd, None))
            return
        v = _f64(values)
        assert len(v) == self.N_DOF - self.N_Active
        self.ctx.check(self.ctx.lib.cdgpu_tcd_set_dirichlet(self.ctx.h, self.tcd, _p(v)))

    def AssembleMRhs(self, sol=None):
        self.ctx.check(self.ctx.lib.cdgpu_tcd_assemble_mass(self.ctx.h, self.tcd))
        if sol is not None:
            sol[self.N_Active:] = self.rhs()[self.N_Active:]

    def AssembleARhs(self):
        self.ctx.check(self.ctx.lib.cdgpu_tcd_assemble_stiffness(self.ctx.h, self.tcd))

    def Step(self, sol, tau, theta1, theta2, theta3, theta4, params=None):
        params = params or solver_params()
        info = SolveInfo()
        x = _f64(sol).copy()
        self.ctx.check(self.ctx.lib.cdgpu_tcd_step(self.ctx.h, self.tcd, C.byref(params), tau, theta1,
                                                   theta2, theta3, theta4, _p(x), C.byref(info)))
        sol[:] = x
        return info


class TSystemTCD3D(TSystemTCD2D):
    """Mirror of TSystemTCD3D (src/System/SystemTCD3D.C:176-330) for theta schemes on the GPU,
    driven like 3DPrograms/TCD3D_ParMooN.C: AssembleMRhs, then per step the old right-hand
    side saved, AssembleARhs, AssembleSystMat + Solve + RestoreMassMat (``Step``).  The device
    path is the 2D one; for a 3D hierarchy it follows the 3D reference's order of the matrix
    updates: M - tau*theta2*A on the finest level only, the coarser levels' system matrices
    M + tau*theta1*A (SystemTCD3D.C:257-278)."""


class TSystemCD2D(TSystemCD3D):
    """2D counterpart.  The reference's TSystemCD2D takes one space and has no multigrid
    branch (src/System/SystemCD2D.C:191-193); here it takes every level's space and
    solves with the same multigrid-preconditioned FGMRES as the 3D system."""

    dim = 2


class Batch:
    """Many independent GMG-FGMRES solves advanced together on one GPU (cdgpu_batch_*).

    ``add_structure`` registers a mesh hierarchy once (pattern, transfers, colour classes);
    ``submit`` adds an instance on a structure with its own coefficients (assembled on
    submission); ``advance`` runs FGMRES iterations of every running instance in grouped
    launches; ``poll`` returns the instances that finished; ``fetch`` reads a solution;
    ``release`` frees an instance's device memory.  The multigrid cycle runs in FP32
    inside FP64 FGMRES with the exact FP64 coarse solve."""

    def __init__(self, params, ctx=None):
        self.ctx = ctx or Context()
        bid = C.c_int()
        self.ctx.check(self.ctx.lib.cdgpu_batch_create(self.ctx.h, C.byref(params), C.byref(bid)))
        self.id = bid.value
        self.structures = []

    def add_structure(self, spaces, parents):
        """Upload a hierarchy (spaces coarsest first); returns its structure id."""
        sids = [self.ctx.upload_space(s) for s in spaces]
        # the patterns of a new mesh are built on the device (bit-identical to the host build)
        nnz = [self.ctx.build_pattern_device(sid) for sid in sids]
        mg = self.ctx.hierarchy(sids, parents)
        self.structures.append(dict(mg=mg, n_dof=int(spaces[-1]["n_dof"]), sids=sids, nnz=nnz))
        return len(self.structures) - 1

    def instance_bytes(self, structure):
        out = C.c_ulonglong()
        self.ctx.check(self.ctx.lib.cdgpu_batch_instance_bytes(self.ctx.h, self.id,
                                                               self.structures[structure]["mg"],
                                                               C.byref(out)))
        return out.value

    def submit(self, structure, coeff, disctype=SUPG, coarse_disctype=None):
        slot = C.c_int()
        st = self.structures[structure]
        cd = disctype if coarse_disctype is None else coarse_disctype
        self.ctx.check(self.ctx.lib.cdgpu_batch_submit(self.ctx.h, self.id, st["mg"], C.byref(coeff),
                                                       disctype, cd, C.byref(slot)))
        return slot.value

    def submit_tcd(self, structure, coeff, tau, theta1, theta2, theta3, theta4, u0, disctype=GALERKIN):
        """A time-dependent instance (theta scheme) with initial solution u0."""
        slot = C.c_int()
        st = self.structures[structure]
        u0 = _f64(u0)
        self.ctx.check(self.ctx.lib.cdgpu_batch_submit_tcd(self.ctx.h, self.id, st["mg"], C.byref(coeff), disctype,
                                                           tau, theta1, theta2, theta3, theta4, _p(u0),
                                                           C.byref(slot)))
        return slot.value

    def tcd_step(self, iterations=4):
        """One time step of every time-dependent instance; returns the iterations given to
        the slowest one."""
        out = C.c_int()
        self.ctx.check(self.ctx.lib.cdgpu_batch_tcd_step(self.ctx.h, self.id, iterations, C.byref(out)))
        return out.value

    def advance(self, iterations=1):
        running = C.c_int()
        self.ctx.check(self.ctx.lib.cdgpu_batch_advance(self.ctx.h, self.id, iterations, C.byref(running)))
        return running.value

    def poll(self, max_slots=65536):
        buf = (C.c_int * max_slots)()
        cnt = C.c_int()
        self.ctx.check(self.ctx.lib.cdgpu_batch_poll(self.ctx.h, self.id, C.cast(buf, C.c_void_p), max_slots,
                                                     C.byref(cnt)))
        return list(buf[:cnt.value])

    def fetch(self, slot, n_dof):
        """(solution, SolveInfo) of a slot; n_dof = 0 reads the statistics only."""
        x = np.zeros(n_dof) if n_dof else None
        info = SolveInfo()
        self.ctx.check(self.ctx.lib.cdgpu_batch_fetch(self.ctx.h, self.id, slot, _p(x) if x is not None else None,
                                                      C.byref(info)))
        return x, info

    def release(self, slot):
        self.ctx.check(self.ctx.lib.cdgpu_batch_release(self.ctx.h, self.id, slot))

    def memory(self):
        out = C.c_ulonglong()
        self.ctx.check(self.ctx.lib.cdgpu_batch_memory(self.ctx.h, self.id, C.byref(out)))
        return out.value

    def loop_info(self):
        """(mode, graph launches, host-loop iterations) of the advance calls so far: mode 1 or
        2 = device-side iteration loop (conditional CUDA graph), 0 = host loop."""
        mode, gl, hi = C.c_int(), C.c_longlong(), C.c_longlong()
        self.ctx.check(self.ctx.lib.cdgpu_batch_loop_info(self.ctx.h, self.id, C.byref(mode), C.byref(gl),
                                                          C.byref(hi)))
        return mode.value, gl.value, hi.value

    def run(self, iterations_per_poll=8):
        """Advance until no instance is running; returns the finished slots in order."""
        done = []
        while True:
            running = self.advance(iterations_per_poll)
            done += self.poll()
            if running == 0:
                return done + self.poll()
