"""neko_b200 -- a B200-native device backend for Neko's pressure/Helmholtz
solve path (ax_helm, gather-scatter add, CG/flexible CG, hsmg).

The compute lives in libnekob200.so (hand-written sm_100a CUDA, C ABI in
include/neko_b200.h).  This module is the host-side mirror of the
reference's operator interfaces, so a solve reads like the reference's
Fortran:

    ax_t%compute(w, u, coef, msh, Xh)        ->  AxHelm().compute(w, u, coef)
    gs_t%op(u, n, GS_OP_ADD)                 ->  coef.gs.op(u, n, GS_OP_ADD)
    bc_list_t%apply(x, n)                    ->  coef.bclst.apply(x, n)
    ksp_t%solve(Ax, x, f, n, coef, blst, gs_h, niter) -> KspMonitor
                                             ->  CG(...).solve(Ax, x, f, n, coef, ...)

(src/math/ax.f90:43-84, src/gs/gather_scatter.f90:82-118,
src/krylov/krylov.f90:136-157, src/krylov/precon.f90:40-66).  Device memory
is handed over as torch CUDA tensors; torch provides allocation and streams.
"""
import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import (NB_ERR_ARG, NB_PC_HSMG, NB_PC_JACOBI, NB_PC_NONE, NekoB200Error,
                   SolveOpts, SolveResult, check, load)

GS_OP_ADD = 1  # src/gs/gs_ops.f90:36

__all__ = ["Problem", "AxHelm", "AxHelmFull", "CoupledCG", "GatherScatter", "BcList", "CG",
           "FCG", "GMRES", "PipeCG",
           "KspMonitor",
           "Jacobi", "Hsmg", "Batch", "Projection", "ortho", "read_nmsh", "write_nmsh",
           "write_fld",
           "GS_OP_ADD", "NekoB200Error",
           "load", "version"]


def version():
    return load().nb_version().decode()


def _stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t):
    if not (t.is_cuda and t.is_contiguous()):
        raise ValueError("expected a contiguous CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


class _DeviceView:
    """__cuda_array_interface__ wrapper so torch can view library memory."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


class Problem:
    """Mesh + GLL space + dofmap + gather-scatter + coefficients (mesh_t,
    space_t, dofmap_t, gs_t, coef_t) of a structured box, resident on the
    current CUDA device."""

    def __init__(self, nel, lx, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                 periodic=(False, False, False), deform=0.0, dirichlet=True):
        L = load()
        ne = (ctypes.c_int * 3)(*nel)
        lo_ = (ctypes.c_double * 3)(*lo)
        hi_ = (ctypes.c_double * 3)(*hi)
        per = (ctypes.c_int * 3)(*[int(bool(p)) for p in periodic])
        h = ctypes.c_void_p()
        torch.cuda.init()
        check(L.nb_problem_create_box(ne, lo_, hi_, per, lx, float(deform), int(bool(dirichlet)),
                                      ctypes.byref(h)))
        self._adopt(h)
        self.nel, self.periodic, self.deform = tuple(nel), tuple(periodic), deform

    @classmethod
    def from_mesh(cls, vertex_ids, vertex_xyz, lx, deform=0.0, dirichlet=True):
        """Problem on an unstructured hex mesh: vertex_ids (nelv, 8) positive
        global ids, vertex_xyz (nelv, 8, 3), symmetric vertex order
        (nb_problem_create_mesh)."""
        import numpy as np
        ids = np.ascontiguousarray(vertex_ids, dtype=np.int32)
        xyz = np.ascontiguousarray(vertex_xyz, dtype=np.float64)
        nelv = ids.shape[0]
        if ids.shape != (nelv, 8) or xyz.shape != (nelv, 8, 3):
            raise ValueError("vertex_ids must be (nelv, 8) and vertex_xyz (nelv, 8, 3)")
        self = cls.__new__(cls)
        h = ctypes.c_void_p()
        torch.cuda.init()
        check(load().nb_problem_create_mesh(
            nelv, ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(lx), float(deform),
            int(bool(dirichlet)), ctypes.byref(h)))
        self._adopt(h)
        self.nel, self.periodic, self.deform = (nelv,), (False, False, False), deform
        return self

    def _adopt(self, h):
        L = load()
        self._h = h
        n = ctypes.c_int64()
        nelv, lxo, nloc, nblk, nmsk = (ctypes.c_int() for _ in range(5))
        check(L.nb_problem_sizes(h, ctypes.byref(n), ctypes.byref(nelv), ctypes.byref(lxo),
                                 ctypes.byref(nloc), ctypes.byref(nblk), ctypes.byref(nmsk)))
        self.n, self.nelv, self.lx = n.value, nelv.value, lxo.value
        self.nlocal, self.nblocks, self.nmask = nloc.value, nblk.value, nmsk.value
        vol = ctypes.c_double()
        check(L.nb_problem_volume(h, ctypes.byref(vol)))
        self.volume = vol.value
        self.gs = GatherScatter(self)
        self.bclst = BcList(self)

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("problem destroyed")
        return self._h

    _SIZES = {"dx": lambda p: p.lx ** 2, "dxt": lambda p: p.lx ** 2, "zg": lambda p: p.lx,
              "dof_gs": lambda p: p.nlocal, "gs_dof": lambda p: p.nlocal,
              "blk_len": lambda p: p.nblocks, "blk_off": lambda p: p.nblocks,
              "msk": lambda p: p.nmask, "err": lambda p: 1}
    _INT_FIELDS = ("dof_gs", "gs_dof", "blk_len", "blk_off", "msk", "err")

    def field(self, name):
        """Zero-copy torch view of a device array of the problem."""
        ptr = ctypes.c_void_p()
        check(load().nb_problem_field(self.handle, name.encode(), ctypes.byref(ptr)))
        size = self._SIZES.get(name, lambda p: p.n)(self)
        typestr = "<i4" if name in self._INT_FIELDS else "<f8"
        if size == 0:
            return torch.empty(0, dtype=torch.int32 if typestr == "<i4" else torch.float64,
                               device="cuda")
        return torch.as_tensor(_DeviceView(ptr.value, size, typestr), device="cuda")

    def set_coefficients(self, h1, h2=None):
        """Helmholtz coefficients: A = -div(h1 grad) + h2 B (ifh2 when h2 given)."""
        h1 = h1.contiguous()
        h2c = h2.contiguous() if h2 is not None else None
        check(load().nb_problem_set_coefficients(self.handle, _ptr(h1),
                                                 _ptr(h2c) if h2c is not None else None,
                                                 int(h2 is not None)))

    def set_coefficients_const(self, h1, h2=0.0, stream=None):
        """Constant h1 > 0, h2 >= 0 set asynchronously on `stream` (h2 = 0:
        no h2 term) -- nb_problem_set_coefficients_const."""
        check(load().nb_problem_set_coefficients_const(self.handle, float(h1), float(h2),
                                                       _stream_handle(stream)))

    def zeros(self):
        return torch.zeros(self.n, dtype=torch.float64, device="cuda")

    def sync(self, stream=None):
        """Wait for `stream` and raise NekoB200Error (NB_ERR_TIMEOUT) when an
        earlier asynchronous call on this problem had a bounded device wait
        expire (nb_problem_sync)."""
        check(load().nb_problem_sync(self.handle, _stream_handle(stream)))

    def close(self):
        if getattr(self, "_h", None) is not None:
            load().nb_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AxHelm:
    """ax_helm_t: w = A u element by element (no assembly)
    (src/math/ax_helm.f90:44-77)."""

    def compute(self, w, u, coef, msh=None, Xh=None, stream=None):
        check(load().nb_ax(coef.handle, _ptr(w), _ptr(u), _stream_handle(stream)))

    def compute_vector(self, au, av, aw, u, v, w, coef, msh=None, Xh=None, stream=None):
        """ax_t%compute_vector: the operator on the three components of a
        vector field with one pass over the coefficients (nb_ax_vector)."""
        check(load().nb_ax_vector(coef.handle, _ptr(au), _ptr(av), _ptr(aw), _ptr(u), _ptr(v),
                                  _ptr(w), _stream_handle(stream)))

    def update_p_compute(self, w, p, z, beta, coef, pap=None, stream=None):
        """p = z + beta p, then w = A p in one streaming pass; pap (a
        one-element float64 CUDA tensor, optional) receives sum(p * w) over
        the local points (nb_ax_update_p)."""
        check(load().nb_ax_update_p(coef.handle, _ptr(w), _ptr(p), _ptr(z), float(beta),
                                    _ptr(pap) if pap is not None else None,
                                    _stream_handle(stream)))


class AxHelmFull:
    """ax_helm_full_t: the full-stress operator of the velocity solve with
    variable viscosity (src/math/ax_helm_full.f90); it acts on the three
    components together only, as the reference's does."""

    op = _lib.NB_AX_STRESS

    def compute(self, w, u, coef, msh=None, Xh=None, stream=None):
        raise NekoB200Error(NB_ERR_ARG, "the full Helmholtz operator cannot be applied to a "
                                        "single field; use compute_vector and a coupled "
                                        "solver (CoupledCG)")

    def compute_vector(self, au, av, aw, u, v, w, coef, msh=None, Xh=None, stream=None):
        check(load().nb_ax_stress(coef.handle, _ptr(au), _ptr(av), _ptr(aw), _ptr(u), _ptr(v),
                                  _ptr(w), _stream_handle(stream)))


class GatherScatter:
    """gs_t of a problem: op(u, n, GS_OP_ADD) sums all local copies."""

    def __init__(self, problem):
        self.problem = problem

    def op(self, u, n=None, op=GS_OP_ADD, stream=None):
        if op != GS_OP_ADD:
            raise NotImplementedError("the native gs supports GS_OP_ADD; use the cuda_* "
                                      "drop-in entry points for mul/min/max")
        check(load().nb_gs_add(self.problem.handle, _ptr(u), _stream_handle(stream)))


class BcList:
    """bc_list_t with the problem's zero-Dirichlet mask."""

    def __init__(self, problem):
        self.problem = problem

    def apply(self, x, n=None, stream=None):
        check(load().nb_bc_apply(self.problem.handle, _ptr(x), _stream_handle(stream)))


@dataclass
class KspMonitor:
    """ksp_monitor_t (src/krylov/krylov.f90:56-70)."""
    iter: int
    res_start: float
    res_final: float
    converged: bool
    launches: int = 0


class Jacobi:
    """pc_jacobi: z = d r with d = 1/gs(diag A) (pc_jacobi.f90:86-170)."""
    kind = NB_PC_JACOBI


class Hsmg:
    """pc_hsmg: additive 3-level Schwarz/FDM multigrid (pc_hsmg.f90).
    `solve(z, r, coef)` is pc_t%solve: z = M r (r masked).  mixed=True runs
    the smoothing levels in FP32 (the coarse CG stays FP64)."""
    kind = NB_PC_HSMG

    def __init__(self, coarse_iter=10, coarse_tol=1e-9, mixed=False):
        self.coarse_iter, self.coarse_tol, self.mixed = coarse_iter, coarse_tol, mixed

    def init(self, coef):
        """hsmg_init: build the levels for this problem (cached until the
        settings change)."""
        check(load().nb_hsmg_init(coef.handle, int(self.mixed), int(self.coarse_iter),
                                  float(self.coarse_tol)))

    def solve(self, z, r, coef, n=None, stream=None):
        self.init(coef)
        kind = _lib.NB_PC_HSMG_MIXED if self.mixed else NB_PC_HSMG
        check(load().nb_pc_apply(coef.handle, kind, _ptr(z), _ptr(r), _stream_handle(stream)))


class Phmg:
    """phmg_t: hybrid ph-multigrid (src/multigrid/phmg.f90).  Polynomial
    levels lx -> schedule + 1 (default lx -> 4 -> 2) smoothed by
    `smoother_iterations` Jacobi-accelerated Chebyshev steps, a tree-AMG
    V-cycle (`coarse_levels` levels, `cheby_degree` Chebyshev steps a
    level, `coarse_iterations` cycles) on the last.  `solve(z, r, coef)` is
    pc_t%solve: z = M r (r masked).  Built for a problem on first use and
    kept, as the reference's phmg_init does (the coarser levels keep the h1
    of that moment)."""
    kind = _lib.NB_PC_PHMG

    def __init__(self, smoother_iterations=3, schedule=(3, 1), coarse_levels=3,
                 coarse_iterations=1, cheby_degree=4):
        self.smoother_iterations = smoother_iterations
        self.schedule = tuple(int(k) for k in schedule)
        self.coarse_levels = coarse_levels
        self.coarse_iterations = coarse_iterations
        self.cheby_degree = cheby_degree

    def _settings(self):
        return (self.smoother_iterations, self.schedule, self.coarse_levels,
                self.coarse_iterations, self.cheby_degree)

    def init(self, coef):
        """phmg_init: build the levels, the aggregation and the eigenvalue
        estimates for this problem (again only when the settings differ from
        those it was built with)."""
        if getattr(coef, "_phmg_settings", None) == self._settings():
            return
        if not 1 <= len(self.schedule) <= 8:
            raise NekoB200Error(NB_ERR_ARG, "phmg: 1 to 8 schedule entries")
        o = _lib.PhmgOpts()
        o.smoother_iterations = self.smoother_iterations
        o.n_schedule = len(self.schedule)
        for i, k in enumerate(self.schedule):
            o.schedule[i] = k
        o.coarse_levels = self.coarse_levels
        o.coarse_iterations = self.coarse_iterations
        o.cheby_degree = self.cheby_degree
        check(load().nb_phmg_init(coef.handle, ctypes.byref(o)))
        coef._phmg_settings = self._settings()

    prepare = init

    def describe(self, coef, what, i=0):
        out = ctypes.c_double()
        check(load().nb_phmg_describe(coef.handle, what, i, ctypes.byref(out)))
        return out.value

    def solve(self, z, r, coef, n=None, stream=None):
        self.init(coef)
        check(load().nb_pc_apply(coef.handle, _lib.NB_PC_PHMG, _ptr(z), _ptr(r),
                                 _stream_handle(stream)))


def tamg_aggregate(nelv, lx, facet_neigh, coarse_levels=3):
    """The tree-AMG aggregation on the host: (levels kept, [aggregates of
    level l], [level-0 point -> 0-based aggregate of level l]) for l = 1 ..
    levels-1."""
    import numpy as np
    fn = np.ascontiguousarray(facet_neigh, dtype=np.int32)
    n0 = nelv * lx ** 3
    nl = ctypes.c_int()
    nn = np.zeros(max(coarse_levels, 1), dtype=np.int32)
    fin = np.zeros(max(coarse_levels, 1) * n0, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    check(load().nb_tamg_aggregate(nelv, lx, fn.ctypes.data_as(ip), coarse_levels,
                                   ctypes.byref(nl), nn.ctypes.data_as(ip),
                                   fin.ctypes.data_as(ip)))
    k = nl.value - 1
    return nl.value, [int(v) for v in nn[:k]], [fin[i * n0:(i + 1) * n0].copy() for i in range(k)]


class CG:
    """ksp_t of type 'cg' with preconditioner M (Jacobi, Hsmg, Phmg or None);
    stops when sqrt(r' mult r / volume) < abs_tol (krylov.f90:411-421).
    flexible=True uses the Polak-Ribiere beta of flexible CG, which keeps
    converging with a non-symmetric preconditioner such as hsmg."""

    ksp = _lib.NB_KSP_CG

    def __init__(self, n=None, max_iter=1000, M=None, abs_tol=1e-9, mixed=False,
                 flexible=False):
        self.max_iter, self.abs_tol, self.mixed = max_iter, abs_tol, mixed
        self.flexible = flexible
        self.M = M if M is not None else Jacobi()

    def solve(self, Ax, x, f, n=None, coef=None, blst=None, gs_h=None, niter=None,
              stream=None):
        o = SolveOpts()
        o.max_iter = niter if niter is not None else self.max_iter
        o.abs_tol = self.abs_tol
        o.pc = getattr(self.M, "kind", NB_PC_NONE) if self.M is not None else NB_PC_NONE
        o.mixed = int(self.mixed or getattr(self.M, "mixed", False))
        o.coarse_iter = getattr(self.M, "coarse_iter", 10)
        o.coarse_tol = getattr(self.M, "coarse_tol", 1e-9)
        o.flexible = int(self.flexible)
        o.ksp = self.ksp
        o.m_restart = getattr(self, "m_restart", 0)
        if hasattr(self.M, "prepare"):
            self.M.prepare(coef)
        r = SolveResult()
        check(load().nb_solve(coef.handle, _ptr(x), _ptr(f), ctypes.byref(o), ctypes.byref(r),
                              _stream_handle(stream)))
        return KspMonitor(r.iter, r.res_start, r.res_final, bool(r.converged), r.launches)


class FCG(CG):
    """Flexible CG: CG with the Polak-Ribiere beta (Notay's FCG(1))."""

    def __init__(self, n=None, max_iter=1000, M=None, abs_tol=1e-9, mixed=False):
        super().__init__(n, max_iter, M, abs_tol, mixed, flexible=True)


class PipeCG(CG):
    """ksp_t of type 'pipecg': pipelined PCG (pipecg_device_t,
    src/krylov/bcknd/device/pipecg_device.F90), one reduction an
    iteration.  For a symmetric preconditioner (Jacobi)."""
    ksp = _lib.NB_KSP_PIPECG


class GMRES(CG):
    """ksp_t of type 'gmres': restarted flexible GMRES with m_restart
    vectors a cycle (gmres_device_t, src/krylov/bcknd/device/gmres_device.F90;
    the reference's default m_restart is 30)."""
    ksp = _lib.NB_KSP_GMRES

    def __init__(self, n=None, max_iter=1000, M=None, abs_tol=1e-9, mixed=False,
                 m_restart=30):
        super().__init__(n, max_iter, M, abs_tol, mixed)
        self.m_restart = m_restart


class CoupledCG:
    """ksp_t of type 'cpldcg' (cg_cpld_device_t,
    src/krylov/bcknd/device/cg_cpld_device.f90): CG on the three velocity
    components with one set of scalars; Ax is AxHelm (ax_helm on each
    component) or AxHelmFull (the full-stress operator); M is Jacobi or
    None.  solve() on one field is refused, as in the reference."""

    def __init__(self, n=None, max_iter=1000, M=None, abs_tol=1e-9):
        self.max_iter, self.abs_tol = max_iter, abs_tol
        self.M = M if M is not None else Jacobi()

    def solve(self, *args, **kwargs):
        raise NekoB200Error(NB_ERR_ARG, "the cpldcg solver is only defined for coupled solves")

    def solve_coupled(self, Ax, x, y, z, fx, fy, fz, n=None, coef=None, blstx=None, blsty=None,
                      blstz=None, gs_h=None, niter=None, stream=None):
        o = SolveOpts()
        o.max_iter = niter if niter is not None else self.max_iter
        o.abs_tol = self.abs_tol
        o.pc = getattr(self.M, "kind", NB_PC_NONE) if self.M is not None else NB_PC_NONE
        op = getattr(Ax, "op", _lib.NB_AX_HELM_VECTOR)
        r = SolveResult()
        check(load().nb_solve_coupled(coef.handle, op, _ptr(x), _ptr(y), _ptr(z), _ptr(fx),
                                      _ptr(fy), _ptr(fz), ctypes.byref(o), ctypes.byref(r),
                                      _stream_handle(stream)))
        mon = KspMonitor(r.iter, r.res_start, r.res_final, bool(r.converged), r.launches)
        return [mon, mon, mon]


class Projection:
    """projection_t (src/common/projection.f90): projects the pressure
    right-hand side onto up to L earlier solutions before the solve and adds
    the projected part back after it.  pre_solving / post_solving act from
    time step activ_step + 1 on, as the reference's fixed-step path does."""

    def __init__(self, coef, L=20, activ_step=5):
        h = ctypes.c_void_p()
        check(load().nb_projection_create(coef.handle, int(L), ctypes.byref(h)))
        self._h, self.coef, self.L, self.activ_step = h, coef, L, activ_step

    def pre_solving(self, b, tstep, stream=None):
        if tstep > self.activ_step and self.L > 0:
            self.project_on(b, stream)

    def post_solving(self, x, tstep, stream=None):
        if tstep > self.activ_step and self.L > 0:
            self.project_back(x, stream)

    def project_on(self, b, stream=None):
        check(load().nb_projection_project_on(self._h, _ptr(b), _stream_handle(stream)))

    def project_back(self, x, stream=None):
        check(load().nb_projection_project_back(self._h, _ptr(x), _stream_handle(stream)))

    def reortho_basis(self, stream=None):
        check(load().nb_projection_reorthogonalize(self._h, _stream_handle(stream)))

    def clear(self, stream=None):
        check(load().nb_projection_clear(self._h, _stream_handle(stream)))

    def info(self, stream=None):
        """(basis size, basis size at the last projection, its residual)."""
        m, pm, pr = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(load().nb_projection_info(self._h, ctypes.byref(m), ctypes.byref(pm),
                                        ctypes.byref(pr), _stream_handle(stream)))
        return m.value, pm.value, pr.value

    def close(self):
        if getattr(self, "_h", None) is not None:
            load().nb_projection_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_nmsh(path):
    """Reads a 3-D .nmsh mesh (nb_mesh_read_nmsh): (vertex ids (nelv, 8),
    coordinates (nelv, 8, 3)) with the periodic zones applied, ready for
    Problem.from_mesh."""
    import numpy as np
    L = load()
    ne = ctypes.c_int()
    check(L.nb_mesh_read_nmsh(str(path).encode(), ctypes.byref(ne), None, None, None, None))
    ids = np.zeros((ne.value, 8), np.int32)
    xyz = np.zeros((ne.value, 8, 3))
    check(L.nb_mesh_read_nmsh(str(path).encode(), ctypes.byref(ne),
                              ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None, None))
    return ids, xyz


def write_nmsh(path, vertex_ids, vertex_xyz):
    """Writes a mesh as a .nmsh file (nb_mesh_write_nmsh)."""
    import numpy as np
    ids = np.ascontiguousarray(vertex_ids, dtype=np.int32)
    xyz = np.ascontiguousarray(vertex_xyz, dtype=np.float64)
    check(load().nb_mesh_write_nmsh(str(path).encode(), ids.shape[0],
                                    ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))


def write_fld(path, coef, p=None, time=0.0, step=0, mesh=True):
    """Writes the problem's coordinates (mesh=True) and the field p (a
    device tensor of n values, written as the pressure) to an fld file
    (nb_fld_write)."""
    import numpy as np
    DP = ctypes.POINTER(ctypes.c_double)
    arrs = [np.ascontiguousarray(coef.field(k).cpu().numpy()) for k in ("x", "y", "z")] \
        if mesh else [None] * 3
    pa = np.ascontiguousarray(p.detach().cpu().numpy(), dtype=np.float64) if p is not None \
        else None
    ptr = lambda a: a.ctypes.data_as(DP) if a is not None else None
    check(load().nb_fld_write(str(path).encode(), coef.nelv, coef.lx, *(ptr(a) for a in arrs),
                              ptr(pa), float(time), int(step)))


def ortho(x, coef, stream=None):
    """device_ortho: x -= mean of x over the local points (nb_ortho)."""
    check(load().nb_ortho(coef.handle, _ptr(x), _stream_handle(stream)))


class Batch:
    """Many Jacobi-PCG solves advanced together (nb_batch_*): one persistent
    Ax launch over every active solve's elements per iteration, replayed
    from a CUDA graph.  Solves may be submitted and released between runs;
    their work vectors are charged against `hbm_budget` bytes (0: none)."""

    def __init__(self, hbm_budget=0):
        h = ctypes.c_void_p()
        check(load().nb_batch_create(int(hbm_budget), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, problem, f, x, abs_tol, max_iter=1000, h1=None, h2=0.0):
        """Adds a solve; with h1 given, the solve uses the constant
        coefficients h1, h2 instead of the problem's fields."""
        slot = ctypes.c_int()
        if h1 is None:
            check(load().nb_batch_submit(self._h, problem.handle, _ptr(f), _ptr(x),
                                         float(abs_tol), int(max_iter), ctypes.byref(slot)))
        else:
            check(load().nb_batch_submit_coef(self._h, problem.handle, _ptr(f), _ptr(x),
                                              float(abs_tol), int(max_iter), float(h1),
                                              float(h2), ctypes.byref(slot)))
        self._keep[slot.value] = (problem, f, x)
        return slot.value

    def submit_solve(self, problem, f, x, abs_tol, max_iter=1000, h1=1.0, h2=0.0, pc="hsmg",
                     mixed=False, flexible=None, coarse_iter=10, coarse_tol=1e-9):
        """Adds a per-problem Krylov solve of the problem instance (which the
        slot owns until release) run concurrently with the other slots:
        pc "hsmg" (flexible CG, FP64 or mixed) or "jacobi" (CG), constant
        coefficients h1, h2 (nb_batch_submit_solve)."""
        o = SolveOpts()
        o.max_iter, o.abs_tol = int(max_iter), float(abs_tol)
        o.pc = {"hsmg": NB_PC_HSMG, "jacobi": NB_PC_JACOBI, "none": NB_PC_NONE}[pc]
        o.mixed = int(bool(mixed))
        o.coarse_iter, o.coarse_tol = int(coarse_iter), float(coarse_tol)
        o.flexible = int(pc == "hsmg" if flexible is None else flexible)
        o.ksp, o.m_restart = _lib.NB_KSP_CG, 0
        slot = ctypes.c_int()
        check(load().nb_batch_submit_solve(self._h, problem.handle, _ptr(f), _ptr(x),
                                           ctypes.byref(o), float(h1), float(h2),
                                           ctypes.byref(slot)))
        self._keep[slot.value] = (problem, f, x)
        return slot.value

    def run(self, max_chunks=0, stream=None):
        """Replays iteration chunks until every solve stopped (or max_chunks);
        returns the number of solves still running."""
        active = ctypes.c_int()
        check(load().nb_batch_run(self._h, int(max_chunks), ctypes.byref(active),
                                  _stream_handle(stream)))
        return active.value

    def result(self, slot):
        done = ctypes.c_int()
        r = SolveResult()
        check(load().nb_batch_result(self._h, int(slot), ctypes.byref(done), ctypes.byref(r)))
        return bool(done.value), KspMonitor(r.iter, r.res_start, r.res_final, bool(r.converged))

    def release(self, slot):
        check(load().nb_batch_release(self._h, int(slot)))
        self._keep.pop(slot, None)

    def tuning(self, lx):
        ks, n = ctypes.c_int(), ctypes.c_int()
        ms = (ctypes.c_float * 4)()
        check(load().nb_batch_tuning(self._h, int(lx), ctypes.byref(ks), ms, ctypes.byref(n)))
        return ks.value, [ms[i] for i in range(min(n.value, 4))]

    def close(self):
        if getattr(self, "_h", None) is not None:
            load().nb_batch_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
