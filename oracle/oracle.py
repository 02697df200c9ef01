"""ctypes front end of the CPU oracle (oracle/libneko_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg.  It is the checker, never part of the
neko_b200 product path.  The shared library restates the reference's CPU
code (see the citations in neko_oracle.cpp / neko_oracle_solve.cpp).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libneko_oracle.so")
_lib = None

_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_int64)


def build():
    """Compile the oracle with its Makefile (g++ only, no GPU needed)."""
    global _lib
    if _lib is None:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        sig = {
            "or_box_create": (_P, [ctypes.c_int] * 3 + [ctypes.c_double] * 6 + [ctypes.c_int] * 4),
            "or_elements_create": (_P, [ctypes.c_int, _I, _D, ctypes.c_int]),
            "or_deform_sine": (None, [_P, ctypes.c_double]),
            "or_coef_init": (None, [_P]),
            "or_bc_boundary": (None, [_P]),
            "or_mark_dirichlet_facets": (None, [_P]),
            "or_destroy": (None, [_P]),
            "or_n": (ctypes.c_long, [_P]),
            "or_nelv": (ctypes.c_int, [_P]),
            "or_lx": (ctypes.c_int, [_P]),
            "or_nlocal": (ctypes.c_int, [_P]),
            "or_local_facet_offset": (ctypes.c_int, [_P]),
            "or_nblks": (ctypes.c_int, [_P]),
            "or_nmsk": (ctypes.c_int, [_P]),
            "or_volume": (ctypes.c_double, [_P]),
            "or_glb_mpts": (ctypes.c_int, [_P]),
            "or_glb_meds": (ctypes.c_int, [_P]),
            "or_dfrmd": (ctypes.c_int, [_P, ctypes.c_int]),
            "or_get_i64": (None, [_P, ctypes.c_char_p, _L]),
            "or_get_i32": (None, [_P, ctypes.c_char_p, _I]),
            "or_get_f64": (None, [_P, ctypes.c_char_p, _D]),
            "or_set_f64": (None, [_P, ctypes.c_char_p, _D]),
            "or_set_ifh2": (None, [_P, ctypes.c_int]),
            "or_gs_add": (None, [_P, _D]),
            "or_ax_helm": (None, [_P, _D, _D]),
            "or_bc_apply": (None, [_P, _D]),
            "or_glsc3": (ctypes.c_double, [_D, _D, _D, ctypes.c_long]),
            "or_jacobi_update": (None, [_P, _D]),
            "or_cg_jacobi": (ctypes.c_int, [_P, _D, _D, ctypes.c_int, ctypes.c_double, _D, _D]),
            "or_fd_weights_full": (None, [ctypes.c_double, _D, ctypes.c_int, ctypes.c_int, _D]),
            "or_zwgll": (None, [ctypes.c_int, _D, _D]),
            "or_dgll": (None, [ctypes.c_int, _D, _D, _D]),
            "or_hsmg_create": (_P, [_P, ctypes.c_int, ctypes.c_double]),
            "or_hsmg_destroy": (None, [_P]),
            "or_hsmg_apply": (None, [_P, _D, _D]),
            "or_hsmg_schwarz_fine": (None, [_P, _D, _D]),
            "or_hsmg_sizes": (ctypes.c_long, [_P, ctypes.c_int]),
            "or_tnsr3d": (None, [_D, ctypes.c_int, _D, ctypes.c_int, _D, _D, _D, ctypes.c_int]),
            "or_fdm_do_fast": (None, [_D, _D, _D, _D, ctypes.c_int, ctypes.c_int]),
            "or_schwarz_extrude": (None, [_D, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int]),
            "or_schwarz_toext3d": (None, [_D, _D, ctypes.c_int, ctypes.c_int]),
            "or_schwarz_toreg3d": (None, [_D, _D, ctypes.c_int, ctypes.c_int]),
            "or_cg_hsmg": (ctypes.c_int, [_P, _P, _D, _D, ctypes.c_int, ctypes.c_double, _D, _D]),
            "or_fcg_hsmg": (ctypes.c_int, [_P, _P, _D, _D, ctypes.c_int, ctypes.c_double, _D, _D]),
            "or_gmres_hsmg": (ctypes.c_int, [_P, _P, _D, _D, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_int, _D, _D]),
            "or_gmres_jacobi": (ctypes.c_int, [_P, _D, _D, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_int, _D, _D]),
            "or_pipecg_jacobi": (ctypes.c_int, [_P, _D, _D, ctypes.c_int, ctypes.c_double, _D, _D]),
            "or_projection_create": (_P, [_P, ctypes.c_int]),
            "or_genmeshbox_nmsh": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 3 +
                                   [ctypes.c_double] * 6 + [ctypes.c_int] * 3),
            "or_projection_destroy": (None, [_P]),
            "or_projection_project_on": (None, [_P, _D]),
            "or_projection_project_back": (None, [_P, _D]),
            "or_projection_m": (ctypes.c_int, [_P]),
            "or_ax_helm_stress": (None, [_P, _D, _D, _D, _D, _D, _D]),
            "or_cg_coupled": (ctypes.c_int, [_P, _D, _D, _D, _D, _D, _D, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int, _D,
                                             _D]),
            "or_phmg_create": (_P, [_P, ctypes.c_int, _I, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int]),
            "or_phmg_destroy": (None, [_P]),
            "or_phmg_apply": (None, [_P, _D, _D]),
            "or_phmg_info": (ctypes.c_double, [_P, ctypes.c_int, ctypes.c_int]),
            "or_phmg_agg_map": (None, [_P, ctypes.c_int, _I]),
            "or_phmg_dinv": (None, [_P, ctypes.c_int, _D]),
            "or_phmg_tamg": (None, [_P, _D, _D]),
            "or_phmg_krylov": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, _D, _D,
                                              ctypes.c_int, ctypes.c_double, _D, _D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


class OracleProblem:
    """Mesh + GLL space + dofmap + gs maps (+ coef, bc) built on the CPU the
    way the reference builds them."""

    def __init__(self, handle):
        self.h = handle
        L = lib()
        self.n = L.or_n(handle)
        self.nelv = L.or_nelv(handle)
        self.lx = L.or_lx(handle)
        self.has_coef = False

    @classmethod
    def box(cls, nel, lx, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), periodic=(False, False, False)):
        nx, ny, nz = nel
        h = lib().or_box_create(nx, ny, nz, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2],
                                int(periodic[0]), int(periodic[1]), int(periodic[2]), lx)
        return cls(h)

    @classmethod
    def from_elements(cls, ids, xyz, lx):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        nelv = ids.shape[0]
        h = lib().or_elements_create(nelv, ids.ctypes.data_as(_I), _dp(xyz), lx)
        return cls(h)

    def deform_sine(self, amp):
        lib().or_deform_sine(self.h, amp)

    def coef(self):
        lib().or_coef_init(self.h)
        self.has_coef = True

    def bc_boundary(self, strong=True):
        """Zero-Dirichlet on every face without a neighbour; with strong=True
        those faces also get facet_type 1 (strong bc) for the FDM."""
        lib().or_bc_boundary(self.h)
        if strong:
            lib().or_mark_dirichlet_facets(self.h)

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- sizes ---------------------------------------------------------
    @property
    def nlocal(self):
        return lib().or_nlocal(self.h)

    @property
    def local_facet_offset(self):
        return lib().or_local_facet_offset(self.h)

    @property
    def nblks(self):
        return lib().or_nblks(self.h)

    @property
    def volume(self):
        return lib().or_volume(self.h)

    @property
    def glb_mpts(self):
        return lib().or_glb_mpts(self.h)

    @property
    def glb_meds(self):
        return lib().or_glb_meds(self.h)

    def dfrmd(self):
        return np.array([lib().or_dfrmd(self.h, e) for e in range(self.nelv)], dtype=bool)

    # --- arrays --------------------------------------------------------
    def dof(self):
        out = np.zeros(self.n, dtype=np.int64)
        lib().or_get_i64(self.h, b"dof", out.ctypes.data_as(_L))
        return out

    def i32(self, name):
        size = {"dof_gs": self.nlocal, "gs_dof": self.nlocal, "blk_len": self.nblks,
                "blk_off": self.nblks, "msk": lib().or_nmsk(self.h),
                "facet_neigh": 6 * self.nelv}[name]
        out = np.zeros(size, dtype=np.int32)
        if size:
            lib().or_get_i32(self.h, name.encode(), out.ctypes.data_as(_I))
        return out

    def f64(self, name):
        size = {"zg": self.lx, "wx": self.lx, "dx": self.lx ** 2, "dxt": self.lx ** 2,
                "w3": self.lx ** 3}.get(name, self.n)
        out = np.zeros(size, dtype=np.float64)
        lib().or_get_f64(self.h, name.encode(), _dp(out))
        return out

    def set_f64(self, name, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        assert arr.size == self.n
        lib().or_set_f64(self.h, name.encode(), _dp(arr))

    def set_ifh2(self, flag):
        lib().or_set_ifh2(self.h, int(bool(flag)))

    # --- operators -----------------------------------------------------
    def gs_add(self, u):
        u = np.array(u, dtype=np.float64, copy=True)
        lib().or_gs_add(self.h, _dp(u))
        return u

    def ax_helm(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        w = np.zeros_like(u)
        lib().or_ax_helm(self.h, _dp(w), _dp(u))
        return w

    def ax_helm_stress(self, u, v, w):
        """Full-stress operator on three components (ax_helm_stress_lx)."""
        u, v, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w))
        au, av, aw = np.zeros_like(u), np.zeros_like(u), np.zeros_like(u)
        lib().or_ax_helm_stress(self.h, _dp(au), _dp(av), _dp(aw), _dp(u), _dp(v), _dp(w))
        return au, av, aw

    def cg_coupled(self, f, max_iter, abs_tol, stress=True, jacobi=True):
        """Coupled CG on three components (cg_cpld_device_solve); f is a
        sequence of three right-hand sides.  Returns ((x, y, z), iterations,
        res_start, res_final)."""
        fx, fy, fz = (np.ascontiguousarray(a, dtype=np.float64) for a in f)
        x, y, z = np.zeros_like(fx), np.zeros_like(fx), np.zeros_like(fx)
        r0 = ctypes.c_double()
        r1 = ctypes.c_double()
        it = lib().or_cg_coupled(self.h, _dp(x), _dp(y), _dp(z), _dp(fx), _dp(fy), _dp(fz),
                                 max_iter, abs_tol, int(stress), int(jacobi), ctypes.byref(r0),
                                 ctypes.byref(r1))
        return (x, y, z), it, r0.value, r1.value

    def bc_apply(self, x):
        x = np.array(x, dtype=np.float64, copy=True)
        lib().or_bc_apply(self.h, _dp(x))
        return x

    def jacobi_diag(self):
        d = np.zeros(self.n)
        lib().or_jacobi_update(self.h, _dp(d))
        return d

    def cg_jacobi(self, f, max_iter, abs_tol):
        f = np.ascontiguousarray(f, dtype=np.float64)
        x = np.zeros_like(f)
        r0 = ctypes.c_double()
        r1 = ctypes.c_double()
        it = lib().or_cg_jacobi(self.h, _dp(x), _dp(f), max_iter, abs_tol,
                                ctypes.byref(r0), ctypes.byref(r1))
        return x, it, r0.value, r1.value

    def pipecg_jacobi(self, f, max_iter, abs_tol):
        """Jacobi-preconditioned pipelined CG (pipecg_device_solve)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        x = np.zeros_like(f)
        r0 = ctypes.c_double()
        r1 = ctypes.c_double()
        it = lib().or_pipecg_jacobi(self.h, _dp(x), _dp(f), max_iter, abs_tol,
                                    ctypes.byref(r0), ctypes.byref(r1))
        return x, it, r0.value, r1.value

    def gmres_jacobi(self, f, max_iter, abs_tol, m_restart=30):
        """Jacobi-preconditioned restarted GMRES (gmres_device_solve)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        x = np.zeros_like(f)
        r0 = ctypes.c_double()
        r1 = ctypes.c_double()
        it = lib().or_gmres_jacobi(self.h, _dp(x), _dp(f), max_iter, abs_tol, m_restart,
                                   ctypes.byref(r0), ctypes.byref(r1))
        return x, it, r0.value, r1.value


class OracleProjection:
    """projection_t of an OracleProblem (device forms of its steps)."""

    def __init__(self, P, L):
        self.P = P
        self.h = lib().or_projection_create(P.h, int(L))

    def project_on(self, b):
        b = np.array(b, dtype=np.float64, copy=True)
        lib().or_projection_project_on(self.h, _dp(b))
        return b

    def project_back(self, x):
        x = np.array(x, dtype=np.float64, copy=True)
        lib().or_projection_project_back(self.h, _dp(x))
        return x

    @property
    def m(self):
        return lib().or_projection_m(self.h)

    def close(self):
        if self.h:
            lib().or_projection_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleHsmg:
    """hsmg_t of an OracleProblem (coef and bc must be set up first)."""

    def __init__(self, P, coarse_iter=10, coarse_tol=1e-9):
        self.P = P
        self.h = lib().or_hsmg_create(P.h, coarse_iter, coarse_tol)

    def apply(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        lib().or_hsmg_apply(self.h, _dp(z), _dp(r))
        return z

    def schwarz_fine(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        e = np.zeros_like(r)
        lib().or_hsmg_schwarz_fine(self.h, _dp(e), _dp(r))
        return e

    @property
    def last_coarse_iter(self):
        return lib().or_hsmg_sizes(self.h, 4)

    def cg(self, f, max_iter, abs_tol, flexible=False):
        f = np.ascontiguousarray(f, dtype=np.float64)
        x = np.zeros_like(f)
        r0 = ctypes.c_double()
        r1 = ctypes.c_double()
        fn = lib().or_fcg_hsmg if flexible else lib().or_cg_hsmg
        it = fn(self.P.h, self.h, _dp(x), _dp(f), max_iter, abs_tol,
                ctypes.byref(r0), ctypes.byref(r1))
        return x, it, r0.value, r1.value

    def gmres(self, f, max_iter, abs_tol, m_restart=30):
        """Restarted flexible GMRES preconditioned by this hsmg
        (gmres_device_solve)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        x = np.zeros_like(f)
        r0 = ctypes.c_double()
        r1 = ctypes.c_double()
        it = lib().or_gmres_hsmg(self.P.h, self.h, _dp(x), _dp(f), max_iter, abs_tol,
                                 m_restart, ctypes.byref(r0), ctypes.byref(r1))
        return x, it, r0.value, r1.value

    def close(self):
        if self.h:
            lib().or_hsmg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def genmeshbox_nmsh(path, nel, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                    periodic=(False, False, False)):
    """Writes the genmeshbox mesh of the box as an .nmsh file (the
    reference's file layout, periodic zones included)."""
    rc = lib().or_genmeshbox_nmsh(str(path).encode(), nel[0], nel[1], nel[2], lo[0], hi[0],
                                  lo[1], hi[1], lo[2], hi[2], int(periodic[0]),
                                  int(periodic[1]), int(periodic[2]))
    assert rc == 0


def fd_weights_full(xi, x, m):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.size - 1
    c = np.zeros((m + 1) * (n + 1))
    lib().or_fd_weights_full(xi, _dp(x), n, m, _dp(c))
    return c.reshape(m + 1, n + 1).T  # c[j, k]


def gll(lx):
    z = np.zeros(lx)
    w = np.zeros(lx)
    lib().or_zwgll(lx, _dp(z), _dp(w))
    d = np.zeros(lx * lx)
    dt = np.zeros(lx * lx)
    lib().or_dgll(lx, _dp(z), _dp(d), _dp(dt))
    return z, w, d.reshape(lx, lx, order="F")


def glsc3(a, b, c):
    a, b, c = (np.ascontiguousarray(v, dtype=np.float64) for v in (a, b, c))
    return lib().or_glsc3(_dp(a), _dp(b), _dp(c), a.size)


# Array-level forms of the reference's device routines (tensor.cu:60,
# fdm.cu:42, schwarz.cu:45-100), used to check the drop-in symbols.
def tnsr3d(u, nu, nv, A, Bt, Ct, nel):
    v = np.zeros(nel * nv ** 3)
    lib().or_tnsr3d(_dp(v), nv, _dp(np.ascontiguousarray(u)), nu, _dp(A), _dp(Bt), _dp(Ct), nel)
    return v


def fdm_do_fast(r, s, d, nl, nel):
    """Returns (e, r_after): the reference overwrites r with d * (first pass)."""
    e = np.zeros(nel * nl ** 3)
    rr = np.array(r, dtype=np.float64)
    lib().or_fdm_do_fast(_dp(e), _dp(rr), _dp(np.ascontiguousarray(s)),
                         _dp(np.ascontiguousarray(d)), nl, nel)
    return e, rr


def schwarz_extrude(a1, l1, f1, a2, l2, f2, nx, nel):
    out = np.array(a1, dtype=np.float64)
    src = out if a2 is a1 else np.ascontiguousarray(a2)
    lib().or_schwarz_extrude(_dp(out), l1, f1, _dp(src), l2, f2, nx, nel)
    return out


def schwarz_toext3d(b, nx, nel):
    a = np.zeros(nel * (nx + 2) ** 3)
    lib().or_schwarz_toext3d(_dp(a), _dp(np.ascontiguousarray(b)), nx, nel)
    return a


def schwarz_toreg3d(a, nx, nel):
    b = np.zeros(nel * nx ** 3)
    lib().or_schwarz_toreg3d(_dp(b), _dp(np.ascontiguousarray(a)), nx, nel)
    return b


class OraclePhmg:
    """phmg_t of an OracleProblem (coef, h1/h2 and bc set up first):
    Jacobi-accelerated Chebyshev smoothing on levels lx -> schedule + 1,
    tree AMG on the last level."""

    def __init__(self, P, smoother_iterations=3, schedule=(3, 1), coarse_levels=3,
                 coarse_iterations=1, cheby_degree=4):
        self.P = P
        sched = (ctypes.c_int * len(schedule))(*schedule)
        self.h = lib().or_phmg_create(P.h, smoother_iterations, sched, len(schedule),
                                      coarse_levels, coarse_iterations, cheby_degree)
        if not self.h:
            raise RuntimeError("phmg set-up failed (the reference stops with an error here)")

    def apply(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        lib().or_phmg_apply(self.h, _dp(z), _dp(r))
        return z

    def info(self, what, i=0):
        return lib().or_phmg_info(self.h, what, i)

    @property
    def levels(self):
        return int(self.info(0))

    def level_lx(self, i):
        return int(self.info(1, i))

    def cheby(self, i):
        """(tha, dlt, lambda_max) of level i's smoother."""
        return self.info(2, i), self.info(3, i), self.info(4, i)

    @property
    def amg_levels(self):
        return int(self.info(5))

    def amg_nodes(self, i):
        return int(self.info(6, i))

    def amg_cheby(self, i):
        return self.info(7, i), self.info(8, i), self.info(9, i)

    def agg_map(self, lvl, n0):
        out = np.zeros(n0, dtype=np.int32)
        lib().or_phmg_agg_map(self.h, lvl, out.ctypes.data_as(_I))
        return out

    def dinv(self, i, n):
        out = np.zeros(n)
        lib().or_phmg_dinv(self.h, i, _dp(out))
        return out

    def tamg(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        lib().or_phmg_tamg(self.h, _dp(z), _dp(r))
        return z

    def krylov(self, f, max_iter, abs_tol, kind="cg", m=30):
        """Solve with M = phmg: kind "cg", "fcg" or "gmres"."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        x = np.zeros_like(f)
        r0 = ctypes.c_double()
        r1 = ctypes.c_double()
        k = {"cg": 0, "fcg": 1, "gmres": 2}[kind]
        it = lib().or_phmg_krylov(self.P.h, self.h, k, m, _dp(x), _dp(f), max_iter, abs_tol,
                                  ctypes.byref(r0), ctypes.byref(r1))
        return x, it, r0.value, r1.value

    def close(self):
        if self.h:
            lib().or_phmg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
