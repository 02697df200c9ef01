"""ctypes binding of libnekob200.so (the C ABI declared in include/neko_b200.h).

The library is built in-tree by ``neko_b200/build.py``.  Loading fails with
an ImportError-style exception when it is missing: there is no fallback
implementation of any operator.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnekob200.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)

NB_OK = 0
STATUS_NAMES = {0: "NB_OK", 1: "NB_ERR_ARG", 2: "NB_ERR_UNSUPPORTED", 3: "NB_ERR_OOM",
                4: "NB_ERR_CUDA", 5: "NB_ERR_NOT_CONVERGED", 6: "NB_ERR_NAN",
                7: "NB_ERR_TIMEOUT"}

NB_PC_JACOBI, NB_PC_HSMG, NB_PC_NONE, NB_PC_HSMG_MIXED, NB_PC_PHMG = 0, 1, 2, 3, 4
NB_KSP_CG, NB_KSP_GMRES, NB_KSP_PIPECG = 0, 1, 2
NB_AX_HELM_VECTOR, NB_AX_STRESS = 0, 1
NB_OK, NB_ERR_ARG, NB_ERR_UNSUPPORTED, NB_ERR_OOM, NB_ERR_CUDA = 0, 1, 2, 3, 4
NB_ERR_NOT_CONVERGED, NB_ERR_NAN, NB_ERR_TIMEOUT = 5, 6, 7


class SolveOpts(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("abs_tol", ctypes.c_double),
                ("pc", ctypes.c_int), ("mixed", ctypes.c_int),
                ("coarse_iter", ctypes.c_int), ("coarse_tol", ctypes.c_double),
                ("flexible", ctypes.c_int), ("ksp", ctypes.c_int), ("m_restart", ctypes.c_int)]


class PhmgOpts(ctypes.Structure):
    _fields_ = [("smoother_iterations", ctypes.c_int), ("n_schedule", ctypes.c_int),
                ("schedule", ctypes.c_int * 8), ("coarse_levels", ctypes.c_int),
                ("coarse_iterations", ctypes.c_int), ("cheby_degree", ctypes.c_int)]


class SolveResult(ctypes.Structure):
    _fields_ = [("iter", ctypes.c_int), ("res_start", ctypes.c_double),
                ("res_final", ctypes.c_double), ("converged", ctypes.c_int),
                ("launches", ctypes.c_int)]


class NekoB200Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


# Signatures of every exported symbol (name -> (restype, argtypes)).
SIGNATURES = {
    # drop-in cuda_* entry points
    "cuda_ax_helm": (None, [_P] * 15 + [_IP, _IP]),
    "cuda_addcol4": (None, [_P, _P, _P, _P, _IP, _P]),
    "cuda_ax_helm_vector": (None, [_P] * 19 + [_IP, _IP]),
    "cuda_ax_helm_vector_part2": (None, [_P] * 8 + [_IP]),
    "cuda_ax_helm_stress_vector": (None, [_P] * 24 + [_IP, _IP]),
    "cuda_ax_helm_stress_vector_part2": (None, [_P] * 8 + [_IP]),
    "cuda_gather_kernel": (None, [_P, _IP, _IP, _P, _P, _IP, _P, _IP, _P, _P, _IP, _P]),
    "cuda_scatter_kernel": (None, [_P, _IP, _P, _P, _IP, _P, _IP, _P, _P, _P]),
    "cuda_glsc3": (ctypes.c_double, [_P, _P, _P, _IP, _P]),
    "cuda_glsc2": (ctypes.c_double, [_P, _P, _IP, _P]),
    "cuda_glsum": (ctypes.c_double, [_P, _IP, _P]),
    "cuda_copy": (None, [_P, _P, _IP, _P]),
    "cuda_rzero": (None, [_P, _IP, _P]),
    "cuda_add2s1": (None, [_P, _P, _DP, _IP, _P]),
    "cuda_add2s2": (None, [_P, _P, _DP, _IP, _P]),
    "cuda_col2": (None, [_P, _P, _IP, _P]),
    "cuda_col3": (None, [_P, _P, _P, _IP, _P]),
    "cuda_addcol3": (None, [_P, _P, _P, _IP, _P]),
    "cuda_invcol1": (None, [_P, _IP, _P]),
    "cuda_radd": (None, [_P, _DP, _IP, _P]),
    "cuda_zero_dirichlet_apply_scalar": (None, [_P, _P, _IP, _P]),
    "cuda_jacobi_update": (None, [_P] * 10 + [_IP, _IP]),
    "cuda_tnsr3d": (None, [_P, _IP, _P, _IP, _P, _P, _P, _IP]),
    "cuda_fdm_do_fast": (None, [_P, _P, _P, _P, _IP, _IP, _P]),
    "cuda_schwarz_extrude": (None, [_P, _IP, _DP, _P, _IP, _DP, _IP, _IP, _P]),
    "cuda_schwarz_toext3d": (None, [_P, _P, _IP, _IP, _P]),
    "cuda_schwarz_toreg3d": (None, [_P, _P, _IP, _IP, _P]),
    "cuda_fusedcg_update_p": (None, [_P, _P, _P, _DP, _IP]),
    "cuda_fusedcg_update_x": (None, [_P, _P, _P, _IP, _IP]),
    "cuda_fusedcg_part2": (ctypes.c_double, [_P, _P, _P, _P, _DP, _IP, _IP]),
    "nb_set_default_stream": (None, [_P]),
    "pnpn_prs_res_part1_cuda": (None, [_P] * 11 + [_DP, _DP, _IP]),
    "pnpn_prs_res_part2_cuda": (None, [_P] * 4 + [_IP]),
    "pnpn_prs_res_part3_cuda": (None, [_P] * 4 + [_DP, _IP]),
    "pnpn_vel_res_update_cuda": (None, [_P] * 9 + [_IP]),
    # native API
    "nb_last_error": (ctypes.c_char_p, []),
    "nb_version": (ctypes.c_char_p, []),
    "nb_gll": (_I, [_I, _DP, _DP, _DP]),
    "nb_box_gs_maps": (_I, [_IP, _IP, _I, _IP, _IP, _IP, _IP, _IP, _IP, _IP]),
    "nb_mesh_read_nmsh": (_I, [ctypes.c_char_p, _IP, _IP, _DP, _IP, _IP]),
    "nb_mesh_write_nmsh": (_I, [ctypes.c_char_p, _I, _IP, _DP]),
    "nb_fld_write": (_I, [ctypes.c_char_p, _I, _I, _DP, _DP, _DP, _DP, ctypes.c_double, _I]),
    "nb_mesh_gs_maps": (_I, [_I, _IP, _I, _IP, _IP, _IP, _IP, _IP, _IP, _IP, _IP]),
    "nb_problem_create_box": (_I, [_IP, _DP, _DP, _IP, _I, ctypes.c_double, _I,
                                   ctypes.POINTER(_P)]),
    "nb_problem_create_mesh": (_I, [_I, _IP, _DP, _I, ctypes.c_double, _I, ctypes.POINTER(_P)]),
    "nb_problem_destroy": (_I, [_P]),
    "nb_problem_sizes": (_I, [_P, ctypes.POINTER(ctypes.c_int64), _IP, _IP, _IP, _IP, _IP]),
    "nb_problem_field": (_I, [_P, ctypes.c_char_p, ctypes.POINTER(_P)]),
    "nb_problem_volume": (_I, [_P, _DP]),
    "nb_problem_set_coefficients": (_I, [_P, _P, _P, _I]),
    "nb_problem_set_coefficients_const": (_I, [_P, ctypes.c_double, ctypes.c_double, _P]),
    "nb_ax": (_I, [_P, _P, _P, _P]),
    "nb_problem_sync": (_I, [_P, _P]),
    "nb_ax_vector": (_I, [_P] * 8),
    "nb_ax_stress": (_I, [_P] * 8),
    "nb_solve_coupled": (_I, [_P, _I] + [_P] * 6 + [ctypes.POINTER(SolveOpts),
                                                  ctypes.POINTER(SolveResult), _P]),
    "nb_ax_update_p": (_I, [_P, _P, _P, _P, ctypes.c_double, _P, _P]),
    "nb_gs_add": (_I, [_P, _P, _P]),
    "nb_bc_apply": (_I, [_P, _P, _P]),
    "nb_solve": (_I, [_P, _P, _P, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveResult), _P]),
    "nb_glsc3_noalloc": (_I, [_P, _P, _P, _I, _DP, _P]),
    "nb_pc_apply": (_I, [_P, _I, _P, _P, _P]),
    "nb_hsmg_init": (_I, [_P, _I, _I, ctypes.c_double]),
    "nb_phmg_init": (_I, [_P, ctypes.POINTER(PhmgOpts)]),
    "nb_phmg_describe": (_I, [_P, _I, _I, _DP]),
    "nb_tamg_aggregate": (_I, [_I, _I, _IP, _I, _IP, _IP, _IP]),
    "nb_projection_create": (_I, [_P, _I, _P]),
    "nb_projection_destroy": (_I, [_P]),
    "nb_projection_clear": (_I, [_P, _P]),
    "nb_projection_project_on": (_I, [_P, _P, _P]),
    "nb_projection_project_back": (_I, [_P, _P, _P]),
    "nb_projection_reorthogonalize": (_I, [_P, _P]),
    "nb_projection_info": (_I, [_P, _IP, _IP, _DP, _P]),
    "nb_ortho": (_I, [_P, _P, _P]),
    "nb_batch_create": (_I, [ctypes.c_int64, _P]),
    "nb_batch_destroy": (None, [_P]),
    "nb_batch_submit": (_I, [_P, _P, _P, _P, ctypes.c_double, _I, _IP]),
    "nb_batch_submit_coef": (_I, [_P, _P, _P, _P, ctypes.c_double, _I, ctypes.c_double,
                                  ctypes.c_double, _IP]),
    "nb_batch_submit_solve": (_I, [_P, _P, _P, _P, ctypes.POINTER(SolveOpts), ctypes.c_double,
                                   ctypes.c_double, _IP]),
    "nb_batch_release": (_I, [_P, _I]),
    "nb_batch_run": (_I, [_P, _I, _IP, _P]),
    "nb_batch_result": (_I, [_P, _I, _IP, _P]),
    "nb_selftest_bounded_waits": (_I, [_IP, _IP]),
    "nb_batch_tuning": (_I, [_P, _I, _IP, ctypes.POINTER(ctypes.c_float), _IP]),
}

_lib = None


def load():
    """Load libnekob200.so and bind every symbol; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} not found: build it with `python neko_b200/build.py` "
            "(there is no fallback implementation)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status):
    if status != NB_OK:
        raise NekoB200Error(status, load().nb_last_error().decode(errors="replace"))
