"""ctypes binding of the falm_b200 C ABI (include/falm_b200.h).

The shared library is built in-tree (``falm_b200/libfalm_b200.so``) by
``falm_b200.build``.  Loading fails loudly when it is missing: there is no
fallback implementation.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfalm_b200.so")

FALM_OK = 0
FALM_ERR_ARG = 1
FALM_ERR_TIMEOUT = 6
STATUS = {0: "ok", 1: "bad argument", 2: "cuda error", 3: "non-finite value", 4: "breakdown",
          5: "maxit", 6: "timeout", 7: "alloc", 8: "state", 9: "no alm", 10: "over capacity"}
FP64, MIXED = 0, 1
ADV = {"Upwind1": 0, "Upwind3": 1, "QUICK": 2, "UTOPIA": 3, "KK": 4}
SGS = {"Empty": 0, "Smagorinsky": 1, "CSM": 2}
LS = {"Empty": 0, "Jacobi": 1, "SOR": 2, "PBiCGStab": 4}
BC_CHANNEL, BC_CAVITY = 0, 1

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)


class Grid(ctypes.Structure):
    _fields_ = [("sx", ctypes.c_int), ("sy", ctypes.c_int), ("sz", ctypes.c_int), ("gc", ctypes.c_int),
                ("x", c_double_p), ("y", c_double_p), ("z", c_double_p),
                ("hx", c_double_p), ("hy", c_double_p), ("hz", c_double_p)]


class AlmDesc(ctypes.Structure):
    _fields_ = [("n_turbine", ctypes.c_int), ("n_blade", ctypes.c_int), ("n_ap_per_blade", ctypes.c_int),
                ("n_attack", ctypes.c_int), ("radius", ctypes.c_double), ("hub_radius", ctypes.c_double),
                ("euler_eps", ctypes.c_double), ("base", c_double_p), ("hub", c_double_p),
                ("tip_rate", c_double_p), ("motion", c_double_p), ("angle_type", c_int_p),
                ("ap_r", c_double_p), ("ap_chord", c_double_p), ("ap_twist", c_double_p),
                ("attack", c_double_p), ("cl", c_double_p), ("cd", c_double_p), ("pitch", ctypes.c_double)]


class Fields(ctypes.Structure):
    _fields_ = [("u", ctypes.c_void_p), ("uu", ctypes.c_void_p), ("p", ctypes.c_void_p),
                ("nut", ctypes.c_void_p), ("ff", ctypes.c_void_p)]


class StepStats(ctypes.Structure):
    _fields_ = [("it", ctypes.c_int), ("err", ctypes.c_double), ("divnorm", ctypes.c_double),
                ("outer", ctypes.c_int), ("status", ctypes.c_int),
                ("torque", ctypes.c_double * 8), ("thrust", ctypes.c_double * 8)]


V, D, I, LL, P = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p


class RmcpDesc(ctypes.Structure):
    _fields_ = [("n_turbine", ctypes.c_int), ("n_blade", ctypes.c_int), ("radius", ctypes.c_double),
                ("hub_radius", ctypes.c_double), ("blade_width", ctypes.c_double), ("blade_thick", ctypes.c_double),
                ("base", c_double_p), ("hub", c_double_p), ("angle", c_double_p), ("angle_type", c_int_p),
                ("tip_rate", c_double_p), ("n_station", ctypes.c_int), ("n_attack", ctypes.c_int),
                ("st_r", c_double_p), ("st_chord", c_double_p), ("st_twist", c_double_p), ("attack", c_double_p),
                ("cl", c_double_p), ("cd", c_double_p)]


class Transport(ctypes.Structure):
    """falm_transport: halo exchange and reductions between the slabs of a grid"""
    _fields_ = [("user", ctypes.c_void_p), ("exchange", ctypes.c_void_p), ("allreduce", ctypes.c_void_p)]

# name -> argtypes (restype is int unless listed in _RESTYPE)
SIGNATURES = {
    "falm_abi_version": [],
    "falm_create": [ctypes.POINTER(Grid), I, ctypes.POINTER(V)],
    "falm_destroy": [V],
    "falm_last_error": [V],
    "falm_kernel_launches": [V],
    "falm_cfd_init": [V, D, I, I, D],
    "falm_cfd_pseudo_u": [V, P, P, P, P, P, P, D, D, P],
    "falm_cfd_utouu": [V, P, P, P],
    "falm_cfd_poisson_rhs": [V, P, P, D, D, P],
    "falm_cfd_project_p": [V, P, P, P, P, P, D, P],
    "falm_cfd_sgs": [V, P, P, P],
    "falm_cfd_divergence": [V, P, P, P],
    "falm_eq_init": [V, I, I, D, D, I, I, D],
    "falm_eq_poisson_operator": [V, I, c_double_p],
    "falm_eq_set_matrix": [V, P],
    "falm_eq_solve": [V, P, P, P, P, c_int_p, c_double_p],
    "falm_eq_res": [V, P, P, P, P],
    "falm_eq_sor_sweep": [V, P, P, D, I, P],
    "falm_mv_mv": [V, P, P, P],
    "falm_mv_dot": [V, P, P, c_double_p, P],
    "falm_mv_dot_static": [I, I, I, I, I, P, P, c_double_p, P],
    "falm_step_adjoint": [V, ctypes.POINTER(Fields), ctypes.POINTER(Fields), D, D, D, P, P, P, P, P],
    "falm_adjoint_set_tol": [V, D],
    "falm_mv_normsq": [V, P, I, c_double_p, P],
    "falm_mv_maxdiag": [V, c_double_p],
    "falm_mv_scale": [V, P, LL, D, P],
    "falm_mv_axby": [V, D, P, D, P, P, LL, P],
    "falm_bc_init": [V, I, D],
    "falm_bc_set_inflow": [V, c_double_p, I, D],
    "falm_bc_ubc": [V, P, P, D, D, P],
    "falm_bc_pbc": [V, P, P],
    "falm_bc_uubc": [V, P, P],
    "falm_alm_init": [V, ctypes.POINTER(AlmDesc)],
    "falm_alm_build_aps": [I, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p, I, I, I, D, D,
                           c_double_p, c_double_p, c_double_p, c_double_p, c_double_p],
    "falm_alm_set_pitch": [V, D],
    "falm_alm_run": [V, P, P, D, P, c_double_p, c_double_p],
    "falm_alm_get_aps": [V, c_double_p, c_double_p, c_double_p, c_double_p],
    "falm_step": [V, ctypes.POINTER(Fields), D, D, P, ctypes.POINTER(StepStats)],
    "falm_bc_set_inlet_plane": [V, c_double_p, P],
    "falm_tavg": [V, P, P, I, LL, P],
    "falm_io_write_vector_file": [V, ctypes.c_char_p, ctypes.POINTER(P), c_int_p, I, ctypes.c_ulonglong, D, I, P],
    "falm_io_read_vector_file": [V, ctypes.c_char_p, ctypes.POINTER(P), c_int_p, I, ctypes.POINTER(ctypes.c_ulonglong),
                                 ctypes.POINTER(D), P],
    "falm_io_wait": [V],
    "falm_io_write_index_file": [ctypes.c_char_p, I, I, I, I, ctypes.POINTER(ctypes.c_ulonglong), c_double_p, c_int_p, I, I],
    "falm_io_write_cv_file": [V, ctypes.c_char_p],
    "falm_io_read_cv_file": [ctypes.c_char_p, c_int_p, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p],
    "falm_mesh_build": [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, I],
    "falm_debug_arm_wait_probe": [V, LL],
    "falm_rmcp_init": [V, ctypes.POINTER(RmcpDesc)],
    "falm_rmcp_run": [V, P, P, D, P, P, c_double_p, c_double_p],
    "falm_slab_init": [V, I, I, I, I, ctypes.POINTER(Transport)],
    "falm_slab_halo": [V, P, I, I, P],
    "falm_local_hub_create": [I, ctypes.POINTER(ctypes.c_void_p)],
    "falm_local_hub_transport": [V, I, ctypes.POINTER(Transport)],
    "falm_local_hub_destroy": [V],
    "falm_nccl_unique_id": [ctypes.POINTER(ctypes.c_ubyte * 128)],
    "falm_nccl_transport_create": [ctypes.POINTER(ctypes.c_ubyte * 128), I, I, ctypes.POINTER(Transport)],
    "falm_nccl_transport_destroy": [ctypes.POINTER(Transport)],
    "falm_profile_enable": [V, I],
    "falm_profile_read": [V, c_double_p, ctypes.POINTER(ctypes.c_longlong), I, I],
}
KERNEL_CLASSES = ["alm", "pseudo_u", "utouu_rhs", "res", "bicg_p", "sor", "mv_dot1", "bicg_s", "mv_dot2",
                  "bicg_xr", "pbc", "project", "ubc", "sgs_div", "other"]
_RESTYPE = {"falm_last_error": ctypes.c_char_p, "falm_kernel_launches": ctypes.c_longlong}

_lib = None


def load():
    """Load libfalm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"falm_b200: CUDA library not built ({LIB_PATH}); run falm_b200.build.build()")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, ctypes.c_int)
    _lib = lib
    return lib


class FalmError(RuntimeError):
    def __init__(self, code, where, detail=""):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)} ({code}) {detail}".strip())
