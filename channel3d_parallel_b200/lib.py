"""ctypes binding of libc3d.so (the C-ABI of include/c3d.h).

The library is built in-tree (``channel3d_parallel_b200/libc3d.so``); loading
fails loudly when it is missing -- there is no CPU fallback.
"""
import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libc3d.so")

# status codes (include/c3d.h)
OK = 0
ERR_PARAM = -1
ERR_CUDA = -2
ERR_NAN = -3
ERR_HANDLE = -4
ERR_IO = -5
ERR_UNSUPPORTED = -6
ERR_NO_DEVICE = -7
WARN_NOT_CONVERGED = 1

FIELD = dict(U=1, V=2, W=3, P=4, RHS_P=5, P_INTERIM=6, RHS_U=7, RHS_V=8, RHS_W=9,
             U_WORK=10, V_WORK=11, W_WORK=12, U_REG=13, V_REG=14, W_REG=15,
             HU_INTERIOR=16, HV_INTERIOR=17, HW_INTERIOR=18, HC_EXTERIOR=19)
MARKER = dict(FB=40, UB=41, XB=42, YB=43, ZB=44, NORMALS=45, SB=46, E1NH_EXT=47, E1NHC_EXT=48)
POISSON_FP64, POISSON_MIXED, POISSON_MIXED_UNREFINED = 0, 1, 2
PRECOND_NONE, PRECOND_JACOBI, PRECOND_LEARNED, PRECOND_SPAI, PRECOND_BAND = 0, 1, 2, 3, 4


class Dims(C.Structure):
    _fields_ = [(n, C.c_int32) for n in
                ("nx", "ny", "nz", "nxg", "nyg", "nzg", "nxp", "nzp", "nym", "nb")]


class Stats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("poisson_solves", C.c_int64),
                ("bicgstab_solves", C.c_int64), ("bicgstab_iters", C.c_int64),
                ("last_bicgstab_iters", C.c_int32), ("refinement_sweeps", C.c_int32),
                ("precond_fallbacks", C.c_int64), ("last_residual", C.c_double),
                ("dPdx", C.c_double), ("dPdy", C.c_double), ("dPdz", C.c_double),
                ("t", C.c_double), ("dt", C.c_double), ("qflow_x_0", C.c_double),
                ("status", C.c_int32), ("precond_mode", C.c_int32),
                ("last_bicgstab_ms", C.c_double), ("bicgstab_ms", C.c_double),
                ("slab_cluster", C.c_int32 * 2), ("slab_narrow", C.c_int32 * 2),
                ("qflow_y_0", C.c_double), ("qflow_z_0", C.c_double),
                ("precond_builds", C.c_int64), ("precond_build_ms", C.c_double),
                ("ib_rows", C.c_int32 * 2)]


_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I64x3 = C.POINTER(C.c_int64)
_INT = C.c_int

# name -> argtypes (all return int unless noted)
PROTOTYPES = {
    "c3d_create": [C.c_char_p, C.POINTER(C.c_int)],
    "c3d_create_from_text": [C.c_char_p, C.POINTER(C.c_int)],
    "c3d_destroy": [_INT],
    "c3d_set_grid": [_INT, _D, _D, _D],
    "c3d_get_dims": [_INT, C.POINTER(Dims)],
    "c3d_get_grid": [_INT, _D, _D, _D, _D, _D, _D],
    "c3d_last_error": [_INT],
    "c3d_upload": [_INT, _INT, _D, _I64x3, _I64x3],
    "c3d_download": [_INT, _INT, _D, _I64x3, _I64x3],
    "c3d_set_scalars": [_INT, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double],
    "c3d_synchronize": [_INT],
    "c3d_time_step_rk3": [_INT, _INT],
    "c3d_time_step_rk3_host": [_INT, _D, _D, _D, _INT],
    "c3d_time_step_euler": [_INT, _INT],
    "c3d_write_snapshot": [_INT, C.c_char_p, _INT],
    "c3d_read_snapshot": [_INT, C.c_char_p],
    "c3d_compute_statistics": [_INT, _D, _D],
    "c3d_write_statistics": [_INT, C.c_char_p, _INT],
    "c3d_monitor": [_INT, _D],
    "c3d_compute_dt": [_INT, _D],
    "c3d_compute_mean_mass_flow_u": [_INT, _D],
    "c3d_compute_mean_mass_flow_v": [_INT, _D],
    "c3d_compute_mean_mass_flow_w": [_INT, _D],
    "c3d_set_flow_targets": [_INT, C.c_double, C.c_double, C.c_double],
    "c3d_compute_rhs_u": [_INT],
    "c3d_compute_rhs_v": [_INT],
    "c3d_compute_rhs_w": [_INT],
    "c3d_solve_poisson_equation": [_INT, _INT],
    "c3d_divergence": [_INT],
    "c3d_compute_non_IB_projection": [_INT, _INT],
    "c3d_apply_boundary_conditions": [_INT, _INT],
    "c3d_compute_dPx_for_constant_mass_flow": [_INT, _D],
    "c3d_compute_dPy_for_constant_mass_flow": [_INT, _D],
    "c3d_compute_dPz_for_constant_mass_flow": [_INT, _D],
    "c3d_compute_pressure": [_INT],
    "c3d_setup_IB_geometry": [_INT],
    "c3d_setup_IB_operators": [_INT],
    "c3d_compute_heaviside": [_INT],
    "c3d_regT": [_INT, _D],
    "c3d_regTc_1n": [_INT, _INT, _D],
    "c3d_regT_1n": [_INT, _D],
    "c3d_reg": [_INT, _INT, _D],
    "c3d_schur": [_INT, _D, _D],
    "c3d_bicgstab": [_INT, _D],
    "c3d_precond_apply": [_INT, _D, _D],
    "c3d_compute_IB_projection": [_INT],
    "c3d_set_mode": [_INT, _INT, _INT],
    "c3d_get_stats": [_INT, C.POINTER(Stats)],
    "c3d_check_divergence": [_INT, _D],
    "c3d_check_finite": [_INT],
    "c3d_last_step_time_ms": [_INT, _D],
    "c3d_kernel_launches": [_INT, C.POINTER(C.c_int64)],
    "c3d_profile_kernels": [_INT, _INT, _D, _INT],
    "c3d_mean_mass_flow_u_noalloc": [C.c_void_p, _INT, _INT, _INT, C.c_void_p, C.c_void_p,
                                     C.c_void_p],
    "c3d_precond_collect": [_INT, _INT, _INT, _INT],
    "c3d_precond_probe": [_INT],
    "c3d_precond_train": [_INT, _INT, C.c_double, _D],
    "c3d_precond_info": [_INT, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(C.c_int), _D],
    "c3d_precond_get_params": [_INT, _F, _INT],
    "c3d_precond_set_params": [_INT, _F, _INT, _F],
    "c3d_precond_eval": [_INT, _F, _F, _INT, _F, _F, _F, _D],
}
PRECOND_NPARAM = 22800
KERNEL_CLASSES = ("rhs_stage", "ghosts", "div_xfft", "spectral_yz", "xfft_inv", "grad_sub",
                  "massflow")

_lib = None


class C3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"c3d error {code}: {msg}")
        self.code = code


def load(path=None):
    """Load libc3d.so once and declare every prototype."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"{p} is missing: build it with `python -m channel3d_parallel_b200._build`")
    lib = C.CDLL(p)
    for name, args in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_char_p if name == "c3d_last_error" else C.c_int
    _lib = lib
    return lib


def check(rc, handle=0):
    if rc < 0:
        msg = load().c3d_last_error(handle)
        raise C3DError(rc, msg.decode() if msg else "")
    return rc


def dptr(a):
    """Pointer to the data of a contiguous float64 numpy array."""
    return a.ctypes.data_as(_D)


def fptr(a):
    """Pointer to the data of a contiguous float32 numpy array."""
    return a.ctypes.data_as(_F)


def box(lb, ub):
    return (C.c_int64 * 3)(*lb), (C.c_int64 * 3)(*ub)
