"""ctypes wrapper and build recipe of the C++/OpenMP restatement
(oracle/cpu_rk3.cpp) -- TEST AND BASELINE INFRASTRUCTURE ONLY.

The restatement advances the same state as ``channel_oracle`` (Fortran-indexed
arrays with an unused index 0) and is used as the timed CPU baseline of
``bench.py`` and checked against ``channel_oracle`` in ``tests/``.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_rk3.cpp")
LIB = os.path.join(HERE, "libc3d_cpu.so")
FLAGS = ["-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
         "-fcx-fortran-rules"]

_lib = None


def build(force=False, verbose=False):
    """g++ build of libc3d_cpu.so beside the source (rebuilt when older)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["g++"] + FLAGS + ["-o", LIB + ".tmp", SRC]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {SRC}:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    D = C.POINTER(C.c_double)
    lib.c3d_cpu_create.restype = C.c_void_p
    lib.c3d_cpu_create.argtypes = [C.c_int] * 3 + [D] * 11 + [C.c_double, C.c_double, C.c_int, C.c_int]
    lib.c3d_cpu_destroy.argtypes = [C.c_void_p]
    lib.c3d_cpu_field_size.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]
    lib.c3d_cpu_set_field.argtypes = [C.c_void_p, C.c_int, D]
    lib.c3d_cpu_get_field.argtypes = [C.c_void_p, C.c_int, D]
    lib.c3d_cpu_set_scalars.argtypes = [C.c_void_p] + [C.c_double] * 5
    lib.c3d_cpu_dpdx.restype = C.c_double
    lib.c3d_cpu_dpdx.argtypes = [C.c_void_p]
    lib.c3d_cpu_steps.argtypes = [C.c_void_p, C.c_int]
    lib.c3d_cpu_threads.argtypes = [C.c_void_p]
    lib.c3d_cpu_fft.argtypes = [C.c_int, D, C.c_int]
    lib.c3d_cpu_zgtsv.argtypes = [C.c_int, D, D, D, D]
    _lib = lib
    return lib


def fft(x, sign=-1):
    """Unnormalised DFT of a complex vector by the restatement's FFT."""
    buf = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).view(np.float64).copy()
    if load().c3d_cpu_fft(len(x), _ptr(buf), int(sign)):
        raise ValueError("length must be 2^a 3^b 5^c")
    return buf.view(np.complex128)


def zgtsv(dl, d, du, b):
    """Solution of the tridiagonal system by the restatement's zgtsv and info."""
    c = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64).copy()
    bl, bd, bu, bb = c(dl), c(d), c(du), c(b)
    info = load().c3d_cpu_zgtsv(len(d), _ptr(bl), _ptr(bd), _ptr(bu), _ptr(bb))
    return bb.view(np.complex128), info


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


FIELDS = {"U": 1, "V": 2, "W": 3, "P": 4, "P_interim": 5}


class CpuChannel:
    """The restatement's state for grid ``g`` (a ``channel_oracle.Grid``)."""

    def __init__(self, g, nthreads=0):
        lib = load()
        self.g = g
        p = g.p
        keep = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (g.x, g.y, g.z, g.xg, g.yg, g.zg, g.kxx, g.kzz, g.Dd, g.Dl, g.Du)]
        self._h = lib.c3d_cpu_create(g.nx, g.ny, g.nz, *[_ptr(a) for a in keep], float(p["nu"]),
                                     float(p["cfl"]), int(p["x_mass_cte"]), int(nthreads))
        if not self._h:
            raise ValueError("nxp and nzp must be products of 2, 3 and 5")
        self.threads = lib.c3d_cpu_threads(self._h)
        self.shapes = {"U": g.u_array().shape, "V": g.v_array().shape, "W": g.w_array().shape,
                       "P": g.p_array().shape, "P_interim": g.rhs_p_array().shape}

    def close(self):
        if self._h:
            load().c3d_cpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_field(self, name, a):
        buf = np.asfortranarray(a, dtype=np.float64).ravel(order="F")
        assert a.shape == self.shapes[name], (name, a.shape)
        if load().c3d_cpu_set_field(self._h, FIELDS[name], _ptr(buf)):
            raise ValueError(name)

    def get_field(self, name):
        n = C.c_int64(0)
        load().c3d_cpu_field_size(self._h, FIELDS[name], C.byref(n))
        buf = np.empty(n.value)
        load().c3d_cpu_get_field(self._h, FIELDS[name], _ptr(buf))
        return buf.reshape(self.shapes[name], order="F")

    def set_state(self, st):
        for name in ("U", "V", "W", "P"):
            self.set_field(name, getattr(st, name))
        load().c3d_cpu_set_scalars(self._h, st.dPdx, st.dPdy, st.dPdz, st.t, st.Qflow_x_0)

    def steps(self, n):
        if load().c3d_cpu_steps(self._h, int(n)):
            raise FloatingPointError("singular tridiagonal mode")

    @property
    def dPdx(self):
        return load().c3d_cpu_dpdx(self._h)
