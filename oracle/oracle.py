"""ctypes wrapper of the CPU oracle (liboracle.so, built from biot_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, to check or time against the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

REF32, FP64 = 0, 1
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        from mixedprecisionfaracoustic_b200._abi import BpConfig, BpMedium
        lib = C.CDLL(str(LIB))
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(BpConfig), C.POINTER(BpMedium), C.c_int]
        lib.orc_run.argtypes = [C.c_void_p, C.c_int]
        lib.orc_get_traces.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.c_size_t]
        lib.orc_get_field.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_size_t]
        lib.orc_get_snapshot.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_size_t]
        lib.orc_get_coef.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_size_t]
        lib.orc_get_profile.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_size_t]
        lib.orc_get_step.argtypes = [C.c_void_p]
        lib.orc_set_z_spacing.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_set_threads.argtypes = [C.c_int]
        lib.orc_medium_reference_borehole.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]
        lib.orc_f2h.restype = C.c_uint16
        lib.orc_f2h.argtypes = [C.c_float]
        lib.orc_h2f.restype = C.c_float
        lib.orc_h2f.argtypes = [C.c_uint16]
        lib.orc_load_ch.restype = C.c_float
        lib.orc_load_ch.argtypes = [C.c_uint16, C.c_int8]
        lib.orc_encode_array.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_uint16),
                                         C.POINTER(C.c_int8)]
        lib.orc_f2h_array.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_uint16)]
        lib.orc_ricker_ref.restype = C.c_float
        lib.orc_ricker_ref.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float]
        lib.orc_comp16_exponents.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int),
                                             C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        _lib = lib
    return _lib


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def borehole_medium(nx: int, ny: int, nz: int) -> np.ndarray:
    out = np.zeros(9 * nx * ny * nz, dtype=np.float32)
    load().orc_medium_reference_borehole(nx, ny, nz, _f(out))
    return out


def set_threads(n: int) -> None:
    load().orc_set_threads(int(n))


class Oracle:
    """CPU restatement of one shot: mode REF32 (the Float build's arithmetic) or FP64."""

    def __init__(self, cfg, medium, mode: int = REF32):
        lib = load()
        self.lib = lib
        self.cfg = cfg
        self._c = cfg.to_c()
        self._m = medium.to_c()
        self.h = lib.orc_create(C.byref(self._c), C.byref(self._m), mode)
        nx, ny, nz = cfg.padded
        self.shape = (nz, ny, nx) if cfg.dim == 3 else (nz, nx)
        self.ncell = nx * ny * nz

    def run(self, n: int) -> None:
        self.lib.orc_run(self.h, int(n))

    def set_z_spacing(self, dz) -> None:
        """Variable grid along z: dz[k] = spacing between padded rows k, k+1."""
        d = np.ascontiguousarray(dz, dtype=np.float64)
        assert self.lib.orc_set_z_spacing(self.h, _d(d), d.size) == 0

    @property
    def step(self) -> int:
        return self.lib.orc_get_step(self.h)

    def traces(self, comp) -> np.ndarray:
        from mixedprecisionfaracoustic_b200._abi import TRACE
        ci = TRACE[comp] if isinstance(comp, str) else int(comp)
        out = np.zeros((self.cfg.nrec, self.cfg.nt), dtype=np.float32)
        assert self.lib.orc_get_traces(self.h, ci, _f(out), out.size) == 0
        return out

    def field(self, name: str) -> np.ndarray:
        from mixedprecisionfaracoustic_b200._abi import FIELD
        out = np.zeros(self.ncell, dtype=np.float64)
        assert self.lib.orc_get_field(self.h, FIELD[name], _d(out), out.size) == 0
        return out.reshape(self.shape)

    def snapshot(self, k: int, name: str) -> np.ndarray:
        from mixedprecisionfaracoustic_b200._abi import FIELD
        nx, ny, nz = self.cfg.padded
        n = nx * nz if (self.cfg.dim == 3 and self.cfg.snap_y >= 0) else self.ncell
        out = np.zeros(n, dtype=np.float32)
        assert self.lib.orc_get_snapshot(self.h, k, FIELD[name], _f(out), out.size) == 0
        return out.reshape((nz, nx) if n == nx * nz else self.shape)

    def coef(self, name: str) -> np.ndarray:
        out = np.zeros(self.ncell, dtype=np.float64)
        rc = self.lib.orc_get_coef(self.h, name.encode(), _d(out), out.size)
        assert rc == 0, rc
        return out.reshape(self.shape)

    def profile(self, axis: int, which: int) -> np.ndarray:
        n = self.cfg.padded[axis]
        out = np.zeros(n, dtype=np.float64)
        assert self.lib.orc_get_profile(self.h, axis, which, _d(out), n) == 0
        return out

    def comp16_exponents(self, mu_padded=None):
        em, epml = C.c_int(), C.c_int()
        km, rm = C.c_float(), C.c_float()
        mp = None
        if mu_padded is not None:
            self._mu = np.ascontiguousarray(mu_padded, dtype=np.float32)
            mp = _f(self._mu)
        assert self.lib.orc_comp16_exponents(self.h, mp, C.byref(em), C.byref(epml), C.byref(km), C.byref(rm)) == 0
        return em.value, epml.value, km.value, rm.value

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def encode_ch(v: np.ndarray):
    """Compensated fp16 encoding of a float32 array (Half/main.cu:94-100)."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    hi = np.zeros(v.size, dtype=np.uint16)
    lo = np.zeros(v.size, dtype=np.int8)
    load().orc_encode_array(_f(v), v.size, hi.ctypes.data_as(C.POINTER(C.c_uint16)),
                            lo.ctypes.data_as(C.POINTER(C.c_int8)))
    return hi, lo


def f2h(v: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(v, dtype=np.float32)
    out = np.zeros(v.size, dtype=np.uint16)
    load().orc_f2h_array(_f(v), v.size, out.ctypes.data_as(C.POINTER(C.c_uint16)))
    return out
