"""The device COMP16 codec is bit-identical to the oracle's restatement of the
reference's store_ch / load_ch (Half/main.cu:59-100), and the COMP16
precompute reproduces the reference medium's scaled coefficients (method.md
section 15, Half/main.cu:967-1045)."""
import ctypes as C

import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Simulation, _abi
from mixedprecisionfaracoustic_b200.presets import reference_compat
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_encode_decode_bit_exact():
    rng = np.random.default_rng(7)
    v = (rng.standard_normal(400000) * 10.0 ** rng.uniform(-14, 4.7, 400000)).astype(np.float32)
    v[:8] = [0.0, -0.0, 1.0, -1.0, 6.1035156e-05, 6.0e-05, 65504.0, 1.0 + 2 ** -12]
    lib = _abi.load()
    hi = np.zeros(v.size, np.uint16)
    lo = np.zeros(v.size, np.int8)
    _abi.check(lib.bp_comp16_encode(_abi.fptr(v), v.size, hi.ctypes.data_as(C.POINTER(C.c_uint16)),
                                    lo.ctypes.data_as(C.POINTER(C.c_int8))), "bp_comp16_encode")
    rhi, rlo = O.encode_ch(v)
    assert np.array_equal(hi, rhi)
    assert np.array_equal(lo, rlo)
    dec = np.zeros(v.size, np.float32)
    _abi.check(lib.bp_comp16_decode(hi.ctypes.data_as(C.POINTER(C.c_uint16)), lo.ctypes.data_as(C.POINTER(C.c_int8)),
                                    v.size, _abi.fptr(dec)), "bp_comp16_decode")
    ol = O.load()
    ref = np.array([ol.orc_load_ch(int(h), int(l)) for h, l in zip(hi[:50000], lo[:50000])], np.float32)
    assert np.array_equal(dec[:50000], ref)


def test_scaled_coefficients_known_answers():
    """method.md 15.1-15.3 for the formation: 2^-em DT rho^-1 = 3.0381276459e-3,
    Aw = 0.9879429575, Bp = 2.0228360646e-4, 2^em DT H = 4.1182637215e-3,
    2^em DT C = 2.4139881134e-4, 2^em DT M = 2.4139881134e-3 (em = -23)."""
    cfg, med = reference_compat(nt=4, n=(32, 32, 24), npml=8, precision="comp16")
    with Simulation(cfg, med) as s:
        assert s.scaling()["em"] == -23
        c = {n: s.coef(n)[12, 9, 9] for n in ("rho_x", "cc1_x", "cc2_x", "H", "C", "M")}
    ref = {"rho_x": 3.0381276459e-3, "cc1_x": 0.9879429575, "cc2_x": 2.0228360646e-4, "H": 4.1182637215e-3,
           "C": 2.4139881134e-4, "M": 2.4139881134e-3}
    for k, v in ref.items():
        assert abs(c[k] / v - 1) < 2e-5, (k, c[k], v)      # hi + lo keeps ~19 bits
