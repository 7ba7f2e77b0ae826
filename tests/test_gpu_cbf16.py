"""Compensated BF16 storage (BP_PREC_CBF16): bf16 hi + 8-bit residual, i.e.
the top 24 bits of the fp32 word rounded to nearest even, with the FP32
path's arithmetic.

  codec      bit-exact: the stored coefficients are the FP32 path's rounded
             to 24 bits (numpy restatement of the rounding), every stored
             field value has a zero low byte, and the kernels' vector and
             scalar encode/decode match the restatement on 2^26 random bit
             patterns plus the inf/NaN, largest-finite and carry cases
  accuracy   seismograms vs the oracle's FP64 run <= 1e-3 (the bound the
             reference-format COMP16 path is held to)
  kernels    the fused step kernel is bit-identical to the register tiles
"""
import numpy as np
import pytest

from conftest import rel_l2
from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.presets import config1
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rne24(a):
    """fp32 -> its top 24 bits, round to nearest even at bit 8 (finite values)."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    w = (b + 0x7F + ((b >> 8) & 1)) >> 8
    return (w << 8).astype(np.uint32).view(np.float32)


def test_stored_coefficients_are_the_fp32_ones_rounded_to_24_bits():
    cfg, med = config1(precision="fp32", nx=120, nz=60, nt=4, npml=8, nrec=10)
    with Simulation(cfg, med) as s:
        ref = {c: s.coef(c) for c in ("rho_x", "rho_z", "rhof", "cc1_x", "cc2_z", "C", "M", "H", "H2u", "mu_xz")}
    cfg.precision = "cbf16"
    with Simulation(cfg, med) as s:
        for c, v in ref.items():
            got = s.coef(c)
            assert np.array_equal(got.view(np.uint32), rne24(v).view(np.uint32)), c


@pytest.mark.parametrize("kind,order", [("2d", 2), ("2d", 4), ("3d", 2)])
def test_cbf16_within_1e3_of_fp64(kind, order):
    if kind == "2d":
        cfg, med = config1(precision="cbf16", nx=96, nz=64, nt=300, npml=10, order=order, nrec=48)
    else:
        from test_gpu_parity import small_3d
        cfg, med = small_3d(order=order, precision="cbf16")
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        tr = {c: s.traces(c) for c in ("txx", "tzz", "vux", "p")}
        f = s.field("txx")
    assert np.all((np.ascontiguousarray(f, dtype=np.float32).view(np.uint32) & 0xFF) == 0)
    c64 = cfg
    c64.precision = "fp64"
    o = O.Oracle(c64, med, O.FP64)
    o.run(c64.nt)
    for c in tr:
        err = rel_l2(tr[c], o.traces(c))
        assert err <= 1e-3, (c, err)
    o.close()


@pytest.mark.parametrize("nx,nz,npml", [(250, 90, 10), (97, 35, 5)])
def test_cbf16_fused_equals_register(nx, nz, npml):
    cfg, med = config1(precision="cbf16", nx=nx, nz=nz, nt=151, npml=npml, nrec=min(64, nx))
    out = {}
    for kern, chunks in (("register", [151]), ("fused", [33, 64, 54])):
        with Simulation(cfg, med) as s:
            s.set_kernel(kern)
            for n in chunks:
                s.run(n)
            out[kern] = ({c: s.traces(c) for c in _abi.TRACES}, s.field("vwz"), s.field("txz"))
    for c in _abi.TRACES:
        assert np.array_equal(out["fused"][0][c], out["register"][0][c]), c
    assert np.array_equal(out["fused"][1], out["register"][1])
    assert np.array_equal(out["fused"][2], out["register"][2])


def b24_host(bits):
    """The CBF16 rounding restated over uint32 bit patterns (all inputs):
    finite values RNE at bit 8; inf and NaN keep their top 24 bits, a NaN
    whose mantissa would vanish keeping bit 8 set."""
    b = bits.astype(np.uint64)
    special = (b & 0x7F800000) == 0x7F800000
    fin = (b + 0x7F + ((b >> 8) & 1)) >> 8
    spec = (b >> 8) | ((b & 0x7FFFFF) != 0).astype(np.uint64)
    w = np.where(special, spec, fin).astype(np.uint32)
    return (w >> 8).astype(np.uint16), (w & 0xFF).astype(np.uint8)


def device_codec(bits):
    import ctypes as C
    lib = _abi.load()
    v = bits.view(np.float32)
    hi = np.zeros(v.size, np.uint16)
    lo = np.zeros(v.size, np.uint8)
    _abi.check(lib.bp_cbf16_encode(_abi.fptr(v), v.size, hi.ctypes.data_as(C.POINTER(C.c_uint16)),
                                   lo.ctypes.data_as(C.POINTER(C.c_uint8))), "bp_cbf16_encode")
    dec = np.zeros(v.size, np.float32)
    _abi.check(lib.bp_cbf16_decode(hi.ctypes.data_as(C.POINTER(C.c_uint16)), lo.ctypes.data_as(C.POINTER(C.c_uint8)),
                                   v.size, _abi.fptr(dec)), "bp_cbf16_decode")
    return hi, lo, dec.view(np.uint32)


@pytest.mark.parametrize("n", [1 << 26, (1 << 20) + 3])
def test_cbf16_codec_bit_exact(n):
    """The kernels' vector and scalar encode/decode against the host rounding:
    random bit patterns (every class) plus every inf/NaN pattern's low 16 bits,
    the largest finite values, and the values whose rounding carries."""
    rng = np.random.default_rng(11)
    parts = [rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)]
    low = np.arange(1 << 16, dtype=np.uint32)
    for top in (0x7F800000, 0xFF800000, 0x7FFF0000, 0xFFFF0000, 0x7F7F0000, 0x00000000, 0x80000000):
        parts.append(top | low)
    parts.append(np.array([0x7F7FFFFF, 0xFF7FFFFF, 0x7F7FFF80, 0x7F7FFE80, 0x3F8000FF, 0x3F800080, 0x3F800180],
                          np.uint32))
    bits = np.concatenate(parts)
    if n % 4:                                          # a ragged tail through the scalar forms
        bits = bits[: bits.size - (bits.size % 4) - 1]
        assert bits.size % 4 == 3
    hi, lo, dec = device_codec(bits)
    eh, el = b24_host(bits)
    assert np.array_equal(hi, eh)
    assert np.array_equal(lo, el)
    expect = (eh.astype(np.uint32) << 16) | (el.astype(np.uint32) << 8)
    assert np.array_equal(dec, expect)
    # NaN stays NaN, inf stays inf, finite stays within half a unit of bit 8
    f = bits.view(np.float32)
    d = dec.view(np.float32)
    assert np.array_equal(np.isnan(d), np.isnan(f))
    fin = np.isfinite(f) & np.isfinite(d)
    err = np.abs(d[fin].astype(np.float64) - f[fin])
    assert np.all(err <= np.maximum(np.abs(f[fin].astype(np.float64)) * 2.0 ** -16, 2.0 ** -142))
