"""Compensated BF16 storage (BP_PREC_CBF16): bf16 hi + 8-bit residual, i.e.
the top 24 bits of the fp32 word rounded to nearest even, with the FP32
path's arithmetic.

  codec      bit-exact: the stored coefficients are the FP32 path's rounded
             to 24 bits (numpy restatement of the rounding), every stored
             field value has a zero low byte
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
