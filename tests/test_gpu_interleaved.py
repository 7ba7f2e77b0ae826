"""The interleaved step kernel (one persistent launch per step; V and T tiles
of bands claimed in order, each T tile waiting for the V tiles of its own and
the neighbouring bands) against the two-phase register kernels: the same
per-chunk code, so every trace and field must be bit-identical (tolerance 0)
in 2D and 3D, at every precision and order, with the source and receivers
recorded by the T tiles or by the post-step kernel, alone and batched."""
import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Batch, Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.presets import config1, config3_shots

pytestmark = pytest.mark.gpu

F2 = ("vux", "vuz", "vwx", "vwz", "p", "txx", "tzz", "txz")
F3 = F2 + ("vuy", "vwy", "tyy", "txy", "tyz")


def run(cfg, med, kernel, chunks, fields):
    with Simulation(cfg, med) as s:
        s.set_kernel(kernel)
        assert s.kernel() == kernel
        for n in chunks:
            s.run(n)
        s.sync()                         # BP_ERR_TIMEOUT here if a band wait ran out
        return {c: s.traces(c) for c in _abi.TRACES}, {f: s.field(f) for f in fields}


def check(cfg, med, fields, nt):
    ref = run(cfg, med, "register", [nt], fields)
    got = run(cfg, med, "interleaved", [1, 32, 33, nt - 66], fields)
    for c in _abi.TRACES:
        assert np.array_equal(got[0][c], ref[0][c]), c
    for f in fields:
        assert np.array_equal(got[1][f], ref[1][f]), f


@pytest.mark.parametrize("prec", ["fp32", "comp16", "cbf16", "fp64"])
@pytest.mark.parametrize("order", [2, 4])
def test_interleaved_2d_equals_two_phase(prec, order):
    cfg, med = config1(precision=prec, nx=300, nz=260, nt=211, npml=10, order=order, nrec=64)
    check(cfg, med, F2, 211)


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
@pytest.mark.parametrize("order", [2, 4])
def test_interleaved_3d_equals_two_phase(prec, order):
    from test_gpu_parity import small_3d
    cfg, med = small_3d(order=order, precision=prec, n=30, nt=130)
    check(cfg, med, F3, 130)


def test_interleaved_reference_rounding_and_post_kernel():
    """FP32 with the reference's rounding, and a receiver on the border (never
    updated), which sends the recording to the post-step kernel."""
    cfg, med = config1(precision="fp32", nx=200, nz=150, nt=120, npml=8, nrec=32)
    cfg.rounding = "reference"
    cfg.rec_x = list(cfg.rec_x) + [0]
    cfg.rec_y = list(cfg.rec_y) + [0]
    cfg.rec_z = list(cfg.rec_z) + [0]
    check(cfg, med, F2, 120)


@pytest.mark.parametrize("prec,tile", [("fp32", (8, 1)), ("comp16", (8, 1)), ("cbf16", (4, 1)), ("fp32", (4, 2))])
def test_interleaved_batch_equals_single_shots(prec, tile):
    """Batches at the tile shapes the kernel takes (at most one unit per warp)."""
    shots = config3_shots(seed=15, nshots=5, nt=140, precision=prec, scale=0.1)
    shots[1][0].nt = 71
    singles = []
    for c, m in shots:
        with Simulation(c, m) as s:
            s.run(c.nt)
            singles.append((s.traces("txx"), s.traces("p")))
    b = Batch([c for c, _ in shots], [m for _, m in shots], steps_per_sync=32, ctas_per_sm=0, tile=tile,
              kernel="interleaved")
    assert b.tune()["kernel"] == "interleaved"
    b.run(140)
    b.sync()
    for i, (tx, tp) in enumerate(singles):
        assert np.array_equal(b.traces(i, "txx"), tx), i
        assert np.array_equal(b.traces(i, "p"), tp), i
    b.close()
