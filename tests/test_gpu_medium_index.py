"""The indexed medium (bp_config.medium = BP_MEDIUM_AUTO): a shot whose cells
hold at most 256 distinct coefficient tuples reads a one-byte index per cell
and a table of the decoded tuples instead of its per-cell coefficient arrays.
The table holds the values the arrays decode to, so every trace and field must
be bit-identical (tolerance 0) to the same shot on its arrays
(BP_MEDIUM_DENSE), for every precision, rounding, order, dimension and kernel
family that reads coefficients; media with more tuples, and FP64 shots, stay
on the arrays."""
import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Batch, Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.biot import MEDIUM_KEYS, Medium
from mixedprecisionfaracoustic_b200.presets import config1, config3_shots

pytestmark = pytest.mark.gpu

F2 = ("vux", "vuz", "vwx", "vwz", "p", "txx", "tzz", "txz")
F3 = F2 + ("vuy", "vwy", "tyy", "txy", "tyz")


def run(cfg, med, medium, kernel="register", fields=F2, chunks=None):
    cfg.medium = medium
    with Simulation(cfg, med) as s:
        s.set_kernel(kernel)
        for n in (chunks or [cfg.nt]):
            s.run(n)
        s.sync()
        return (s.medium_tuples(), {c: s.traces(c) for c in _abi.TRACES}, {f: s.field(f) for f in fields},
                s.algorithmic_bytes()[0])


def same(a, b):
    for c in _abi.TRACES:
        assert np.array_equal(a[1][c], b[1][c]), c
    for f in a[2]:
        assert np.array_equal(a[2][f], b[2][f]), f


@pytest.mark.parametrize("prec,rounding", [("fp32", "fast"), ("fp32", "reference"), ("comp16", "fast"),
                                          ("cbf16", "fast")])
@pytest.mark.parametrize("order", [2, 4])
def test_indexed_2d_equals_dense(prec, rounding, order):
    cfg, med = config1(precision=prec, nx=300, nz=260, nt=181, npml=10, order=order, nrec=64)
    cfg.rounding = rounding
    dense = run(cfg, med, "dense")
    idx = run(cfg, med, "auto")
    assert dense[0] == 0
    assert 0 < idx[0] <= 256, idx[0]
    same(idx, dense)
    # the coefficient bytes drop to one index byte per cell and phase
    nvc = 7
    cb = 4 if prec == "fp32" else 3
    assert idx[3][0] == pytest.approx(dense[3][0] - nvc * cb + 1)


@pytest.mark.parametrize("prec", ["fp32", "comp16", "cbf16"])
@pytest.mark.parametrize("order", [2, 4])
def test_indexed_3d_equals_dense(prec, order):
    from test_gpu_parity import small_3d
    cfg, med = small_3d(order=order, precision=prec, n=30, nt=120)
    dense = run(cfg, med, "dense", fields=F3)
    idx = run(cfg, med, "auto", fields=F3)
    assert 0 < idx[0] <= 256
    same(idx, dense)


@pytest.mark.parametrize("kernel,prec", [("interleaved", "fp32"), ("interleaved", "comp16"), ("fused", "fp32"),
                                         ("fused", "cbf16"), ("fused", "comp16")])
def test_indexed_other_kernel_families(kernel, prec):
    cfg, med = config1(precision=prec, nx=260, nz=200, nt=130, npml=10, nrec=40)
    dense = run(cfg, med, "dense")
    idx = run(cfg, med, "auto", kernel=kernel, chunks=[1, 32, 33, 64])
    assert idx[0] > 0
    same(idx, dense)


def test_many_tuples_stay_dense_and_fp64_is_never_indexed():
    cfg, med = config1(precision="fp32", nx=120, nz=90, nt=60, npml=8, nrec=16)
    rng = np.random.default_rng(3)
    noisy = Medium({k: (v * (1 + 1e-3 * rng.standard_normal(v.shape))).astype(np.float32) for k, v in med.items()})
    a = run(cfg, noisy, "auto")
    b = run(cfg, noisy, "dense")
    assert a[0] == 0 and b[0] == 0
    same(a, b)
    cfg.precision = "fp64"
    assert run(cfg, med, "auto")[0] == 0


def test_indexed_batch_equals_single_dense_shots():
    shots = config3_shots(seed=21, nshots=4, nt=120, precision="cbf16", scale=0.1)
    singles = []
    for c, m in shots:
        singles.append(run(c, m, "dense")[1])
        c.medium = "auto"
    b = Batch([c for c, _ in shots], [m for _, m in shots], steps_per_sync=32)
    assert all(b.medium_tuples(i) > 0 for i in range(len(shots)))
    b.run(120)
    b.sync()
    for i, tr in enumerate(singles):
        for comp in ("txx", "p", "vux"):
            assert np.array_equal(b.traces(i, comp), tr[comp]), (i, comp)
    assert b.algorithmic_bytes() > 0
    b.close()


def test_staged_and_march_refuse_an_indexed_shot():
    cfg, med = config1(precision="fp32", nx=200, nz=100, nt=20, npml=8, nrec=8)
    cfg.medium = "auto"
    with Simulation(cfg, med) as s:
        assert s.medium_tuples() > 0
        for k in ("staged", "march"):
            with pytest.raises(RuntimeError):
                s.set_kernel(k)
