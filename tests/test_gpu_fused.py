"""The fused step kernel (one launch per step, two copies of the state)
against the two-phase register kernels: the same per-cell arithmetic, so every
seismogram and every field must be bit-identical (tolerance 0), whatever the
grid's fit to the kernel's 120-cell columns and row segments, the chunking of
the steps into pairs and odd tails, the order, the precision and the COMP16
rescale steps (one in a hundred)."""
import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.presets import config1

pytestmark = pytest.mark.gpu

FIELDS = ("vux", "vuz", "vwx", "vwz", "p", "txx", "tzz", "txz")


def run(cfg, med, kernel, chunks):
    with Simulation(cfg, med) as s:
        s.set_kernel(kernel)
        assert s.kernel() == kernel
        for n in chunks:
            s.run(n)
        s.sync()
        return {c: s.traces(c) for c in _abi.TRACES}, {f: s.field(f) for f in FIELDS}


CASES = [
    # (precision, order, physical nx, nz, npml)
    ("fp32", 2, 250, 90, 10),       # 3 columns, the last one partial; 7 row segments
    ("comp16", 2, 250, 90, 10),
    ("fp32", 4, 233, 77, 8),
    ("comp16", 4, 233, 77, 8),
    ("fp32", 2, 1100, 300, 20),     # more columns than one warp row
    ("comp16", 2, 97, 35, 5),       # one column
]


@pytest.mark.parametrize("prec,order,nx,nz,npml", CASES)
def test_fused_step_equals_the_two_phase_kernels(prec, order, nx, nz, npml):
    nt = 231                                            # crosses the rescale steps 100 and 200
    cfg, med = config1(precision=prec, nx=nx, nz=nz, nt=nt, npml=npml, order=order, nrec=min(64, nx))
    ref_tr, ref_f = run(cfg, med, "register", [nt])
    got_tr, got_f = run(cfg, med, "fused", [37, 64, 1, 2, 127])   # odd tails, graph replays, pairs
    for c in _abi.TRACES:
        assert np.array_equal(got_tr[c], ref_tr[c]), c
    for f in FIELDS:
        assert np.array_equal(got_f[f], ref_f[f]), f
    assert np.abs(ref_tr["txx"]).max() > 0


def test_fused_step_launch_count_and_profile():
    cfg, med = config1(precision="fp32", nx=300, nz=120, nt=100, npml=10, nrec=20)
    with Simulation(cfg, med) as s:
        s.set_kernel("fused")
        assert s.launches_per_step() == 1
        l0 = s.launch_count()
        s.run(64)                    # two replays of a 32-step graph: 32 fused launches + 1 advance each
        s.sync()
        assert s.launch_count() - l0 == 66
        ms, bpc = s.profile_fused(10)
        # fields once each way, coefficients once: one index byte for the
        # layered (indexed) medium, 12 words on the per-cell arrays
        assert ms > 0 and bpc == 2 * 8 * 4 + (1 if s.medium_tuples() else 12 * 4)
    cfg.medium = "dense"
    with Simulation(cfg, med) as s:
        s.set_kernel("fused")
        assert s.profile_fused(4)[1] == 2 * 8 * 4 + 12 * 4


def test_fused_refused_where_it_does_not_apply():
    from mixedprecisionfaracoustic_b200._abi import BiotError
    from mixedprecisionfaracoustic_b200.presets import config0
    cfg, med = config0(precision="fp32", order=2, n=16, nt=10)
    with Simulation(cfg, med) as s:
        with pytest.raises(BiotError) as e:
            s.set_kernel("fused")
        assert e.value.code == _abi.BP_ERR_ARG
    cfg, med = config1(precision="fp32", nx=100, nz=50, nt=10, npml=5, nrec=10)
    cfg.rounding = "reference"
    with Simulation(cfg, med) as s:
        with pytest.raises(BiotError):
            s.set_kernel("fused")
