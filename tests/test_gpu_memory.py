"""Reuse of device memory across simulations (the per-device arena cache):
results do not depend on whether a shot gets a fresh or a reused block, and
bp_release_cached_memory hands the cached blocks back to the device."""
import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.presets import config1

pytestmark = pytest.mark.gpu


def run(cfg, med):
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        return {c: s.traces(c) for c in _abi.TRACES}, s.field("vwx")


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
def test_reused_blocks_give_identical_results(prec):
    lib = _abi.load()
    assert lib.bp_release_cached_memory(-1) == _abi.BP_OK
    cfg, med = config1(precision=prec, nx=300, nz=120, nt=150, npml=10, nrec=30)
    fresh = run(cfg, med)              # new block, cached on destroy
    reused = run(cfg, med)             # the cached block, dirty from the first run
    for c in _abi.TRACES:
        assert np.array_equal(fresh[0][c], reused[0][c]), c
    assert np.array_equal(fresh[1], reused[1])
    # a smaller shot may take a slightly larger cached block; a much smaller one gets its own
    small, smed = config1(precision=prec, nx=290, nz=118, nt=150, npml=10, nrec=30)
    a = run(small, smed)
    assert lib.bp_release_cached_memory(0) == _abi.BP_OK
    b = run(small, smed)
    for c in _abi.TRACES:
        assert np.array_equal(a[0][c], b[0][c]), c


def test_release_returns_the_memory():
    import torch
    lib = _abi.load()
    lib.bp_release_cached_memory(-1)
    cfg, med = config1(precision="fp32", nx=2000, nz=1000, nt=4, npml=20, nrec=10)
    with Simulation(cfg, med) as s:
        s.run(2)
        s.sync()
    torch.cuda.synchronize()
    free_cached, _ = torch.cuda.mem_get_info()
    assert lib.bp_release_cached_memory(0) == _abi.BP_OK
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after - free_cached > 100 << 20          # the ~250 MB arena came back
    assert lib.bp_release_cached_memory(-2) == _abi.BP_ERR_ARG
