"""bp_rel_l2_device_noalloc (static device scratch, no allocation) against
bp_rel_l2_device (allocating) through the C ABI.

The file name sorts last so the entry point also runs after every other GPU
test in one process, with the library's device state already used; it passes
alone as well.  Both calls of a pair must agree to 1e-12 relative (the two
reductions sum in different orders in FP64), and with numpy to 1e-9.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2
from mixedprecisionfaracoustic_b200 import _abi

pytestmark = pytest.mark.gpu


def _call(fn, x, r):
    v = C.c_double()
    rc = fn(C.c_void_p(x.data_ptr()), C.c_void_p(r.data_ptr()), x.numel(), C.byref(v))
    return rc, v.value


@pytest.mark.parametrize("n", [1, 1000, (1 << 20) + 3, 16_777_216])
def test_noalloc_matches_allocating_entry_point_twice(n):
    import torch
    lib = _abi.load()
    g = torch.Generator(device="cuda").manual_seed(n)
    for rep in range(2):
        x = torch.randn(n, device="cuda", dtype=torch.float32, generator=g)
        r = x + 1e-3 * (rep + 1) * torch.randn(n, device="cuda", dtype=torch.float32, generator=g)
        rc_a, a = _call(lib.bp_rel_l2_device, x, r)
        rc_b, b = _call(lib.bp_rel_l2_device_noalloc, x, r)
        assert rc_a == _abi.BP_OK and rc_b == _abi.BP_OK, (rc_a, rc_b, lib.bp_last_error())
        assert abs(a - b) <= 1e-12 * a, (rep, a, b)
        ref = rel_l2(x.cpu().numpy(), r.cpu().numpy())
        assert abs(b - ref) <= 1e-9 * ref, (rep, b, ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = _abi.load()
    n = 16_777_216 + 1
    x = torch.zeros(n, device="cuda", dtype=torch.float32)
    rc, _ = _call(lib.bp_rel_l2_device_noalloc, x, x)
    assert rc == _abi.BP_ERR_ARG
    assert b"no-allocation limit" in lib.bp_last_error()
    # the allocating entry point still takes it
    rc, v = _call(lib.bp_rel_l2_device, x, x)
    assert rc == _abi.BP_OK and v == 0.0


def test_noalloc_on_seismograms():
    """Trace arrays of two runs of a small shot, compared both ways."""
    import torch
    from mixedprecisionfaracoustic_b200 import Simulation
    from mixedprecisionfaracoustic_b200.presets import config1
    lib = _abi.load()
    out = []
    for prec in ("fp32", "comp16"):
        cfg, med = config1(precision=prec, nx=96, nz=64, nt=200, npml=10, nrec=32)
        with Simulation(cfg, med) as s:
            s.run(cfg.nt)
            out.append(torch.from_numpy(np.ascontiguousarray(s.traces("txx"), dtype=np.float32)).cuda())
    rc_a, a = _call(lib.bp_rel_l2_device, out[1], out[0])
    rc_b, b = _call(lib.bp_rel_l2_device_noalloc, out[1], out[0])
    assert rc_a == 0 and rc_b == 0
    assert 0 < a < 1e-3
    assert abs(a - b) <= 1e-12 * a


def test_noalloc_works_with_no_device_memory_left():
    """The property the entry point exists for: it needs no device memory of
    its own.  After a first call (which loads the kernels and looks up the
    scratch array), the test takes every free byte of the device through torch,
    as a process that hands all memory to its own pool does; the call must
    still succeed and give the same value twice.  The allocating entry point
    is then expected to fail for lack of memory (reported, not required: the
    last partial page may still hold its small scratch)."""
    import torch
    lib = _abi.load()
    n = 1 << 20
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(n, device="cuda", dtype=torch.float32, generator=g)
    r = x + 1e-3 * torch.randn(n, device="cuda", dtype=torch.float32, generator=g)
    rc, want = _call(lib.bp_rel_l2_device_noalloc, x, r)
    assert rc == _abi.BP_OK
    torch.cuda.synchronize()
    hold = []
    try:
        for chunk in (1 << 30, 1 << 26, 1 << 22, 1 << 20):     # bytes; the last from 2 MB segments
            while True:
                try:
                    hold.append(torch.empty(chunk, dtype=torch.uint8, device="cuda"))
                except torch.OutOfMemoryError:
                    break
        free, _ = torch.cuda.mem_get_info()
        assert free < (64 << 20), free
        got = []
        for _ in range(2):
            rc, v = _call(lib.bp_rel_l2_device_noalloc, x, r)
            assert rc == _abi.BP_OK, lib.bp_last_error()
            got.append(v)
        assert got[0] == want and got[1] == want, (got, want)
        rc_alloc, _ = _call(lib.bp_rel_l2_device, x, r)
        print(f"free bytes while full: {free}; allocating entry point rc = {rc_alloc}")
    finally:
        hold.clear()
        torch.cuda.empty_cache()
