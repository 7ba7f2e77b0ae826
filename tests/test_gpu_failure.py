"""Blow-up detection: a shot whose time step is above the stability limit (the
CFL check switched off) overflows within a few dozen steps; the library reports
BP_ERR_UNSTABLE at the next sync of a single shot or a batch, and the server
ends such a request as failed while the healthy requests of the same mix
finish with their usual results.  Nothing here faults the GPU: the failure is
plain floating-point overflow to inf/NaN."""
import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Batch, Server, Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200._abi import BiotError
from mixedprecisionfaracoustic_b200.biot import cfl_limit
from mixedprecisionfaracoustic_b200.presets import config1

pytestmark = pytest.mark.gpu


def unstable(prec="fp32"):
    cfg, med = config1(precision=prec, nx=200, nz=90, nt=300, npml=10, nrec=40)
    dt_lim, _ = cfl_limit(cfg, med)
    cfg.dt = float(3.0 * dt_lim)
    cfg.check_cfl = 0
    return cfg, med


def healthy(prec="fp32"):
    return config1(precision=prec, nx=180, nz=80, nt=120, npml=10, nrec=30)


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
def test_single_shot_reports_unstable(prec):
    cfg, med = unstable(prec)
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        with pytest.raises(BiotError) as e:
            s.sync()
        assert e.value.code == _abi.BP_ERR_UNSTABLE
        assert "step" in str(e.value)
    cfg, med = healthy(prec)
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.sync()                         # a stable run stays silent


def test_batch_reports_the_unstable_shot():
    (c1, m1), (c2, m2) = healthy(), unstable()
    c2.nx = c1.nx
    c2.nz = c1.nz
    c2.rec_x, c2.rec_y, c2.rec_z = c1.rec_x, c1.rec_y, c1.rec_z
    c2.src = c1.src
    m2 = m1
    b = Batch([c1, c2], [m1, m2])
    b.run(c1.nt)
    with pytest.raises(BiotError) as e:
        b.sync()
    assert e.value.code == _abi.BP_ERR_UNSTABLE and "shot 1" in str(e.value)
    b.close()


def test_server_fails_the_unstable_request_only():
    good, bad = healthy("comp16"), unstable("comp16")
    with Simulation(*good) as s:
        s.run(good[0].nt)
        ref = s.traces("txx")
    srv = Server(hbm_budget_bytes=4 << 30, steps_per_sync=20)
    r_bad = srv.submit(*bad)
    r_good = srv.submit(*good)
    srv.wait(r_bad, 300)
    srv.wait(r_good, 300)
    assert srv.poll(r_bad) == "failed"
    assert srv.poll(r_good) == "done"
    assert np.array_equal(srv.traces(r_good, "txx"), ref)
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
    srv.close()


def test_create_refuses_a_time_step_above_the_stability_limit():
    """With the check on, bp_create refuses dt above the limit (the check runs
    beside the device set-up, which is then undone), and a healthy shot created
    right after runs as usual."""
    cfg, med = unstable()
    cfg.check_cfl = 1
    with pytest.raises(BiotError) as e:
        Simulation(cfg, med)
    assert e.value.code == _abi.BP_ERR_CFL
    assert "stability limit" in str(e.value)
    cfg, med = healthy()
    cfg.check_cfl = 1
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.sync()
        assert np.isfinite(s.traces("txx")).all() and np.abs(s.traces("txx")).max() > 0


# ---- injected allocation failures (host-side fake of an exhausted device) ----
def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def leak_sized(prec="fp32"):
    """A shot whose arena (~100 MB) dwarfs the driver's own small allocations."""
    return config1(precision=prec, nx=1400, nz=700, nt=40, npml=10, nrec=30)


LEAK_SLACK = 8 << 20     # bytes of device memory the driver may take for itself (streams, events)


@pytest.mark.parametrize("nth", [1, 2])
def test_create_out_of_memory_leaves_nothing_behind(nth):
    """bp_create whose arena block (nth = 1) or medium staging block (nth = 2)
    cannot be had returns BP_ERR_OOM and holds no device memory afterwards; the
    next create on the same device works and gives the usual results."""
    lib = _abi.load()
    cfg, med = leak_sized()
    with Simulation(cfg, med) as s:      # first: loads the kernels, fills the cache
        s.run(cfg.nt)
        want = s.traces("txx")
    assert lib.bp_release_cached_memory(-1) == _abi.BP_OK
    before = _free_bytes()
    assert lib.bp_debug_fail_allocation(nth) == _abi.BP_OK
    try:
        with pytest.raises(BiotError) as e:
            Simulation(cfg, med)
        assert e.value.code == _abi.BP_ERR_OOM, str(e.value)
    finally:
        lib.bp_debug_fail_allocation(0)
    assert lib.bp_release_cached_memory(-1) == _abi.BP_OK
    assert abs(_free_bytes() - before) <= LEAK_SLACK
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        assert np.array_equal(s.traces("txx"), want)


def test_batch_create_out_of_memory_releases_the_shots_already_made():
    lib = _abi.load()
    shots = [leak_sized() for _ in range(3)]
    Batch([c for c, _ in shots[:1]], [m for _, m in shots[:1]]).close()     # warm: kernels, streams
    assert lib.bp_release_cached_memory(-1) == _abi.BP_OK
    before = _free_bytes()
    assert lib.bp_debug_fail_allocation(5) == _abi.BP_OK   # the third shot's arena block
    try:
        with pytest.raises(BiotError) as e:
            Batch([c for c, _ in shots], [m for _, m in shots])
        assert e.value.code == _abi.BP_ERR_OOM, str(e.value)
    finally:
        lib.bp_debug_fail_allocation(0)
    assert lib.bp_release_cached_memory(-1) == _abi.BP_OK
    assert abs(_free_bytes() - before) <= LEAK_SLACK


def test_server_request_fails_on_allocation_failure_and_the_rest_run():
    """A request whose shot cannot get its device memory at admission ends as
    failed and gives its budget back; the requests after it run normally and
    give the results they give alone."""
    lib = _abi.load()
    cfg, med = healthy()
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        want = s.traces("txx")
    srv = Server(hbm_budget_bytes=4 << 30, steps_per_sync=20)
    try:
        assert lib.bp_debug_fail_allocation(1) == _abi.BP_OK
        bad = srv.submit(cfg, med)
        srv.wait(bad, 120)
        assert srv.poll(bad) == "failed"
        lib.bp_debug_fail_allocation(0)
        good = srv.submit(cfg, med)
        srv.wait(good, 120)
        assert srv.poll(good) == "done"
        assert np.array_equal(srv.traces(good, "txx"), want)
        st = srv.stats()
        assert st["failed"] == 1 and st["completed"] == 1 and st["hbm_in_use"] == 0
    finally:
        lib.bp_debug_fail_allocation(0)
        srv.close()


def test_server_cancel_of_a_queued_and_of_a_resident_request():
    """bp_server_cancel on a request that is still queued (the budget holds one
    request at a time) and on one that is resident: both end as cancelled,
    their budget comes back, and the request that was not cancelled finishes
    with the result it gives alone."""
    from mixedprecisionfaracoustic_b200.biot import shot_bytes
    import time
    long_cfg, long_med = config1(precision="fp32", nx=400, nz=200, nt=4000, npml=10, nrec=20)
    cfg, med = healthy()
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        want = s.traces("txx")
    budget = max(shot_bytes(long_cfg), shot_bytes(cfg)) + (1 << 20)
    srv = Server(hbm_budget_bytes=budget, steps_per_sync=10)
    try:
        resident = srv.submit(long_cfg, long_med)
        queued = srv.submit(long_cfg, long_med)
        ok = srv.submit(cfg, med)
        t0 = time.time()
        while srv.poll(resident) != "running":
            assert time.time() - t0 < 60
            time.sleep(0.01)
        assert srv.poll(queued) == "queued"
        srv.cancel(queued)
        srv.cancel(resident)
        for rid in (resident, queued, ok):
            srv.wait(rid, 300)
        assert srv.poll(resident) == "cancelled" and srv.poll(queued) == "cancelled"
        assert srv.poll(ok) == "done"
        assert np.array_equal(srv.traces(ok, "txx"), want)
        with pytest.raises(BiotError) as e:
            srv.traces(resident, "txx")
        assert e.value.code == _abi.BP_ERR_STATE
        st = srv.stats()
        assert st["cancelled"] == 2 and st["completed"] == 1 and st["hbm_in_use"] == 0
    finally:
        srv.close()
