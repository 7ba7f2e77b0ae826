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
