"""Batched shots and the serving loop.

A shot's arithmetic depends only on its own arrays, so its traces are
bit-identical alone, in a batch, and in a server mix (the tolerance is 0).
"""
import time

import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Batch, Server, Simulation
from mixedprecisionfaracoustic_b200.presets import config3_shots, config4_requests

pytestmark = pytest.mark.gpu


def alone(cfg, med):
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        return s.traces("txx"), s.traces("p")


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
def test_batch_equals_single_shots(prec):
    shots = config3_shots(seed=3, nshots=5, nt=160, precision=prec, scale=0.08)
    b = Batch([c for c, _ in shots], [m for _, m in shots])
    b.run(160)
    b.sync()
    for i, (cfg, med) in enumerate(shots):
        tx, tp = alone(cfg, med)
        assert np.array_equal(b.traces(i, "txx"), tx), i
        assert np.array_equal(b.traces(i, "p"), tp), i
    t = b.tune()
    assert t["steps_per_sync"] > 0 and t["tile_rows"] > 0
    assert b.cell_updates() == sum(c.nt * (c.nx + 2 * c.npml - 2) * (c.nz + 2 * c.npml - 2) for c, _ in shots)
    b.close()


def test_batch_shots_with_different_lengths():
    shots = config3_shots(seed=5, nshots=3, nt=100, precision="fp32", scale=0.06)
    shots[1][0].nt = 40
    shots[2][0].nt = 130
    b = Batch([c for c, _ in shots], [m for _, m in shots], steps_per_sync=16, ctas_per_sm=2)
    b.run(200)
    for i, (cfg, med) in enumerate(shots):
        tx, _ = alone(cfg, med)
        assert np.array_equal(b.traces(i, "txx"), tx), i
    b.close()


def test_server_invariance_and_admission():
    """Requests submitted together into a budget that holds about three of them:
    some queue until others finish (admission), several are resident at once
    (continuous batching, 2D and 3D classes overlapping), and every result is
    bit-identical to the same shot run alone."""
    from mixedprecisionfaracoustic_b200.biot import shot_bytes
    reqs = config4_requests(seed=4, n=8, precision="fp32", scale=0.05, steps=(60, 200), include_3d=True)
    singles = [alone(c, m)[0] for c, m in reqs]
    sizes = [shot_bytes(c) for c, _ in reqs]
    budget = max(max(sizes), sum(sizes) // 3)
    assert sum(sizes) > budget
    srv = Server(hbm_budget_bytes=budget, steps_per_sync=20)
    ids = [srv.submit(c, m) for c, m in reqs]
    for rid in ids:
        srv.wait(rid, 300)
    for rid, ref in zip(ids, singles):
        assert srv.poll(rid) == "done"
        assert np.array_equal(srv.traces(rid, "txx"), ref)
        assert srv.latency(rid) > 0
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0
    assert st["max_resident"] >= 2
    assert st["hbm_in_use"] == 0
    srv.close()


def test_server_rejects_oversized_request():
    (c, m), = config4_requests(seed=9, n=1, scale=0.05, steps=(50, 60), include_3d=False)
    srv = Server(hbm_budget_bytes=1 << 20, steps_per_sync=10)
    from mixedprecisionfaracoustic_b200._abi import BiotError, BP_ERR_BUDGET
    with pytest.raises(BiotError) as e:
        srv.submit(c, m)
    assert e.value.code == BP_ERR_BUDGET
    srv.close()


def test_sharded_server_on_the_visible_devices():
    """The shot-sharded router over every visible GPU (one here): results are
    bit-identical to single runs, and the per-device totals add up."""
    import torch
    from mixedprecisionfaracoustic_b200.sharded import ShardedServer
    reqs = config4_requests(seed=6, n=5, precision="comp16", scale=0.05, steps=(60, 150), include_3d=True)
    singles = [alone(c, m)[0] for c, m in reqs]
    devs = list(range(torch.cuda.device_count()))
    srv = ShardedServer(devs, hbm_budget_bytes=8 << 30, steps_per_sync=20)
    ids = [srv.submit(c, m) for c, m in reqs]
    for gid in ids:
        srv.wait(gid, 300)
    for gid, ref in zip(ids, singles):
        assert srv.poll(gid) == "done"
        assert np.array_equal(srv.traces(gid, "txx"), ref)
        assert srv.device_of(gid) in devs
    assert srv.stats()["completed"] == len(reqs)
    for gid in ids:
        srv.release(gid)
    assert all(v == 0 for v in srv.outstanding.values())
    srv.close()


SHAPES_2D = [(8, 1), (4, 2), (16, 1), (8, 2), (4, 1), (32, 1), (4, 4)]
SHAPES_3D = [(8, 1, 1), (8, 1, 2), (8, 1, 4), (8, 1, 8), (16, 1, 4), (16, 1, 8), (4, 2, 2), (4, 1, 4)]


def _shots_3d(prec, n=2, nt=90):
    from mixedprecisionfaracoustic_b200.presets import c0_coefficients, uniform_medium
    from mixedprecisionfaracoustic_b200.biot import ShotConfig
    from mixedprecisionfaracoustic_b200 import _abi
    out = []
    for i, e in enumerate((22, 27)[:n]):
        npml = 6
        nxe = e + 2 * npml
        c = nxe // 2
        cfg = ShotConfig(dim=3, nx=e, ny=e + 3, nz=e - 2, npml=npml, order=2 + 2 * i, precision=prec, nt=nt,
                         dx=5.0, dt=4e-4, f0=30.0, pml_v0=3300.0, pml_r=1e-6, src=(c, c, c - 2),
                         src_mask=_abi.SRC_TAU | _abi.SRC_P, rec_x=list(range(npml, npml + e)),
                         rec_y=[c] * e, rec_z=[npml + 2] * e)
        out.append((cfg, uniform_medium((e - 2, e + 3, e), c0_coefficients())))
    return out


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
def test_every_tile_shape_gives_the_single_shot_results_2d(prec):
    """The autotuner's tile shapes only change which warp takes which 4-cell
    chunk: every shape gives bit-identical seismograms to the single runs."""
    shots = config3_shots(seed=11, nshots=3, nt=120, precision=prec, scale=0.07)
    singles = [alone(c, m) for c, m in shots]
    for shape in SHAPES_2D:
        b = Batch([c for c, _ in shots], [m for _, m in shots], steps_per_sync=16, ctas_per_sm=2, tile=shape,
                  kernel="register")
        b.run(120)
        b.sync()
        t = b.tune()
        assert (t["tile_rows"], t["tile_segs"]) == shape
        for i, (tx, tp) in enumerate(singles):
            assert np.array_equal(b.traces(i, "txx"), tx), (shape, i)
            assert np.array_equal(b.traces(i, "p"), tp), (shape, i)
        b.close()


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
def test_every_tile_shape_gives_the_single_shot_results_3d(prec):
    for order_shots in ([s] for s in _shots_3d(prec)):       # a batch holds one order
        singles = [alone(c, m) for c, m in order_shots]
        for shape in SHAPES_3D:
            b = Batch([c for c, _ in order_shots], [m for _, m in order_shots], steps_per_sync=16, ctas_per_sm=2,
                      tile=shape, kernel="register")
            b.run(90)
            b.sync()
            t = b.tune()
            assert (t["tile_rows"], t["tile_segs"], t["tile_tz"]) == shape
            for i, (tx, tp) in enumerate(singles):
                assert np.array_equal(b.traces(i, "txx"), tx), (shape, i)
                assert np.array_equal(b.traces(i, "p"), tp), (shape, i)
            b.close()


def test_autotune_picks_a_shape_and_keeps_results():
    shots = config3_shots(seed=12, nshots=4, nt=600, precision="fp32", scale=0.1)
    singles = [alone(c, m) for c, m in shots]
    b = Batch([c for c, _ in shots], [m for _, m in shots])
    t = b.autotune(560)
    assert t["tile_rows"] in (4, 8, 16, 32) and t["tile_segs"] in (1, 2, 4) and t["steps_per_sync"] > 0
    b.run(600)
    b.sync()
    for i, (tx, _) in enumerate(singles):
        assert np.array_equal(b.traces(i, "txx"), tx), i
    b.close()


def test_batch_rejects_a_bad_tile_shape():
    from mixedprecisionfaracoustic_b200._abi import BiotError, BP_ERR_ARG
    shots = config3_shots(seed=13, nshots=1, nt=20, precision="fp32", scale=0.05)
    for bad in ((3, 1), (8, 8), (64, 1), (2, 1)):
        with pytest.raises(BiotError) as e:
            Batch([c for c, _ in shots], [m for _, m in shots], tile=bad)
        assert e.value.code == BP_ERR_ARG


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
def test_fused_kernel_batch_equals_single_shots(prec):
    """The fused step kernel over a batch of shots of different sizes and
    lengths (tasks of every shot in one launch): bit-identical to single runs."""
    shots = config3_shots(seed=14, nshots=4, nt=150, precision=prec, scale=0.09)
    shots[2][0].nt = 67                     # finishes mid-chunk, on an odd step
    singles = [alone(c, m) for c, m in shots]
    b = Batch([c for c, _ in shots], [m for _, m in shots], steps_per_sync=32, ctas_per_sm=0, tile=(8, 1),
              kernel="fused")
    assert b.tune()["kernel"] == "fused"
    b.run(150)
    b.sync()
    for i, (tx, tp) in enumerate(singles):
        assert np.array_equal(b.traces(i, "txx"), tx), i
        assert np.array_equal(b.traces(i, "p"), tp), i
    b.close()
