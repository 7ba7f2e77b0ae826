"""Checkpoint/restore of resident shot state, binary outputs and streamed trace
windows, through the C ABI (no counterpart in the reference; they serve the
batching/serving layer and large receiver sets)."""
import numpy as np
import pytest

from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200._abi import BiotError
from mixedprecisionfaracoustic_b200.presets import config0, config1

pytestmark = pytest.mark.gpu

FIELDS2 = ("vux", "vuz", "vwx", "vwz", "p", "txx", "tzz", "txz")


def case(kind, prec):
    if kind == "2d":
        cfg, med = config1(precision=prec, nx=200, nz=90, nt=240, npml=10, nrec=40)
        cfg.snap_steps, cfg.snap_fields = [60, 200], ["txx", "vux"]
    else:
        cfg, med = config0(precision=prec, order=4, n=24, npml=8, nt=120, nrec=16)
        cfg.snap_steps, cfg.snap_fields = [30, 100], ["txx", "vwz"]
    return cfg, med


def state(s, cfg):
    tr = {c: s.traces(c) for c in _abi.TRACES}
    fl = {f: s.field(f) for f in (FIELDS2 if cfg.dim == 2 else _abi.FIELDS)}
    sn = {(k, f): s.snapshot(k, f) for k in range(len(cfg.snap_steps)) for f in cfg.snap_fields}
    return tr, fl, sn


def same(a, b):
    for d1, d2 in zip(a, b):
        assert d1.keys() == d2.keys()
        for k in d1:
            assert np.array_equal(d1[k], d2[k]), k


@pytest.mark.parametrize("kind,prec", [("2d", "fp32"), ("2d", "comp16"), ("3d", "fp32"), ("3d", "fp64")])
def test_restore_continues_bit_identically(kind, prec):
    cfg, med = case(kind, prec)
    cut = cfg.nt // 3 + 7          # between the two snapshot steps of the 2D case, after the first
    with Simulation(cfg, med) as a:
        a.run(cut)
        img = a.checkpoint()
        a.run(cfg.nt - cut)
        ref = state(a, cfg)
        # rewind the same simulation and run the tail again
        a.restore(img)
        assert a.step == cut
        a.run(cfg.nt - cut)
        same(state(a, cfg), ref)
    with Simulation(cfg, med) as b:       # a fresh simulation picks up the image
        b.restore(img)
        b.run(cfg.nt - cut)
        same(state(b, cfg), ref)


def test_restore_rejects_another_configuration():
    cfg, med = case("2d", "fp32")
    with Simulation(cfg, med) as a:
        a.run(5)
        img = a.checkpoint()
    other, om = config1(precision="fp32", nx=208, nz=90, nt=240, npml=10, nrec=40)
    with Simulation(other, om) as b:
        with pytest.raises(BiotError) as e:
            b.restore(img)
        assert e.value.code == _abi.BP_ERR_ARG
        with pytest.raises(BiotError):
            b.restore(img[:100])


def _read_bin(path):
    raw = path.read_bytes()
    assert raw[:8] == b"BPBIN001"
    ver, dtype, ndims = np.frombuffer(raw[8:20], dtype="<i4")
    dims = np.frombuffer(raw[20:32], dtype="<i4")[:ndims]
    assert ver == 1 and dtype == 0
    return np.frombuffer(raw[32:], dtype="<f4").reshape(tuple(dims))


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_binary_outputs_equal_the_getters(kind, tmp_path):
    cfg, med = case(kind, "fp32")
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.write_binary_outputs(tmp_path)
        tr = _read_bin(tmp_path / "traces.bin")
        assert tr.shape == (5, cfg.nrec, cfg.nt)
        for i, c in enumerate(_abi.TRACES):
            assert np.array_equal(tr[i], s.traces(c))
        for k, st in enumerate(cfg.snap_steps):
            for f in cfg.snap_fields:
                a = _read_bin(tmp_path / f"{f}{st}.bin")
                assert np.array_equal(a, s.snapshot(k, f).reshape(a.shape)), (f, st)


def test_streamed_trace_windows_equal_the_final_traces():
    import torch
    cfg, med = case("2d", "fp32")
    cfg.rec_x = list(cfg.rec_x) + list(cfg.rec_x[:5])      # repeated receiver cells
    cfg.rec_z = list(cfg.rec_z) + list(cfg.rec_z[:5])
    cfg.rec_y = list(cfg.rec_y) + list(cfg.rec_y[:5])
    win = 48
    with Simulation(cfg, med) as s:
        nu, umap = s.receiver_map()
        assert nu == cfg.nrec - 5 and np.array_equal(umap[-5:], umap[:5])
        pinned = torch.empty((cfg.nt // win + 1, nu, win), dtype=torch.float32, pin_memory=True).numpy()
        it, k = 0, 0
        while it < cfg.nt:
            n = min(win, cfg.nt - it)
            s.run(n)
            buf = pinned[k]
            if n < win:
                buf = np.ascontiguousarray(buf[:, :n])
            s.copy_traces_async("vux", it, buf)
            if n < win:
                s.sync()
                pinned[k][:, :n] = buf
            it += n
            k += 1
        s.sync()
        full = s.traces("vux")
    got = np.concatenate([pinned[i][:, :min(win, cfg.nt - i * win)] for i in range(k)], axis=1)
    assert np.array_equal(got[umap], full)


def test_traces_into_caller_buffers():
    """traces(c, out=...) fills a caller's buffer (pinned host memory here)
    with the same values, and refuses a buffer of the wrong size or type."""
    import torch
    cfg, med = case("2d", "fp32")
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.sync()
        for c in _abi.TRACES:
            buf = torch.empty(cfg.nrec * cfg.nt, dtype=torch.float32, pin_memory=True).numpy()
            got = s.traces(c, out=buf)
            assert got.shape == (cfg.nrec, cfg.nt)
            assert np.shares_memory(got, buf)
            assert np.array_equal(got, s.traces(c))
        with pytest.raises(ValueError):
            s.traces("txx", out=np.zeros(cfg.nrec * cfg.nt - 1, dtype=np.float32))
        with pytest.raises(ValueError):
            s.traces("txx", out=np.zeros(cfg.nrec * cfg.nt, dtype=np.float64))
