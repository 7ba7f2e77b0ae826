"""Routing of the shot-sharded server (host logic, fake per-device servers)."""
import pytest

from mixedprecisionfaracoustic_b200.sharded import RoutingError, ShardedServer
from mixedprecisionfaracoustic_b200._abi import BP_ERR_BUDGET, BP_ERR_NOT_FOUND


class FakeCfg:
    def __init__(self, n, nt, nbytes=100):
        self.padded = (n, 1, n)
        self.nt = nt
        self.nbytes = nbytes


class FakeServer:
    def __init__(self, budget, steps, device):
        self.device, self.reqs, self.n = device, {}, 0

    def submit(self, cfg, med):
        self.n += 1
        self.reqs[self.n] = "queued"
        return self.n

    def poll(self, rid):
        return self.reqs[rid]

    def finish(self, rid):
        self.reqs[rid] = "done"

    def wait(self, rid, t):
        self.reqs[rid] = "done"

    def cancel(self, rid):
        self.reqs[rid] = "cancelled"

    def traces(self, rid, comp):
        return (self.device, rid, comp)

    def latency(self, rid):
        return 0.5

    def release(self, rid):
        del self.reqs[rid]

    def stats(self):
        return {"submitted": self.n, "admitted": self.n, "completed": sum(v == "done" for v in self.reqs.values()),
                "failed": 0, "cancelled": 0, "cell_updates": 0}

    def close(self):
        pass


def make(devs=(0, 1, 2), budget=1000):
    return ShardedServer(devs, budget, server_factory=FakeServer, bytes_of=lambda c: c.nbytes)


def test_least_outstanding_work_routing():
    s = make()
    big, small = FakeCfg(100, 100), FakeCfg(10, 100)
    g0 = s.submit(big, None)
    assert s.device_of(g0) == 0
    g1, g2 = s.submit(small, None), s.submit(small, None)
    assert (s.device_of(g1), s.device_of(g2)) == (1, 2)
    g3 = s.submit(small, None)                      # devices 1 and 2 each hold one small request
    assert s.device_of(g3) == 1
    assert s.outstanding == {0: 100 * 100 * 100, 1: 2 * 10 * 10 * 100, 2: 10 * 10 * 100}


def test_finished_requests_stop_counting():
    s = make(devs=(0, 1))
    g0 = s.submit(FakeCfg(100, 100), None)
    g1 = s.submit(FakeCfg(100, 50), None)
    assert s.device_of(g1) == 1
    s.servers[0].finish(s.route[g0][1])
    assert s.pick(FakeCfg(5, 5)) == 0               # device 0 has nothing left
    s.release(g1)
    assert s.outstanding[1] == 0
    assert s.traces(g0, "txx") == (0, s.route[g0][1], "txx")
    st = s.stats()
    assert st["submitted"] == 2 and set(st["devices"]) == {0, 1}


def test_budget_and_unknown_ids():
    s = make(budget=50)
    with pytest.raises(RoutingError) as e:
        s.submit(FakeCfg(10, 10, nbytes=51), None)
    assert e.value.code == BP_ERR_BUDGET
    with pytest.raises(RoutingError) as e:
        s.poll(12345)
    assert e.value.code == BP_ERR_NOT_FOUND
    with pytest.raises(ValueError):
        ShardedServer([], 10, server_factory=FakeServer, bytes_of=lambda c: 1)
