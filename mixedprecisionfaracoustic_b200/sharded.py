"""Shot-sharded serving over the GPUs of one process.

Shots are independent, so serving on several GPUs needs no data exchange: one
continuous-batching Server (bp_server) per device, and a router that sends
each request to the device with the least outstanding work, counted in
cell-updates (padded cells x steps) of the requests it holds that have not
finished, among the devices whose HBM budget can hold the request at all.
Request ids returned here are global; every other call is forwarded to the
device that owns the request.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

from ._abi import BP_ERR_BUDGET, BP_ERR_NOT_FOUND
from .replicas import shot_cost

_FINISHED = ("done", "failed", "cancelled")


class RoutingError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class ShardedServer:
    """One Server per device; least-outstanding-work routing."""

    def __init__(self, devices: Sequence[int], hbm_budget_bytes: int, steps_per_sync: int = 100,
                 server_factory: Optional[Callable] = None, bytes_of: Optional[Callable] = None):
        if not devices:
            raise ValueError("at least one device")
        if server_factory is None:
            from .biot import Server as server_factory
        if bytes_of is None:
            from .biot import shot_bytes as bytes_of
        self.devices = list(devices)
        self.budget = int(hbm_budget_bytes)
        self.servers = {d: server_factory(hbm_budget_bytes, steps_per_sync, d) for d in self.devices}
        self.bytes_of = bytes_of
        self.outstanding = {d: 0 for d in self.devices}
        self.route = {}            # global id -> (device, local id, cost, finished)
        self._next = 0

    def _settle(self) -> None:
        for gid, (d, rid, cost, fin) in list(self.route.items()):
            if not fin and self.servers[d].poll(rid) in _FINISHED:
                self.outstanding[d] -= cost
                self.route[gid] = (d, rid, cost, True)

    def pick(self, cfg) -> int:
        """The device a request would go to now."""
        if self.bytes_of(cfg) > self.budget:
            raise RoutingError(BP_ERR_BUDGET, "request can never fit the per-device HBM budget")
        self._settle()
        return min(self.devices, key=lambda d: (self.outstanding[d], d))

    def submit(self, cfg, medium) -> int:
        d = self.pick(cfg)
        rid = self.servers[d].submit(cfg, medium)
        cost = shot_cost(cfg)
        gid = self._next
        self._next += 1
        self.route[gid] = (d, rid, cost, False)
        self.outstanding[d] += cost
        return gid

    def _owner(self, gid: int):
        if gid not in self.route:
            raise RoutingError(BP_ERR_NOT_FOUND, f"unknown request {gid}")
        d, rid, _, _ = self.route[gid]
        return self.servers[d], rid

    def device_of(self, gid: int) -> int:
        self._owner(gid)
        return self.route[gid][0]

    def poll(self, gid: int) -> str:
        srv, rid = self._owner(gid)
        return srv.poll(rid)

    def wait(self, gid: int, timeout_s: float = 600.0) -> None:
        srv, rid = self._owner(gid)
        srv.wait(rid, timeout_s)

    def cancel(self, gid: int) -> None:
        srv, rid = self._owner(gid)
        srv.cancel(rid)

    def traces(self, gid: int, comp):
        srv, rid = self._owner(gid)
        return srv.traces(rid, comp)

    def latency(self, gid: int) -> float:
        srv, rid = self._owner(gid)
        return srv.latency(rid)

    def release(self, gid: int) -> None:
        srv, rid = self._owner(gid)
        d, _, cost, fin = self.route.pop(gid)
        if not fin:
            self.outstanding[d] -= cost
        srv.release(rid)

    def stats(self) -> dict:
        per = {d: s.stats() for d, s in self.servers.items()}
        tot = {}
        for k in ("submitted", "admitted", "completed", "failed", "cancelled", "cell_updates"):
            tot[k] = sum(p[k] for p in per.values())
        return {"devices": per, **tot}

    def close(self) -> None:
        for s in self.servers.values():
            s.close()
        self.servers = {}
