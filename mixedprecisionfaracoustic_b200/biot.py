"""Python host mirror of the reference program's interface, over the C ABI.

The reference (Float/main.cu, Half/main.cu) is one program: set up the
medium, run NT steps of Source -> FD_V -> FD_T, record five seismogram
components and some snapshots, write text files.  ``Simulation`` exposes the
same steps one call each (``run``, ``traces``, ``snapshot``,
``write_reference_outputs``); ``Batch`` and ``Server`` add multi-shot
execution and continuous-batching serving.  Every call goes through
``lib/libbiot_b200.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import BpConfig, BpMedium, BpServerStats, BpTune, check, fptr, iptr, load

MEDIUM_KEYS = ("rho", "rhof", "M", "C", "H", "H2mu", "mu", "C1", "C2")


@dataclass
class ShotConfig:
    """bp_config as a Python object (coordinates are padded, i.e. include the CPML)."""
    dim: int = 3
    nx: int = 128
    ny: int = 128
    nz: int = 128
    npml: int = 32
    order: int = 2
    precision: str = "fp32"
    nt: int = 3500
    dx: float = 0.01
    dt: float = 0.9e-6
    f0: float = 3000.0
    t0: float = 0.0
    pml_v0: float = 4000.0
    pml_r: float = 1e-6
    src: tuple = (96, 96, 52)            # (x, y, z), y ignored in 2D
    src_mask: int = _abi.SRC_TAU
    rec_x: Sequence[int] = ()
    rec_y: Sequence[int] = ()
    rec_z: Sequence[int] = ()
    snap_steps: Sequence[int] = ()
    snap_fields: Sequence[str] = ()
    snap_masks: Optional[Sequence[Sequence[str]]] = None
    snap_y: int = -1
    device: int = 0
    comp_coef_lo: int = 1
    dyn_scale: int = 1
    check_cfl: int = 0
    rounding: str = "fast"                # FP32: "fast" or "reference" (bp_config.rounding)
    medium: str = "auto"                  # "auto" (indexed where <= 256 tuples) or "dense" (bp_config.medium)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def padded(self) -> tuple:
        ny = self.ny + 2 * self.npml if self.dim == 3 else 1
        return (self.nx + 2 * self.npml, ny, self.nz + 2 * self.npml)

    @property
    def nrec(self) -> int:
        return len(self.rec_x)

    def to_c(self) -> BpConfig:
        c = BpConfig()
        c.dim, c.nx, c.ny, c.nz, c.npml = self.dim, self.nx, self.ny if self.dim == 3 else 1, self.nz, self.npml
        c.order, c.precision, c.nt = self.order, _abi.PREC[self.precision], self.nt
        c.dx, c.dt, c.f0, c.t0 = self.dx, self.dt, self.f0, self.t0
        c.pml_v0, c.pml_r = self.pml_v0, self.pml_r
        c.src_x, c.src_y, c.src_z = self.src[0], self.src[1], self.src[2]
        c.src_mask = self.src_mask
        rx = np.ascontiguousarray(self.rec_x, dtype=np.int32)
        rz = np.ascontiguousarray(self.rec_z, dtype=np.int32)
        ry = np.ascontiguousarray(self.rec_y if self.dim == 3 else np.zeros(len(rx)), dtype=np.int32)
        ss = np.ascontiguousarray(self.snap_steps, dtype=np.int32)
        self._keep = [rx, ry, rz, ss]
        c.nrec = len(rx)
        c.rec_x, c.rec_y, c.rec_z = iptr(rx), iptr(ry), iptr(rz)
        c.nsnap = len(ss)
        c.snap_steps = iptr(ss)
        c.snap_fields = _mask(self.snap_fields)
        if self.snap_masks is not None:
            sm = np.ascontiguousarray([_mask(m) for m in self.snap_masks], dtype=np.uint32)
            self._keep.append(sm)
            c.snap_masks = sm.ctypes.data_as(_abi.UIntP)
        c.snap_y = self.snap_y
        c.device, c.comp_coef_lo, c.dyn_scale, c.check_cfl = self.device, self.comp_coef_lo, self.dyn_scale, self.check_cfl
        c.rounding = _abi.ROUND[self.rounding]
        c.medium = _abi.MEDIUM[self.medium]
        return c


def _mask(names) -> int:
    m = 0
    for n in names:
        m |= 1 << _abi.FIELD[n]
    return m


class Medium(dict):
    """The nine cell-centred Biot coefficient arrays (float32, physical grid)."""

    def to_c(self) -> BpMedium:
        m = BpMedium()
        arrs = []
        for k in MEDIUM_KEYS:
            a = np.ascontiguousarray(self[k], dtype=np.float32)
            arrs.append(a)
            setattr(m, k, fptr(a))
        self._keep = arrs
        return m

    @staticmethod
    def from_stack(stack: np.ndarray, shape: tuple) -> "Medium":
        n = int(np.prod(shape))
        return Medium({k: stack[i * n:(i + 1) * n].reshape(shape) for i, k in enumerate(MEDIUM_KEYS)})


def reference_borehole_medium(nx: int, ny: int, nz: int) -> Medium:
    """create_model of the reference (Float/main.cu:1590-1655), built by the library."""
    lib = load()
    out = np.zeros(9 * nx * ny * nz, dtype=np.float32)
    check(lib.bp_medium_reference_borehole(nx, ny, nz, fptr(out)), "bp_medium_reference_borehole")
    return Medium.from_stack(out, (nz, ny, nx))


def biot_from_moduli(Ks, Kb, mu, Kf, rhos, rhof, phi, tort, eta, kappa, m_shape=8.0) -> dict:
    lib = load()
    out = (C.c_double * 9)()
    check(lib.bp_biot_from_moduli(Ks, Kb, mu, Kf, rhos, rhof, phi, tort, eta, kappa, m_shape, out),
          "bp_biot_from_moduli")
    return dict(zip(MEDIUM_KEYS, list(out)))


def shot_bytes(cfg: ShotConfig) -> int:
    """Device bytes the shot occupies while resident (what serving admission charges)."""
    lib = load()
    c = cfg.to_c()
    n = C.c_size_t()
    check(lib.bp_shot_bytes(C.byref(c), C.byref(n)), "bp_shot_bytes")
    return n.value


def cfl_limit(cfg: ShotConfig, medium: Medium) -> tuple:
    lib = load()
    c, m = cfg.to_c(), medium.to_c()
    dt, v = C.c_double(), C.c_double()
    check(lib.bp_cfl_limit(C.byref(c), C.byref(m), C.byref(dt), C.byref(v)), "bp_cfl_limit")
    return dt.value, v.value


class Simulation:
    """One shot resident on the GPU (bp_sim)."""

    def __init__(self, cfg: ShotConfig, medium: Medium):
        self.lib = load()
        self.cfg = cfg
        c, m = cfg.to_c(), medium.to_c()
        h = C.c_void_p()
        check(self.lib.bp_create(C.byref(c), C.byref(m), C.byref(h)), "bp_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.bp_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nsteps: int) -> None:
        check(self.lib.bp_run(self.h, int(nsteps)), "bp_run")

    def sync(self) -> None:
        check(self.lib.bp_sync(self.h), "bp_sync")

    def run_timed(self, nsteps: int) -> float:
        """Runs nsteps steps; returns their device time in ms (CUDA events on the sim's stream)."""
        ms = C.c_float()
        check(self.lib.bp_run_timed(self.h, int(nsteps), C.byref(ms)), "bp_run_timed")
        return ms.value

    def set_kernel(self, variant: str) -> None:
        """Kernel family: 'auto', 'register', 'staged', 'march' or 'fused' (the
        last three 2D FP32/COMP16 only)."""
        check(self.lib.bp_set_kernel(self.h, _abi.KERNELS[variant]), "bp_set_kernel")

    def kernel(self) -> str:
        """The kernel family that runs the steps."""
        v = C.c_int()
        check(self.lib.bp_get_kernel(self.h, C.byref(v)), "bp_get_kernel")
        return {k: n for n, k in _abi.KERNELS.items()}[v.value]

    def profile_fused(self, nsteps: int) -> tuple:
        """(ms per fused-kernel launch, algorithmic bytes per cell of one fused step)."""
        ms, b = C.c_float(), C.c_double()
        check(self.lib.bp_profile_fused(self.h, int(nsteps), C.byref(ms), C.byref(b)), "bp_profile_fused")
        return ms.value, b.value

    def set_graph_steps(self, steps: int) -> None:
        """Steps per captured CUDA graph (0: direct launches)."""
        check(self.lib.bp_set_graph_steps(self.h, int(steps)), "bp_set_graph_steps")

    @property
    def step(self) -> int:
        v = C.c_int()
        check(self.lib.bp_get_step(self.h, C.byref(v)), "bp_get_step")
        return v.value

    @property
    def dims(self) -> tuple:
        x, y, z = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.bp_get_dims(self.h, C.byref(x), C.byref(y), C.byref(z)), "bp_get_dims")
        return x.value, y.value, z.value

    def traces(self, comp, out: np.ndarray = None) -> np.ndarray:
        """(nrec, nt) float32 seismogram of component 'txx','tzz','vux','vwx','p'.

        out: a C-contiguous float32 array of nrec * nt elements to fill (for
        instance pinned host memory, which the copy reaches at full speed);
        a new array otherwise."""
        ci = _abi.TRACE[comp] if isinstance(comp, str) else int(comp)
        if out is None:
            out = np.zeros((self.cfg.nrec, self.cfg.nt), dtype=np.float32)
        elif out.dtype != np.float32 or not out.flags.c_contiguous or out.size != self.cfg.nrec * self.cfg.nt:
            raise ValueError("out must be a C-contiguous float32 array of nrec * nt elements")
        check(self.lib.bp_get_traces(self.h, ci, fptr(out), out.size), "bp_get_traces")
        return out.reshape(self.cfg.nrec, self.cfg.nt)

    def snapshot(self, k: int, fld: str) -> np.ndarray:
        n = C.c_size_t()
        check(self.lib.bp_snapshot_size(self.h, C.byref(n)), "bp_snapshot_size")
        out = np.zeros(n.value, dtype=np.float32)
        check(self.lib.bp_get_snapshot(self.h, k, _abi.FIELD[fld], fptr(out), out.size), "bp_get_snapshot")
        nx, ny, nz = self.dims
        return out.reshape((nz, nx) if out.size == nx * nz else (nz, ny, nx))

    def field(self, fld: str, f64: bool = True) -> np.ndarray:
        nx, ny, nz = self.dims
        if f64:
            out = np.zeros(nx * ny * nz, dtype=np.float64)
            check(self.lib.bp_get_field_f64(self.h, _abi.FIELD[fld], out.ctypes.data_as(_abi.DoubleP), out.size),
                  "bp_get_field_f64")
        else:
            out = np.zeros(nx * ny * nz, dtype=np.float32)
            check(self.lib.bp_get_field(self.h, _abi.FIELD[fld], fptr(out), out.size), "bp_get_field")
        return out.reshape((nz, ny, nx) if self.cfg.dim == 3 else (nz, nx))

    def coef(self, name: str) -> np.ndarray:
        """Device coefficient array (decoded to float) over the padded grid."""
        nx, ny, nz = self.dims
        out = np.zeros(nx * ny * nz, dtype=np.float32)
        check(self.lib.bp_get_coef(self.h, _abi.COEF[name], fptr(out), out.size), "bp_get_coef")
        return out.reshape((nz, ny, nx) if self.cfg.dim == 3 else (nz, nx))

    def energy(self) -> float:
        v = C.c_double()
        check(self.lib.bp_field_energy(self.h, C.byref(v)), "bp_field_energy")
        return v.value

    def scaling(self) -> dict:
        em, es, dyn, km, rm = C.c_int(), C.c_int(), C.c_float(), C.c_double(), C.c_double()
        check(self.lib.bp_get_scaling(self.h, C.byref(em), C.byref(es), C.byref(dyn), C.byref(km), C.byref(rm)),
              "bp_get_scaling")
        return {"em": em.value, "es": es.value, "dyn": dyn.value, "kmax": km.value, "rmax": rm.value}

    def profile_phases(self, nsteps: int) -> tuple:
        ms = (C.c_float * 3)()
        check(self.lib.bp_profile_phases(self.h, int(nsteps), ms), "bp_profile_phases")
        return tuple(ms)

    def algorithmic_bytes(self) -> tuple:
        b = (C.c_double * 2)()
        cells = C.c_longlong()
        check(self.lib.bp_algorithmic_bytes(self.h, b, C.byref(cells)), "bp_algorithmic_bytes")
        return (b[0], b[1]), cells.value

    def medium_tuples(self) -> int:
        """Distinct coefficient tuples of the indexed medium (0: per-cell arrays)."""
        n = C.c_int()
        check(self.lib.bp_get_medium_tuples(self.h, C.byref(n)), "bp_get_medium_tuples")
        return n.value

    def set_z_spacing(self, dz) -> None:
        """Variable grid along z: dz[k] = spacing (m) between padded rows k and
        k+1, nz + 2 npml - 1 values; FP32, order 2, before the first step."""
        d = np.ascontiguousarray(dz, dtype=np.float64)
        check(self.lib.bp_set_z_spacing(self.h, d.ctypes.data_as(_abi.DoubleP), d.size), "bp_set_z_spacing")

    def launches_per_step(self) -> int:
        """Kernels one step launches: 3, or 2 where the T phase records the
        receivers and injects the source itself."""
        n = C.c_int()
        check(self.lib.bp_launches_per_step(self.h, C.byref(n)), "bp_launches_per_step")
        return n.value

    def launch_count(self) -> int:
        n = C.c_longlong()
        check(self.lib.bp_launch_count(self.h, C.byref(n)), "bp_launch_count")
        return n.value

    def trace_rel_l2(self, ref: "Simulation", comp) -> float:
        ci = _abi.TRACE[comp] if isinstance(comp, str) else int(comp)
        v = C.c_double()
        check(self.lib.bp_trace_rel_l2(self.h, ref.h, ci, C.byref(v)), "bp_trace_rel_l2")
        return v.value

    def write_reference_outputs(self, directory: str) -> None:
        check(self.lib.bp_write_reference_outputs(self.h, str(directory).encode()), "bp_write_reference_outputs")

    def write_binary_outputs(self, directory: str) -> None:
        check(self.lib.bp_write_binary_outputs(self.h, str(directory).encode()), "bp_write_binary_outputs")

    def receiver_map(self) -> tuple:
        """(number of distinct receiver cells, distinct-cell index of each receiver)."""
        n = C.c_int()
        m = np.zeros(self.cfg.nrec, dtype=np.int32)
        check(self.lib.bp_receiver_map(self.h, C.byref(n), _abi.iptr(m)), "bp_receiver_map")
        return n.value, m

    def copy_traces_async(self, comp, it0: int, out: np.ndarray) -> None:
        """Enqueues the copy of steps [it0, it0 + out.shape[1]) of one component for
        every distinct receiver cell into out (float32 [nurec, n], C order); sync() waits."""
        ci = _abi.TRACE[comp] if isinstance(comp, str) else int(comp)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.ndim == 2
        check(self.lib.bp_copy_traces_async(self.h, ci, int(it0), int(out.shape[1]), _abi.fptr(out)),
              "bp_copy_traces_async")

    def checkpoint(self) -> bytes:
        """Image of the evolving state (fields, CPML memory, traces, snapshots, step)."""
        n = C.c_size_t()
        check(self.lib.bp_checkpoint_size(self.h, C.byref(n)), "bp_checkpoint_size")
        buf = (C.c_char * n.value)()
        check(self.lib.bp_checkpoint(self.h, buf, n.value), "bp_checkpoint")
        return bytes(buf)

    def restore(self, image: bytes) -> None:
        buf = C.create_string_buffer(image, len(image))
        check(self.lib.bp_restore(self.h, buf, len(image)), "bp_restore")


class Batch:
    """Many shots advanced by the same launches (bp_batch)."""

    def __init__(self, cfgs: Sequence[ShotConfig], media: Sequence[Medium], steps_per_sync: int = 0,
                 ctas_per_sm: int = 0, tile: Optional[tuple] = None, kernel: str = "auto"):
        """tile = (rows, segs[, tz]) fixes the register kernels' tile shape and
        kernel the family ('register', 'fused'); None / 'auto' (and any other 0
        setting) leave it to the autotuner."""
        self.lib = load()
        self.cfgs = list(cfgs)
        carr = (BpConfig * len(cfgs))(*[c.to_c() for c in cfgs])
        marr = (BpMedium * len(media))(*[m.to_c() for m in media])
        t = BpTune()
        t.steps_per_sync, t.ctas_per_sm = steps_per_sync, ctas_per_sm
        if tile is not None:
            t.tile_rows, t.tile_segs = tile[0], tile[1]
            t.tile_tz = tile[2] if len(tile) > 2 else 0
        t.kernel = _abi.KERNELS[kernel]
        h = C.c_void_p()
        check(self.lib.bp_batch_create(carr, marr, len(cfgs), C.byref(t), C.byref(h)), "bp_batch_create")
        self.h = h

    def run(self, nsteps: int) -> None:
        check(self.lib.bp_batch_run(self.h, int(nsteps)), "bp_batch_run")

    def sync(self) -> None:
        check(self.lib.bp_batch_sync(self.h), "bp_batch_sync")

    def run_timed(self, nsteps: int) -> float:
        """Runs nsteps and returns their device time in ms (CUDA events on the batch's stream)."""
        ms = C.c_float()
        check(self.lib.bp_batch_run_timed(self.h, int(nsteps), C.byref(ms)), "bp_batch_run_timed")
        return ms.value

    def traces(self, shot: int, comp) -> np.ndarray:
        ci = _abi.TRACE[comp] if isinstance(comp, str) else int(comp)
        c = self.cfgs[shot]
        out = np.zeros((c.nrec, c.nt), dtype=np.float32)
        check(self.lib.bp_batch_get_traces(self.h, shot, ci, fptr(out), out.size), "bp_batch_get_traces")
        return out

    def tune(self) -> dict:
        t = BpTune()
        check(self.lib.bp_batch_get_tune(self.h, C.byref(t)), "bp_batch_get_tune")
        return {"tile_rows": t.tile_rows, "tile_segs": t.tile_segs, "tile_tz": t.tile_tz,
                "steps_per_sync": t.steps_per_sync, "ctas_per_sm": t.ctas_per_sm,
                "kernel": {k: n for n, k in _abi.KERNELS.items()}[t.kernel]}

    def autotune(self, budget_steps: int) -> dict:
        """Runs the autotuner now within budget_steps (real) steps; returns the choice."""
        check(self.lib.bp_batch_autotune(self.h, int(budget_steps)), "bp_batch_autotune")
        return self.tune()

    def cell_updates(self) -> int:
        n = C.c_longlong()
        check(self.lib.bp_batch_cell_updates(self.h, C.byref(n)), "bp_batch_cell_updates")
        return n.value

    def medium_tuples(self, shot: int) -> int:
        n = C.c_int()
        check(self.lib.bp_batch_medium_tuples(self.h, int(shot), C.byref(n)), "bp_batch_medium_tuples")
        return n.value

    def algorithmic_bytes(self) -> float:
        """Algorithmic HBM bytes of one step of the whole batch."""
        v = C.c_double()
        check(self.lib.bp_batch_algorithmic_bytes(self.h, C.byref(v)), "bp_batch_algorithmic_bytes")
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.bp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching shot server with HBM-budget admission (bp_server)."""

    def __init__(self, hbm_budget_bytes: int, steps_per_sync: int = 100, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.bp_server_create(device, int(hbm_budget_bytes), steps_per_sync, C.byref(h)),
              "bp_server_create")
        self.h = h
        self.cfgs = {}

    def submit(self, cfg: ShotConfig, medium: Medium) -> int:
        c, m = cfg.to_c(), medium.to_c()
        rid = C.c_uint64()
        check(self.lib.bp_server_submit(self.h, C.byref(c), C.byref(m), C.byref(rid)), "bp_server_submit")
        self.cfgs[rid.value] = cfg
        return rid.value

    def poll(self, rid: int) -> str:
        s = C.c_int()
        check(self.lib.bp_server_poll(self.h, rid, C.byref(s)), "bp_server_poll")
        return _abi.REQ_STATES[s.value]

    def wait(self, rid: int, timeout_s: float = 600.0) -> None:
        check(self.lib.bp_server_wait(self.h, rid, float(timeout_s)), "bp_server_wait")

    def cancel(self, rid: int) -> None:
        check(self.lib.bp_server_cancel(self.h, rid), "bp_server_cancel")

    def traces(self, rid: int, comp) -> np.ndarray:
        ci = _abi.TRACE[comp] if isinstance(comp, str) else int(comp)
        c = self.cfgs[rid]
        out = np.zeros((c.nrec, c.nt), dtype=np.float32)
        check(self.lib.bp_server_get_traces(self.h, rid, ci, fptr(out), out.size), "bp_server_get_traces")
        return out

    def latency(self, rid: int) -> float:
        v = C.c_double()
        check(self.lib.bp_server_latency(self.h, rid, C.byref(v)), "bp_server_latency")
        return v.value

    def release(self, rid: int) -> None:
        check(self.lib.bp_server_release(self.h, rid), "bp_server_release")
        self.cfgs.pop(rid, None)

    def stats(self) -> dict:
        s = BpServerStats()
        check(self.lib.bp_server_get_stats(self.h, C.byref(s)), "bp_server_get_stats")
        return {k: getattr(s, k) for k, _ in BpServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.bp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
