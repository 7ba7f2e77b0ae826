"""The CUDA path against the CPU oracle at the benchmark configurations' real
sizes (the small-grid parity tests are in test_gpu_parity.py).

  c1   2D layered 4040 x 2040 (4000 x 2000 + 20-cell CPML), order 2, 200 steps:
       FP32 vs oracle REF32 <= 1e-5 on all five seismogram components, and
       <= 1e-5 on the final fields (the relative fluid velocities <= 1e-4, see
       test_gpu_parity.py); COMP16 vs oracle FP64 <= 1e-3; FP64 vs oracle FP64
       <= 1e-10.
  c0   3D homogeneous 200^3 (160^3 + 20-cell CPML), order 4, 60 steps: the
       wave has not reached the receivers yet, so the whole 3D fields are
       compared: FP32 vs REF32 <= 1e-5, COMP16 vs FP64 <= 1e-3.
  c2   the 128^3 crop of the 3D log-normal model (168^3 padded), 300 steps:
       FP32 vs REF32 <= 1e-5 and COMP16 vs FP64 <= 1e-3 on the seismograms of
       the surface receivers inside the crop.

Each oracle run is made once per session (fixtures) and shared.
"""
import numpy as np
import pytest

from conftest import rel_l2
from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200 import _abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS_2D = ("vux", "vuz", "vwx", "vwz", "p", "txx", "tzz", "txz")
FIELDS_3D = ("vux", "vuy", "vuz", "vwx", "vwy", "vwz", "p", "txx", "tyy", "tzz", "txy", "txz", "tyz")
FLUID = ("vwx", "vwy", "vwz")


def gpu_run(cfg, med, fields):
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.sync()
        return {c: s.traces(c) for c in _abi.TRACES}, {f: s.field(f) for f in fields}


def oracle_run(cfg, med, mode, fields):
    o = O.Oracle(cfg, med, mode)
    o.run(cfg.nt)
    out = {c: o.traces(c) for c in _abi.TRACES}, {f: o.field(f).reshape(-1) for f in fields}
    o.close()
    return out


def _with(cfg, precision):
    import copy
    c = copy.copy(cfg)
    c.precision = precision
    return c


# ---- c1 ---------------------------------------------------------------------
@pytest.fixture(scope="module")
def c1():
    from mixedprecisionfaracoustic_b200.presets import config1
    cfg, med = config1(precision="fp32", nt=200)
    assert cfg.padded == (4040, 1, 2040)
    return cfg, med, {"ref32": oracle_run(cfg, med, O.REF32, FIELDS_2D),
                      "fp64": oracle_run(cfg, med, O.FP64, FIELDS_2D)}


def test_c1_fp32_matches_oracle_at_full_size(c1):
    cfg, med, orc = c1
    tr, fl = gpu_run(cfg, med, FIELDS_2D)
    otr, ofl = orc["ref32"]
    for c in _abi.TRACES:
        if np.any(otr[c]):
            assert rel_l2(tr[c], otr[c]) <= 1e-5, (c, rel_l2(tr[c], otr[c]))
    for f in FIELDS_2D:
        tol = 1e-4 if f in FLUID else 1e-5
        assert rel_l2(fl[f].reshape(-1), ofl[f]) <= tol, (f, rel_l2(fl[f].reshape(-1), ofl[f]))


def test_c1_comp16_and_fp64_against_oracle_fp64_at_full_size(c1):
    cfg, med, orc = c1
    otr, ofl = orc["fp64"]
    tr16, _ = gpu_run(_with(cfg, "comp16"), med, ())
    for c in ("txx", "tzz", "vux", "vwx", "p"):
        assert rel_l2(tr16[c], otr[c]) <= 1e-3, (c, rel_l2(tr16[c], otr[c]))
    tr64, fl64 = gpu_run(_with(cfg, "fp64"), med, ("vux", "txx", "p"))
    for c in ("txx", "tzz", "vux", "vwx", "p"):
        assert rel_l2(tr64[c], otr[c]) <= 1e-10, c
    for f in ("vux", "txx", "p"):
        assert rel_l2(fl64[f].reshape(-1), ofl[f]) <= 1e-10, f


# ---- c0 ---------------------------------------------------------------------
@pytest.fixture(scope="module")
def c0():
    from mixedprecisionfaracoustic_b200.presets import config0
    cfg, med = config0(precision="fp32", order=4, nt=60)
    assert cfg.padded == (200, 200, 200)
    return cfg, med, {"ref32": oracle_run(cfg, med, O.REF32, FIELDS_3D),
                      "fp64": oracle_run(cfg, med, O.FP64, FIELDS_3D)}


def test_c0_order4_fp32_fields_match_oracle_at_full_size(c0):
    cfg, med, orc = c0
    _, fl = gpu_run(cfg, med, FIELDS_3D)
    _, ofl = orc["ref32"]
    for f in FIELDS_3D:
        assert np.linalg.norm(ofl[f]) > 0, f
        tol = 1e-4 if f in FLUID else 1e-5
        assert rel_l2(fl[f].reshape(-1), ofl[f]) <= tol, (f, rel_l2(fl[f].reshape(-1), ofl[f]))


def test_c0_order4_comp16_fields_within_1e3_of_oracle_fp64(c0):
    cfg, med, orc = c0
    _, fl = gpu_run(_with(cfg, "comp16"), med, FIELDS_3D)
    _, ofl = orc["fp64"]
    for f in FIELDS_3D:
        assert rel_l2(fl[f].reshape(-1), ofl[f]) <= 1e-3, (f, rel_l2(fl[f].reshape(-1), ofl[f]))


# ---- c2 crop ------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2crop():
    from mixedprecisionfaracoustic_b200.presets import config2, config2_crop
    base, med = config2(precision="fp32", nt=300)
    cfg, cm = config2_crop(base, med, size=128, precision="fp32", nt=300)
    del med
    assert cfg.padded == (168, 168, 168) and cfg.nrec > 100
    return cfg, cm, {"ref32": oracle_run(cfg, cm, O.REF32, ()), "fp64": oracle_run(cfg, cm, O.FP64, ())}


def test_c2_crop_fp32_and_comp16_against_oracle(c2crop):
    cfg, med, orc = c2crop
    tr, _ = gpu_run(cfg, med, ())
    tr16, _ = gpu_run(_with(cfg, "comp16"), med, ())
    otr, o64 = orc["ref32"][0], orc["fp64"][0]
    for c in ("txx", "tzz", "vux", "vwx", "p"):
        assert np.any(o64[c]), c
        assert rel_l2(tr[c], otr[c]) <= 1e-5, (c, rel_l2(tr[c], otr[c]))
        assert rel_l2(tr16[c], o64[c]) <= 1e-3, (c, rel_l2(tr16[c], o64[c]))
