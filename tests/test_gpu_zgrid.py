"""Variable grid along z (bp_set_z_spacing): the z differences divide by the
local spacing (forward: dz[z]; backward: the mean of dz[z-1], dz[z]).  Checked
against the oracle's restatement of the same scheme (REF32 within the FP32
bound, FP64 within 1e-4), against the uniform path when every spacing is dx,
for its effect on the wavefield, and for every refusal the entry point makes."""
import numpy as np
import pytest

from conftest import rel_l2
from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.presets import config1, z_spacing_step
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def graded_2d(nt=260):
    cfg, med = config1(precision="fp32", nx=160, nz=120, nt=nt, npml=10, order=2, nrec=64)
    cfg.dt = float(np.float32(cfg.dt / 2))      # the fine rows halve the stable step
    dz = z_spacing_step(cfg, z_fine=12, z_coarse=90, ratio=2.0)
    return cfg, med, dz


def gpu(cfg, med, dz=None, kernel="auto"):
    with Simulation(cfg, med) as s:
        if dz is not None:
            s.set_z_spacing(dz)
        s.set_kernel(kernel)
        s.run(cfg.nt)
        return {c: s.traces(c) for c in _abi.TRACES}, s.kernel()


def oracle(cfg, med, dz, mode):
    o = O.Oracle(cfg, med, mode)
    if dz is not None:
        o.set_z_spacing(dz)
    o.run(cfg.nt)
    return {c: o.traces(c) for c in _abi.TRACES}


def test_graded_2d_matches_oracle():
    cfg, med, dz = graded_2d()
    got, kern = gpu(cfg, med, dz)
    assert kern == "register"
    ref = oracle(cfg, med, dz, O.REF32)
    f64 = oracle(cfg, med, dz, O.FP64)
    for c in ("txx", "tzz", "vux", "vwx", "p"):
        assert np.abs(ref[c]).max() > 0, c
        assert rel_l2(got[c], ref[c]) <= 1e-5, (c, rel_l2(got[c], ref[c]))
        assert rel_l2(got[c], f64[c]) <= 1e-4, (c, rel_l2(got[c], f64[c]))


def test_graded_3d_matches_oracle():
    from test_gpu_parity import small_3d
    cfg, med = small_3d(order=2, precision="fp32", n=24, nt=100)
    cfg.dt = float(np.float32(cfg.dt / 2))
    dz = z_spacing_step(cfg, z_fine=10, z_coarse=26, ratio=2.0)
    got, _ = gpu(cfg, med, dz)
    ref = oracle(cfg, med, dz, O.REF32)
    for c in ("txx", "tzz", "vux", "p"):
        assert rel_l2(got[c], ref[c]) <= 1e-5, (c, rel_l2(got[c], ref[c]))


def test_uniform_spacing_equals_the_uniform_path_and_refinement_matters():
    cfg, med, dz = graded_2d(nt=200)
    flat = np.full_like(dz, float(np.float32(cfg.dx)))
    a, _ = gpu(cfg, med, flat)
    b, _ = gpu(cfg, med)
    c, _ = gpu(cfg, med, dz)
    for k in ("txx", "p", "vux"):
        # multiplying by the row factor 1/dx against dividing by dx: an ulp per difference
        assert rel_l2(a[k], b[k]) <= 1e-6, (k, rel_l2(a[k], b[k]))
    # the refined band changes what the receivers record
    assert max(rel_l2(c[k], b[k]) for k in ("txx", "tzz", "vux", "vwx")) >= 1e-3


def test_refusals():
    from mixedprecisionfaracoustic_b200._abi import BiotError
    cfg, med, dz = graded_2d(nt=20)
    with Simulation(cfg, med) as s:
        with pytest.raises(BiotError):
            s.set_z_spacing(dz[:-1])                 # wrong length
        bad = dz.copy()
        bad[2] = bad[2] / 2                          # a CPML row
        with pytest.raises(BiotError):
            s.set_z_spacing(bad)
        neg = dz.copy()
        neg[50] = -1.0
        with pytest.raises(BiotError):
            s.set_z_spacing(neg)
        s.set_z_spacing(dz)
        with pytest.raises(BiotError):
            s.set_kernel("fused")
        with pytest.raises(BiotError):
            s.set_z_spacing(dz)                      # once only
    with Simulation(cfg, med) as s:
        s.run(1)
        with pytest.raises(BiotError):
            s.set_z_spacing(dz)                      # before the first step
    for change in ({"order": 4}, {"precision": "comp16"}, {"rounding": "reference"}):
        c2, m2, d2 = graded_2d(nt=20)
        for k, v in change.items():
            setattr(c2, k, v)
        with Simulation(c2, m2) as s:
            with pytest.raises(BiotError):
                s.set_z_spacing(d2)
    # with the stability check on, dt is checked against the finest spacing
    from mixedprecisionfaracoustic_b200.biot import cfl_limit
    c3, m3, d3 = graded_2d(nt=20)
    c3.check_cfl = 1
    c3.dt = float(np.float32(0.9 * cfl_limit(c3, m3)[0]))    # stable for dx, not for dx / 2
    with Simulation(c3, m3) as s:
        with pytest.raises(BiotError) as e:
            s.set_z_spacing(d3)
        assert e.value.code == _abi.BP_ERR_CFL
