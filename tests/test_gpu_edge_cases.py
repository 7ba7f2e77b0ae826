"""Degenerate and ragged configurations on the GPU against the oracle: no CPML,
the smallest grids the stencil allows, no receivers, no source, and 3D extents
that leave partial tiles in every direction."""
import numpy as np
import pytest

from conftest import rel_l2
from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.biot import ShotConfig
from mixedprecisionfaracoustic_b200.presets import DT, DX, c0_coefficients, uniform_medium
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def shot(dim, n, npml, order=2, prec="fp32", nt=60, nrec=None, src_mask=_abi.SRC_TAU | _abi.SRC_P):
    nx, ny, nz = n
    px, py, pz = nx + 2 * npml, (ny + 2 * npml) if dim == 3 else 1, nz + 2 * npml
    sx, sy, sz = px // 2, py // 2, pz // 2
    if nrec is None:
        nrec = max(1, nx // 2)
    rx = [npml + (i * nx) // max(nrec, 1) for i in range(nrec)]
    cfg = ShotConfig(dim=dim, nx=nx, ny=ny if dim == 3 else 1, nz=nz, npml=npml, order=order, precision=prec, nt=nt,
                     dx=DX, dt=DT, f0=30.0, pml_v0=4000.0, pml_r=1e-6, src=(sx, sy, sz), src_mask=src_mask,
                     rec_x=rx, rec_y=[sy] * nrec, rec_z=[min(sz + 1, pz - 1)] * nrec)
    shape = (nz, ny, nx) if dim == 3 else (nz, nx)
    return cfg, uniform_medium(shape, c0_coefficients())


def compare(cfg, med, tol):
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.sync()
        got = {c: s.traces(c) for c in _abi.TRACES}
    o = O.Oracle(cfg, med, O.FP64 if cfg.precision in ("fp64", "comp16") else O.REF32)
    o.run(cfg.nt)
    for c in ("txx", "tzz", "vux", "p"):
        ref = o.traces(c)
        assert np.all(np.isfinite(got[c])), c
        if np.abs(ref).max() == 0:
            assert np.abs(got[c]).max() == 0, c
        else:
            assert rel_l2(got[c], ref) <= tol, (c, rel_l2(got[c], ref))


TOL = {"fp32": 1e-5, "fp64": 1e-10, "comp16": 1e-3}


@pytest.mark.parametrize("prec", ["fp32", "fp64", "comp16"])
@pytest.mark.parametrize("order", [2, 4])
def test_no_cpml_2d(prec, order):
    cfg, med = shot(2, (40, 1, 30), npml=0, order=order, prec=prec)
    compare(cfg, med, TOL[prec])


def test_no_cpml_3d():
    cfg, med = shot(3, (16, 14, 12), npml=0)
    compare(cfg, med, TOL["fp32"])


@pytest.mark.parametrize("dim,order", [(2, 2), (2, 4), (3, 2), (3, 4)])
def test_smallest_grids(dim, order):
    """One physical cell per axis inside a CPML just wide enough for the stencil."""
    npml = order // 2
    cfg, med = shot(dim, (1, 1, 1), npml=npml, order=order, nt=30, nrec=1)
    cfg.rec_z = [cfg.src[2]]                 # the single updated cell, which holds the source
    compare(cfg, med, TOL["fp32"])


@pytest.mark.parametrize("prec", ["fp32", "comp16"])
def test_ragged_3d_extents(prec):
    """x not a multiple of 4 or 128, y and z leaving partial tiles of both 3D tile shapes."""
    cfg, med = shot(3, (37, 11, 13), npml=6, order=4, prec=prec, nt=50)
    compare(cfg, med, TOL[prec])


def test_no_receivers_and_no_source():
    cfg, med = shot(2, (64, 1, 48), npml=8, nrec=0)
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.sync()
        assert s.traces("txx").shape == (0, cfg.nt)
        assert np.abs(s.field("txx")).max() > 0
    cfg, med = shot(2, (64, 1, 48), npml=8, src_mask=0)
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        s.sync()
        for f in ("vux", "vwz", "p", "txx", "txz"):
            assert np.abs(s.field(f)).max() == 0, f
        assert np.abs(s.traces("p")).max() == 0


def test_receivers_sharing_cells_and_out_of_order():
    """Receivers listed out of order and several on one cell each get that
    cell's seismogram: the same rows as a run with the distinct cells in order."""
    cfg, med = shot(2, (64, 1, 48), npml=8, nrec=6)
    order = [3, 0, 3, 5, 1, 0, 2, 4, 3]
    dup = shot(2, (64, 1, 48), npml=8, nrec=6)[0]
    dup.rec_x = [cfg.rec_x[i] for i in order]
    dup.rec_y = [cfg.rec_y[i] for i in order]
    dup.rec_z = [cfg.rec_z[i] for i in order]
    with Simulation(cfg, med) as a, Simulation(dup, med) as b:
        a.run(cfg.nt)
        b.run(cfg.nt)
        a.sync()
        b.sync()
        for c in _abi.TRACES:
            ta, tb = a.traces(c), b.traces(c)
            assert tb.shape == (len(order), cfg.nt)
            assert np.array_equal(tb, ta[order]), c


@pytest.mark.parametrize("dim,prec", [(2, "fp32"), (2, "comp16"), (3, "fp32"), (2, "fp64")])
def test_recording_in_the_t_phase_equals_the_post_kernel(dim, prec):
    """Where every receiver and the source lie in cells the T phase visits, the
    T phase records and injects itself; a receiver in the outermost row (z = 0,
    which no phase updates or visits) makes the library use the separate post
    kernel instead.  The receivers both runs share get bit-identical seismograms."""
    n = (40, 1, 30) if dim == 2 else (16, 14, 12)
    cfg, med = shot(dim, n, npml=4, prec=prec, nt=120, nrec=6)
    border = shot(dim, n, npml=4, prec=prec, nt=120, nrec=6)[0]
    border.rec_x = list(cfg.rec_x) + [cfg.rec_x[0]]
    border.rec_y = list(cfg.rec_y) + [cfg.rec_y[0]]
    border.rec_z = list(cfg.rec_z) + [0]
    with Simulation(cfg, med) as a, Simulation(border, med) as b:
        assert (a.launches_per_step(), b.launches_per_step()) == (2, 3)
        a.run(cfg.nt)
        b.run(cfg.nt)
        a.sync()
        b.sync()
        for c in _abi.TRACES:
            ta, tb = a.traces(c), b.traces(c)
            assert np.abs(ta).max() > 0, c
            assert np.array_equal(ta, tb[:cfg.nrec]), c
