"""Synthetic workload generators: seeded, with the configurations' shapes,
sizes and value distributions."""
import numpy as np

from mixedprecisionfaracoustic_b200.biot import cfl_limit
from mixedprecisionfaracoustic_b200.presets import (config0, config1, config2, config3_shots, config4_requests,
                                                    layered_coefficients, lognormal_field, reference_compat_config)


def test_reference_compat_geometry():
    c = reference_compat_config()
    assert c.padded == (192, 192, 192) and c.nt == 3500 and c.src == (96, 96, 52)
    assert c.nrec == 192 and set(c.rec_x) == {96} and list(c.rec_z) == list(range(192))
    assert list(c.snap_steps) == [500, 1000, 1500, 2000, 2500, 3000]


def test_config1_layers():
    coefs, thick = layered_coefficients(1)
    assert len(coefs) == 6 and np.all((thick >= 200) & (thick <= 500))
    cfg, med = config1()
    assert cfg.padded == (4040, 1, 2040) and cfg.nrec == 2000 and cfg.nt == 8000
    assert cfg.src == (2020, 0, 30) and set(cfg.rec_z) == {30}
    rho = med["rho"]
    assert np.all(rho == rho[:, :1])                       # horizontal layers
    assert 2 <= len(np.unique(rho[:, 0])) <= 6
    dt, v = cfl_limit(cfg, med)
    assert cfg.dt < dt


def test_config0_and_2():
    cfg, med = config0(n=24, npml=6, nt=20, nrec=16)
    assert cfg.order == 4 and cfg.src_mask == 3 and cfg.padded == (36, 36, 36)
    cfg2, med2 = config2(n=(40, 36, 32), nrec_side=8, nt=10)
    assert cfg2.nrec == 64 and cfg2.padded == (80, 76, 72)
    assert cfg2.dt < cfl_limit(cfg2, med2)[0]


def test_config2_crop_is_a_crop():
    from mixedprecisionfaracoustic_b200.presets import config2_crop
    cfg, med = config2(n=(40, 36, 32), nrec_side=8, nt=10)
    c, m = config2_crop(cfg, med, size=16)
    assert c.padded == (56, 56, 56) and c.precision == "fp64"
    x0, y0 = 20 - 8, 18 - 8                              # columns centred on the source (20, 18)
    full = np.asarray(med["H"]).reshape(32, 36, 40)
    assert np.array_equal(np.asarray(m["H"]).reshape(16, 16, 16), full[:16, y0:y0 + 16, x0:x0 + 16])
    assert c.src == (cfg.npml + 8, cfg.npml + 8, cfg.npml + 1)
    assert c.nrec > 0 and all(cfg.npml <= x < cfg.npml + 16 for x in c.rec_x)


def test_lognormal_statistics():
    rng = np.random.default_rng(2)
    f = lognormal_field((48, 64, 64), 0.1, 10.0, rng)
    g = np.log(f)
    assert abs(g.std() - 0.1) < 0.01
    assert abs(np.mean(f) - 1.0) < 0.02
    # neighbours are strongly correlated, cells 30 apart much less
    c1 = np.corrcoef(g[:, :, :-1].ravel(), g[:, :, 1:].ravel())[0, 1]
    c30 = np.corrcoef(g[:, :, :-30].ravel(), g[:, :, 30:].ravel())[0, 1]
    assert c1 > 0.9 and c30 < 0.5


def test_config3_and_4():
    shots = config3_shots(nshots=64, nt=4000, scale=0.02)
    assert len(shots) == 64
    f0 = [c.f0 for c, _ in shots]
    assert 15 <= min(f0) and max(f0) <= 40
    reqs = config4_requests(n=40, scale=0.05)
    nts = [c.nt for c, _ in reqs]
    assert 1000 <= min(nts) and max(nts) <= 6000
    assert {c.dim for c, _ in reqs} == {2, 3}


def test_host_builder_is_bit_identical_to_the_library():
    """The benchmark's CPU reference arm forms its medium without the CUDA
    library; its values must be the library's bit for bit."""
    from mixedprecisionfaracoustic_b200.presets import c0_coefficients
    for seed in (1, 2, 3, 1000, 5000):
        h, _ = layered_coefficients(seed, host=True)
        lib, _ = layered_coefficients(seed, host=False)
        assert h == lib, seed
    assert c0_coefficients(host=True) == c0_coefficients(host=False)
    a, _ = config1(nx=64, nz=48, nt=10, host=True)
    b, mb = config1(nx=64, nz=48, nt=10)
    _, ma = config1(nx=64, nz=48, nt=10, host=True)
    assert a.pml_v0 == b.pml_v0
    for k in ma:
        assert np.array_equal(ma[k], mb[k]), k


def test_z_spacing_step():
    """The variable z grid helper: dx outside the band, dx / ratio inside, the
    CPML rows untouched, one spacing per pair of padded rows."""
    import numpy as np
    from mixedprecisionfaracoustic_b200.presets import config1, z_spacing_step
    cfg, _ = config1(precision="fp32", nx=40, nz=50, nt=4, npml=6, nrec=4, host=True)
    dz = z_spacing_step(cfg, 10, 30, 4.0)
    assert dz.shape == (cfg.padded[2] - 1,)
    assert np.all(dz[:10] == np.float32(cfg.dx)) and np.all(dz[30:] == np.float32(cfg.dx))
    assert np.allclose(dz[10:30], np.float32(cfg.dx) / 4.0)
