"""Unit pins of the oracle's pieces against independent restatements and the
reference's worked numbers (method.md)."""
import math

import numpy as np
import pytest

from mixedprecisionfaracoustic_b200.biot import Medium
from mixedprecisionfaracoustic_b200.presets import reference_compat_config
from oracle import oracle as O


def test_f2h_matches_numpy_rne():
    rng = np.random.default_rng(0)
    v = np.concatenate([
        rng.standard_normal(200000).astype(np.float32) * np.float32(10.0) ** rng.integers(-9, 6, 200000),
        np.array([0.0, -0.0, 65504.0, 65519.0, 65520.0, 1e9, -1e9, 6.1e-5, 5.96e-8, 2.98e-8, 2.99e-8,
                  1.0 + 2 ** -11, 1.0 + 3 * 2 ** -11, np.inf, -np.inf], dtype=np.float32)]).astype(np.float32)
    mine = O.f2h(v)
    with np.errstate(over="ignore"):
        ref = v.astype(np.float16).view(np.uint16)
    assert np.array_equal(mine, ref)


def test_compensated_codec_error_bound():
    rng = np.random.default_rng(1)
    v = (rng.standard_normal(100000) * 10.0 ** rng.uniform(-12, 4, 100000)).astype(np.float32)
    hi, lo = O.encode_ch(v)
    lib = O.load()
    dec = np.array([lib.orc_load_ch(int(h), int(l)) for h, l in zip(hi[:20000], lo[:20000])], dtype=np.float64)
    h = hi[:20000].view(np.float16).astype(np.float64)
    a = np.abs(h)
    e = np.floor(np.log2(np.where(a > 0, a, 1.0))) + 1            # frexp exponent
    unit = np.where(a < 2.0 ** -14, 2.0 ** -32, 2.0 ** (e - 19))
    err = np.abs(dec - v[:20000].astype(np.float64))
    assert np.all(err <= unit * 1.0 + 1e-45)
    # about 19 significant bits for normal-range values
    big = np.abs(v[:20000]) > 1e-3
    assert np.max(err[big] / np.abs(v[:20000][big])) < 2.0 ** -17


def test_ricker_matches_reference_formula():
    lib = O.load()
    DT, F0 = np.float32(0.9e-6), np.float32(3000.0)
    T0 = np.float32(1.2 / 3000.0)
    for it in (0, 1, 100, 444, 445, 1000, 3499):
        tt = np.float32(it) * DT
        a = float(np.float32(tt - T0))
        pi = 3.1415926535
        ref = np.float32(-(1 - 2 * pi * pi * float(F0) ** 2 * a * a) * math.exp(-pi * pi * float(F0) ** 2 * a * a))
        assert lib.orc_ricker_ref(it, DT, F0, T0) == ref


@pytest.fixture(scope="module")
def ref_oracle_small():
    # the reference medium (borehole radius^2 <= 100 cells) with the reference's
    # 32-cell CPML, few cells in z to keep it small
    cfg = reference_compat_config(nt=4, n=(32, 32, 8), npml=32)
    med = Medium.from_stack(O.borehole_medium(32, 32, 8), (8, 32, 32))
    return cfg, med, O.Oracle(cfg, med, O.REF32)


def test_profile_region_and_values(ref_oracle_small):
    cfg, _, o = ref_oracle_small
    n = cfg.padded[0]
    H, DT = np.float32(cfg.dx), np.float32(cfg.dt)
    DP = np.float32(32) * H
    oright = np.float32(n - 1) * H - DP
    d0 = np.float32(3.0 * 4000.0 * math.log(1.0 / float(np.float32(1e-6))) / (2.0 * float(DP)))
    d = o.profile(0, 0)
    left = [i for i in range(n) if np.float32(i) * H < DP]
    right = [i for i in range(n) if np.float32(i) * H >= oright]
    assert len(left) == 32 and len(right) == 33        # asymmetric like Float/main.cu:597-614
    for i in left:
        x = np.float32(i) * H
        assert d[i] == float(np.float32(float(d0) * float(np.float32(np.float32(DP - x) / DP)) ** 2))
    assert np.all(d[max(left) + 1:min(right)] == 0.0)
    e = o.profile(0, 1)
    assert np.allclose(e[left], np.exp(-d[left] * float(DT)), rtol=1e-6)


def test_exponent_scaling_known_answers(ref_oracle_small):
    """method.md 14.3-14.5: K_max = H = 3.8385e10, e_m = -23; the code's R_max
    also sees the borehole's rho^-1 = 1e-3 (Half/main.cu:767-769)."""
    cfg, med, o = ref_oracle_small
    np_ = cfg.npml
    mu = np.pad(med["mu"], ((np_, np_), (np_, np_), (np_, np_)), mode="edge")
    em, epml, kmax, rmax = o.comp16_exponents(mu)
    assert em == -23
    assert abs(kmax / 3.8385e10 - 1) < 1e-4
    assert abs(rmax - 1e-3) < 1e-9
    # e_r and the unrounded e_m of method.md for the formation (R = 1/2485)
    er = 1.0 / math.sqrt(float(cfg.dt) ** 2 * 3.8385e10 / 2485.0)
    assert abs(er - 282.709) < 0.01
    assert abs(-math.log2(er * float(cfg.dt) * 3.8385e10) - (-23.2194268667)) < 1e-4
    # PML exponent: floor(log2(2048 / (DT d0))) with d0 at the outermost cell
    assert epml == 13


def test_medium_formation_values():
    m = O.borehole_medium(32, 32, 4).reshape(9, 4, 32, 32)
    rho, rhof, M, C, H, H2u, mu, C1, C2 = (m[i, 0, 0, 0] for i in range(9))
    assert rho == np.float32(2485.0)
    assert M == np.float32(2.25e10)
    assert abs(H / 3.8385e10 - 1) < 1e-4
    assert C1 == np.float32(5e8) and C2 == np.float32(37500.0)
    # borehole cell: fluid, C = M = H = H-2mu = Kf, C1 = 0
    b = m[:, 0, 16, 16]
    assert b[0] == 1000.0 and b[6] == 0.0 and b[7] == 0.0 and b[2] == b[3] == b[4] == b[5] == np.float32(2.25e9)


@pytest.mark.parametrize("dim,order", [(2, 2), (2, 4), (3, 2), (3, 4)])
def test_ref32_close_to_fp64(dim, order):
    """The Float arithmetic and the FP64 oracle agree on small grids."""
    from mixedprecisionfaracoustic_b200 import _abi
    from mixedprecisionfaracoustic_b200.biot import ShotConfig
    n = 20
    shape = (n, n, n) if dim == 3 else (n, n)
    med = Medium.from_stack(O.borehole_medium(n, n if dim == 3 else 1, n), shape)
    c = (n + 12) // 2
    cfg = ShotConfig(dim=dim, nx=n, ny=n, nz=n, npml=6, order=order, nt=80, dx=0.01, dt=0.9e-6, f0=3000.0,
                     pml_v0=4000.0, pml_r=1e-6, src=(c, c, c), src_mask=_abi.SRC_TAU | _abi.SRC_P,
                     rec_x=list(range(2, n + 10)), rec_y=[c] * (n + 8), rec_z=[c + 2] * (n + 8))
    a = O.Oracle(cfg, med, O.REF32)
    b = O.Oracle(cfg, med, O.FP64)
    a.run(80)
    b.run(80)
    for comp in ("txx", "vux", "p"):
        x, y = a.traces(comp), b.traces(comp)
        assert np.abs(y).max() > 0
        assert np.linalg.norm(x - y) / np.linalg.norm(y) < 1e-5


def test_oracle_variable_z_grid():
    """The oracle's variable z grid: every spacing dx reproduces the uniform
    grid (FP64 to rounding; REF32 within an ulp per difference, since it
    multiplies by 1/dx where the uniform path divides by dx), and a refined
    band changes the wavefield."""
    import numpy as np
    from mixedprecisionfaracoustic_b200.presets import config1, z_spacing_step
    cfg, med = config1(precision="fp32", nx=60, nz=50, nt=120, npml=6, order=2, nrec=16, host=True)
    cfg.dt = float(np.float32(cfg.dt / 2))
    flat = np.full(cfg.padded[2] - 1, float(np.float32(cfg.dx)))
    fine = z_spacing_step(cfg, 8, 40, 2.0)          # the source and receivers' rows lie in the band

    def run(mode, dz):
        o = O.Oracle(cfg, med, mode)
        if dz is not None:
            o.set_z_spacing(dz)
        o.run(cfg.nt)
        t = o.traces("txx").astype(np.float64)
        o.close()
        return t

    def rel(a, b):
        return np.linalg.norm(a - b) / np.linalg.norm(b)

    base64, base32 = run(O.FP64, None), run(O.REF32, None)
    assert rel(run(O.FP64, flat), base64) <= 1e-12
    assert rel(run(O.REF32, flat), base32) <= 1e-6
    assert rel(run(O.FP64, fine), base64) >= 1e-3
