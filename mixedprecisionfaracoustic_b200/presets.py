"""Shot presets: the reference program's run and the workload configurations.

``reference_compat`` reproduces the reference run (Float/main.cu:300-345,
1590-1655): 128^3 cells + a 32-cell CPML, H = 0.01 m, DT = 0.9 us, NT = 3500,
a 3 kHz Ricker on txx/tyy/tzz at (NX_ext/2, NY_ext/2, 20+NP), a vertical line
of NZ_ext receivers through the source column and the snapshots of
Float/main.cu:1094-1163.

The workload presets (c0..c4) are seeded synthetic inputs with the shapes,
sizes and value distributions of the benchmark configurations:
  c0  3D homogeneous 160^3, dx 5 m, dt 0.4 ms, 1000 steps, 20-cell CPML,
      30 Hz source on txx/tyy/tzz and p at the centre, 128 receivers along x
      at depth 20 cells, snapshots every 500 steps
  c1  2D x-z 4000 x 2000 with 6 layers (thickness U[200, 500] cells,
      porosity U[0.1, 0.35], permeability log-U[1e-14, 1e-11] m^2,
      frame bulk U[5, 20] GPa, shear U[3, 12] GPa), 25 Hz at (2000, 10),
      2000 receivers at depth 10, 8000 steps
  c2  3D 512 x 512 x 384 log-normal (sigma 0.1, 10-cell correlation) on the
      c0 moduli and permeability, 20 Hz at the surface centre, 256 x 256
      surface receivers, 3000 steps
  c3  64 2D shots, sizes from {1024^2, 1536x1024, 2048^2, 3072x1536}, random
      source position, 15-40 Hz, layered media with per-shot seeds, 4000 steps
  c4  Poisson stream of shot requests (2D 512^2..2048^2, 3D 128^3..320^3,
      1000..6000 steps)
The c0 medium: solid density 2650, fluid density 1000 kg/m^3, porosity 0.2,
tortuosity 2.0, grain bulk 36 GPa, frame bulk 9.6 GPa, shear 5.1 GPa, fluid
bulk 2.25 GPa, viscosity 1e-3 Pa s, permeability 1e-12 m^2, pore-shape factor
m = 8 (the reference's porousm, Float/main.cu:1599).
"""
from __future__ import annotations

import functools
import math

import numpy as np

from . import _abi
from .biot import MEDIUM_KEYS, Medium, ShotConfig, biot_from_moduli, reference_borehole_medium

C0 = dict(Ks=36e9, Kb=9.6e9, mu=5.1e9, Kf=2.25e9, rhos=2650.0, rhof=1000.0, phi=0.2, tort=2.0,
          eta=1e-3, kappa=1e-12, m_shape=8.0)
DX, DT = 5.0, 4e-4


def reference_compat(nt: int = 3500, precision: str = "fp32", n=(128, 128, 128), npml: int = 32,
                     rounding: str = None):
    """The reference program's run, returned as (ShotConfig, Medium)."""
    return reference_compat_config(nt, precision, n, npml, rounding), reference_borehole_medium(*n)


def reference_compat_config(nt: int = 3500, precision: str = "fp32", n=(128, 128, 128), npml: int = 32,
                            rounding: str = None):
    """ShotConfig of the reference program's run (no library call).  FP32 runs
    round like the reference's Float build unless rounding="fast"."""
    NX, NY, NZ = n
    NXe, NYe, NZe = NX + 2 * npml, NY + 2 * npml, NZ + 2 * npml
    sx, sy, sz = NXe // 2, NYe // 2, 20 + npml
    snaps = [s for s in range(500, 3001, 500) if s < nt]
    masks = [["txx", "vux", "vwx", "vuz", "vwz"] if s == 500 else ["txx"] for s in snaps]
    dt = float(np.float32(0.9 * 10.0 ** -6))
    cfg = ShotConfig(dim=3, nx=NX, ny=NY, nz=NZ, npml=npml, order=2, precision=precision, nt=nt,
                     dx=float(np.float32(0.01)), dt=dt, f0=3000.0, t0=float(np.float32(1.2 / 3000.0)),
                     pml_v0=4000.0, pml_r=float(np.float32(1e-6)), src=(sx, sy, sz), src_mask=_abi.SRC_TAU,
                     rec_x=[sx] * NZe, rec_y=[sy] * NZe, rec_z=list(range(NZe)),
                     snap_steps=snaps, snap_masks=masks, snap_y=NYe // 2,
                     rounding=rounding or ("reference" if precision == "fp32" else "fast"))
    return cfg


def uniform_medium(shape: tuple, coef: dict) -> Medium:
    return Medium({k: np.full(shape, coef[k], dtype=np.float32) for k in MEDIUM_KEYS})


def biot_from_moduli_host(Ks, Kb, mu, Kf, rhos, rhof, phi, tort, eta, kappa, m_shape=8.0) -> dict:
    """The nine Biot coefficients of one material, in Python double arithmetic:
    the formation branch of create_model (Float/main.cu:1635-1650), the same
    operations in the same order as bp_biot_from_moduli, so the values are
    bit-identical to the library's.  For callers that must not load the CUDA
    library (the CPU reference arm of the benchmark)."""
    alpha = 1 - Kb / Ks
    M = Kf * Ks / (phi * Ks + (alpha - phi) * Kf)
    H = alpha * alpha * M + Kb + mu * 4.0 / 3.0
    vals = ((1 - phi) * rhos + phi * rhof, rhof, M, alpha * M, H, H - 2 * mu, mu, eta / kappa,
            (1 + 2 / m_shape) * tort * rhof / phi)
    return dict(zip(MEDIUM_KEYS, (float(v) for v in vals)))


def _builder(host: bool):
    return biot_from_moduli_host if host else biot_from_moduli


def c0_coefficients(host: bool = False) -> dict:
    p = C0
    return _builder(host)(p["Ks"], p["Kb"], p["mu"], p["Kf"], p["rhos"], p["rhof"], p["phi"], p["tort"],
                          p["eta"], p["kappa"], p["m_shape"])


def _vmax(coefs: list) -> float:
    v = 0.0
    for c in coefs:
        a = c["rho"] * c["C2"] - c["rhof"] ** 2
        b = -(c["H"] * c["C2"] + c["M"] * c["rho"] - 2 * c["C"] * c["rhof"])
        cc = c["H"] * c["M"] - c["C"] ** 2
        lam = c["H"] / c["rho"]
        if a > 1e-9 * abs(c["rho"] * c["C2"]):
            lam = max(lam, (-b + math.sqrt(max(b * b - 4 * a * cc, 0.0))) / (2 * a))
        v = max(v, math.sqrt(lam))
    return v


def config0(precision: str = "fp32", order: int = 4, n: int = 160, npml: int = 20, nt: int = 1000,
            nrec: int = 128):
    """c0: 3D homogeneous Biot medium (scaled by n for tests)."""
    co = c0_coefficients()
    NXe = n + 2 * npml
    ctr = NXe // 2
    depth = npml + min(20, n // 2)
    x0 = npml + (n - nrec) // 2 if n >= nrec else npml
    rx = [min(x0 + i, npml + n - 1) for i in range(nrec)]
    snaps = [s for s in range(500, nt, 500)] + [nt - 1]
    cfg = ShotConfig(dim=3, nx=n, ny=n, nz=n, npml=npml, order=order, precision=precision, nt=nt, dx=DX, dt=DT,
                     f0=30.0, pml_v0=_vmax([co]), pml_r=1e-6, src=(ctr, ctr, ctr),
                     src_mask=_abi.SRC_TAU | _abi.SRC_P, rec_x=rx, rec_y=[ctr] * nrec, rec_z=[depth] * nrec,
                     snap_steps=snaps, snap_fields=["txx", "vux", "vuz", "vwx", "vwz"], snap_y=ctr, check_cfl=1)
    return cfg, uniform_medium((n, n, n), co)


def layered_coefficients(seed: int, nlayers: int = 6, host: bool = False):
    """Per-layer Biot coefficients and thicknesses (cells) of the c1 layered model
    (host=True: formed without the CUDA library, bit-identical values)."""
    rng = np.random.default_rng(seed)
    thick = rng.integers(200, 501, size=nlayers)
    phi = rng.uniform(0.1, 0.35, nlayers)
    kappa = 10.0 ** rng.uniform(-14.0, -11.0, nlayers)
    kb = rng.uniform(5e9, 20e9, nlayers)
    mu = rng.uniform(3e9, 12e9, nlayers)
    p = C0
    build = _builder(host)
    coefs = [build(p["Ks"], float(kb[i]), float(mu[i]), p["Kf"], p["rhos"], p["rhof"], float(phi[i]),
                   p["tort"], p["eta"], float(kappa[i]), p["m_shape"]) for i in range(nlayers)]
    return coefs, thick


def layered_medium(nx: int, nz: int, seed: int, depth_scale: float = 1.0, host: bool = False) -> tuple:
    """2D layered medium (nz, nx); layer thicknesses are scaled by depth_scale."""
    coefs, thick = layered_coefficients(seed, host=host)
    bounds = np.cumsum(np.maximum(1, np.round(thick * depth_scale).astype(int)))
    z = np.arange(nz)
    layer = np.searchsorted(bounds, z, side="right")
    layer = np.minimum(layer, len(coefs) - 1)
    med = Medium()
    for k in MEDIUM_KEYS:
        col = np.array([coefs[l][k] for l in layer], dtype=np.float32)
        med[k] = np.ascontiguousarray(np.broadcast_to(col[:, None], (nz, nx)))
    return med, _vmax(coefs)


def _layered_only(nx: int, nz: int, seed: int, depth_scale: float) -> Medium:
    return layered_medium(nx, nz, seed, depth_scale=depth_scale)[0]


def config1(precision: str = "fp32", seed: int = 1, nx: int = 4000, nz: int = 2000, nt: int = 8000,
            npml: int = 20, order: int = 2, nrec: int = 2000, host: bool = False):
    """c1: 2D x-z layered model (scaled by nx, nz for tests).  host=True forms
    the medium without loading the CUDA library (same values)."""
    scale = nz / 2000.0
    med, vmax = layered_medium(nx, nz, seed, depth_scale=scale, host=host)
    sx = npml + int(round(2000 * nx / 4000.0))
    sz = npml + max(1, int(round(10 * scale)))
    rz = npml + max(1, int(round(10 * scale)))
    step = max(1, nx // nrec)
    rx = [npml + min(i * step, nx - 1) for i in range(nrec)]
    cfg = ShotConfig(dim=2, nx=nx, ny=1, nz=nz, npml=npml, order=order, precision=precision, nt=nt, dx=DX, dt=DT,
                     f0=25.0, pml_v0=vmax, pml_r=1e-6, src=(sx, 0, sz), src_mask=_abi.SRC_TAU | _abi.SRC_P,
                     rec_x=rx, rec_y=[0] * nrec, rec_z=[rz] * nrec, check_cfl=1)
    return cfg, med


def lognormal_field(shape: tuple, sigma: float, corr: float, rng) -> np.ndarray:
    """exp(sigma g - sigma^2/2) with g a unit-variance Gaussian field of correlation
    length `corr` cells: white noise on a grid coarsened by corr/2, smoothed with a
    Gaussian of one coarse cell, trilinearly upsampled and renormalised."""
    from scipy import ndimage
    step = max(1, int(round(corr / 2)))
    cshape = tuple(s // step + 3 for s in shape)
    g = ndimage.gaussian_filter(rng.standard_normal(cshape).astype(np.float32), sigma=1.0, mode="wrap")
    g = ndimage.zoom(g, step, order=1)[tuple(slice(0, s) for s in shape)]
    g = (g - g.mean()) / max(float(g.std()), 1e-12)
    return np.exp(sigma * g - 0.5 * sigma * sigma).astype(np.float32)


def config2(precision: str = "comp16", seed: int = 2, n=(512, 512, 384), npml: int = 20, nt: int = 3000,
            order: int = 2, nrec_side: int = 256, sigma: float = 0.1, corr: float = 10.0):
    """c2: 3D log-normal perturbation of the c0 moduli and permeability (scaled by n for tests)."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    shape = (nz, ny, nx)
    fkb, fmu, fks, fkap = (lognormal_field(shape, sigma, corr, rng) for _ in range(4))
    p = C0
    # per-cell Biot coefficients (the same formulas as bp_biot_from_moduli, vectorised)
    Ks = p["Ks"] * fks.astype(np.float64)
    Kb = np.minimum(p["Kb"] * fkb.astype(np.float64), 0.95 * Ks)
    mu = p["mu"] * fmu.astype(np.float64)
    kappa = p["kappa"] * fkap.astype(np.float64)
    phi, Kf, rhos, rhof, tort, eta, m = p["phi"], p["Kf"], p["rhos"], p["rhof"], p["tort"], p["eta"], p["m_shape"]
    alpha = 1 - Kb / Ks
    M = Kf * Ks / (phi * Ks + (alpha - phi) * Kf)
    H = alpha * alpha * M + Kb + mu * 4.0 / 3.0
    med = Medium({"rho": np.full(shape, (1 - phi) * rhos + phi * rhof, np.float32),
                  "rhof": np.full(shape, rhof, np.float32), "M": M.astype(np.float32),
                  "C": (alpha * M).astype(np.float32), "H": H.astype(np.float32),
                  "H2mu": (H - 2 * mu).astype(np.float32), "mu": mu.astype(np.float32),
                  "C1": (eta / kappa).astype(np.float32),
                  "C2": np.full(shape, (1 + 2 / m) * tort * rhof / phi, np.float32)})
    vmax = float(np.sqrt(np.max(H) / ((1 - phi) * rhos + phi * rhof))) * 1.05
    cx, cy = npml + nx // 2, npml + ny // 2
    side = min(nrec_side, nx, ny)
    xs = [npml + (i * nx) // side for i in range(side)]
    ys = [npml + (j * ny) // side for j in range(side)]
    rx = [x for y in ys for x in xs]
    ry = [y for y in ys for _ in xs]
    cfg = ShotConfig(dim=3, nx=nx, ny=ny, nz=nz, npml=npml, order=order, precision=precision, nt=nt, dx=DX, dt=DT,
                     f0=20.0, pml_v0=vmax, pml_r=1e-6, src=(cx, cy, npml + 1), src_mask=_abi.SRC_TAU | _abi.SRC_P,
                     rec_x=rx, rec_y=ry, rec_z=[npml + 1] * len(rx), check_cfl=1)
    return cfg, med


def config2_crop(cfg, med, size: int = 128, precision: str = "fp64", nt: int = None):
    """A size^3 crop of a c2 model: the top `size` cells in depth of the size x size
    columns centred on the source, the same medium values cell for cell, the same
    source cell and the surface receivers that fall inside the crop."""
    nx, ny, nz, np_ = cfg.nx, cfg.ny, cfg.nz, cfg.npml
    sx, sy, sz = (c - np_ for c in cfg.src)            # physical source cell
    x0 = min(max(sx - size // 2, 0), nx - size)
    y0 = min(max(sy - size // 2, 0), ny - size)
    z0 = 0
    sl = (slice(z0, z0 + size), slice(y0, y0 + size), slice(x0, x0 + size))
    cm = Medium({k: np.ascontiguousarray(np.asarray(v).reshape(nz, ny, nx)[sl]) for k, v in med.items()})
    keep = [i for i in range(cfg.nrec)
            if x0 <= cfg.rec_x[i] - np_ < x0 + size and y0 <= cfg.rec_y[i] - np_ < y0 + size
            and z0 <= cfg.rec_z[i] - np_ < z0 + size]
    out = ShotConfig(dim=3, nx=size, ny=size, nz=size, npml=np_, order=cfg.order, precision=precision,
                     nt=cfg.nt if nt is None else nt, dx=cfg.dx, dt=cfg.dt, f0=cfg.f0, pml_v0=cfg.pml_v0,
                     pml_r=cfg.pml_r, src=(np_ + sx - x0, np_ + sy - y0, np_ + sz - z0), src_mask=cfg.src_mask,
                     rec_x=[cfg.rec_x[i] - x0 for i in keep], rec_y=[cfg.rec_y[i] - y0 for i in keep],
                     rec_z=[cfg.rec_z[i] - z0 for i in keep], check_cfl=cfg.check_cfl)
    return out, cm


def config3_shots(seed: int = 3, nshots: int = 64, nt: int = 4000, precision: str = "fp32", npml: int = 20,
                  sizes=((1024, 1024), (1536, 1024), (2048, 2048), (3072, 1536)), order: int = 2,
                  scale: float = 1.0):
    """c3: batched 2D shots with random sizes, sources and layered media."""
    rng = np.random.default_rng(seed)
    shots = []
    for s in range(nshots):
        nx, nz = sizes[int(rng.integers(0, len(sizes)))]
        nx, nz = max(16, int(nx * scale)), max(16, int(nz * scale))
        f0 = float(rng.uniform(15.0, 40.0))
        sx = npml + int(rng.integers(0, nx))
        sz = npml + int(rng.integers(0, nz))
        med, vmax = layered_medium(nx, nz, seed=1000 + s, depth_scale=nz / 2000.0)
        nrec = min(256, nx)
        rx = [npml + (i * nx) // nrec for i in range(nrec)]
        rz = npml + min(10, nz - 1)
        cfg = ShotConfig(dim=2, nx=nx, ny=1, nz=nz, npml=npml, order=order, precision=precision, nt=nt, dx=DX,
                         dt=DT, f0=f0, pml_v0=vmax, pml_r=1e-6, src=(sx, 0, sz),
                         src_mask=_abi.SRC_TAU | _abi.SRC_P, rec_x=rx, rec_y=[0] * nrec, rec_z=[rz] * nrec)
        shots.append((cfg, med))
    return shots


def config4_requests(seed: int = 4, n: int = 1000, precision: str = "fp32", scale: float = 1.0,
                     steps=(1000, 6000), include_3d: bool = True, npml: int = 20, lazy: bool = False):
    """c4: request list (cfg, medium) for the serving stream; sizes are scaled by `scale`.
    lazy=True gives, in place of each medium, a function that builds it (the
    full-size stream's media add up to hundreds of GB on the host; built one
    at a time at submission, each is freed once the server holds its copy).
    The configurations and media are the same either way."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        nt = int(rng.integers(steps[0], steps[1] + 1))
        if include_3d and rng.uniform() < 0.25:
            e = int(rng.integers(128, 321) * scale)
            e = max(8, e)
            co = c0_coefficients()
            ctr = (e + 2 * npml) // 2
            cfg = ShotConfig(dim=3, nx=e, ny=e, nz=e, npml=npml, order=2, precision=precision, nt=nt, dx=DX,
                             dt=DT, f0=float(rng.uniform(15, 40)), pml_v0=_vmax([co]), src=(ctr, ctr, npml + 2),
                             src_mask=_abi.SRC_TAU | _abi.SRC_P, rec_x=list(range(npml, npml + e, max(1, e // 64))),
                             rec_y=None or [], rec_z=[])
            nr = len(cfg.rec_x)
            cfg.rec_y, cfg.rec_z = [ctr] * nr, [npml + 2] * nr
            build = functools.partial(uniform_medium, (e, e, e), co)
            reqs.append((cfg, build if lazy else build()))
        else:
            nx = max(16, int(rng.integers(512, 2049) * scale))
            nz = max(16, int(rng.integers(512, 2049) * scale))
            coefs, _ = layered_coefficients(5000 + i)
            vmax = _vmax(coefs)
            build = functools.partial(_layered_only, nx, nz, 5000 + i, nz / 2000.0)
            nrec = min(256, nx)
            rx = [npml + (k * nx) // nrec for k in range(nrec)]
            cfg = ShotConfig(dim=2, nx=nx, ny=1, nz=nz, npml=npml, order=2, precision=precision, nt=nt, dx=DX,
                             dt=DT, f0=float(rng.uniform(15, 40)), pml_v0=vmax,
                             src=(npml + nx // 2, 0, npml + 2), src_mask=_abi.SRC_TAU | _abi.SRC_P,
                             rec_x=rx, rec_y=[0] * nrec, rec_z=[npml + 2] * nrec)
            reqs.append((cfg, build if lazy else build()))
    return reqs


def z_spacing_step(cfg: ShotConfig, z_fine: int, z_coarse: int, ratio: float) -> np.ndarray:
    """Spacings of a variable z grid (bp_set_z_spacing) shaped like the
    reference's unused variable-grid constants (Float/main.cu:24-25,76-89: the
    spacing H drops by a factor m at a depth): dx down to padded row z_fine,
    dx / ratio between rows z_fine and z_coarse, dx below; z_fine and z_coarse
    must leave the CPML rows at dx.  Returns nz + 2 npml - 1 spacings."""
    nzp = cfg.padded[2]
    dz = np.full(nzp - 1, float(np.float32(cfg.dx)), dtype=np.float64)
    dz[z_fine:z_coarse] /= ratio
    return dz
