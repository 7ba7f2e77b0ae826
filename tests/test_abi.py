"""The C-ABI library on the host: loads, exports every declared entry point,
validates arguments and builds media (no GPU compute here)."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from mixedprecisionfaracoustic_b200 import _abi
from mixedprecisionfaracoustic_b200.biot import Medium, ShotConfig, biot_from_moduli, cfl_limit, reference_borehole_medium
from mixedprecisionfaracoustic_b200.presets import c0_coefficients, config0, config1, reference_compat
from oracle import oracle as O


def header_functions():
    txt = (ROOT / "include" / "biot.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bp_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_abi.LIB_PATH))
    names = header_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_abi.declared_symbols()) == names


def test_error_strings():
    lib = _abi.load()
    for code in range(11):
        assert lib.bp_error_string(code)
    assert lib.bp_error_string(99) == b"unknown error"


def _create(cfg, med):
    lib = _abi.load()
    h = C.c_void_p()
    c, m = cfg.to_c(), med.to_c()
    return lib.bp_create(C.byref(c), C.byref(m), C.byref(h)), h


@pytest.mark.parametrize("bad", [dict(dim=4), dict(order=3), dict(nt=0), dict(dx=0.0), dict(src=(1000, 0, 0)),
                                 dict(npml=-1), dict(precision="fp64", nx=0)])
def test_create_rejects_bad_config(bad):
    cfg, med = config1(nx=64, nz=48, nt=10, npml=6, nrec=8)
    for k, v in bad.items():
        if k == "precision":
            cfg.precision = v
        else:
            setattr(cfg, k, v)
    rc, _ = _create(cfg, med)
    assert rc == _abi.BP_ERR_ARG


def test_create_rejects_grids_of_2_31_cells():
    """Arrays are addressed with 32-bit cell offsets: a padded grid (row pitch x
    ny x nz) of 2^31 cells or more is refused before any device work; one just
    below the limit passes the check (and, without a GPU, fails at the device
    check that follows)."""
    cfg, med = config0(n=16, npml=4, nt=10, nrec=8)
    lib = _abi.load()
    # pitch 2048 (nx + 2 npml = 2048), ny = 1024, nz = 1024: exactly 2^31 cells
    cfg.nx, cfg.ny, cfg.nz, cfg.npml = 2040, 1016, 1016, 4
    rc, _ = _create(cfg, med)
    assert rc == _abi.BP_ERR_ARG
    assert b"2^31" in lib.bp_last_error()
    if not has_gpu():                               # the medium here is far smaller than that grid
        cfg.nz = 1015                               # 2^31 - 2^21 cells
        rc, _ = _create(cfg, med)
        assert rc == _abi.BP_ERR_NO_DEVICE


def test_create_without_gpu_fails_loudly():
    if has_gpu():
        pytest.skip("a GPU is present")
    cfg, med = config1(nx=64, nz=48, nt=10, npml=6, nrec=8)
    rc, _ = _create(cfg, med)
    assert rc == _abi.BP_ERR_NO_DEVICE


def test_library_borehole_medium_matches_oracle():
    a = reference_borehole_medium(40, 36, 6)
    b = O.borehole_medium(40, 36, 6)
    n = 40 * 36 * 6
    for i, k in enumerate(("rho", "rhof", "M", "C", "H", "H2mu", "mu", "C1", "C2")):
        assert np.array_equal(a[k].ravel(), b[i * n:(i + 1) * n]), k


def test_biot_from_moduli_c0():
    c = c0_coefficients()
    alpha = 1 - 9.6 / 36
    M = 2.25e9 * 36e9 / (0.2 * 36e9 + (alpha - 0.2) * 2.25e9)
    assert abs(c["M"] / M - 1) < 1e-12
    assert abs(c["rho"] - 2320.0) < 1e-9
    assert abs(c["H"] - (alpha ** 2 * M + 9.6e9 + 4 * 5.1e9 / 3)) < 1.0
    assert abs(c["C1"] - 1e9) < 1e-3
    assert abs(c["C2"] - 1.25 * 2.0 * 1000 / 0.2) < 1e-9


def test_cfl_limits():
    cfg, med = reference_compat(nt=10, n=(24, 24, 24), npml=4)
    dt, v = cfl_limit(cfg, med)
    assert 3500 < v < 4300 and cfg.dt < dt
    cfg, med = config0(n=16, npml=4, nt=10, nrec=8)
    dt, v = cfl_limit(cfg, med)
    assert 3000 < v < 3500 and cfg.dt < dt
    cfg.dt = 1.5 * dt
    cfg.check_cfl = 1
    if not has_gpu():
        rc, _ = _create(cfg, med)
        assert rc in (_abi.BP_ERR_CFL, _abi.BP_ERR_NO_DEVICE)


def _vmax_numpy(med):
    """Fast P velocity bound of every cell (the largest root of the Biot
    dispersion determinant, or sqrt(H / rho) for a singular mass matrix)."""
    rho, rhof, M, C, H, C2 = (np.asarray(med[k], dtype=np.float64).ravel() for k in ("rho", "rhof", "M", "C", "H", "C2"))
    v2 = np.where(rho > 0, H / rho, 0.0)
    a = rho * C2 - rhof * rhof
    b = -(H * C2 + M * rho - 2 * C * rhof)
    c = H * M - C * C
    with np.errstate(all="ignore"):
        root = (-b + np.sqrt(np.maximum(b * b - 4 * a * c, 0))) / (2 * a)
    v2 = np.where((a > 1e-9 * np.abs(rho * C2)) & (root > v2), root, v2)
    return float(np.sqrt(np.maximum(v2, 0)).max())


def test_cfl_scan_on_threads_matches_every_cell():
    """The threaded scan with reuse of repeated cells finds the same maximum
    as an evaluation of every cell: a layered medium (runs of equal cells) with
    its fastest cell alone in the middle of a run, over several scan ranges."""
    cfg, med = config0(n=16, npml=4, nt=10, nrec=8)
    nx, nz = 1500, 1100                      # 1.65 M cells: several 2^18-cell ranges
    cfg.dim, cfg.nx, cfg.ny, cfg.nz = 2, nx, 1, nz
    rng = np.random.default_rng(7)
    layers = rng.integers(0, 4, nz)
    lay = {k: np.asarray(v, dtype=np.float32).ravel()[:4] for k, v in med.items()}
    m = Medium({k: np.ascontiguousarray(np.repeat(v[layers][:, None], nx, axis=1)) for k, v in lay.items()})
    base = _vmax_numpy(m)
    m["H"][nz // 2, nx // 3] *= np.float32(1.7)        # one fast cell
    dt, v = cfl_limit(cfg, m)
    assert v == pytest.approx(_vmax_numpy(m), rel=1e-12)
    assert v > 1.05 * base


def test_struct_layout_matches_header(tmp_path):
    """The ctypes mirror has the C structs' sizes and field offsets."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    structs = {"bp_config": _abi.BpConfig, "bp_medium": _abi.BpMedium, "bp_tune": _abi.BpTune,
               "bp_server_stats": _abi.BpServerStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "biot.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(out[name]) == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert int(out[f"{name}.{f}"]) == getattr(cls, f).offset, (name, f)
