"""The drop-in run: the reference program's configuration on the GPU.

Checks the FP32 path against the reference's own golden slices (state after
step 500, Float/*.dat) and the text files the drop-in writes against the
reference's format (wfile / wfile3d, Float/main.cu:1501-1516,1563-1588).
"""
import numpy as np
import pytest

from conftest import rel_l2
from mixedprecisionfaracoustic_b200 import Simulation
from mixedprecisionfaracoustic_b200.presets import reference_compat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_run(tmp_path_factory):
    cfg, med = reference_compat(nt=501)
    s = Simulation(cfg, med)
    s.run(501)
    out = tmp_path_factory.mktemp("refout")
    s.write_reference_outputs(out)
    yield s, out
    s.close()


@pytest.mark.parametrize("field", ["txx", "vux", "vuz", "vwx", "vwz"])
def test_fp32_matches_reference_golden(ref_run, golden, field):
    s, _ = ref_run
    a = s.snapshot(0, field)
    assert a.shape == (192, 192)
    err = rel_l2(a, golden[field + "500"])
    assert err <= 1e-5, f"{field}500 rel L2 {err:.3e}"


def _parse(path):
    return np.array([[float(v) for v in ln.split()] for ln in path.read_text().splitlines() if ln.strip()])


def test_reference_text_format(ref_run, golden):
    _, out = ref_run
    names = sorted(p.name for p in out.iterdir())
    for n in ["sisx.dat", "sisz.dat", "sisvu.dat", "sisvw.dat", "sisp.dat", "txx500.dat", "vux500.dat",
              "vwx500.dat", "vuz500.dat", "vwz500.dat", "txx.dat"]:
        assert n in names, n
    raw = (out / "txx500.dat").read_text()
    rows = raw.split("\n")
    # 192 rows of 192 "%e " values, each row terminated by "\n\n"
    assert raw.count("\n") == 2 * 192
    assert rows[0].endswith(" ") and len(rows[0].split()) == 192 and rows[1] == ""
    a = _parse(out / "txx500.dat")
    assert a.shape == (192, 192)
    assert rel_l2(a, golden["txx500"]) <= 1e-5
    sis = _parse(out / "sisx.dat")
    assert sis.shape == (192, 501)


def _reference_run_traces(precision, rounding=None):
    from conftest import GOLDEN
    rows = np.load(GOLDEN / "float_ref_seismograms.npz")["rows"]
    cfg, med = reference_compat(nt=3500, precision=precision, rounding=rounding)
    with Simulation(cfg, med) as s:
        s.run(3500)
        return {k: s.traces(c)[rows].astype(np.float64) for k, c in COMPS}


COMPS = (("sisx", "txx"), ("sisz", "tzz"), ("sisvu", "vux"), ("sisvw", "vwx"), ("sisp", "p"))


def test_fp32_seismograms_match_reference_run():
    """Full 3500-step drop-in run vs the reference's own sis*.dat (regenerated by
    running the unmodified reference Float program on a B200;
    tests/golden/float_ref_seismograms.npz keeps 25 of the 192 receiver rows,
    every 8th and the source row 52).

    With the reference's rounding (the drop-in's default for FP32) every
    component matches to <= 1e-6 over all steps (measured <= 1.5e-7, the text
    files' own 7-digit rounding).  The fast rounding is held to the FP64
    solution instead: sisvu's late coda is at float noise level, and the
    reference itself moves by 1.3e-5 on sisvu when it is only recompiled
    without FMA contraction (test_oracle_golden.py); the fast form is closer
    to FP64 than the reference on sisvu and within 1e-5 of it elsewhere."""
    from conftest import GOLDEN
    g = np.load(GOLDEN / "float_ref_seismograms.npz")
    ref = _reference_run_traces("fp32", "reference")
    for k, _ in COMPS:
        if k == "sisvw":
            continue
        err = rel_l2(ref[k], g[k])
        assert err <= 1e-6, f"reference rounding {k}: rel L2 {err:.3e}"
    fast = _reference_run_traces("fp32", "fast")
    f64 = _reference_run_traces("fp64")
    for k in ("sisx", "sisz", "sisp"):
        assert rel_l2(fast[k], g[k]) <= 1e-5, k
        assert rel_l2(fast[k], f64[k]) <= 1e-5, k
    mine, theirs = rel_l2(fast["sisvu"], f64["sisvu"]), rel_l2(g["sisvu"], f64["sisvu"])
    assert mine <= theirs, (mine, theirs)
    assert np.all(fast["sisvw"] == 0) and np.all(g["sisvw"] == 0)   # receivers in the fluid borehole


def test_comp16_as_close_to_fp64_as_the_reference_half_build():
    """COMP16 (the reference's compensated fp16 storage) over the full 3500-step
    reference run, against the unmodified reference Half build's own outputs
    (tests/golden/half_ref_seismograms.npz, same rows): per component, the
    distance to the FP64 solution is at most 1.5 x the Half build's (measured
    0.18 x on sisx and sisz, 1.04 x on sisvu, 1.42 x on sisp), and the two
    agree with each other to <= 3e-4 on the stress traces."""
    from conftest import GOLDEN
    h = np.load(GOLDEN / "half_ref_seismograms.npz")
    c16 = _reference_run_traces("comp16")
    f64 = _reference_run_traces("fp64")
    for k in ("sisx", "sisz", "sisvu", "sisp"):
        mine, theirs = rel_l2(c16[k], f64[k]), rel_l2(h[k], f64[k])
        assert mine <= 1.5 * theirs and mine <= 1e-3, (k, mine, theirs)
    for k in ("sisx", "sisz", "sisp"):
        assert rel_l2(c16[k], h[k]) <= 3e-4, k


def test_comp16_reference_run_vs_fp64():
    cfg, med = reference_compat(nt=301, precision="comp16")
    c64, _ = reference_compat(nt=301, precision="fp64")
    with Simulation(cfg, med) as a, Simulation(c64, med) as b:
        a.run(301)
        b.run(301)
        for c in ("txx", "tzz", "vux", "p"):
            assert a.trace_rel_l2(b, c) <= 1e-3, c
        sc = a.scaling()
    assert sc["em"] == -23          # method.md worked example for this medium


def test_dropin_binary_writes_the_reference_files(ref_run, golden, tmp_path):
    """The shipped drop-in program (bin/biot_reference_run, the C++ driver over
    the C ABI) run for 501 steps: its snapshot files match the reference's
    golden slices, and every file it writes is byte-identical to the files
    bp_write_reference_outputs wrote for the same run through Python."""
    import subprocess
    from conftest import ROOT
    exe = ROOT / "mixedprecisionfaracoustic_b200" / "bin" / "biot_reference_run"
    assert exe.exists(), exe
    r = subprocess.run([str(exe), "--nt", "501", "--out", str(tmp_path)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    assert "time loop" in r.stdout
    _, py_out = ref_run
    names = sorted(p.name for p in py_out.iterdir())
    assert sorted(p.name for p in tmp_path.iterdir()) == names
    for n in names:
        assert (tmp_path / n).read_bytes() == (py_out / n).read_bytes(), n
    for f in ("txx", "vux", "vuz", "vwx", "vwz"):
        assert rel_l2(_parse(tmp_path / f"{f}500.dat"), golden[f + "500"]) <= 1e-5, f
