"""Turns the text outputs of one run of a reference program into a small .npz
golden file.

    python tests/golden/make_seismogram_golden.py <run dir> <out.npz> [--all-rows]

<run dir> holds the files the reference's Float or Half program writes in its
working directory (wfile / wfile3d, Float/main.cu:1501-1516,1563-1588,
Half/main.cu:1875-1960): sisx.dat, sisz.dat, sisvu.dat, sisvw.dat, sisp.dat
(NZ_ext receiver rows of NT "%e " values, each row ended by "\\n\\n").

The runs are made with the reference's own programs, unmodified, compiled for
sm_100a by `make -C oracle ref REF_DIR=<reference checkout>` into oracle/_ref/
(float_ref: the Float build; float_ref_nofma: the same source compiled with
-fmad=false; half_ref: the Half build) and run on a B200 in an empty directory,
e.g. `cd <run dir> && <repo>/oracle/_ref/float_ref`.

Kept: the seismograms of every 8th receiver row plus the source row 52
(25 of 192 rows) unless --all-rows, as float32 (the text holds 7 significant
digits).  Made this way: float_ref_seismograms.npz (float_ref),
float_ref_nofma_seismograms.npz (float_ref_nofma), half_ref_seismograms.npz
(half_ref).
"""
import sys
from pathlib import Path

import numpy as np

SIS = ("sisx", "sisz", "sisvu", "sisvw", "sisp")
SOURCE_ROW = 52


def read_dat(path: Path) -> np.ndarray:
    rows = [ln.split() for ln in path.read_text().splitlines() if ln.strip()]
    return np.array([[float(v) for v in r] for r in rows], dtype=np.float64)


def main(run: Path, out: Path, all_rows: bool) -> None:
    first = read_dat(run / "sisx.dat")
    nrow = first.shape[0]
    rows = np.arange(nrow) if all_rows else np.array(sorted(set(range(0, nrow, 8)) | {SOURCE_ROW}), np.int32)
    res = {"rows": rows.astype(np.int32)}
    for k in SIS:
        a = first if k == "sisx" else read_dat(run / f"{k}.dat")
        assert a.shape == first.shape, (k, a.shape)
        res[k] = a[rows].astype(np.float32)
    np.savez_compressed(out, **res)
    print(out, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if len(args) != 2:
        sys.exit("usage: make_seismogram_golden.py <run dir> <out.npz> [--all-rows]")
    main(Path(args[0]), Path(args[1]), "--all-rows" in sys.argv)
