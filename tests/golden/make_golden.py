"""Regenerates tests/golden/float_snapshots.npz from the reference's shipped
golden snapshots (Float/*.dat: 192 x 192 y-mid slices written with "%e ").

    python tests/golden/make_golden.py <reference checkout>

The reference project is read here, in the build container; the GPU box and
the tests only read the committed .npz.
"""
import sys
from pathlib import Path

import numpy as np

NAMES = ["txx500", "txx1000", "txx1500", "txx2000", "txx2500", "txx3000", "txx",
         "vux500", "vuz500", "vwx500", "vwz500"]


def read_dat(path: Path) -> np.ndarray:
    rows = [ln.split() for ln in path.read_text().splitlines() if ln.strip()]
    return np.array([[float(v) for v in r] for r in rows], dtype=np.float64)


def main(ref: Path) -> None:
    out = {}
    for n in NAMES:
        a = read_dat(ref / "Float" / f"{n}.dat")
        assert a.shape == (192, 192), (n, a.shape)
        # %e keeps 7 significant digits: float32 holds them exactly enough
        out[n] = a.astype(np.float32)
    dst = Path(__file__).resolve().parent / "float_snapshots.npz"
    np.savez_compressed(dst, **out)
    print(dst, {k: float(np.abs(v).max()) for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout holding Float/*.dat>")
    main(Path(sys.argv[1]))
