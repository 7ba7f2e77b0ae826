"""Large 3D FP32 grids launch the same per-cell arithmetic under looser
register caps (PolF32W, from 16 M updated cells per launch).  A child process
with BP_WIDE_CELLS=0 takes that path on small grids: its traces and fields
must equal the default kernels' bit for bit (tolerance 0), at orders 2 and 4,
alone and batched."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = Path(__file__).resolve().parent

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
from mixedprecisionfaracoustic_b200 import Batch, Simulation
from test_gpu_parity import small_3d
out = {}
for order in (2, 4):
    cfg, med = small_3d(order=order, precision="fp32", n=30, nt=90)
    with Simulation(cfg, med) as s:
        s.run(cfg.nt)
        out[f"o{order}"] = {c: s.traces(c).tolist() for c in ("txx", "vux", "p")}
        out[f"o{order}_txz"] = s.field("txz").ravel()[::97].tolist()
cfgs, meds = [], []
for n in (22, 30):
    c, m = small_3d(order=2, precision="fp32", n=n, nt=60)
    cfgs.append(c); meds.append(m)
b = Batch(cfgs, meds, steps_per_sync=16)
b.run(60); b.sync()
out["batch"] = [b.traces(i, "txx").tolist() for i in range(2)]
b.close()
print(json.dumps(out))
"""


def child(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD, str(HERE.parent), str(HERE)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_large_grid_caps_are_bit_identical():
    wide = child({"BP_WIDE_CELLS": "0"})
    base = child({"BP_WIDE_CELLS": str(1 << 40)})
    def same(a, b):                       # exact, element by element
        if isinstance(a, dict):
            return a.keys() == b.keys() and all(same(a[k], b[k]) for k in a)
        if isinstance(a, list):
            return len(a) == len(b) and all(same(x, y) for x, y in zip(a, b))
        return a == b
    for k in base:
        assert same(wide[k], base[k]), k
    assert np.abs(np.asarray(base["o2"]["txx"])).max() > 0
