"""Pin the CPU oracle to the reference itself: golden vectors produced by the
reference's own CUDA kernels (compiled from the reference sources for
sm_100a, each operation rounded on its own) on race-free seeded inputs
(tests/golden/make_golden.py).  The oracle, fed the stored inputs, must
reproduce the reference's allocated block set, every voxel and every ray-cast
depth / position / colour map bit for bit (SHA-256 of the canonical
export).  CPU only."""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def test_fixtures_present():
    assert len(FIXTURES) >= 3


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_reproduces_reference_kernels(oracle_mod, path):
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden

    g = np.load(path)
    W, H, n = int(g["W"]), int(g["H"]), int(g["frames"])
    voxel, trunc = float(g["voxel"]), float(g["trunc"])
    fx, fy, cx, cy = (float(g[k]) for k in ("fx", "fy", "cx", "cy"))
    orc = oracle_mod.OracleScene(voxel)
    for i in range(n):
        orc.integrate(g[f"pointmap_{i}"], g[f"rgb_{i}"], trunc, g[f"pose_{i}"], fx, fy, cx, cy)
        r = orc.render(W, H, g[f"pose_{i}"], fx, fy, cx, cy, float(g["min_depth"]), float(g["max_depth"]))
        assert np.array_equal(r["depth"].view(np.uint32), g[f"ref_depth_{i}"].view(np.uint32)), i
        assert make_golden.render_digest(r["depth"], r["position"], r["color"]) == str(g[f"ref_render_sha256_{i}"])
    coords, vox = orc.export()
    assert coords.shape[0] == int(g["ref_blocks"]) == int(g["reffma_blocks"])
    assert make_golden.volume_digest(coords, vox["raw"]) == str(g["ref_volume_sha256"])
