"""Point-cloud splat on the GPU (vsg_splat_points) against the oracle's
restatement of CustomDepthMapGenerator::generateFromPointCloud, bit for bit
on every output, in both modes (needs a GPU)."""
import numpy as np
import pytest

from test_oracle_splat import CX, CY, FX, FY, H, W, _cloud

pytestmark = pytest.mark.gpu


def _check(cuda, oracle_mod, pts, w, h, fx, fy, cx, cy, nrm=None, col=None, mode=0, **kw):
    import vsg

    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a)).cuda() if a is not None else None
    got = vsg.splat_points(t(pts), w, h, fx, fy, cx, cy, normals=t(nrm), colors=t(col), mode=mode, **kw)
    want = oracle_mod.splat_points(pts, w, h, fx, fy, cx, cy, normals=nrm, colors=col, mode=mode, **kw)
    for k in ("depth", "pointmap", "normalmap", "colormap"):
        g = got[k].cpu().numpy()
        assert np.array_equal(g.view(np.uint8), want[k].view(np.uint8)), (k, mode)
    assert got["n_valid"] == int((want["depth"] > 0).sum())
    return got


@pytest.mark.parametrize("mode", [0, 1])
def test_small_cloud_every_rule(cuda, oracle_mod, mode):
    rng = np.random.default_rng(11)
    pts = _cloud(rng)
    pts[9] = [np.nan, 0.0, 1.0]
    pts[10] = [0.0, 0.0, np.nan]
    nrm = rng.normal(size=(250, 3)).astype(np.float32)
    col = rng.integers(0, 256, size=(300, 3)).astype(np.uint8)
    _check(cuda, oracle_mod, pts, W, H, FX, FY, CX, CY, nrm, col, mode)
    _check(cuda, oracle_mod, pts, W, H, FX, FY, CX, CY, None, None, mode)
    _check(cuda, oracle_mod, pts, W, H, FX, FY, CX, CY, nrm, col, mode, min_depth=1.0, max_depth=1.5)


@pytest.mark.parametrize("mode", [0, 1])
def test_overlapping_scans_640x480(cuda, oracle_mod, synth_mod, mode):
    """Two tabletop frames' points seen from the first camera (many pixels
    receive several points), with per-point normals and colours."""
    fr, K = synth_mod.tabletop_stream(5, 2, 640, 480)
    T0, T1 = (np.asarray(f.pose, np.float64) for f in fr)
    clouds, normals, colors = [], [], []
    for f, T in zip(fr, (T0, T1)):
        m = np.any(f.pointmap != 0, -1)
        p = f.pointmap[m].astype(np.float64)
        M = np.linalg.inv(T0) @ T
        clouds.append((p @ M[:3, :3].T + M[:3, 3]).astype(np.float32))
        normals.append((f.normals[m].astype(np.float64) @ M[:3, :3].T).astype(np.float32))
        colors.append(f.rgb[m])
    pts, nrm, col = np.concatenate(clouds), np.concatenate(normals), np.concatenate(colors)
    got = _check(cuda, oracle_mod, pts, K.width, K.height, K.fx, K.fy, K.cx, K.cy, nrm, col, mode)
    assert got["n_valid"] > 100000
    _check(cuda, oracle_mod, pts, K.width, K.height, K.fx, K.fy, K.cx, K.cy, None, col[: len(col) // 2], mode)


def test_empty_cloud(cuda, oracle_mod):
    got = _check(cuda, oracle_mod, np.zeros((0, 3), np.float32), 32, 24, 20.0, 20.0, 16.0, 12.0)
    assert got["n_valid"] == 0
