"""Depth image -> point map and normals (vsg_depth_to_pointmap) against a
float32 numpy restatement of the back-projection and of the normal fallback
of CustomDepthMapGenerator.cpp:163-209, bit for bit; and a frame integrated
from the back-projected depth equals the oracle's from the same point map
(needs a GPU)."""
import numpy as np
import pytest

from parity_util import compare_volumes

pytestmark = pytest.mark.gpu


def _restate(depth, fx, fy, cx, cy):
    f32 = np.float32
    H, W = depth.shape
    x = np.arange(W, dtype=f32)[None, :].repeat(H, 0)
    y = np.arange(H, dtype=f32)[:, None].repeat(W, 1)
    fx, fy, cx, cy = f32(fx), f32(fy), f32(cx), f32(cy)

    def bp(xx, yy, d):
        return np.stack([(xx - cx) * d / fx, (yy - cy) * d / fy, d], -1)

    valid = (depth > 0) & np.isfinite(depth)
    pm = np.where(valid[..., None], bp(x, y, depth), f32(0))
    nm = np.zeros((H, W, 3), f32)
    c = bp(x[1:-1, 1:-1], y[1:-1, 1:-1], depth[1:-1, 1:-1])
    r = bp(x[1:-1, 1:-1] + f32(1), y[1:-1, 1:-1], depth[1:-1, 2:])
    w = bp(x[1:-1, 1:-1], y[1:-1, 1:-1] + f32(1), depth[2:, 1:-1])
    a, b = r - c, w - c
    cr = np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                   a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)
    ln = np.sqrt((cr[..., 0] * cr[..., 0] + cr[..., 1] * cr[..., 1]) + cr[..., 2] * cr[..., 2])
    with np.errstate(divide="ignore", invalid="ignore"):
        n = cr * (f32(1) / ln)[..., None]
    ok = (depth[1:-1, 1:-1] > 0) & (ln > 0)
    nm[1:-1, 1:-1] = np.where(ok[..., None], n, f32(0))
    return pm.astype(f32), nm


def test_depth_to_pointmap_matches_restatement(cuda, synth_mod):
    import vsg

    fr, K = synth_mod.tabletop_stream(5, 2, 320, 240)
    depth = np.ascontiguousarray(fr[1].pointmap[..., 2]).astype(np.float32)
    depth[10, 10] = np.nan
    depth[11, 10] = -1.0
    depth[12, 10] = np.inf
    pm, nm = vsg.depth_to_pointmap(cuda.from_numpy(depth).cuda(), K.fx, K.fy, K.cx, K.cy)
    want_pm, want_nm = _restate(depth, K.fx, K.fy, K.cx, K.cy)
    assert np.array_equal(pm.cpu().numpy().view(np.uint32), want_pm.view(np.uint32))
    got_nm = nm.cpu().numpy()
    fin = np.isfinite(want_nm).all(-1)
    assert np.array_equal(got_nm[fin].view(np.uint32), want_nm[fin].view(np.uint32))
    assert np.all(pm.cpu().numpy()[10:13, 10] == 0)


def test_integrating_backprojected_depth_matches_oracle(cuda, synth_mod, oracle_mod):
    import vsg

    fr, K = synth_mod.tabletop_stream(6, 3, 160, 120)
    sc = vsg.Scene(voxel_size=0.004, truncation=0.02, hash_num_slots=20011, num_sdf_blocks=40000)
    o = oracle_mod.OracleScene(0.004)
    for f in fr:
        depth = cuda.from_numpy(np.ascontiguousarray(f.pointmap[..., 2])).cuda()
        pm, nm = vsg.depth_to_pointmap(depth, K.fx, K.fy, K.cx, K.cy)
        rgb = cuda.from_numpy(f.rgb).cuda()
        sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        o.integrate(pm.cpu().numpy(), f.rgb, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
    gc, gv = sc.export()
    oc, ov = o.export()
    v = compare_volumes(gc, gv, oc, ov["raw"])
    assert v["same_blocks"] and v["bit_exact"], v
