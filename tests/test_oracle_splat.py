"""The oracle's point-cloud splat (CustomDepthMapGenerator::
generateFromPointCloud, CustomDepthMapGenerator.cpp:81-222) against a
plain-Python float32 restatement of that loop on a small cloud built to hit
every rule: several points per pixel, shorter normal / colour lists, points
behind the camera, outside the image and on its edges, and the depth-map
normal fallback (no GPU)."""
import numpy as np

f32 = np.float32
W, H, FX, FY, CX, CY = 12, 9, f32(10.0), f32(11.0), f32(5.5), f32(4.0)


def _cloud(rng, n=400):
    z = rng.uniform(0.5, 2.0, n).astype(f32)
    u = rng.uniform(-1.5, W + 1.5, n).astype(f32)
    v = rng.uniform(-1.5, H + 1.5, n).astype(f32)
    pts = np.stack([(u - CX) * z / FX, (v - CY) * z / FY, z], 1).astype(f32)
    pts[::37, 2] *= -1  # behind the camera
    pts[5] = pts[3]      # exact duplicates: equal z
    pts[6] = pts[3]
    pts[7] = [0.0, 0.0, 1.0]  # the principal point
    pts[8] = [(f32(W) - CX) / FX, 0.0, 1.0]  # u == W exactly: outside
    return pts


def _restate(pts, nrm, col, mode):
    depth = np.zeros((H, W), f32)
    pm = np.zeros((H, W, 3), f32)
    nm = np.zeros((H, W, 3), f32)
    cm = np.zeros((H, W, 3), np.uint8)
    for i, (x, y, z) in enumerate(pts):
        if not z > 0:
            continue
        u = f32(f32(x * FX) / z) + CX
        v = f32(f32(y * FY) / z) + CY
        if not (0 <= u < W and 0 <= v < H):
            continue
        px, py = int(np.floor(u)), int(np.floor(v))
        if mode == 1 and depth[py, px] > 0 and depth[py, px] < z:
            continue
        depth[py, px] = z
        pm[py, px] = (x, y, z)
        if i < len(nrm):
            nm[py, px] = nrm[i]
        elif mode == 1:
            nm[py, px] = 0
        if i < len(col):
            cm[py, px] = col[i]
        elif mode == 1:
            cm[py, px] = 0
    return depth, pm, nm, cm


def _fallback(depth):
    nm = np.zeros((H, W, 3), f32)
    for y in range(1, H - 1):
        for x in range(1, W - 1):
            d = depth[y, x]
            if not d > 0:
                continue
            dr, dd = depth[y, x + 1], depth[y + 1, x]

            def bp(xx, yy, dz):
                return [f32(f32(f32(xx) - CX) * dz) / FX, f32(f32(f32(yy) - CY) * dz) / FY, dz]

            c, r, w = bp(x, y, d), bp(x + 1, y, dr), bp(x, y + 1, dd)
            a = [r[k] - c[k] for k in range(3)]
            b = [w[k] - c[k] for k in range(3)]
            cr = [f32(a[1] * b[2]) - f32(a[2] * b[1]), f32(a[2] * b[0]) - f32(a[0] * b[2]),
                  f32(a[0] * b[1]) - f32(a[1] * b[0])]
            ln = np.sqrt(f32(f32(cr[0] * cr[0]) + f32(cr[1] * cr[1])) + f32(cr[2] * cr[2]))
            if ln > 0:
                inv = f32(1.0) / ln
                nm[y, x] = [f32(cr[k] * inv) for k in range(3)]
    return nm


def test_splat_matches_generator_loop(oracle_mod):
    rng = np.random.default_rng(11)
    pts = _cloud(rng)
    nrm = rng.normal(size=(250, 3)).astype(f32)   # shorter than the cloud
    col = rng.integers(0, 256, size=(300, 3)).astype(np.uint8)
    for mode in (0, 1):
        got = oracle_mod.splat_points(pts, W, H, FX, FY, CX, CY, normals=nrm, colors=col, mode=mode)
        want = _restate(pts, nrm, col, mode)
        for g, w in zip((got["depth"], got["pointmap"], got["normalmap"], got["colormap"]), want):
            assert np.array_equal(g.view(np.uint8), w.view(np.uint8)), mode
        assert (got["depth"] > 0).sum() > W * H // 2
    # last-wins and nearest differ on this cloud
    a = oracle_mod.splat_points(pts, W, H, FX, FY, CX, CY, mode=0)["depth"]
    b = oracle_mod.splat_points(pts, W, H, FX, FY, CX, CY, mode=1)["depth"]
    assert not np.array_equal(a, b) and np.all(b[b > 0] <= a[b > 0])
    # no normals: the depth-map fallback
    got = oracle_mod.splat_points(pts, W, H, FX, FY, CX, CY, mode=0)
    assert np.array_equal(got["normalmap"].view(np.uint32), _fallback(got["depth"]).view(np.uint32))
    # depth range
    r = oracle_mod.splat_points(pts, W, H, FX, FY, CX, CY, mode=1, min_depth=1.0, max_depth=1.5)["depth"]
    assert np.all((r == 0) | ((r >= 1.0) & (r <= 1.5)))
