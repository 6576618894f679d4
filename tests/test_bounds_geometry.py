"""The geometry behind the ray caster's per-tile distance bounds (CPU).

k_tile_bounds (csrc/vsg_raycast_core.cuh, tile_bounds_range) takes every
block with a weighted voxel as the box of its weighted 2x2x2 sub-cubes grown
by 2 voxels, clips it at half the minimum depth, projects it onto 8x4 pixel
tiles (64x32 tiles for large boxes, one shared entry beyond that) and keeps
the box's nearest and farthest camera distance per tile; apply_bounds then
starts each ray at its tile's nearest distance minus a margin and stops it
after the farthest plus the margin.  The claim that makes this exact: every
march sample with a weighted voxel among its 8 taps lies inside that range.

This test restates the bounds in numpy and checks the claim sample by sample
on the march the kernel takes (RayCastRender.cu:447-500 ray setup, :389-392
FP32 chain, :17-25 and :127-170 tap voxels, all in float32 without
contraction) over an oracle volume, from random poses inside and around it,
with fields of view from very wide to narrow and minimum depths down to 1 cm.
The CUDA code itself is checked against the oracle on the GPU
(tests/test_gpu_render_bounds.py and the parity suites).
"""
import warnings

import numpy as np
import pytest

W, H = 40, 30
VOX = np.float32(0.004)
TRUNC = 0.02
OFF = 1 << 20  # voxel-index offset for packing keys (21 bits per axis)


def _pack(gx, gy, gz):
    return ((gx + OFF) << 42) | ((gy + OFF) << 21) | (gz + OFF)


@pytest.fixture(scope="module")
def volume(oracle_mod, synth_mod):
    fr, K = synth_mod.tabletop_stream(5, 3, 160, 120)
    orc = oracle_mod.OracleScene(float(VOX))
    for f in fr:
        orc.integrate(f.pointmap, f.rgb, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
    coords, vox = orc.export()
    w = vox["weight"]
    bi, li = np.nonzero(w > 0)
    lx, ly, lz = li % 8, (li // 8) % 8, li // 64
    c = coords.astype(np.int64)
    gx, gy, gz = c[bi, 0] * 8 + lx, c[bi, 1] * 8 + ly, c[bi, 2] * 8 + lz
    assert np.abs(np.concatenate([gx, gy, gz])).max() < OFF
    keys = np.unique(_pack(gx, gy, gz))
    # per weighted block: bounding box of its weighted sub-cubes
    blocks, first = np.unique(bi, return_index=True)
    smin = np.stack([np.minimum.reduceat(a // 2, first) for a in (lx, ly, lz)], 1)
    smax = np.stack([np.maximum.reduceat(a // 2, first) for a in (lx, ly, lz)], 1)
    base = c[blocks] * 8
    v = float(VOX)
    lo = (base + 2 * smin - 2).astype(np.float64) * v
    hi = (base + 2 * smax + 4).astype(np.float64) * v
    wlo = np.array([gx.min(), gy.min(), gz.min()]) * v
    whi = np.array([gx.max(), gy.max(), gz.max()]) * v
    sel = np.random.default_rng(0).choice(gx.size, 4096, replace=False)
    pts = (np.stack([gx[sel], gy[sel], gz[sel]], 1) + 0.5) * v  # weighted voxel centres to aim at
    return keys, lo, hi, wlo, whi, pts


def _tile_bounds(lo, hi, R, cam, fx, fy, cx, cy, min_d):
    """Restatement of tile_bounds_range: per 8x4 tile, per 64x32 tile and a
    shared entry, the min of the boxes' nearest and max of their farthest
    camera distances (inf / -inf: no box)."""
    t1x, t1y, t2x, t2y = (W + 7) // 8, (H + 3) // 4, (W + 63) // 64, (H + 31) // 32
    l1n, l1f = np.full((t1y, t1x), np.inf), np.full((t1y, t1x), -np.inf)
    l2n, l2f = np.full((t2y, t2x), np.inf), np.full((t2y, t2x), -np.inf)
    gn, gf = np.inf, -np.inf
    dl, dh = lo - cam, hi - cam
    dmin = np.linalg.norm(np.maximum(np.maximum(dl, -dh), 0.0), axis=1)
    dmax = np.linalg.norm(np.maximum(np.abs(dl), np.abs(dh)), axis=1)
    corners = np.stack([np.where([(k >> a) & 1 for a in range(3)], hi, lo) for k in range(8)], 1)  # (n,8,3)
    P = (corners - cam) @ R  # camera coordinates: R^T (X - cam)
    zc = 0.5 * min_d
    front = P[:, :, 2] >= zc
    with np.errstate(divide="ignore", invalid="ignore"):
        u = np.where(front, fx * (P[:, :, 0] / P[:, :, 2]) + cx, np.nan)
        w = np.where(front, fy * (P[:, :, 1] / P[:, :, 2]) + cy, np.nan)
        us, ws = [u], [w]
        for k in range(8):
            for ax in (1, 2, 4):
                if k & ax:
                    continue
                j = k | ax
                cross = front[:, k] != front[:, j]
                t = (zc - P[:, k, 2]) / (P[:, j, 2] - P[:, k, 2])
                q = P[:, k] + t[:, None] * (P[:, j] - P[:, k])
                us.append(np.where(cross, fx * (q[:, 0] / zc) + cx, np.nan)[:, None])
                ws.append(np.where(cross, fy * (q[:, 1] / zc) + cy, np.nan)[:, None])
        U, Wv = np.concatenate(us, 1), np.concatenate(ws, 1)
    with warnings.catch_warnings():  # boxes wholly nearer than the clip plane: all NaN, dropped below
        warnings.simplefilter("ignore", RuntimeWarning)
        u0, u1 = np.nanmin(U, 1) - 2.0, np.nanmax(U, 1) + 2.0
        w0, w1 = np.nanmin(Wv, 1) - 2.0, np.nanmax(Wv, 1) + 2.0
    keep = front.any(1) & (u1 >= 0) & (w1 >= 0) & (u0 <= W - 1) & (w0 <= H - 1)
    for i in np.nonzero(keep)[0]:
        x0, x1 = int(max(u0[i], 0.0)), int(min(u1[i], W - 1.0))
        y0, y1 = int(max(w0[i], 0.0)), int(min(w1[i], H - 1.0))
        a = (slice(y0 >> 2, (y1 >> 2) + 1), slice(x0 >> 3, (x1 >> 3) + 1))
        b = (slice(y0 >> 5, (y1 >> 5) + 1), slice(x0 >> 6, (x1 >> 6) + 1))
        if ((x1 >> 3) - (x0 >> 3) + 1) * ((y1 >> 2) - (y0 >> 2) + 1) <= 64:
            l1n[a] = np.minimum(l1n[a], dmin[i])
            l1f[a] = np.maximum(l1f[a], dmax[i])
        elif ((x1 >> 6) - (x0 >> 6) + 1) * ((y1 >> 5) - (y0 >> 5) + 1) <= 4096:
            l2n[b] = np.minimum(l2n[b], dmin[i])
            l2f[b] = np.maximum(l2f[b], dmax[i])
        else:
            gn, gf = min(gn, dmin[i]), max(gf, dmax[i])
    ys, xs = np.mgrid[0:H, 0:W]
    near = np.minimum(np.minimum(l1n[ys >> 2, xs >> 3], l2n[ys >> 5, xs >> 6]), gn)
    far = np.maximum(np.maximum(l1f[ys >> 2, xs >> 3], l2f[ys >> 5, xs >> 6]), gf)
    return near.astype(np.float32), far.astype(np.float32)


def _tap(q):
    sg = np.sign(q).astype(np.float32)
    return np.floor(q + np.float32(0.5) * sg).astype(np.int64)


def _weighted_tap(keys, px, py, pz):
    """Does any of the sample's 8 tap voxels hold a weight?"""
    v, half = VOX, VOX / np.float32(2)
    dx, dy, dz = px - half, py - half, pz - half
    ax = (_tap(dx / v), _tap((dx + v) / v))
    ay = (_tap(dy / v), _tap((dy + v) / v))
    az = (_tap(dz / v), _tap((dz + v) / v))
    hit = np.zeros(px.shape, bool)
    for i in range(8):
        k = _pack(ax[i & 1], ay[(i >> 1) & 1], az[i >> 2])
        pos = np.minimum(np.searchsorted(keys, k), keys.size - 1)
        hit |= keys[pos] == k
    return hit


def _random_pose(rng, wlo, whi, pts):
    """A camera anywhere in the volume's box grown by 0.5 m, looking at a
    random weighted voxel, with a random roll."""
    cam = rng.uniform(wlo - 0.5, whi + 0.5)
    z = pts[rng.integers(len(pts))] - cam
    z /= np.linalg.norm(z)
    up = rng.normal(size=3)
    x = np.cross(up, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    T = np.eye(4)
    T[:3, :3] = np.stack([x, y, z], 1)
    T[:3, 3] = cam
    return T.astype(np.float32)


@pytest.mark.parametrize("seed", range(12))
def test_weighted_samples_lie_within_their_tile_bounds(volume, seed):
    keys, lo, hi, wlo, whi, pts = volume
    rng = np.random.default_rng(seed)
    T = _random_pose(rng, wlo, whi, pts)
    fx = fy = float(rng.choice([15.0, 40.0, 150.0, 900.0]))
    cx, cy = (W - 1) / 2 + rng.uniform(-5, 5), (H - 1) / 2 + rng.uniform(-5, 5)
    min_d, max_d = float(rng.choice([0.01, 0.05, 0.2])), 2.5
    f32 = np.float32
    R32, cam32 = T[:3, :3], T[:3, 3].copy()
    near, far = _tile_bounds(lo, hi, R32.astype(np.float64), cam32.astype(np.float64), fx, fy, cx, cy, min_d)
    # ray setup in float32, no contraction (renderKernel, RayCastRender.cu:447-500)
    ys, xs = np.mgrid[0:H, 0:W]
    cdx = (xs.astype(f32) - f32(cx)) / f32(fx)
    cdy = (ys.astype(f32) - f32(cy)) / f32(fy)
    cdz = np.ones_like(cdx)
    cl = np.sqrt((cdx * cdx + cdy * cdy) + cdz * cdz)
    cdx, cdy, cdz = cdx / cl, cdy / cl, cdz / cl
    wd = [(R32[i, 0] * cdx + R32[i, 1] * cdy) + R32[i, 2] * cdz for i in range(3)]
    wl = np.sqrt((wd[0] * wd[0] + wd[1] * wd[1]) + wd[2] * wd[2])
    wd = [c / wl for c in wd]
    d2r = f32(1.0) / cdz
    rc = d2r * f32(min_d)
    re = d2r * f32(max_d)
    h = VOX * f32(0.5)
    cm = f32(np.abs(cam32).max())
    with np.errstate(invalid="ignore"):  # inf - inf: a tile without boxes admits no sample
        first = near - (f32(1e-4) + f32(1e-4) * near + f32(1e-6) * (cm + near))
        last = far + (f32(1e-4) + f32(1e-4) * far + f32(1e-6) * (cm + far))
    checked = 0
    with np.errstate(invalid="ignore"):
        while True:
            live = rc < re
            if not live.any():
                break
            px = cam32[0] + rc * wd[0]
            py = cam32[1] + rc * wd[1]
            pz = cam32[2] + rc * wd[2]
            wt = _weighted_tap(keys, px, py, pz) & live
            checked += int(wt.sum())
            bad = wt & ~((rc >= first) & (rc < last))
            assert not bad.any(), (seed, np.argwhere(bad)[:5], rc[bad][:5], first[bad][:5], last[bad][:5])
            rc = np.where(live, rc + h, rc)
    assert checked > 0  # the pose looks at the surface: some samples read weighted voxels
