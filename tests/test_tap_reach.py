"""How far a ray-cast sample reaches for its trilinear taps (CPU).

The ray caster's distance bounds grow each block's weighted sub-cubes by 2
voxels on the premise that a sample at p reads voxel i only when p lies in
[(i - 1) v, (i + 2) v], i.e. within one voxel of the voxel's cell.  This
checks that premise on the tap arithmetic of trilinearInterpolationSimpleFastFast
(RayCastRender.cu:127-170; worldToVirtualVoxelPos, :17-25: x0 = round half
away from zero of (p - v/2) / v, x1 the same of (p + v/2) / v), evaluated in
FP32 like the kernel, over positions of both signs and of several magnitudes.
"""
import numpy as np
import pytest


def _tap(q):
    q = q.astype(np.float32)
    sg = np.sign(q).astype(np.float32)
    return np.floor((q + np.float32(0.5) * sg).astype(np.float32)).astype(np.int64)


@pytest.mark.parametrize("voxel", [0.0005, 0.002, 0.004, 0.01])
def test_taps_lie_within_one_voxel_of_the_sample(voxel):
    rng = np.random.default_rng(int(voxel * 1e5))
    v = np.float32(voxel)
    n = 1_000_000
    p = (rng.uniform(-50.0, 50.0, n) * rng.choice([1.0, 0.01, 0.001], n)).astype(np.float32)
    dx = (p - v / np.float32(2)).astype(np.float32)
    x0 = _tap((dx / v).astype(np.float32))
    x1 = _tap(((dx + v).astype(np.float32) / v).astype(np.float32))
    pv = p.astype(np.float64) / float(v)
    for i in (x0, x1):
        # p / v in [i - 1, i + 2] up to FP32 rounding of p / v
        assert (pv - (i - 1)).min() > -0.01
        assert ((i + 2) - pv).min() > -0.01
    # the taps are floor(p / v) - 1 .. floor(p / v) + 1
    fl = np.floor(pv).astype(np.int64)
    ok = np.abs(pv - np.round(pv)) > 1e-4 + 1e-6 * np.abs(pv)  # away from the rounding boundaries
    assert np.all((x0[ok] >= fl[ok] - 1) & (x1[ok] <= fl[ok] + 1))
    assert np.all((x1 - x0 >= 0) & (x1 - x0 <= 2))


@pytest.mark.parametrize("voxel", [0.0005, 0.002, 0.004, 0.01])
def test_taps_lie_within_one_subcube_of_the_sample(voxel):
    """The march's skip test (dwm: a weighted voxel within one 2x2x2
    sub-cube) takes the sample's sub-cube as the kernel computes it,
    q = floor(RN(p * RN(1 / RN(2 v)))), and reads the bit dilated by one
    sub-cube.  Every tap voxel's sub-cube is q - 1 .. q + 1, for every
    sample: the taps span 3 voxels, the dilated range 6, and the voxel of
    slack on each side absorbs the rounding of q at the sub-cube faces."""
    rng = np.random.default_rng(int(voxel * 1e5) + 1)
    v = np.float32(voxel)
    n = 1_000_000
    p = (rng.uniform(-50.0, 50.0, n) * rng.choice([1.0, 0.01, 0.001], n)).astype(np.float32)
    # positions on and next to sub-cube faces too
    faces = (rng.integers(-20000, 20000, n // 4) * (2 * float(voxel))).astype(np.float32)
    p = np.concatenate([p, faces, np.nextafter(faces, np.float32(-np.inf)), np.nextafter(faces, np.float32(np.inf))])
    dx = (p - v / np.float32(2)).astype(np.float32)
    x0 = _tap((dx / v).astype(np.float32))
    x1 = _tap(((dx + v).astype(np.float32) / v).astype(np.float32))
    inv_c2 = np.float32(1.0) / (np.float32(2.0) * v)
    q = np.floor((p * inv_c2).astype(np.float32)).astype(np.int64)
    for i in (x0, x1):
        s = i >> 1
        assert np.all((s >= q - 1) & (s <= q + 1))
