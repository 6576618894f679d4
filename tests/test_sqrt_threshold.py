"""The integration's squared-distance threshold (CPU).

Integration negates a voxel's SDF when RN(sqrt(D_voxel)) < w, w the pixel's
camera distance (VoxelScene.cu:1055-1066).  The library instead compares
D_voxel with D* = the smallest float with RN(sqrt(D*)) >= w, stored per
pixel (sqrt_threshold in csrc/vsg_device.cuh).  RN(sqrt(.)) is
non-decreasing over the floats, so the two tests agree for every D >= 0.
This restates the threshold search in C with the C library's correctly
rounded sqrtf and checks the equivalence on random and boundary values of w
and D, including tiny, huge, zero, infinite and NaN distances.  (The GPU
parity tests check the volumes bit for bit.)
"""
import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def thr(hosttest_lib):
    f = hosttest_lib.vsg_test_sqrt_threshold
    f.argtypes = [ctypes.c_float]
    f.restype = ctypes.c_float
    return f


def _ws(rng):
    w = np.concatenate([rng.uniform(0.05, 6.0, 3000), 10.0 ** rng.uniform(-40, 36, 2000),
                        [0.0, np.inf, np.nan, 1e-45, 2e-38, 3.4e38, 1.0, 2.0, 0.25]]).astype(np.float32)
    return w


def test_threshold_reproduces_the_sqrt_comparison(thr):
    rng = np.random.default_rng(4)
    for w in _ws(rng):
        t = np.float32(thr(float(w)))
        if np.isnan(w):
            assert np.isnan(t)
            continue
        # candidate squared distances around the threshold and at random
        with np.errstate(over="ignore"):
            base = np.float32(w) * np.float32(w) if np.isfinite(w) else np.float32(3e38)
            cand = [t, base] + [np.nextafter(t, np.float32(-1)), np.nextafter(t, np.float32(np.inf))]
            cand += list((np.float64(base) * rng.uniform(0.5, 1.5, 40)).astype(np.float32))
        for d in cand:
            d = np.float32(d)
            if not d >= 0:
                continue
            with np.errstate(invalid="ignore"):
                assert (np.sqrt(d) < w) == (d < t), (w, t, d)


def test_threshold_is_the_least_float_reaching_w(thr):
    rng = np.random.default_rng(5)
    for w in rng.uniform(0.05, 6.0, 2000).astype(np.float32):
        t = np.float32(thr(float(w)))
        assert np.sqrt(t) >= w and np.sqrt(np.nextafter(t, np.float32(-1))) < w
