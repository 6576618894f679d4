"""The running average's division shortcut (CPU).

Integration divides four running sums per updated voxel by the new weight d,
which takes only the values 1..256 (VoxelScene.cu:1101-1110).  The library
replaces x / d by one Markstein correction of x * RN(1/d) (avg_div in
csrc/vsg_device.cuh), enabled per divisor only where a verification on the
GPU at scene creation found it equal to IEEE division for every dividend in
[1, 2) -- which covers every 2^-100 <= |x| < 2^100, since the three
operations commute with scaling by powers of two there.  This restates the
correction with the C library's correctly rounded fmaf and checks it against
IEEE division: every dividend in [1, 2) for a spread of divisors, every
4099th dividend for all 256.  (The GPU tests then check the volumes bit for
bit and that all 256 divisors passed on the device.)
"""
import ctypes

import pytest


@pytest.fixture(scope="module")
def mism(hosttest_lib):
    f = hosttest_lib.vsg_test_avg_div_mismatches
    f.argtypes = [ctypes.c_int, ctypes.c_int]
    f.restype = ctypes.c_long
    return f


@pytest.mark.parametrize("d", [2, 3, 7, 10, 49, 100, 127, 129, 191, 200, 251, 255, 256])
def test_every_dividend_of_one_binade(mism, d):
    assert mism(d, 1) == 0


def test_all_divisors_sampled(mism):
    assert all(mism(d, 4099) == 0 for d in range(1, 257))
