"""Closed-form replay of the ray caster's FP32 step chain (vsg_fpchain.h)
against serial additions: it must land on the identical float after the
identical number of steps.  Host build of the same header; no GPU."""
import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def L(hosttest_lib):
    lib = hosttest_lib
    for f in (lib.vsg_test_chain_advance, lib.vsg_test_chain_serial):
        f.restype = ctypes.c_float
        f.argtypes = [ctypes.c_float] * 3 + [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    return lib


def _both(L, r, h, tgt, ms):
    s1, s2 = ctypes.c_int(), ctypes.c_int()
    a = L.vsg_test_chain_advance(r, h, tgt, ms, ctypes.byref(s1))
    b = L.vsg_test_chain_serial(r, h, tgt, ms, ctypes.byref(s2))
    return np.float32(a), np.float32(b), s1.value, s2.value


def test_random_chains_match_serial(L):
    rng = np.random.default_rng(1)
    for i in range(30000):
        v = np.float32(rng.choice([0.004, 0.002, 0.003, 0.005, 0.001, 0.0037, 0.01, 0.0123]))
        h = float(np.float32(v * np.float32(0.5)))
        r = float(np.float32(rng.uniform(0.05, 4.0) if i % 3 else rng.uniform(1e-4, 0.3)))
        tgt = float(np.float32(r + rng.uniform(-0.01, 3.5)))
        ms = int(rng.integers(1, 3000)) if i % 4 == 0 else 1 << 22
        a, b, s1, s2 = _both(L, r, h, tgt, ms)
        assert a.view(np.uint32) == b.view(np.uint32) and s1 == s2, (r, h, tgt, ms, a, b, s1, s2)


def test_binade_boundaries_and_ties(L):
    # chains that start just below a power of two, and steps whose ulp count is
    # an exact half (ties to even)
    for r0 in (0.25, 0.5, 1.0, 2.0):
        for d in range(1, 40):
            r = float(np.nextafter(np.float32(r0), np.float32(0)) - np.float32(d * 1e-6))
            for h in (0.002, float(np.float32(2.0 ** -9)), float(np.float32(3 * 2.0 ** -25)), 1e-3):
                a, b, s1, s2 = _both(L, r, h, r0 + 0.05, 1 << 22)
                assert a.view(np.uint32) == b.view(np.uint32) and s1 == s2, (r, h)


def test_no_progress_and_below_target(L):
    a, b, s1, s2 = _both(L, 1.0, 1e-9, 2.0, 100)  # r + h == r: stuck
    assert s1 <= 100 and a == np.float32(1.0)
    a, b, s1, s2 = _both(L, 2.0, 0.002, 1.0, 100)  # already past target
    assert a == b and s1 == s2 == 0
