"""Marching cubes (vsg_mc_*) against the oracle's restatement of
MarchingCubes.cu:352-467 on the same volume, bit for bit: the GPU volume is
read back and loaded into the oracle, which extracts with the case table of
the library's header built on the host (its reference rows and generated rows
are pinned on the CPU by test_mc_table.py).  Triangle order is unspecified on both
sides (the reference appends through an atomic counter), so triangles are
compared as sorted multisets of their 18 floats (needs a GPU)."""
import ctypes

import numpy as np
import pytest


pytestmark = pytest.mark.gpu


def _table(hosttest_lib):
    t = np.zeros((256, 16), np.uint8)
    hosttest_lib.vsg_test_mc_table.argtypes = [ctypes.c_void_p]
    hosttest_lib.vsg_test_mc_table(t.ctypes.data)
    return t


def _rows(v, n):
    m = v.shape[0]
    a = np.concatenate([v.reshape(m, 9).view(np.uint32), n.reshape(m, 9).view(np.uint32)], 1)
    return a[np.lexsort(a.T[::-1])]


def _scene(vsg, cuda, synth_mod, seed, W, H, frames, voxel=0.004, trunc=0.02):
    fr, K = synth_mod.tabletop_stream(seed, frames, W, H)
    sc = vsg.Scene(voxel_size=voxel, truncation=trunc, hash_num_slots=20011, num_sdf_blocks=60000)
    for f in fr:
        pm, rgb, nm = (cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals))
        sc.integrate(pm, rgb, nm, K.width, K.height, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
    return sc


def _oracle_of(oracle_mod, sc, voxel):
    coords, vox = sc.export()
    o = oracle_mod.OracleScene(voxel)
    o.load(coords, vox)
    return o


@pytest.mark.parametrize("iso,voxel_override", [(0.0, 0.0), (0.004, 0.0), (-0.003, 0.005)])
def test_mc_matches_oracle(cuda, synth_mod, oracle_mod, hosttest_lib, iso, voxel_override):
    import vsg

    sc = _scene(vsg, cuda, synth_mod, 21, 160, 120, 4)
    probe = vsg.MarchingCubes(1)  # learn the count, then size the output to it
    probe.run(sc, iso=iso, voxel_size=voxel_override)
    need = probe.count()
    probe.close()
    mc = vsg.MarchingCubes(need)
    mc.run(sc, iso=iso, voxel_size=voxel_override)
    n, v, nrm = mc.download()
    o = _oracle_of(oracle_mod, sc, 0.004)
    on, ov, onrm = o.marching_cubes(_table(hosttest_lib), iso, voxel_override if voxel_override > 0 else 0.004, need)
    assert n == on == need == v.shape[0] > 1000
    assert np.array_equal(_rows(v, nrm), _rows(ov, onrm))
    # every normal is unit length or zero
    ln = np.linalg.norm(nrm[:, 0].astype(np.float64), axis=1)
    assert np.all((np.abs(ln - 1) < 1e-5) | (ln == 0))
    mc.close()
    sc.close()


def test_mc_capacity_and_empty(cuda, synth_mod, oracle_mod, hosttest_lib):
    import vsg

    sc = vsg.Scene(voxel_size=0.004, hash_num_slots=5003, num_sdf_blocks=8000)
    mc = vsg.MarchingCubes(64)
    mc.run(sc)  # no block allocated: count 0, like the reference's early return
    n, v, _ = mc.download()
    assert n == 0 and v.shape[0] == 0
    sc.close()
    sc = _scene(vsg, cuda, synth_mod, 22, 96, 72, 2)
    mc.run(sc)
    n, v, nrm = mc.download()
    o = _oracle_of(oracle_mod, sc, 0.004)
    on, ov, onrm = o.marching_cubes(_table(hosttest_lib), 0.0, 0.004, n)
    assert n == on > 64 and v.shape[0] == 64
    full = {r.tobytes() for r in _rows(ov, onrm)}
    assert all(r.tobytes() in full for r in _rows(v, nrm))  # the written ones are genuine
    buf = mc.buffers()
    assert buf["max_triangles"] == 64 and buf["vertices"] and buf["count"]
    # the device int counter (MarchingCubesOutput.d_triangleCount) holds the total too
    assert int(_dev_int32(cuda, buf["count"])) == n
    mc.close()
    sc.close()


class _DevInt32:
    def __init__(self, ptr):
        self.__cuda_array_interface__ = {"shape": (1,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def _dev_int32(torch, ptr):
    torch.cuda.synchronize()
    return torch.as_tensor(_DevInt32(ptr), device="cuda").item()
