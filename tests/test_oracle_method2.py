"""The oracle's normal-direction allocation (Method 2) against a plain-Python
float32 restatement on a small frame (no GPU): the block set and each
block's parent pixel after allocBlocksFromDepthMapMethod2Kernel
(VoxelScene.cu:768-912), and the parent-pixel branch of the integration
(VoxelScene.cu:1015-1035) for the voxels of parent blocks."""
import ctypes

import numpy as np

f32 = np.float32
TRUNC, VOXEL = 0.02, 0.004


def _xform(T, p):
    return [f32(f32(f32(T[4 * r] * p[0]) + f32(T[4 * r + 1] * p[1])) + f32(T[4 * r + 2] * p[2])) + T[4 * r + 3]
            for r in range(3)]


def _rot(T, n):
    return [f32(f32(T[4 * r] * n[0]) + f32(T[4 * r + 1] * n[1])) + f32(T[4 * r + 2] * n[2]) for r in range(3)]


def _norm(v):
    return np.sqrt(f32(f32(v[0] * v[0]) + f32(v[1] * v[1])) + f32(v[2] * v[2]))


def _dda(L, s, e):
    out = np.zeros(3 * 1024, np.int32)
    n = L.orc_dda_blocks(np.asarray(s, f32).ctypes.data_as(ctypes.c_void_p),
                         np.asarray(e, f32).ctypes.data_as(ctypes.c_void_p), f32(VOXEL),
                         out.ctypes.data_as(ctypes.c_void_p))
    return [tuple(out[3 * i:3 * i + 3]) for i in range(n)]


def test_method2_blocks_parents_and_parent_integration(oracle_mod, synth_mod):
    fr, K = synth_mod.tabletop_stream(1, 1, 40, 30)
    f = fr[0]
    T = np.asarray(f.pose, f32).reshape(16)
    cam = [T[3], T[7], T[11]]
    L = oracle_mod.lib()
    blocks, parents = set(), {}
    tr = f32(TRUNC)
    for y in range(K.height):
        for x in range(K.width):
            p = [f32(c) for c in f.pointmap[y, x]]
            if p == [0, 0, 0]:
                continue
            nc = [f32(c) for c in f.normals[y, x]]
            nl = _norm(nc)
            if nl < f32(0.1):
                continue
            n = [c / nl for c in nc]
            w = _xform(T, p)
            nw = _rot(T, n)
            nl = _norm(nw)
            if nl > f32(1e-6):
                nw = [c / nl for c in nw]
            rd = [w[k] - cam[k] for k in range(3)]
            rl = _norm(rd)
            if rl > 0:
                rd = [c / rl for c in rd]
                blocks.update(_dda(L, w, [w[k] + f32(rd[k] * tr) for k in range(3)]))
            for b in _dda(L, w, [w[k] - f32(nw[k] * tr) for k in range(3)]):
                blocks.add(b)
                parents[b] = max(parents.get(b, 0), (1 << 32) | (y << 16) | x)
    o = oracle_mod.OracleScene(VOXEL)
    o.set_alloc_method(2)
    o.integrate(f.pointmap, f.rgb, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy, normals=f.normals)
    coords, vox = o.export()
    got = [tuple(c) for c in coords.tolist()]
    assert set(got) == blocks and len(got) == len(blocks)
    tags = o.export_parents()
    assert {b: int(t) for b, t in zip(got, tags) if t} == parents
    assert len(parents) > 10

    # parent blocks: every voxel integrates the parent pixel's point
    sdf = np.ascontiguousarray(vox["sdf"]).reshape(len(got), 512)
    wgt = np.asarray(vox["weight"]).reshape(len(got), 512)
    checked = 0
    for bi, b in enumerate(got):
        t = parents.get(b)
        if not t:
            continue
        px, py = t & 0xFFFF, (t >> 16) & 0xFFFF
        P = _xform(T, [f32(c) for c in f.pointmap[py, px]])
        cdist = _norm([P[k] - cam[k] for k in range(3)])
        for li in range(0, 512, 7):
            lx, ly, lz = li % 8, (li // 8) % 8, li // 64
            wv = [f32(int(b[k]) * 8 + (lx, ly, lz)[k]) * f32(VOXEL) for k in range(3)]
            s = _norm([wv[k] - P[k] for k in range(3)])
            if _norm([wv[k] - cam[k] for k in range(3)]) < cdist:
                s = -s
            if s < -tr or s > tr:
                assert wgt[bi, li] == 0
            else:
                assert wgt[bi, li] == 1 and sdf[bi, li].view(np.uint32) == f32(s).view(np.uint32)
                checked += 1
    assert checked > 100
