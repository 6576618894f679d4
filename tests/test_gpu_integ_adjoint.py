"""Adjoint of one frame's integration (vsg_integrate_backward) against float64
central differences of the updated voxels' SDF as a function of the frame's
pose and point map, with the forward's decisions (each voxel's pixel, sign
and truncation test) frozen by a float32 retrace of integrateDepthMapIntoBlocks
(VoxelScene.cu:954-1126) that must reproduce exactly which voxels the GPU
updated (needs a GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VOXEL, TRUNC = 0.004, 0.02


def _ctz(x):
    """CUDA float -> int conversion (round toward zero, saturating, NaN -> 0)."""
    x = np.where(np.isnan(x), 0.0, x)
    return np.clip(np.trunc(x), -2147483648.0, 2147483647.0).astype(np.int64)


def _retrace(coords, T, pm, K, parents=None):
    """Float32 retrace of the forward's per-voxel projection and tests; a
    block with a parent tag (normal-direction allocation) whose pixel is in
    the image and holds a point uses that pixel for all its voxels.
    Returns per voxel (n, 512): updated mask, pixel index, negative flag and
    the float32 voxel centre."""
    f32 = np.float32
    T = np.asarray(T, f32).reshape(16)
    v = f32(VOXEL)
    n = len(coords)
    li = np.arange(512)
    lx, ly, lz = li & 7, (li >> 3) & 7, li >> 6
    wx = (((coords[:, 0:1] * 8 + lx[None]).astype(np.int64)).astype(f32) * v)
    wy = (((coords[:, 1:2] * 8 + ly[None]).astype(np.int64)).astype(f32) * v)
    wz = (((coords[:, 2:3] * 8 + lz[None]).astype(np.int64)).astype(f32) * v)
    rx, ry, rz = wx - T[3], wy - T[7], wz - T[11]
    cxp = (T[0] * rx + T[4] * ry) + T[8] * rz
    cyp = (T[1] * rx + T[5] * ry) + T[9] * rz
    czp = (T[2] * rx + T[6] * ry) + T[10] * rz
    with np.errstate(all="ignore"):
        sx = (cxp * f32(K.fx)) / czp + f32(K.cx)
        sy = (cyp * f32(K.fy)) / czp + f32(K.cy)
    ix, iy = _ctz(sx + f32(0.5)), _ctz(sy + f32(0.5))
    inb = (ix >= 0) & (ix < K.width) & (iy >= 0) & (iy < K.height)
    pix = np.where(inb, iy * K.width + ix, 0)
    if parents is not None:
        px = (parents & 0xFFFF).astype(np.int64)
        py = ((parents >> 16) & 0xFFFF).astype(np.int64)
        pp = np.where((parents != 0) & (px < K.width) & (py < K.height), py * K.width + px, -1)
        flat = pm.reshape(-1, 3)
        pp = np.where((pp >= 0) & np.any(flat[np.maximum(pp, 0)] != 0, -1), pp, -1)
        inb = np.where(pp[:, None] >= 0, True, inb)
        pix = np.where(pp[:, None] >= 0, pp[:, None], pix)
    p = pm.reshape(-1, 3)[pix]
    valid = inb & np.any(p != 0, -1)
    P = [((T[4 * r] * p[..., 0] + T[4 * r + 1] * p[..., 1]) + T[4 * r + 2] * p[..., 2]) + T[4 * r + 3] for r in range(3)]
    ex, ey, ez = P[0] - T[3], P[1] - T[7], P[2] - T[11]
    pdist = np.sqrt((ex * ex + ey * ey) + ez * ez)
    dx, dy, dz = wx - P[0], wy - P[1], wz - P[2]
    sdf = np.sqrt((dx * dx + dy * dy) + dz * dz)
    vdist = np.sqrt(((wx - T[3]) * (wx - T[3]) + (wy - T[7]) * (wy - T[7])) + (wz - T[11]) * (wz - T[11]))
    neg = vdist < pdist
    sdf = np.where(neg, -sdf, sdf)
    upd = valid & ~((sdf < -f32(TRUNC)) | (sdf > f32(TRUNC)))
    return upd, pix, neg, np.stack([wx, wy, wz], -1).astype(np.float64)


@pytest.mark.parametrize("alloc_method", [1, 2])
def test_integration_gradient_matches_central_differences(cuda, synth_mod, oracle_mod, alloc_method):
    import vsg

    fr, K = synth_mod.tabletop_stream(8, 4, 160, 120)
    sc = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=20011, num_sdf_blocks=40000)
    sc.set_alloc_method(alloc_method)
    orc = oracle_mod.OracleScene(VOXEL)  # lock-step oracle: the blocks' parent pixels
    orc.set_alloc_method(alloc_method)
    for f in fr[:3]:
        pm, rgb, nm = (cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals))
        sc.integrate(pm, rgb, nm, K.width, K.height, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
        orc.integrate(f.pointmap, f.rgb, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy, normals=f.normals)
    c0, v0 = sc.export()
    f = fr[3]
    pm, rgb, nm = (cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals))
    sc.integrate(pm, rgb, nm, K.width, K.height, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
    orc.integrate(f.pointmap, f.rgb, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy, normals=f.normals)
    c1, v1 = sc.export()
    oc, _ = orc.export(with_voxels=False)
    assert np.array_equal(oc, c1)
    parents = orc.export_parents()
    assert (parents != 0).any() == (alloc_method == 2)
    # volume before the frame on the block set after it (new blocks start empty)
    before = {tuple(c): i for i, c in enumerate(c0.tolist())}
    old = np.zeros((len(c1), 512, 8), np.uint8)
    for i, c in enumerate(c1.tolist()):
        j = before.get(tuple(c))
        if j is not None:
            old[i] = v0[j].reshape(512, 8)
    old_sdf = np.ascontiguousarray(old[..., :4]).view(np.float32)[..., 0].astype(np.float64)
    old_w = old[..., 7].astype(np.float64)
    new_w = v1.reshape(-1, 512, 8)[..., 7].astype(np.float64)
    new_sdf = np.ascontiguousarray(v1.reshape(-1, 512, 8)[..., :4]).view(np.float32)[..., 0]

    upd, pix, neg, w = _retrace(c1, f.pose, f.pointmap, K, parents)
    # the retrace reproduces the forward's decisions exactly
    assert np.array_equal(new_w != old_w, upd)
    assert np.all(new_w[upd] == np.minimum(255, old_w[upd] + 1))

    rng = np.random.default_rng(3)
    g = rng.normal(size=(len(c1), 512)).astype(np.float32)
    ptrs = sc.lookup_blocks(c1)
    gbuf = np.zeros((sc.params.num_sdf_blocks, 512), np.float32)
    gbuf[ptrs] = g
    gdev = cuda.from_numpy(gbuf.reshape(-1)).cuda()
    gpm = cuda.zeros((K.height, K.width, 3), dtype=cuda.float32, device="cuda")
    gT, n_upd = sc.integrate_backward(pm, K.width, K.height, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy, gdev,
                                      grad_pointmap=gpm)
    assert n_upd == int(upd.sum())
    g_old = gdev.view(-1, 512).cpu().numpy()[ptrs]
    want_old = np.where(upd, g.astype(np.float64) * old_w / (old_w + 1), g)
    assert np.allclose(g_old, want_old, rtol=1e-6, atol=1e-12)

    # float64 function of the frozen decisions
    gu, pu, su, wu = g[upd].astype(np.float64), pix[upd], np.where(neg[upd], -1.0, 1.0), w[upd]
    ou, Wu = old_sdf[upd], old_w[upd]
    pm64 = f.pointmap.reshape(-1, 3).astype(np.float64)

    def loss(T, pmap=pm64):
        T = np.asarray(T, np.float64)
        P = pmap[pu] @ T[:3, :3].T + T[:3, 3]
        s = su * np.linalg.norm(wu - P, axis=1)
        return float((gu * (ou * Wu + s) / (Wu + 1)).sum())

    # the float64 function agrees with the stored float32 result
    T64 = np.asarray(f.pose, np.float32).astype(np.float64)
    P = pm64[pu] @ T64[:3, :3].T + T64[:3, 3]
    s64 = su * np.linalg.norm(wu - P, axis=1)
    assert np.abs((ou * Wu + s64) / (Wu + 1) - new_sdf[upd]).max() < 1e-6
    h = 1e-6
    fd = np.zeros((3, 4))
    for r in range(3):
        for c in range(4):
            Tp, Tm = T64.copy(), T64.copy()
            Tp[r, c] += h
            Tm[r, c] -= h
            fd[r, c] = (loss(Tp) - loss(Tm)) / (2 * h)
    rel = np.linalg.norm(gT - fd) / np.linalg.norm(fd)
    assert rel <= 1e-4, (rel, gT, fd)
    # point-map gradient at the pixels feeding the most updated voxels
    G = gpm.cpu().numpy().reshape(-1, 3)
    top = np.bincount(pu, minlength=K.width * K.height).argsort()[-5:]
    for px in top:
        for j in range(3):
            pp, pq = pm64.copy(), pm64.copy()
            pp[px, j] += h
            pq[px, j] -= h
            fdp = (loss(T64, pp) - loss(T64, pq)) / (2 * h)
            assert abs(G[px, j] - fdp) <= 1e-3 * abs(fdp) + 1e-6, (px, j, G[px, j], fdp)
