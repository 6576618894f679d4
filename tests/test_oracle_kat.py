"""Analytic known answers for the oracle (CPU): a noise-free fronto-parallel
plane seen head-on.  The reference's SDF is the distance from the voxel
centre to the back-projected point of the pixel the voxel projects to,
negative in front of the surface (VoxelScene.cu:1052-1066), so for a plane
at depth Z it equals the signed depth difference up to the lateral offset
inside one pixel footprint."""
import math

import numpy as np


def plane_frame(W=96, H=72, f=80.0, Z=1.0):
    cx, cy = (W - 1) / 2.0, (H - 1) / 2.0
    u, v = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    pm = np.stack([(u - cx) * Z / f, (v - cy) * Z / f, np.full_like(u, Z)], -1).astype(np.float32)
    rgb = np.full((H, W, 3), 200, np.uint8)
    return pm, rgb, np.eye(4, dtype=np.float32), (f, f, cx, cy)


def test_plane_sdf_matches_signed_depth(oracle_mod):
    voxel, trunc, Z = 0.004, 0.02, 1.0
    pm, rgb, T, (fx, fy, cx, cy) = plane_frame(Z=Z)
    orc = oracle_mod.OracleScene(voxel)
    st = orc.integrate(pm, rgb, trunc, T, fx, fy, cx, cy)
    assert st["new_blocks"] > 0 and st["updated_voxels"] > 0
    coords, vox = orc.export()
    w = vox["weight"]
    assert set(np.unique(w)) <= {0, 1}  # one frame: every updated voxel has weight 1
    idx = np.nonzero(w == 1)
    b = coords[idx[0]]
    local = idx[1]
    lx, ly, lz = local % 8, (local // 8) % 8, local // 64
    zv = (b[:, 2] * 8 + lz) * voxel
    sdf = vox["sdf"][idx]
    footprint = math.sqrt(2) * 0.5 * Z / fx + 2 * voxel  # lateral offset bound
    signed = zv - Z  # in front of the plane (closer to the camera) is negative
    assert np.all(np.abs(sdf) <= trunc + 1e-7)
    assert np.all(np.abs(np.abs(sdf) - np.abs(signed)) <= footprint)
    inside = np.abs(signed) > footprint
    assert np.all(np.sign(sdf[inside]) == np.sign(signed[inside]))
    assert np.all(vox["rgb"][idx] == 200)


def test_plane_raycast_depth(oracle_mod):
    voxel, trunc, Z = 0.004, 0.02, 1.0
    pm, rgb, T, (fx, fy, cx, cy) = plane_frame(Z=Z)
    orc = oracle_mod.OracleScene(voxel)
    for _ in range(3):
        orc.integrate(pm, rgb, trunc, T, fx, fy, cx, cy)
    r = orc.render(96, 72, T, fx, fy, cx, cy, 0.2, 3.0)
    hit = r["depth"] < 1e9
    assert hit.mean() > 0.9
    # depth of a plane at Z, within a voxel
    assert np.abs(r["depth"][hit] - Z).max() < voxel
    # colour: the trilinear average truncated to uint8 (RayCastRender.cu:205-209)
    # lands on 200 or, after FP rounding just below it, 199
    c = np.round(r["color"][hit][:, :3] * 255.0)
    assert set(np.unique(c)) <= {199.0, 200.0}
