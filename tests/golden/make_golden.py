"""Generate golden vectors from the reference's own kernels (run on a GPU).

    python tests/golden/make_golden.py OUT_DIR

Builds nothing: needs oracle/_ref/libvsgref_nofma.so and libvsgref.so (built
from the reference sources by oracle/ref_build.py).  For each case it picks
seeded synthetic frames for which the reference's allocation is race-free
(no two new blocks of a frame share a hash bucket -- the reference takes each
bucket's lock once per frame and drops the rest, VoxelScene.cu:176-203; its
bucket hash repeats for some small coordinate triples whatever the bucket
count, so only some seeds qualify),
runs the reference's integrate + ray cast per frame, and saves the inputs and
the reference's outputs: final allocated block set + voxels, and every
frame's depth / position / colour maps.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "real-time-depth-fusion-directional-tsdf_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

CASES = [
    # name, scene seed, frames, W, H, voxel, trunc, buckets, pool blocks
    ("tabletop_64x48_4mm", 13, 3, 64, 48, 0.004, 0.02, 1 << 24, 20000),
    ("tabletop_80x60_6mm", 13, 2, 80, 60, 0.006, 0.03, 1 << 24, 20000),
    ("tabletop_64x48_5mm", 54, 2, 64, 48, 0.005, 0.02, 1 << 24, 20000),
]


def bucket_collision(oracle, frames, K, voxel, trunc, buckets) -> bool:
    """True if some frame allocates two new blocks in one bucket (the
    reference would drop one of them)."""
    orc = oracle.OracleScene(voxel)
    prev = set()
    for f in frames:
        orc.alloc(f.pointmap, trunc, f.pose)
        coords, _ = orc.export(with_voxels=False)
        cur = {tuple(c) for c in coords.tolist()}
        new = cur - prev
        seen = {}
        for c in new:
            b = oracle.bucket_hash(c[0], c[1], c[2], buckets)
            if b in seen:
                return True
            seen[b] = c
        prev = cur
    return False


def make_case(name, seed, nframes, W, H, voxel, trunc, buckets, blocks):
    import torch

    import oracle
    import ref
    import synth

    for s in range(seed, seed + 50):
        frames, K = synth.tabletop_stream(s, nframes, W, H)
        if not bucket_collision(oracle, frames, K, voxel, trunc, buckets):
            break
    else:
        raise RuntimeError(f"{name}: no race-free seed found")
    out = {"seed": s, "W": W, "H": H, "voxel": voxel, "trunc": trunc, "buckets": buckets, "blocks": blocks,
           "fx": K.fx, "fy": K.fy, "cx": K.cx, "cy": K.cy, "min_depth": 0.2, "max_depth": 3.0}
    for i, f in enumerate(frames):
        out[f"pointmap_{i}"] = f.pointmap
        out[f"rgb_{i}"] = f.rgb
        out[f"pose_{i}"] = f.pose
    for nofma, tag in ((True, "ref"), (False, "reffma")):
        rs = ref.RefScene(buckets, blocks, voxel, trunc, nofma=nofma)
        for i, f in enumerate(frames):
            pm = torch.from_numpy(f.pointmap).cuda()
            rgb = torch.from_numpy(f.rgb).cuda()
            nm = torch.from_numpy(f.normals).cuda()
            rs.integrate(pm.data_ptr(), rgb.data_ptr(), nm.data_ptr(), W, H, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
            r = rs.render(W, H, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
            for k in ("depth", "position", "color"):
                out[f"{tag}_{k}_{i}"] = r[k]
        coords, vox = rs.export()
        out[f"{tag}_coords"] = coords
        out[f"{tag}_voxels"] = vox
        rs.close()
    out["frames"] = nframes
    return out


def volume_digest(coords: np.ndarray, vox_bytes: np.ndarray) -> str:
    """SHA-256 of the allocated block set and its voxels, blocks sorted by
    (x, y, z), voxels as 8-byte records (float sdf, r, g, b, weight)."""
    import hashlib

    h = hashlib.sha256()
    h.update(np.ascontiguousarray(coords, dtype="<i4").tobytes())
    h.update(np.ascontiguousarray(vox_bytes, dtype=np.uint8).tobytes())
    return h.hexdigest()


def render_digest(depth, position, color) -> str:
    import hashlib

    h = hashlib.sha256()
    for a in (depth, position, color):
        h.update(np.ascontiguousarray(a, dtype="<f4").tobytes())
    return h.hexdigest()


def compact(data: dict) -> dict:
    """Small fixture: inputs, digests of the reference outputs, depth maps
    and the block count (the full volumes are megabytes)."""
    out = {k: v for k, v in data.items() if not k.startswith(("ref", "reffma"))}
    n = int(data["frames"])
    for tag in ("ref", "reffma"):
        out[f"{tag}_volume_sha256"] = volume_digest(data[f"{tag}_coords"], data[f"{tag}_voxels"])
        out[f"{tag}_blocks"] = int(data[f"{tag}_coords"].shape[0])
        for i in range(n):
            out[f"{tag}_render_sha256_{i}"] = render_digest(data[f"{tag}_depth_{i}"], data[f"{tag}_position_{i}"],
                                                            data[f"{tag}_color_{i}"])
    for i in range(n):
        out[f"ref_depth_{i}"] = data[f"ref_depth_{i}"]
    return out


def main(out_dir: str):
    os.makedirs(out_dir, exist_ok=True)
    for case in CASES:
        data = compact(make_case(*case))
        path = os.path.join(out_dir, case[0] + ".npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in data.items()})
        print(path, "seed", data["seed"], "blocks", data["ref_blocks"], os.path.getsize(path))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden.py OUT_DIR")
    main(sys.argv[1])
