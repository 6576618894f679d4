"""Comparison helpers between the CUDA path and the CPU oracle."""
from __future__ import annotations

import numpy as np

MINF = 1e10


def split(vox_bytes: np.ndarray) -> dict:
    v = np.ascontiguousarray(vox_bytes).reshape(-1, 512, 8)
    sdf = np.ascontiguousarray(v[:, :, :4]).view(np.float32).reshape(-1, 512)
    return {"sdf": sdf, "rgb": v[:, :, 4:7], "weight": v[:, :, 7]}


def compare_volumes(gc, gv, oc, ov) -> dict:
    """Block sets must be equal; voxel fields compared per block."""
    res = {"gpu_blocks": int(gc.shape[0]), "oracle_blocks": int(oc.shape[0])}
    res["same_blocks"] = bool(gc.shape == oc.shape and np.array_equal(gc, oc))
    if not res["same_blocks"]:
        gs = {tuple(r) for r in gc.tolist()}
        os_ = {tuple(r) for r in oc.tolist()}
        res["only_gpu"] = len(gs - os_)
        res["only_oracle"] = len(os_ - gs)
        return res
    g, o = split(gv), split(ov)
    res["weight_mismatch"] = int((g["weight"] != o["weight"]).sum())
    res["rgb_mismatch"] = int((g["rgb"] != o["rgb"]).any(-1).sum())
    m = o["weight"] > 0
    d = np.abs(g["sdf"].astype(np.float64) - o["sdf"].astype(np.float64))[m]
    res["sdf_max_err"] = float(d.max()) if d.size else 0.0
    res["sdf_rms_err"] = float(np.sqrt((d ** 2).mean())) if d.size else 0.0
    res["bit_exact"] = bool(np.array_equal(np.ascontiguousarray(gv), np.ascontiguousarray(ov)))
    res["updated_voxels"] = int(m.sum())
    return res


def compare_renders(g: dict, o: dict, tol: float = 1e-4) -> dict:
    gd, od = g["depth"], o["depth"]
    gh, oh = gd < MINF * 0.5, od < MINF * 0.5
    both = gh & oh
    err = np.abs(gd.astype(np.float64) - od.astype(np.float64))
    ok = (gh == oh) & np.where(both, err <= tol, True)
    e = err[both]
    return {
        "pixels": int(gd.size),
        "hits_gpu": int(gh.sum()),
        "hits_oracle": int(oh.sum()),
        "hit_mask_mismatch": int((gh != oh).sum()),
        "frac_within_tol": float(ok.mean()),
        "depth_max_err": float(e.max()) if e.size else 0.0,
        "depth_rms_err": float(np.sqrt((e ** 2).mean())) if e.size else 0.0,
        "bit_exact_depth": bool(np.array_equal(gd.view(np.uint32), od.view(np.uint32))),
        "bit_exact_all": bool(all(np.array_equal(g[k].view(np.uint32), o[k].view(np.uint32))
                                  for k in ("depth", "position", "color", "normal"))),
    }
