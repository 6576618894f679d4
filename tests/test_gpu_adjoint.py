"""Adjoint of the ray cast (vsg_render_backward, vsg_render_normals) against
float64 central finite differences of the same depth function with the
march's discrete decisions held fixed (adjoint_fd.Evaluator): gradients with
respect to the 3x4 camera pose and to individual voxel SDF values, through
depth and position outputs; normals against the float64 SDF gradient; and a
pose-refinement run through the torch autograd wrapper (needs a GPU)."""
import numpy as np
import pytest

from adjoint_fd import Evaluator, Volume

pytestmark = pytest.mark.gpu

VOXEL, TRUNC, MIN_D, MAX_D = 0.004, 0.02, 0.2, 3.0
POSE_TOL = 1e-4  # relative error of the pose gradient against FP64 central differences
SDF_TOL = 1e-3   # relative error per voxel SDF gradient
# Central-difference steps.  The fixed-decision depth has large third
# derivatives (three regula-falsi divisions, trilinear weights renormalised
# over the valid taps), so the truncation error of a central difference is
# about 1e-2 relative at h = 1e-4 and falls as h^2: 1e-4 at 1e-5, 1e-6 at
# 1e-6 (measured on this scene); float64 round-off stays below 1e-9 there.
H_POSE, H_SDF = 1e-6, 1e-7
# Pixels whose samples renormalise over valid taps with total weight below
# this are left out: there the depth is so steep that no step resolves it.
MIN_WEIGHT_SUM = 0.05


def _setup(cuda, synth_mod, oracle_mod, frames=4, W=160, H=120):
    import vsg

    fr, K = synth_mod.tabletop_stream(3, frames, W, H)
    sc = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=20011, num_sdf_blocks=60000)
    for f in fr:
        pm, rgb, nm = (cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals))
        sc.integrate(pm, rgb, nm, W, H, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
    rr = vsg.Renderer(W, H)
    rr.record(True)
    coords, vox = sc.export()
    o = oracle_mod.OracleScene(VOXEL)
    o.load(coords, vox)
    return vsg, fr, K, sc, rr, o, Volume(coords, vox)


def _pose(fr, i=-1, rot_deg=2.0, shift=(0.01, -0.005, 0.004)):
    """A pose near frame i's (a view the volume was not built from)."""
    T = np.array(fr[i].pose, np.float64)
    a = np.deg2rad(rot_deg)
    Rz = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    T[:3, :3] = T[:3, :3] @ Rz
    T[:3, 3] += np.array(shift)
    return T.astype(np.float32)


def _subset(depth, n, rng):
    hit = np.argwhere(depth < 1e9)
    sel = hit[rng.choice(len(hit), size=min(n, len(hit)), replace=False)]
    return sel[:, ::-1].copy()  # (x, y)


def _well_conditioned(vol, K, depth, T, o, n, rng):
    """n hit pixels whose crossing samples all have weight sum >= MIN_WEIGHT_SUM,
    with their brackets and a base-pose evaluator."""
    pix = _subset(depth, 3 * n, rng)
    br = o.brackets(K.width, K.height, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)[pix[:, 1], pix[:, 0]]
    ev = Evaluator(vol, VOXEL, K, pix, br)
    d32 = ev.freeze_fp32(T)  # the GPU's decisions, retraced in float32
    assert np.array_equal(d32.view(np.uint32), depth[pix[:, 1], pix[:, 0]].view(np.uint32))
    keep = np.nonzero(ev.weight_sums(T.astype(np.float64)) >= MIN_WEIGHT_SUM)[0][:n]
    pix, br = pix[keep], br[keep]
    ev = Evaluator(vol, VOXEL, K, pix, br)
    ev.freeze_fp32(T)
    return pix, ev


def test_pose_and_sdf_gradients_match_fp64_central_differences(cuda, synth_mod, oracle_mod):
    vsg, fr, K, sc, rr, o, vol = _setup(cuda, synth_mod, oracle_mod)
    T = _pose(fr)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
    out = rr.download()
    depth = out["depth"]
    rng = np.random.default_rng(0)
    pix, ev = _well_conditioned(vol, K, depth, T, o, 600, rng)
    assert len(pix) >= 500
    g = rng.normal(size=len(pix)).astype(np.float32).astype(np.float64)
    gpos = (rng.normal(size=(len(pix), 3)) * 0.5).astype(np.float32).astype(np.float64)
    gd = np.zeros_like(depth)
    gd[pix[:, 1], pix[:, 0]] = g
    gp = np.zeros((K.height, K.width, 4), np.float32)
    gp[pix[:, 1], pix[:, 0], :3] = gpos
    n_vox = sc.params.num_sdf_blocks * 512
    gsdf = cuda.zeros(n_vox, dtype=cuda.float32, device="cuda")
    gT, skipped = rr.backward(sc, T, K.fx, K.fy, K.cx, K.cy, grad_depth=cuda.from_numpy(gd).cuda(),
                              grad_position=cuda.from_numpy(gp).cuda(), grad_sdf=gsdf)
    assert skipped == 0

    T64 = T.astype(np.float64)

    def loss(Tm, sdf=None):
        d, _, alpha, wd, org = ev.depth(Tm, sdf, want_normal=True)
        pos = org + alpha[:, None] * wd
        return float((g * d).sum() + (gpos * pos).sum())

    base_depth = ev.depth(T64)
    assert np.abs(base_depth - depth[pix[:, 1], pix[:, 0]]).max() < 1e-4  # FP64 restatement agrees
    h = H_POSE
    fd = np.zeros((3, 4))
    for r in range(3):
        for c in range(4):
            Tp, Tm = T64.copy(), T64.copy()
            Tp[r, c] += h
            Tm[r, c] -= h
            fd[r, c] = (loss(Tp) - loss(Tm)) / (2 * h)
    rel = np.linalg.norm(gT - fd) / np.linalg.norm(fd)
    assert rel <= POSE_TOL, (rel, gT, fd)

    # voxel SDF gradients: the GPU buffer is indexed by pool block
    ptrs = sc.lookup_blocks(vol.coords)
    assert np.all(ptrs >= 0)
    G = gsdf.view(-1, 512).cpu().numpy()[ptrs]
    top = np.argsort(-np.abs(G).ravel())[:20]
    hs = H_SDF
    for flat in top:
        sp, sm = vol.sdf.copy(), vol.sdf.copy()
        sp.ravel()[flat] += hs
        sm.ravel()[flat] -= hs
        fdv = (loss(T64, sp) - loss(T64, sm)) / (2 * hs)
        assert abs(G.ravel()[flat] - fdv) <= SDF_TOL * abs(fdv) + 1e-6, (flat, G.ravel()[flat], fdv)


def test_normals_match_fp64_sdf_gradient(cuda, synth_mod, oracle_mod):
    vsg, fr, K, sc, rr, o, vol = _setup(cuda, synth_mod, oracle_mod)
    T = _pose(fr, rot_deg=-1.0)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
    depth = rr.download()["depth"]
    nrm, skipped = rr.normals(sc, T, K.fx, K.fy, K.cx, K.cy)
    assert skipped == 0
    nrm = nrm.cpu().numpy()
    miss = depth >= 1e9
    assert np.all(nrm[miss] == 1e10)
    rng = np.random.default_rng(1)
    pix, ev = _well_conditioned(vol, K, depth, T, o, 400, rng)
    _, n64, _, _, _ = ev.depth(T.astype(np.float64), want_normal=True)
    ok = np.all(np.isfinite(n64), 1)
    assert ok.mean() > 0.95
    got = nrm[pix[:, 1], pix[:, 0], :3].astype(np.float64)
    assert np.abs(got[ok] - n64[ok]).max() < 1e-4
    assert np.all(nrm[pix[:, 1], pix[:, 0], 3] == 0.0)


def test_pose_refinement_with_autograd(cuda, synth_mod, oracle_mod):
    """20 Adam steps on a robust (Huber) depth loss bring a pose perturbed by
    about 1 cm and 1 degree back towards the one that rendered the target."""
    import torch

    vsg, fr, K, sc, rr, o, vol = _setup(cuda, synth_mod, oracle_mod, frames=6)
    T_true = torch.tensor(np.array(fr[-1].pose, np.float32), dtype=torch.float64)
    target = vsg.render_depth(sc, rr, T_true.float(), K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D).detach()

    def hat(w):
        z = torch.zeros((), dtype=w.dtype)
        return torch.stack([torch.stack([z, -w[2], w[1]]), torch.stack([w[2], z, -w[0]]),
                            torch.stack([-w[1], w[0], z])])

    def exp_se3(xi):
        w, t = xi[:3], xi[3:]
        th = torch.sqrt((w * w).sum() + 1e-18)
        W = hat(w)
        R = torch.eye(3, dtype=xi.dtype) + torch.sin(th) / th * W + (1 - torch.cos(th)) / th ** 2 * (W @ W)
        T = torch.eye(4, dtype=xi.dtype)
        T = torch.cat([torch.cat([R, t[:, None]], 1), T[3:]], 0)
        return T

    rng = np.random.default_rng(2)
    d0 = np.concatenate([rng.normal(size=3) / np.sqrt(3) * np.deg2rad(1.0), rng.normal(size=3) / np.sqrt(3) * 0.01])
    xi = torch.tensor(d0, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([xi], lr=2e-3)
    err0 = None
    for _ in range(20):
        opt.zero_grad()
        T = T_true @ exp_se3(xi)
        d = vsg.render_depth(sc, rr, T.float(), K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
        m = (d < 1e9) & (target < 1e9)
        loss = torch.nn.functional.huber_loss(d[m], target[m], delta=0.01)
        loss.backward()
        if err0 is None:
            err0 = float(xi.detach().norm())
        opt.step()
    assert float(xi.detach().norm()) < 0.5 * err0


def test_pose_normal_equations_match_fp64_central_differences(cuda, synth_mod, oracle_mod):
    """vsg_render_pose_normal_equations: H = sum w J J^T and b = sum w J r,
    J = d depth / d xi for T exp(xi), against per-pixel float64 central
    differences of the frozen-decision depth along the six twist axes."""
    import torch

    vsg, fr, K, sc, rr, o, vol = _setup(cuda, synth_mod, oracle_mod)
    T = _pose(fr)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
    depth = rr.download()["depth"]
    rng = np.random.default_rng(4)
    pix, ev = _well_conditioned(vol, K, depth, T, o, 600, rng)
    assert len(pix) >= 500
    r = (rng.normal(size=len(pix)) * 0.01).astype(np.float32)
    w = rng.uniform(0.2, 1.0, size=len(pix)).astype(np.float32)
    R = np.zeros_like(depth)
    Wt = np.zeros_like(depth)
    R[pix[:, 1], pix[:, 0]] = r
    Wt[pix[:, 1], pix[:, 0]] = w
    Hm, b, skipped = rr.pose_normal_equations(sc, T, K.fx, K.fy, K.cx, K.cy, torch.from_numpy(R).cuda(),
                                              torch.from_numpy(Wt).cuda(), MIN_WEIGHT_SUM)
    assert skipped == 0
    T64 = T.astype(np.float64)
    J = np.zeros((len(pix), 6))
    for k in range(6):
        e = np.zeros(6)
        e[k] = H_POSE
        J[:, k] = (ev.depth(T64 @ vsg.se3_exp(e)) - ev.depth(T64 @ vsg.se3_exp(-e))) / (2 * H_POSE)
    w64, r64 = w.astype(np.float64), r.astype(np.float64)
    H_fd = (J * w64[:, None]).T @ J
    b_fd = J.T @ (w64 * r64)
    assert np.linalg.norm(Hm - H_fd) <= POSE_TOL * np.linalg.norm(H_fd), (Hm, H_fd)
    assert np.linalg.norm(b - b_fd) <= POSE_TOL * np.linalg.norm(b_fd), (b, b_fd)
    # pixels with zero weight and misses contribute nothing
    Hz, bz, _ = rr.pose_normal_equations(sc, T, K.fx, K.fy, K.cx, K.cy, torch.from_numpy(R).cuda(),
                                         torch.zeros_like(torch.from_numpy(Wt)).cuda(), MIN_WEIGHT_SUM)
    assert not Hz.any() and not bz.any()


def test_gauss_newton_pose_refinement(cuda, synth_mod, oracle_mod):
    """vsg.refine_pose: 8 Gauss-Newton steps (Huber-weighted depth residuals
    against the render at the true pose) bring poses perturbed by about 1 cm
    and 1 degree to within a small fraction of their initial error."""
    vsg, fr, K, sc, rr, o, vol = _setup(cuda, synth_mod, oracle_mod, frames=6)
    rng = np.random.default_rng(5)
    ratios = []
    for i in (-1, -3):
        T_true = np.array(fr[i].pose, np.float32).astype(np.float64)
        rr.render(sc, T_true.astype(np.float32), K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
        target = rr.depth_tensor().clone()
        d0 = np.concatenate([rng.normal(size=3) / np.sqrt(3) * np.deg2rad(1.0),
                             rng.normal(size=3) / np.sqrt(3) * 0.01])
        T0 = T_true @ vsg.se3_exp(d0)
        T, rms = vsg.refine_pose(sc, rr, target, T0, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D, steps=8)
        D = np.linalg.inv(T_true) @ T
        ang = np.arccos(np.clip((np.trace(D[:3, :3]) - 1) / 2, -1, 1))
        err = np.hypot(ang, np.linalg.norm(D[:3, 3]))
        ratios.append(err / np.hypot(np.linalg.norm(d0[:3]), np.linalg.norm(d0[3:])))
        assert rms[-1] < rms[0]
    assert max(ratios) < 0.1, ratios
