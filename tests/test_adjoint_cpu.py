"""The adjoint's algorithm on the CPU (no GPU): the float64 reverse mode of
adjoint_fd.Evaluator.analytic_grad -- the steps the GPU kernel
k_render_backward takes -- against float64 central differences of the same
fixed-decision depth, on an oracle-built volume.  Also pins the
finite-difference methodology the GPU test relies on: the difference error
falls as h^2 (truncation-dominated), so h = 1e-6 resolves the gradient to
far below the 1e-4 bar."""
import numpy as np

from adjoint_fd import Evaluator, Volume


def test_reverse_mode_matches_central_differences(oracle_mod, synth_mod):
    fr, K = synth_mod.tabletop_stream(3, 3, 128, 96)
    o = oracle_mod.OracleScene(0.004)
    for f in fr:
        o.integrate(f.pointmap, f.rgb, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
    T = np.array(fr[-1].pose, np.float64)
    T[:3, 3] += (0.006, -0.004, 0.003)
    T = T.astype(np.float32)
    depth = o.render(K.width, K.height, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)["depth"]
    br_all = o.brackets(K.width, K.height, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    rng = np.random.default_rng(4)
    hit = np.argwhere(depth < 1e9)
    pix = hit[rng.choice(len(hit), 900, replace=False)][:, ::-1].copy()
    coords, vox = o.export()
    vol = Volume(coords, vox["raw"])
    T64 = T.astype(np.float64)
    ev = Evaluator(vol, 0.004, K, pix, br_all[pix[:, 1], pix[:, 0]])
    # the float32 retrace reproduces the oracle's (and the GPU's) depth bit for bit
    d32 = ev.freeze_fp32(T)
    assert np.array_equal(d32.view(np.uint32), depth[pix[:, 1], pix[:, 0]].view(np.uint32))
    keep = ev.weight_sums(T64) >= 0.05
    pix = pix[keep][:400]
    ev = Evaluator(vol, 0.004, K, pix, br_all[pix[:, 1], pix[:, 0]])
    ev.freeze_fp32(T)
    base = ev.depth(T64)
    assert np.abs(base - depth[pix[:, 1], pix[:, 0]]).max() < 1e-4
    g = rng.normal(size=len(pix))
    gpos = rng.normal(size=(len(pix), 3))

    def loss(Tm):
        d, _, alpha, wd, org = ev.depth(Tm, want_normal=True)
        return float((g * d).sum() + (gpos * (org + alpha[:, None] * wd)).sum())

    an = ev.analytic_grad(T64, g, gpos)
    rel = {}
    for h in (1e-5, 1e-6):
        fd = np.zeros((3, 4))
        for r in range(3):
            for c in range(4):
                Tp, Tm = T64.copy(), T64.copy()
                Tp[r, c] += h
                Tm[r, c] -= h
                fd[r, c] = (loss(Tp) - loss(Tm)) / (2 * h)
        rel[h] = np.linalg.norm(an - fd) / np.linalg.norm(fd)
    assert rel[1e-6] <= 1e-4, rel
    assert 30 < rel[1e-5] / rel[1e-6] < 300, rel  # truncation error ~ h^2
