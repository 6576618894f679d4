"""Float64 restatement of a hit pixel's ray-cast depth as a function of the
camera pose and the voxel SDF values, with the march's discrete decisions
held fixed -- test infrastructure for the adjoint (vsg_render_backward).

Per pixel: ray direction wd = normalize(R cd) from the pixel's normalised
camera direction cd, origin o = translation (RayCastRender.cu:447-470); the
zero-crossing bracket [a, b] (march parameters, pose-independent) comes from
the oracle's FP32 march; f(t) is the trilinear SDF at o + t wd
(RayCastRender.cu:127-215) with each sample's 8 tap voxels, their weights'
integer bases and validity frozen at the base pose; three regula-falsi steps
RF(a, fa, b, fb) = a + fa / (fa - fb) (b - a) (:229-271), the side each step
keeps frozen at the base pose; depth = alpha * cd_z.  Central differences of
this function in float64 are what the GPU gradient is checked against.
"""
import numpy as np


class Volume:
    """Exported blocks: sdf (n,512) float64, weight (n,512), coord -> row."""

    def __init__(self, coords, vox_bytes):
        v = np.ascontiguousarray(vox_bytes).reshape(-1, 512, 8)
        self.sdf = np.ascontiguousarray(v[:, :, :4]).view(np.float32).reshape(-1, 512).astype(np.float64)
        self.w = v[:, :, 7].astype(np.int64)
        self.coords = np.asarray(coords)
        self.row = {tuple(c): i for i, c in enumerate(self.coords.tolist())}


def _tap(q):
    return np.floor(q + 0.5 * np.sign(q)).astype(np.int64)


class Evaluator:
    def __init__(self, vol: Volume, voxel: float, K, pix, brackets):
        self.vol = vol
        self.v = float(np.float32(voxel))
        self.K = K
        self.pix = np.asarray(pix, np.float64)
        self.br = np.asarray(brackets, np.float64)
        self.frozen = None

    def freeze_fp32(self, T):
        """Fix the discrete decisions by retracing the crossing in float32
        with the GPU kernel's operation order (k_render_backward's recompute:
        ray setup, tap rounding, trilinear sums, regula-falsi steps and their
        sign tests), so finite differences follow exactly the branch the GPU
        differentiated.  Returns the float32 depths."""
        f32 = np.float32
        K = self.K
        T = np.asarray(T, np.float32)
        x = self.pix[:, 0].astype(f32)
        y = self.pix[:, 1].astype(f32)
        cdx = (x - f32(K.cx)) / f32(K.fx)
        cdy = (y - f32(K.cy)) / f32(K.fy)
        cdz = np.ones_like(cdx)
        cl = np.sqrt((cdx * cdx + cdy * cdy) + cdz * cdz)
        m = cl > f32(1e-6)
        cdx, cdy, cdz = np.where(m, cdx / cl, cdx), np.where(m, cdy / cl, cdy), np.where(m, cdz / cl, cdz)
        wd = [(T[i, 0] * cdx + T[i, 1] * cdy) + T[i, 2] * cdz for i in range(3)]
        wl = np.sqrt((wd[0] * wd[0] + wd[1] * wd[1]) + wd[2] * wd[2])
        m = wl > f32(1e-6)
        wd = [np.where(m, w / wl, w) for w in wd]
        o = [T[0, 3], T[1, 3], T[2, 3]]
        v = f32(self.v)
        N = len(self.pix)
        rows = np.arange(N)
        P = np.zeros((N, 4), f32)
        F = np.zeros((N, 4), f32)
        P[:, 0], P[:, 1] = self.br[:, 0].astype(f32), self.br[:, 1].astype(f32)
        taps, sides = [], []

        def tapv(q):
            sg = np.where(q > 0, f32(1), np.where(q < 0, f32(-1), f32(0)))
            return np.floor(q + f32(0.5) * sg).astype(np.int64)

        def sample(t):
            p = [o[i] + t * wd[i] for i in range(3)]
            dq = [p[i] - v / f32(2.0) for i in range(3)]
            fq = [dq[i] / v for i in range(3)]
            fl = np.stack([np.floor(q) for q in fq], 1).astype(np.float64)
            t0 = np.stack([tapv(q) for q in fq], 1)
            t1 = np.stack([tapv((dq[i] + v) / v) for i in range(3)], 1)
            w = [q - np.floor(q) for q in fq]
            idx = np.full((N, 8), -1, np.int64)
            valid = np.zeros((N, 8), bool)
            d = np.zeros(N, f32)
            ws = np.zeros(N, f32)
            for i in range(8):
                vx = np.stack([t1[:, 0] if i & 1 else t0[:, 0], t1[:, 1] if i & 2 else t0[:, 1],
                               t1[:, 2] if i & 4 else t0[:, 2]], 1)
                blk, loc = vx >> 3, vx & 7
                s = np.zeros(N, f32)
                for n in range(N):
                    r = self.vol.row.get(tuple(blk[n].tolist()))
                    if r is not None:
                        li = loc[n, 0] + 8 * loc[n, 1] + 64 * loc[n, 2]
                        idx[n, i] = r * 512 + li
                        valid[n, i] = self.vol.w[r, li] > 0
                        s[n] = f32(self.vol.sdf[r, li])
                tw = ((w[0] if i & 1 else f32(1) - w[0]) * (w[1] if i & 2 else f32(1) - w[1])) * \
                     (w[2] if i & 4 else f32(1) - w[2])
                d = np.where(valid[:, i], d + tw * s, d)
                ws = np.where(valid[:, i], ws + tw, ws)
            taps.append({"fl": fl, "idx": idx, "valid": valid})
            return d * (f32(1.0) / ws)

        F[:, 0] = sample(P[:, 0])
        F[:, 1] = sample(P[:, 1])
        ia = np.zeros(N, np.int64)
        ib = np.ones(N, np.int64)
        for k in (2, 3):
            a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
            P[:, k] = a + (fa / (fa - fb)) * (b - a)
            F[:, k] = sample(P[:, k])
            keep = F[rows, ia] * F[:, k] > f32(0)
            sides.append(keep)
            ia = np.where(keep, k, ia)
            ib = np.where(keep, ib, k)
        a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
        alpha = a + (fa / (fa - fb)) * (b - a)
        d2r = f32(1.0) / cdz
        self.frozen = {"taps": taps, "side": sides}
        hit_p = np.stack([o[i] + alpha * wd[i] for i in range(3)], 1).astype(np.float64)
        self.frozen["hit_taps"] = self._taps(hit_p)
        return alpha / d2r

    def rays(self, T):
        K = self.K
        x, y = self.pix[:, 0], self.pix[:, 1]
        cd = np.stack([(x - K.cx) / K.fx, (y - K.cy) / K.fy, np.ones_like(x)], 1)
        cd /= np.linalg.norm(cd, axis=1, keepdims=True)
        u = cd @ np.asarray(T, np.float64)[:3, :3].T
        wd = u / np.linalg.norm(u, axis=1, keepdims=True)
        o = np.asarray(T, np.float64)[:3, 3]
        return cd, wd, o

    def _taps(self, p):
        v = self.v
        q = (p - v / 2) / v
        fl = np.floor(q)
        t0, t1 = _tap(q), _tap(q + 1.0)
        N = p.shape[0]
        idx = np.full((N, 8), -1, np.int64)
        valid = np.zeros((N, 8), bool)
        for i in range(8):
            vx = np.stack([t1[:, 0] if i & 1 else t0[:, 0], t1[:, 1] if i & 2 else t0[:, 1],
                           t1[:, 2] if i & 4 else t0[:, 2]], 1)
            blk, loc = vx >> 3, vx & 7
            for n in range(N):
                r = self.vol.row.get(tuple(blk[n].tolist()))
                if r is not None:
                    li = loc[n, 0] + 8 * loc[n, 1] + 64 * loc[n, 2]
                    idx[n, i] = r * 512 + li
                    valid[n, i] = self.vol.w[r, li] > 0
        return {"fl": fl, "idx": idx, "valid": valid}

    def _f(self, p, tp, sdf):
        v = self.v
        w = (p - v / 2) / v - tp["fl"]
        tw = np.ones((p.shape[0], 8))
        for i in range(8):
            for a, bit in enumerate((1, 2, 4)):
                tw[:, i] *= w[:, a] if i & bit else (1.0 - w[:, a])
        tw = tw * tp["valid"]
        s = sdf.reshape(-1)[np.maximum(tp["idx"], 0)]
        return (tw * s).sum(1) / tw.sum(1)

    def _f_and_grad(self, p, tp, sdf):
        """f and its analytic position gradient (frozen taps)."""
        v = self.v
        w = (p - v / 2) / v - tp["fl"]
        valid = tp["valid"]
        s = sdf.reshape(-1)[np.maximum(tp["idx"], 0)]
        terms = [[w[:, a] if i & bit else 1.0 - w[:, a] for a, bit in enumerate((1, 2, 4))] for i in range(8)]
        tw = np.stack([terms[i][0] * terms[i][1] * terms[i][2] for i in range(8)], 1) * valid
        W = tw.sum(1)
        f = (tw * s).sum(1) / W
        g = np.zeros_like(p)
        for a, bit in enumerate((1, 2, 4)):
            dtw = np.stack([(1.0 if i & bit else -1.0) * np.prod([terms[i][b] for b in range(3) if b != a], 0)
                            for i in range(8)], 1) * valid
            g[:, a] = (dtw * (s - f[:, None])).sum(1) / W / v
        return f, g, tw / W[:, None]

    def analytic_grad(self, T, gd, gpos):
        """Reverse mode through the fixed-decision depth (the GPU kernel's
        algorithm in float64): dL/dT (3,4) for L = sum gd*depth + gpos.pos."""
        cd, wd, o = self.rays(T)
        T = np.asarray(T, np.float64)
        N = len(self.pix)
        rows = np.arange(N)
        P = np.zeros((N, 4))
        F = np.zeros((N, 4))
        G = np.zeros((N, 4, 3))
        P[:, 0], P[:, 1] = self.br[:, 0], self.br[:, 1]
        ia = np.zeros(N, np.int64)
        ib = np.ones(N, np.int64)
        steps = []
        for k in range(4):
            if k >= 2:
                steps.append((ia.copy(), ib.copy()))
                a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
                P[:, k] = a + fa / (fa - fb) * (b - a)
            F[:, k], G[:, k], _ = self._f_and_grad(o + P[:, k:k + 1] * wd, self.frozen["taps"][k], self.vol.sdf)
            if k >= 2:
                keep = self.frozen["side"][k - 2]
                ia = np.where(keep, k, ia)
                ib = np.where(keep, ib, k)
        steps.append((ia.copy(), ib.copy()))
        a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
        alpha = a + fa / (fa - fb) * (b - a)
        g_alpha = gd * cd[:, 2] + (gpos * wd).sum(1)
        go = gpos.copy()
        gw = alpha[:, None] * gpos
        gP = np.zeros((N, 4))
        gF = np.zeros((N, 4))

        def rf_back(ia, ib, g):
            a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
            den = fa - fb
            t = fa / den
            np.add.at(gP, (rows, ia), (1 - t) * g)
            np.add.at(gP, (rows, ib), t * g)
            np.add.at(gF, (rows, ia), (b - a) * (-fb / den ** 2) * g)
            np.add.at(gF, (rows, ib), (b - a) * (fa / den ** 2) * g)

        rf_back(*steps[2], g_alpha)
        for k in (3, 2, 1, 0):
            gf = gF[:, k]
            go += gf[:, None] * G[:, k]
            gw += (gf * P[:, k])[:, None] * G[:, k]
            gP[:, k] += gf * (G[:, k] * wd).sum(1)
            if k >= 2:
                rf_back(*steps[k - 2], gP[:, k])
        u = cd @ T[:3, :3].T
        wl = np.linalg.norm(u, axis=1)
        gu = (gw - wd * (gw * wd).sum(1, keepdims=True)) / wl[:, None]
        out = np.zeros((3, 4))
        out[:, :3] = gu.T @ cd
        out[:, 3] = go.sum(0)
        return out

    def weight_sums(self, T):
        """Per pixel, the smallest normalising weight (sum of the valid taps'
        trilinear weights) over the crossing's samples: where it is small the
        depth is a steep function of the pose and finite differences need a
        tiny step."""
        cd, wd, o = self.rays(T)
        N = len(self.pix)
        rows = np.arange(N)
        P = np.zeros((N, 4))
        F = np.zeros((N, 4))
        P[:, 0], P[:, 1] = self.br[:, 0], self.br[:, 1]
        ia = np.zeros(N, np.int64)
        ib = np.ones(N, np.int64)
        wmin = np.full(N, np.inf)
        for k in range(4):
            if k >= 2:
                a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
                P[:, k] = a + fa / (fa - fb) * (b - a)
            p = o + P[:, k:k + 1] * wd
            tp = self.frozen["taps"][k]
            v = self.v
            w = (p - v / 2) / v - tp["fl"]
            tw = np.ones((N, 8))
            for i in range(8):
                for ax, bit in enumerate((1, 2, 4)):
                    tw[:, i] *= w[:, ax] if i & bit else (1.0 - w[:, ax])
            tw = tw * tp["valid"]
            wmin = np.minimum(wmin, tw.sum(1))
            F[:, k] = self._f(p, tp, self.vol.sdf)
            if k >= 2:
                keep = self.frozen["side"][k - 2]
                ia = np.where(keep, k, ia)
                ib = np.where(keep, ib, k)
        return wmin

    def _grad_f(self, p, tp, sdf):
        eps = 1e-7
        g = np.zeros_like(p)
        for a in range(3):
            d = np.zeros(3)
            d[a] = eps
            g[:, a] = (self._f(p + d, tp, sdf) - self._f(p - d, tp, sdf)) / (2 * eps)
        return g

    def depth(self, T, sdf=None, want_normal=False):
        """Depth of every pixel; the first call fixes the decisions."""
        sdf = self.vol.sdf if sdf is None else sdf
        cd, wd, o = self.rays(T)
        N = len(self.pix)
        first = self.frozen is None
        if first:
            self.frozen = {"taps": [], "side": []}
        P = np.zeros((N, 4))
        F = np.zeros((N, 4))
        P[:, 0], P[:, 1] = self.br[:, 0], self.br[:, 1]
        ia = np.zeros(N, np.int64)
        ib = np.ones(N, np.int64)
        rows = np.arange(N)

        def sample(k):
            p = o + P[:, k:k + 1] * wd
            if first:
                self.frozen["taps"].append(self._taps(p))
            F[:, k] = self._f(p, self.frozen["taps"][k], sdf)

        sample(0)
        sample(1)
        for k in (2, 3):
            a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
            P[:, k] = a + fa / (fa - fb) * (b - a)
            sample(k)
            if first:
                self.frozen["side"].append(F[rows, ia] * F[:, k] > 0)
            keep = self.frozen["side"][k - 2]
            ia = np.where(keep, k, ia)
            ib = np.where(keep, ib, k)
        a, fa, b, fb = P[rows, ia], F[rows, ia], P[rows, ib], F[rows, ib]
        alpha = a + fa / (fa - fb) * (b - a)
        out = alpha * cd[:, 2]
        if want_normal:
            p = o + alpha[:, None] * wd
            if "hit_taps" not in self.frozen:
                self.frozen["hit_taps"] = self._taps(p)
            g = self._grad_f(p, self.frozen["hit_taps"], sdf)
            return out, g / np.linalg.norm(g, axis=1, keepdims=True), alpha, wd, o
        return out
