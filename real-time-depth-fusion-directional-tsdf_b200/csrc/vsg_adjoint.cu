// vsg_adjoint.cu -- gradients of the ray cast with respect to the camera pose
// and the voxel SDF values (no counterpart in the reference), and ray-cast
// normals.
//
// A hit pixel's depth is a smooth function of the pose and of the SDF values
// of the voxels its samples interpolate, once the march's discrete decisions
// are fixed: the bracket [a, b] of the zero crossing (march parameters that
// do not depend on the pose: the ray parameter chain starts at minDepth /
// camDir.z and steps by 0.5 voxel), each sample's 8 tap voxels, which taps
// carry weight, and the side each regula-falsi step keeps.  With those fixed:
//   o = T[:3,3], wd = normalize(R cd)       (RayCastRender.cu:447-470)
//   f(t) = trilinear SDF at o + t wd        (:127-215)
//   c1 = RF(a, f(a), b, f(b)), c2 = RF(bracket, ...), alpha = c3
//   RF(a, fa, b, fb) = a + fa / (fa - fb) * (b - a)   (:229-271)
//   depth = alpha * camDir.z, position = o + alpha wd
// The forward pass records [a, b] per pixel (vsg_renderer_record); the
// backward kernel recomputes the samples with the forward's exact FP32
// operations (and checks that it lands on the recorded depth bit for bit),
// then runs reverse mode through the three regula-falsi steps and the
// trilinear interpolations: d(trilinear)/d(position) is the weight
// derivative, d/d(voxel sdf) is the tap's normalised weight.
//
// The recomputation is FP32: it retraces the forward's decisions (tap voxels,
// weight bases, regula-falsi sides) and checks the depth.  The smooth
// function those decisions define is then evaluated again in double --
// ray, sample points, trilinear values, regula-falsi steps -- and
// differentiated there: near the root a sample's FP32 value carries a large
// relative rounding error that would otherwise enter the regula-falsi
// derivatives.
//
// Work layout: one thread per pixel on the forward's 8x4 warp tiles; pose
// gradients reduced per warp by shuffles, per CTA in shared memory, then
// across CTAs in a fixed order (deterministic), all in double; voxel SDF
// gradients accumulated with float atomics into the caller's buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"
#include "vsg_raycast_core.cuh"

namespace vsg {
namespace {

struct BackArgs {
    SceneDev s;
    int W, H;
    Pose pose;
    float fx, fy, cx, cy;
    const float* depth;
    const float2* rec;
    const float* g_depth;   // may be null
    const float4* g_pos;    // may be null
    float* g_sdf;           // may be null
    const float* resid;     // normal equations: per-pixel residual
    const float* wts;       // normal equations: per-pixel weight (null = 1)
    float4* normals;        // vsg_render_normals output (null in backward)
    double* partials;       // per CTA 12 doubles
    float min_w;            // leave out pixels whose samples renormalise over less weight
    unsigned int* skipped;
};

// One trilinear sample with the forward's exact arithmetic (trilinear,
// vsg_raycast_core.cuh) plus its gradient with respect to the sample
// position and, on request, the scatter of g_f into the taps' SDF gradients.
struct Sample {
    float f;
    double gx, gy, gz;  // d f / d position
    bool ok;
};

// The frozen decisions of one sample: tap voxel coordinates and the integer
// base of its trilinear weights.
struct NodeTaps {
    int t0[3], t1[3];
    float fl[3];
};

__device__ Sample sample_grad(const SceneDev& s, float px, float py, float pz, float* g_sdf, float g_f,
                              NodeTaps* nt = nullptr) {
    Sample out{0.0f, 0.0, 0.0, 0.0, false};
    const float off = s.voxel;
    const float v = s.voxel;
    const float dx = px - off / 2.0f, dy = py - off / 2.0f, dz = pz - off / 2.0f;
    const bool fast = s.div_fast;
    const float y = s.inv_voxel;
    const float fx = div_v(dx, v, y, fast), fy = div_v(dy, v, y, fast), fz = div_v(dz, v, y, fast);
    const float wx = frac01(fx), wy = frac01(fy), wz = frac01(fz);
    const int ax0 = tap_voxel(fx), ay0 = tap_voxel(fy), az0 = tap_voxel(fz);
    const int ax1 = tap_voxel(div_v(dx + off, v, y, fast)), ay1 = tap_voxel(div_v(dy + off, v, y, fast)),
              az1 = tap_voxel(div_v(dz + off, v, y, fast));
    if (nt) {
        nt->t0[0] = ax0;
        nt->t0[1] = ay0;
        nt->t0[2] = az0;
        nt->t1[0] = ax1;
        nt->t1[1] = ay1;
        nt->t1[2] = az1;
        nt->fl[0] = floorf(fx);
        nt->fl[1] = floorf(fy);
        nt->fl[2] = floorf(fz);
    }
    float d = 0.0f, vws = 0.0f;
    float sdfv[8];
    size_t idx[8];
    bool valid[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int vx = (i & 1) ? ax1 : ax0, vy = (i & 2) ? ay1 : ay0, vz = (i & 4) ? az1 : az0;
        const int p = block_ptr(s, vox_to_block(vx), vox_to_block(vy), vox_to_block(vz));
        valid[i] = false;
        sdfv[i] = 0.0f;
        idx[i] = 0;
        if (p >= 0) {
            idx[i] = (size_t)p * kVoxPerBlock + vox_local(vx) + vox_local(vy) * kBlock + vox_local(vz) * kBlock * kBlock;
            const uint2 raw = __ldg(reinterpret_cast<const uint2*>(s.voxels + idx[i]));
            if ((raw.y >> 24) != 0u) {
                valid[i] = true;
                sdfv[i] = __uint_as_float(raw.x);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        const float w = ((i & 1) ? wx : (1.0f - wx)) * ((i & 2) ? wy : (1.0f - wy)) * ((i & 4) ? wz : (1.0f - wz));
        d += w * sdfv[i];
        vws += w;
    }
    if (vws <= 1e-6f) return out;
    const float inv = 1.0f / vws;
    out.f = d * inv;
    out.ok = true;
    // derivatives in double at the FP32 point
    double W = 0.0, D = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        const double tw = ((i & 1) ? (double)wx : 1.0 - wx) * ((i & 2) ? (double)wy : 1.0 - wy) *
                          ((i & 4) ? (double)wz : 1.0 - wz);
        W += tw;
        D += tw * sdfv[i];
    }
    const double f = D / W;
    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        const double tx = (i & 1) ? (double)wx : 1.0 - wx, ty = (i & 2) ? (double)wy : 1.0 - wy,
                     tz = (i & 4) ? (double)wz : 1.0 - wz;
        const double r = ((double)sdfv[i] - f) / W;
        gx += ((i & 1) ? 1.0 : -1.0) * ty * tz * r;
        gy += ((i & 2) ? 1.0 : -1.0) * tx * tz * r;
        gz += ((i & 4) ? 1.0 : -1.0) * tx * ty * r;
        if (g_sdf && g_f != 0.0f) atomicAdd(g_sdf + idx[i], (float)((double)g_f * (tx * ty * tz) / W));
    }
    const double iv = 1.0 / (double)v;  // d(frac(p / v - 1/2)) / dp
    out.gx = gx * iv;
    out.gy = gy * iv;
    out.gz = gz * iv;
    return out;
}

// The same trilinear sample in double at a double position, with the taps and
// weight bases frozen: value, position gradient, and (on request) the
// scatter of g_f into the taps' SDF gradients.
__device__ bool sample64(const SceneDev& s, const double p[3], const NodeTaps& nt, double& f, double g[3],
                         float* g_sdf, double g_f, double* wsum = nullptr) {
    const double v = s.voxel;
    double w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) w[a] = (p[a] - v / 2.0) / v - (double)nt.fl[a];
    double sdfv[8];
    size_t idx[8];
    bool valid[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int vx = (i & 1) ? nt.t1[0] : nt.t0[0], vy = (i & 2) ? nt.t1[1] : nt.t0[1],
                  vz = (i & 4) ? nt.t1[2] : nt.t0[2];
        const int b = block_ptr(s, vox_to_block(vx), vox_to_block(vy), vox_to_block(vz));
        valid[i] = false;
        sdfv[i] = 0.0;
        idx[i] = 0;
        if (b >= 0) {
            idx[i] = (size_t)b * kVoxPerBlock + vox_local(vx) + vox_local(vy) * kBlock + vox_local(vz) * kBlock * kBlock;
            const uint2 raw = __ldg(reinterpret_cast<const uint2*>(s.voxels + idx[i]));
            if ((raw.y >> 24) != 0u) {
                valid[i] = true;
                sdfv[i] = (double)__uint_as_float(raw.x);
            }
        }
    }
    double W = 0.0, D = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        const double tw = ((i & 1) ? w[0] : 1.0 - w[0]) * ((i & 2) ? w[1] : 1.0 - w[1]) * ((i & 4) ? w[2] : 1.0 - w[2]);
        W += tw;
        D += tw * sdfv[i];
    }
    if (wsum) *wsum = W;
    if (!(W > 0.0)) return false;
    f = D / W;
    g[0] = g[1] = g[2] = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!valid[i]) continue;
        const double tx = (i & 1) ? w[0] : 1.0 - w[0], ty = (i & 2) ? w[1] : 1.0 - w[1],
                     tz = (i & 4) ? w[2] : 1.0 - w[2];
        const double r = (sdfv[i] - f) / W;
        g[0] += ((i & 1) ? 1.0 : -1.0) * ty * tz * r;
        g[1] += ((i & 2) ? 1.0 : -1.0) * tx * tz * r;
        g[2] += ((i & 4) ? 1.0 : -1.0) * tx * ty * r;
        if (g_sdf && g_f != 0.0) atomicAdd(g_sdf + idx[i], (float)(g_f * (tx * ty * tz) / W));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) g[a] /= v;
    return true;
}

// Regula falsi step, RayCastRender.cu:238-240, and its partial derivatives.
__device__ __forceinline__ float rf(float a, float fa, float b, float fb) { return a + (fa / (fa - fb)) * (b - a); }
__device__ __forceinline__ double rf64(double a, double fa, double b, double fb) { return a + (fa / (fa - fb)) * (b - a); }

__device__ __forceinline__ void rf_back(double a, double fa, double b, double fb, double g, double& ga, double& gfa,
                                        double& gb, double& gfb) {
    const double den = fa - fb;
    const double t = fa / den;
    const double ba = b - a;
    ga += (1.0 - t) * g;
    gb += t * g;
    gfa += ba * (-fb / (den * den)) * g;
    gfb += ba * (fa / (den * den)) * g;
}

struct Ray {
    float cdx, cdy, cdz;     // normalised camera-space direction
    float ux, uy, uz, wl;    // R cd and its length
    float wdx, wdy, wdz;     // normalised world direction
    float ox, oy, oz;
};

// renderKernel's ray setup, RayCastRender.cu:447-470 (same operations as
// render_pixel)
__device__ __forceinline__ Ray make_ray(const BackArgs& a, int x, int y) {
    const float* T = a.pose.T;
    Ray r;
    float cdx = ((float)x - a.cx) / a.fx, cdy = ((float)y - a.cy) / a.fy, cdz = 1.0f;
    const float cl = sqrtf(cdx * cdx + cdy * cdy + cdz * cdz);
    if (cl > 1e-6f) {
        cdx /= cl;
        cdy /= cl;
        cdz /= cl;
    }
    r.cdx = cdx;
    r.cdy = cdy;
    r.cdz = cdz;
    float wdx = T[0] * cdx + T[1] * cdy + T[2] * cdz;
    float wdy = T[4] * cdx + T[5] * cdy + T[6] * cdz;
    float wdz = T[8] * cdx + T[9] * cdy + T[10] * cdz;
    r.ux = wdx;
    r.uy = wdy;
    r.uz = wdz;
    const float wl = sqrtf(wdx * wdx + wdy * wdy + wdz * wdz);
    r.wl = wl;
    if (wl > 1e-6f) {
        wdx /= wl;
        wdy /= wl;
        wdz /= wl;
    }
    r.wdx = wdx;
    r.wdy = wdy;
    r.wdz = wdz;
    r.ox = T[3];
    r.oy = T[7];
    r.oz = T[11];
    return r;
}

// Recompute the crossing of one hit pixel: nodes P[0..3] = a, b, c1, c2 with
// values F[0..3], bracket indices of steps 2 and 3, alpha.  false when a
// sample is invalid (cannot happen for a hit recorded by the same scene).
struct Crossing {
    float P[4], F[4];
    double G[4][3];  // d F / d position at each node
    NodeTaps taps[4];
    int ia[3], ib[3];  // bracket (node indices) of regula-falsi steps 1..3
    float alpha;
};

__device__ bool recompute(const SceneDev& s, const Ray& r, float a0, float b0, Crossing& c) {
    c.P[0] = a0;
    c.P[1] = b0;
    int ia = 0, ib = 1;
    for (int k = 0; k < 4; ++k) {
        if (k >= 2) {
            c.ia[k - 2] = ia;
            c.ib[k - 2] = ib;
            c.P[k] = rf(c.P[ia], c.F[ia], c.P[ib], c.F[ib]);
        }
        const float t = c.P[k];
        const Sample sm = sample_grad(s, r.ox + t * r.wdx, r.oy + t * r.wdy, r.oz + t * r.wdz, nullptr, 0.0f,
                                      &c.taps[k]);
        if (!sm.ok) return false;
        c.F[k] = sm.f;
        c.G[k][0] = sm.gx;
        c.G[k][1] = sm.gy;
        c.G[k][2] = sm.gz;
        if (k >= 2) {
            if (c.F[ia] * c.F[k] > 0.0f)
                ia = k;
            else
                ib = k;
        }
    }
    c.ia[2] = ia;
    c.ib[2] = ib;
    c.alpha = rf(c.P[ia], c.F[ia], c.P[ib], c.F[ib]);
    return true;
}

// One hit pixel's reverse pass: dL/dT (12 entries, written to gT) for
// dL/ddepth = gd and dL/dposition = gp.  false (and counted in a.skipped)
// when the pixel is left out; gT is then untouched.
__device__ bool pixel_grad(const BackArgs& a, int x, int y, size_t pi, float depth, float gd, float4 gp,
                           double gT[12]) {
    const Ray r = make_ray(a, x, y);
    const float2 br = a.rec[pi];
    Crossing c;
    const float d2r = 1.0f / r.cdz;
    if (!recompute(a.s, r, br.x, br.y, c) ||
        __float_as_uint(c.alpha / d2r) != __float_as_uint(depth)) {
        atomicAdd(a.skipped, 1u);
        return false;
    } else {
        // the smooth function of the frozen decisions, in double
        double cd[3] = {((double)x - a.cx) / a.fx, ((double)y - a.cy) / a.fy, 1.0};
        {
            const double cl = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
            cd[0] /= cl;
            cd[1] /= cl;
            cd[2] /= cl;
        }
        const float* T = a.pose.T;
        double u[3], wd[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            u[i] = (double)T[4 * i] * cd[0] + (double)T[4 * i + 1] * cd[1] + (double)T[4 * i + 2] * cd[2];
        const double wl = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
#pragma unroll
        for (int i = 0; i < 3; ++i) wd[i] = u[i] / wl;
        const double o[3] = {T[3], T[7], T[11]};
        double P[4] = {0.0, 0.0, 0.0, 0.0}, F[4] = {0.0, 0.0, 0.0, 0.0}, G[4][3] = {};
        P[0] = br.x;
        P[1] = br.y;
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k >= 2) {
                const int s = k - 2;
                ok = ok && F[c.ia[s]] != F[c.ib[s]];
                P[k] = rf64(P[c.ia[s]], F[c.ia[s]], P[c.ib[s]], F[c.ib[s]]);
            }
            const double q[3] = {o[0] + P[k] * wd[0], o[1] + P[k] * wd[1], o[2] + P[k] * wd[2]};
            double wsum = 0.0;
            ok = ok && sample64(a.s, q, c.taps[k], F[k], G[k], nullptr, 0.0, &wsum);
            ok = ok && wsum >= (double)a.min_w;
        }
        // a step whose two values coincide in exact arithmetic (e.g. both
        // samples read truncation-clamped voxels only) has no derivative:
        // the forward's step there was decided by rounding noise
        ok = ok && F[c.ia[2]] != F[c.ib[2]];
        const double alpha = ok ? rf64(P[c.ia[2]], F[c.ia[2]], P[c.ib[2]], F[c.ib[2]]) : 0.0;
        ok = ok && isfinite(alpha);
        if (!ok) {
            atomicAdd(a.skipped, 1u);
            return false;
        }
        // outputs: depth = alpha cd_z, position = o + alpha wd
        double g_alpha = (double)gd * cd[2] + (double)gp.x * wd[0] + (double)gp.y * wd[1] +
                         (double)gp.z * wd[2];
        double go[3] = {gp.x, gp.y, gp.z};
        double gw[3] = {alpha * gp.x, alpha * gp.y, alpha * gp.z};
        double gP[4] = {0.0, 0.0, 0.0, 0.0}, gF[4] = {0.0, 0.0, 0.0, 0.0};
        if (ok) {
            rf_back(P[c.ia[2]], F[c.ia[2]], P[c.ib[2]], F[c.ib[2]], g_alpha, gP[c.ia[2]], gF[c.ia[2]],
                    gP[c.ib[2]], gF[c.ib[2]]);
            // nodes 3, 2 (regula-falsi points), then 1, 0 (bracket ends)
#pragma unroll
            for (int k = 3; k >= 0; --k) {
                const double gf = gF[k];
                if (gf != 0.0) {
                    if (a.g_sdf) {
                        const double q[3] = {o[0] + P[k] * wd[0], o[1] + P[k] * wd[1], o[2] + P[k] * wd[2]};
                        double fdummy, gdummy[3];
                        sample64(a.s, q, c.taps[k], fdummy, gdummy, a.g_sdf, gf);
                    }
                    go[0] += gf * G[k][0];
                    go[1] += gf * G[k][1];
                    go[2] += gf * G[k][2];
                    gw[0] += gf * P[k] * G[k][0];
                    gw[1] += gf * P[k] * G[k][1];
                    gw[2] += gf * P[k] * G[k][2];
                    gP[k] += gf * (G[k][0] * wd[0] + G[k][1] * wd[1] + G[k][2] * wd[2]);
                }
                if (k >= 2) {  // node k = RF of step k-1's bracket
                    const int s = k - 2;
                    rf_back(P[c.ia[s]], F[c.ia[s]], P[c.ib[s]], F[c.ib[s]], gP[k], gP[c.ia[s]], gF[c.ia[s]],
                            gP[c.ib[s]], gF[c.ib[s]]);
                }
            }
            // wd = u / |u|, u = R cd
            double gu[3];
            {
                const double dot = gw[0] * wd[0] + gw[1] * wd[1] + gw[2] * wd[2];
                gu[0] = (gw[0] - dot * wd[0]) / wl;
                gu[1] = (gw[1] - dot * wd[1]) / wl;
                gu[2] = (gw[2] - dot * wd[2]) / wl;
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
#pragma unroll
                for (int j = 0; j < 3; ++j) gT[4 * i + j] = gu[i] * cd[j];
                gT[4 * i + 3] = go[i];
            }
        }
    }
    return true;
}

__global__ void __launch_bounds__(128) k_render_backward(BackArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int y = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    double gT[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) gT[i] = 0.0;
    if (x < a.W && y < a.H) {
        const size_t pi = (size_t)y * a.W + x;
        const float depth = a.depth[pi];
        const float gd = a.g_depth ? a.g_depth[pi] : 0.0f;
        const float4 gp = a.g_pos ? a.g_pos[pi] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (depth < 0.5f * kMinf && (gd != 0.0f || gp.x != 0.0f || gp.y != 0.0f || gp.z != 0.0f))
            pixel_grad(a, x, y, pi, depth, gd, gp, gT);
    }
    // deterministic reduction: warp shuffles, then the CTA's four warps
    __shared__ double red[4][12];
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        double v = gT[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        if (lane == 0) red[warp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        const int i = threadIdx.x;
        a.partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 12 + i] =
            ((red[0][i] + red[1][i]) + red[2][i]) + red[3][i];
    }
}

// Gauss-Newton normal equations of a weighted depth least-squares problem in
// the pose's right-perturbation coordinates xi = (omega, v): T exp(xi),
// dR = R [omega]x, dt = R v.  Per hit pixel the reverse pass with dL/ddepth
// = 1 gives the depth's Jacobian J_T (12); J_xi follows by the chain rule,
// and the pixel adds w J J^T and w J r.  Output per CTA: H's upper triangle
// (21, row-major) then b (6), in double.
constexpr int kNeVals = 27;

__global__ void __launch_bounds__(128) k_pose_normal_equations(BackArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int y = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    double acc[kNeVals];
#pragma unroll
    for (int i = 0; i < kNeVals; ++i) acc[i] = 0.0;
    if (x < a.W && y < a.H) {
        const size_t pi = (size_t)y * a.W + x;
        const float depth = a.depth[pi];
        const float w = a.wts ? a.wts[pi] : 1.0f;
        const float res = a.resid[pi];
        double gT[12];
        if (depth < 0.5f * kMinf && w != 0.0f && isfinite(res) &&
            pixel_grad(a, x, y, pi, depth, 1.0f, make_float4(0.0f, 0.0f, 0.0f, 0.0f), gT)) {
            const float* T = a.pose.T;
            double J[6];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                // d depth / d omega_k = sum_ij J_T[i][j] (R (e_k x e_j))_i
                double sum = 0.0;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double c[3] = {0.0, 0.0, 0.0};  // e_k x e_j
                    const int m = 3 - k - j;        // the remaining axis when k != j
                    if (k != j) c[m] = ((j - k + 3) % 3 == 1) ? 1.0 : -1.0;
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const double Rc = (double)T[4 * i] * c[0] + (double)T[4 * i + 1] * c[1] +
                                          (double)T[4 * i + 2] * c[2];
                        sum += gT[4 * i + j] * Rc;
                    }
                }
                J[k] = sum;
                // d depth / d v_k = sum_i J_t[i] R[i][k]
                J[3 + k] = gT[3] * (double)T[k] + gT[7] * (double)T[4 + k] + gT[11] * (double)T[8 + k];
            }
            int n = 0;
#pragma unroll
            for (int p = 0; p < 6; ++p)
#pragma unroll
                for (int q = p; q < 6; ++q) acc[n++] += (double)w * J[p] * J[q];
#pragma unroll
            for (int p = 0; p < 6; ++p) acc[21 + p] += (double)w * J[p] * (double)res;
        }
    }
    __shared__ double red[4][kNeVals];
#pragma unroll
    for (int i = 0; i < kNeVals; ++i) {
        double v = acc[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        if (lane == 0) red[warp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < kNeVals) {
        const int i = threadIdx.x;
        a.partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * kNeVals + i] =
            ((red[0][i] + red[1][i]) + red[2][i]) + red[3][i];
    }
}

// Sum nv values (nv <= 32) over n partial records in a fixed order (four
// independent accumulators per lane keep four loads in flight).
__global__ void k_reduce_records(const double* partials, int n, int nv, double* out) {
    __shared__ double red[32][33];
    const int i = threadIdx.x / 32, lane = threadIdx.x % 32;
    double s = 0.0;
    if (i < nv) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int k = lane;
        for (; k + 96 < n; k += 128) {
            s0 += partials[(size_t)k * nv + i];
            s1 += partials[(size_t)(k + 32) * nv + i];
            s2 += partials[(size_t)(k + 64) * nv + i];
            s3 += partials[(size_t)(k + 96) * nv + i];
        }
        for (; k < n; k += 32) s0 += partials[(size_t)k * nv + i];
        s = (s0 + s1) + (s2 + s3);
    }
    red[i][lane] = s;
    __syncthreads();
    if (lane == 0 && i < nv) {
        double t = 0.0;
        for (int k = 0; k < 32; ++k) t += red[i][k];
        out[i] = t;
    }
}

__global__ void k_reduce_pose(const double* partials, int n, double* out) {
    __shared__ double red[12][32];
    const int i = threadIdx.x / 32, lane = threadIdx.x % 32;  // 384 threads: 12 x 32
    double s = 0.0;
    for (int k = lane; k < n; k += 32) s += partials[(size_t)k * 12 + i];
    red[i][lane] = s;
    __syncthreads();
    if (lane == 0) {
        double t = 0.0;
        for (int k = 0; k < 32; ++k) t += red[i][k];
        out[i] = t;
    }
}

// Normal at the hit: the normalised trilinear SDF gradient at o + alpha wd.
__global__ void __launch_bounds__(128) k_render_normals(BackArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int y = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    if (x >= a.W || y >= a.H) return;
    const size_t pi = (size_t)y * a.W + x;
    float4 n = make_float4(kMinf, kMinf, kMinf, kMinf);
    const float depth = a.depth[pi];
    if (depth < 0.5f * kMinf) {
        const Ray r = make_ray(a, x, y);
        const float2 br = a.rec[pi];
        Crossing c;
        const float d2r = 1.0f / r.cdz;
        if (recompute(a.s, r, br.x, br.y, c) && __float_as_uint(c.alpha / d2r) == __float_as_uint(depth)) {
            const float t = c.alpha;
            const Sample sm = sample_grad(a.s, r.ox + t * r.wdx, r.oy + t * r.wdy, r.oz + t * r.wdz, nullptr, 0.0f);
            const float len = sqrtf(sm.gx * sm.gx + sm.gy * sm.gy + sm.gz * sm.gz);
            if (sm.ok && len > 0.0f) n = make_float4(sm.gx / len, sm.gy / len, sm.gz / len, 0.0f);
        } else {
            atomicAdd(a.skipped, 1u);
        }
    }
    a.normals[pi] = n;
}

__global__ void k_lookup_blocks(SceneDev s, const int* coords, uint32_t n, int* ptrs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        ptrs[i] = block_ptr(s, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
}

int prepare(const Renderer& r, const Scene& sc, const float pose[16], float fx, float fy, float cx, float cy,
            BackArgs& a) {
    if (!r.record || !r.bracket) return VSG_ERR_NOT_ALLOCATED;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != sc.device || dev != r.device) return VSG_ERR_INVALID_ARG;
    std::memset(&a, 0, sizeof(a));
    a.s = sc.dev;
    a.W = r.w;
    a.H = r.h;
    std::memcpy(a.pose.T, pose, sizeof(a.pose.T));
    a.fx = fx;
    a.fy = fy;
    a.cx = cx;
    a.cy = cy;
    a.depth = r.depth;
    a.rec = r.bracket;
    a.partials = r.partials;
    a.skipped = r.skipped;
    return VSG_OK;
}

int read_skipped(const Renderer& r, uint32_t* n, cudaStream_t st) {
    if (!n) return VSG_OK;
    if (cudaMemcpyAsync(n, r.skipped, sizeof(unsigned int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return VSG_ERR_CUDA;
    return VSG_OK;
}

}  // namespace
}  // namespace vsg

extern "C" {

int vsg_renderer_record(vsg_renderer* rh, int enable) {
    if (!rh) return VSG_ERR_INVALID_ARG;
    vsg::Renderer& r = rh->impl;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != r.device) return VSG_ERR_INVALID_ARG;  // buffers go on r's device
    if (enable && !r.bracket) {
        const size_t n = (size_t)r.w * r.h;
        const size_t ctas = (size_t)((r.w + 15) / 16) * ((r.h + 7) / 8);
        if (cudaMalloc(&r.bracket, n * sizeof(float2)) != cudaSuccess ||
            cudaMalloc(&r.partials, ctas * vsg::kNeVals * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&r.skipped, sizeof(unsigned int)) != cudaSuccess) {
            cudaFree(r.bracket);
            cudaFree(r.partials);
            cudaFree(r.skipped);
            r.bracket = nullptr;
            r.partials = nullptr;
            r.skipped = nullptr;
            return VSG_ERR_OUT_OF_MEMORY;
        }
    }
    r.record = enable != 0;
    return VSG_OK;
}

int vsg_render_backward(const vsg_renderer* rh, const vsg_scene* s, const float pose[16], float fx, float fy,
                        float cx, float cy, const float* grad_depth, const float* grad_position, double* grad_pose,
                        float* grad_sdf, float min_weight_sum, uint32_t* n_skipped, vsg_stream_t stream) {
    if (!rh || !s || !pose || !grad_pose || !(min_weight_sum >= 0.0f)) return VSG_ERR_INVALID_ARG;
    const vsg::Renderer& r = rh->impl;
    vsg::BackArgs a;
    const int rc = vsg::prepare(r, s->impl, pose, fx, fy, cx, cy, a);
    if (rc != VSG_OK) return rc;
    a.g_depth = grad_depth;
    a.g_pos = reinterpret_cast<const float4*>(grad_position);
    a.g_sdf = grad_sdf;
    a.min_w = min_weight_sum;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(r.skipped, 0, sizeof(unsigned int), st) != cudaSuccess) return VSG_ERR_CUDA;
    const dim3 grid((r.w + 15) / 16, (r.h + 7) / 8);
    vsg::k_render_backward<<<grid, 128, 0, st>>>(a);
    vsg::k_reduce_pose<<<1, 384, 0, st>>>(r.partials, (int)(grid.x * grid.y), grad_pose);
    if (cudaGetLastError() != cudaSuccess) return VSG_ERR_CUDA;
    return vsg::read_skipped(r, n_skipped, st);
}

int vsg_scene_lookup_blocks(const vsg_scene* s, const int32_t* coords, uint32_t n, int32_t* ptrs) {
    if (!s || (n && (!coords || !ptrs))) return VSG_ERR_INVALID_ARG;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != s->impl.device) return VSG_ERR_INVALID_ARG;
    if (n == 0) return VSG_OK;
    int* d = nullptr;
    if (cudaMalloc(&d, (size_t)n * 4 * sizeof(int)) != cudaSuccess) return VSG_ERR_OUT_OF_MEMORY;
    int rc = VSG_OK;
    if (cudaMemcpy(d, coords, (size_t)n * 3 * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = VSG_ERR_CUDA;
    } else {
        const int grid = (int)std::min<uint32_t>((n + 255) / 256, 4096u);
        vsg::k_lookup_blocks<<<grid, 256>>>(s->impl.dev, d, n, d + (size_t)n * 3);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(ptrs, d + (size_t)n * 3, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = VSG_ERR_CUDA;
    }
    cudaFree(d);
    return rc;
}

int vsg_render_pose_normal_equations(const vsg_renderer* rh, const vsg_scene* s, const float pose[16], float fx,
                                     float fy, float cx, float cy, const float* residual, const float* weights,
                                     float min_weight_sum, double* normal_eq, uint32_t* n_skipped,
                                     vsg_stream_t stream) {
    if (!rh || !s || !pose || !residual || !normal_eq || !(min_weight_sum >= 0.0f)) return VSG_ERR_INVALID_ARG;
    const vsg::Renderer& r = rh->impl;
    vsg::BackArgs a;
    const int rc = vsg::prepare(r, s->impl, pose, fx, fy, cx, cy, a);
    if (rc != VSG_OK) return rc;
    a.resid = residual;
    a.wts = weights;
    a.min_w = min_weight_sum;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(r.skipped, 0, sizeof(unsigned int), st) != cudaSuccess) return VSG_ERR_CUDA;
    const dim3 grid((r.w + 15) / 16, (r.h + 7) / 8);
    vsg::k_pose_normal_equations<<<grid, 128, 0, st>>>(a);
    vsg::k_reduce_records<<<1, 32 * 32, 0, st>>>(r.partials, (int)(grid.x * grid.y), vsg::kNeVals, normal_eq);
    if (cudaGetLastError() != cudaSuccess) return VSG_ERR_CUDA;
    return vsg::read_skipped(r, n_skipped, st);
}

int vsg_render_normals(const vsg_renderer* rh, const vsg_scene* s, const float pose[16], float fx, float fy,
                       float cx, float cy, float* normals, uint32_t* n_skipped, vsg_stream_t stream) {
    if (!rh || !s || !pose || !normals) return VSG_ERR_INVALID_ARG;
    const vsg::Renderer& r = rh->impl;
    vsg::BackArgs a;
    const int rc = vsg::prepare(r, s->impl, pose, fx, fy, cx, cy, a);
    if (rc != VSG_OK) return rc;
    a.normals = reinterpret_cast<float4*>(normals);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(r.skipped, 0, sizeof(unsigned int), st) != cudaSuccess) return VSG_ERR_CUDA;
    const dim3 grid((r.w + 15) / 16, (r.h + 7) / 8);
    vsg::k_render_normals<<<grid, 128, 0, st>>>(a);
    if (cudaGetLastError() != cudaSuccess) return VSG_ERR_CUDA;
    return vsg::read_skipped(r, n_skipped, st);
}

}  // extern "C"
