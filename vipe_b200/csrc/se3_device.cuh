// Device SE3 helpers for the bundle-adjustment kernels.
//
// Poses are stored [tx ty tz qx qy qz qw] (reference layout, poses (N,7)).
// These follow the formulas of the reference's fused BA helpers
// (vipe: csrc/slam_ext/geom_kernels.cu:69-177) so that FP32 results agree with
// the reference to rounding; they are written here as small inline functions on
// register arrays.
#pragma once

namespace vipe {

// Y = R(q) X
__device__ __forceinline__ void qrot(const float* q, const float* X, float* Y) {
    const float u0 = 2.0f * (q[1] * X[2] - q[2] * X[1]);
    const float u1 = 2.0f * (q[2] * X[0] - q[0] * X[2]);
    const float u2 = 2.0f * (q[0] * X[1] - q[1] * X[0]);
    Y[0] = X[0] + q[3] * u0 + (q[1] * u2 - q[2] * u1);
    Y[1] = X[1] + q[3] * u1 + (q[2] * u0 - q[0] * u2);
    Y[2] = X[2] + q[3] * u2 + (q[0] * u1 - q[1] * u0);
}

// homogeneous action Y = [R X + X3 t, X3]
__device__ __forceinline__ void act_h(const float* t, const float* q, const float* X, float* Y) {
    qrot(q, X, Y);
    Y[3] = X[3];
    Y[0] += X[3] * t[0];
    Y[1] += X[3] * t[1];
    Y[2] += X[3] * t[2];
}

// pulls a target-pose Jacobian row back to the source pose: Y = Ad^T X
__device__ __forceinline__ void adj_t(const float* t, const float* q, const float* X, float* Y) {
    const float qi[4] = {-q[0], -q[1], -q[2], q[3]};
    qrot(qi, X, Y);
    qrot(qi, X + 3, Y + 3);
    const float u[3] = {t[2] * X[1] - t[1] * X[2], t[0] * X[2] - t[2] * X[0], t[1] * X[0] - t[0] * X[1]};
    float v[3];
    qrot(qi, u, v);
    Y[3] += v[0];
    Y[4] += v[1];
    Y[5] += v[2];
}

// Tij = Tj * Ti^-1
__device__ __forceinline__ void rel_pose(const float* Ti, const float* Tj, float* tij, float* qij) {
    const float* qi = Ti + 3;
    const float* qj = Tj + 3;
    qij[0] = -qj[3] * qi[0] + qj[0] * qi[3] - qj[1] * qi[2] + qj[2] * qi[1];
    qij[1] = -qj[3] * qi[1] + qj[1] * qi[3] - qj[2] * qi[0] + qj[0] * qi[2];
    qij[2] = -qj[3] * qi[2] + qj[2] * qi[3] - qj[0] * qi[1] + qj[1] * qi[0];
    qij[3] = qj[3] * qi[3] + qj[0] * qi[0] + qj[1] * qi[1] + qj[2] * qi[2];
    float r[3];
    qrot(qij, Ti, r);
    tij[0] = Tj[0] - r[0];
    tij[1] = Tj[1] - r[1];
    tij[2] = Tj[2] - r[2];
}

// relative pose of an edge; ii == jj is a stereo edge with a fixed baseline
__device__ __forceinline__ void edge_pose(const float* poses, int a, int b, float* tij, float* qij) {
    if (a == b) {
        tij[0] = -0.1f; tij[1] = 0.f; tij[2] = 0.f;
        qij[0] = 0.f; qij[1] = 0.f; qij[2] = 0.f; qij[3] = 1.f;
    } else {
        float Ti[7], Tj[7];
#pragma unroll
        for (int n = 0; n < 7; n++) {
            Ti[n] = __ldg(poses + 7 * a + n);
            Tj[n] = __ldg(poses + 7 * b + n);
        }
        rel_pose(Ti, Tj, tij, qij);
    }
}

// SE3 exponential (tangent [tau, phi]) -> (t, q)
__device__ __forceinline__ void se3_exp(const float* xi, float* t, float* q) {
    const float* phi = xi + 3;
    const float th2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
    const float th = sqrtf(th2);
    float im, re;
    if (th2 < 1e-8f) {
        im = 0.5f - (1.0f / 48.0f) * th2 + (1.0f / 3840.0f) * th2 * th2;
        re = 1.0f - (1.0f / 8.0f) * th2 + (1.0f / 384.0f) * th2 * th2;
    } else {
        im = sinf(0.5f * th) / th;
        re = cosf(0.5f * th);
    }
    q[0] = im * phi[0];
    q[1] = im * phi[1];
    q[2] = im * phi[2];
    q[3] = re;
    t[0] = xi[0];
    t[1] = xi[1];
    t[2] = xi[2];
    if (th > 1e-4f) {
        const float c1[3] = {phi[1] * xi[2] - phi[2] * xi[1], phi[2] * xi[0] - phi[0] * xi[2],
                             phi[0] * xi[1] - phi[1] * xi[0]};
        const float c2[3] = {phi[1] * c1[2] - phi[2] * c1[1], phi[2] * c1[0] - phi[0] * c1[2],
                             phi[0] * c1[1] - phi[1] * c1[0]};
        const float A = (1.0f - cosf(th)) / th2;
        const float B = (th - sinf(th)) / (th * th2);
        t[0] += A * c1[0];
        t[1] += A * c1[1];
        t[2] += A * c1[2];
        t[0] += B * c2[0];
        t[1] += B * c2[1];
        t[2] += B * c2[2];
    }
}

// left retraction T <- Exp(xi) T, in place on a (7,) pose
__device__ __forceinline__ void retract_pose(const float* xi, float* T) {
    float dt[3], dq[4];
    se3_exp(xi, dt, dq);
    const float q[4] = {T[3], T[4], T[5], T[6]};
    const float t[3] = {T[0], T[1], T[2]};
    float t1[3];
    qrot(dq, t, t1);
    T[0] = t1[0] + dt[0];
    T[1] = t1[1] + dt[1];
    T[2] = t1[2] + dt[2];
    T[3] = dq[3] * q[0] + dq[0] * q[3] + dq[1] * q[2] - dq[2] * q[1];
    T[4] = dq[3] * q[1] + dq[1] * q[3] + dq[2] * q[0] - dq[0] * q[2];
    T[5] = dq[3] * q[2] + dq[2] * q[3] + dq[0] * q[1] - dq[1] * q[0];
    T[6] = dq[3] * q[3] - dq[0] * q[0] - dq[1] * q[1] - dq[2] * q[2];
}

// Linearisation of one edge at one pixel (both flow channels).  Follows the
// per-pixel body of the reference kernel (geom_kernels.cu:298-435): MIN_DEPTH
// mask, 0.001 weight scale, stereo rule, optional focal derivative.
struct PixelLin {
    float Ji[2][6];   // source-pose Jacobian per channel
    float Jj[2][6];   // target-pose Jacobian per channel
    float Jz[2];      // inverse-depth Jacobian per channel
    float w[2];       // pose weight (0 for stereo edges)
    float wd[2];      // depth weight (w * depth_active, before the stereo rule)
    float we[2];      // energy weight (masked and scaled, before the stereo rule)
    float r[2];       // residual
    float Jf[2];      // focal Jacobian (when requested)
};

// Robust reweighting of the reprojection residuals, per flow channel, at the linearisation
// point (the reference's generic solver: vipe/slam/ba/kernel.py:40-162, applied as
// w <- w * kernel(r) by ConcreteTermEvalReturn.apply_robust_kernel, terms.py:73-75):
//   kind 1 Huber    1 if |r| <= c else c / max(|r|, 1e-8)
//   kind 2 Tukey    max(1 - (r/c)^2, 0)^2
//   kind 3 GNC-TLS  at scalar mu: 1 below mu/(mu+1) c^2, 0 above (mu+1)/mu c^2, between
//                   max(sqrt(c^2 mu (mu+1) / r^2) - mu, 0); mu = +inf: the hard TLS 1{r^2 < c^2}
// kind 0: no reweighting.
// Also carried here: the camera model of the frames (cam 0 pinhole; cam 1 the unified
// (MEI) model of vipe/utils/cameras.py:220-330 with distortion k1, fx fy cx cy as for pinhole),
// and per-view intrinsics of a multi-view rig: nview > 1 means the intrinsics array holds
// nview rows (fx, fy, cx, cy) and depth frame f is seen by view f % nview (the generic
// solver's intrinsics (Q, 4) indexed by the terms' rig indices, vipe/slam/ba/terms.py:175-206).
struct RobustSpec {
    int kind = 0;
    float c = 1.0f;
    float mu = 1.0f;
    int cam = 0;
    float k1 = 0.0f;
    int nview = 0;
    const float* k1v = nullptr;  // per-view MEI distortion (nview entries), or one k1 for all
};

// Intrinsics of the source view of a term when they differ from the target view's (per-view
// intrinsics of a rig): the pixel is unprojected with these, projected with the target's
// (the fx, fy, cx, cy arguments of the linearisation).  on == 0: one camera for both.
struct SrcIntr {
    int on = 0;
    float fx = 1.0f, fy = 1.0f, cx = 0.0f, cy = 0.0f;
    float k1 = 0.0f;  // the source view's MEI distortion
};

// per-view intrinsics: the target view's row of depth frame b into fx..cy and the source
// view's row of depth frame a into si
__device__ __forceinline__ void view_intrinsics(const float* intr, int nview, int a, int b, float& fx, float& fy,
                                                float& cx, float& cy, SrcIntr& si) {
    const float* ki = intr + 4 * (a % nview);
    const float* kj = intr + 4 * (b % nview);
    fx = kj[0];
    fy = kj[1];
    cx = kj[2];
    cy = kj[3];
    si.on = 1;
    si.fx = ki[0];
    si.fy = ki[1];
    si.cx = ki[2];
    si.cy = ki[3];
}

// the per-view camera of a term from source frame a into target frame b: the target's
// intrinsics into fx..cy and its MEI distortion into rb.k1, the source's into si
__device__ __forceinline__ void view_camera(const float* intr, RobustSpec& rb, int a, int b, float& fx, float& fy,
                                            float& cx, float& cy, SrcIntr& si) {
    view_intrinsics(intr, rb.nview, a, b, fx, fy, cx, cy, si);
    if (rb.k1v) {
        si.k1 = rb.k1v[a % rb.nview];
        rb.k1 = rb.k1v[b % rb.nview];
    } else {
        si.k1 = rb.k1;
    }
}

__device__ __forceinline__ float robust_weight(const RobustSpec& rb, float r) {
    if (rb.kind == 1) {
        const float a = fabsf(r);
        return a <= rb.c ? 1.0f : rb.c / fmaxf(a, 1e-8f);
    }
    if (rb.kind == 2) {
        const float t = fmaxf(1.0f - (r / rb.c) * (r / rb.c), 0.0f);
        return t * t;
    }
    if (rb.kind == 3) {
        const float r2 = r * r, c2 = rb.c * rb.c, mu = rb.mu;
        if (!(mu < INFINITY)) return r2 < c2 ? 1.0f : 0.0f;
        if (r2 < (mu / (mu + 1.0f)) * c2) return 1.0f;
        if (r2 <= ((mu + 1.0f) / mu) * c2) return fmaxf(sqrtf(c2 * mu * (mu + 1.0f) / fmaxf(r2, 1e-12f)) - mu, 0.0f);
        return 0.0f;
    }
    return 1.0f;
}

// The unified (MEI) camera, as the reference's MeiCameraModel (vipe/utils/cameras.py:220-330):
// unprojection of pixel (u, v) to (X, Y, 1) with u_b = (u - cx) / fx, v_b = (v - cy) / fy,
// r2 = u_b^2 + v_b^2, q = sqrt(1 + (1 - k1^2) r2), s = (k1 + q) / (1 + r2):
// X = u_b s / (s - k1), Y = v_b s / (s - k1); projection of P: x = fx P0 / (P2 + k1 |P|) + cx,
// y = fy P1 / (P2 + k1 |P|) + cy, with the projection gradient g_c (row c of its Jacobian in P).
// The pose and depth rows follow from g_c as for any central camera: target pose
// (h g_c, P x g_c), source pose -Ad(Tij)^T of it, inverse depth g_c . t.  The focal
// derivative is not formed (the solver refuses optimize_intrinsics with this camera).
template <bool kResidual>
__device__ __forceinline__ void linearize_mei(const float* tij, const float* qij, bool stereo, float fx, float fy,
                                              float cx, float cy, float u, float v, float disp, float wu_in,
                                              float wv_in, float tu, float tv, float act, PixelLin& L,
                                              const RobustSpec& rb, const SrcIntr& si) {
    const float k1 = rb.k1;                 // the target view's (projection)
    const float k1s = si.on ? si.k1 : k1;   // the source view's (unprojection)
    const float ub = si.on ? (u - si.cx) / si.fx : (u - cx) / fx;
    const float vb = si.on ? (v - si.cy) / si.fy : (v - cy) / fy;
    const float r2 = ub * ub + vb * vb;
    const float qq = sqrtf(1.0f + (1.0f - k1s * k1s) * r2);
    const float fac = (k1s + qq) / (1.0f + r2);
    const float Xi[4] = {ub * fac / (fac - k1s), vb * fac / (fac - k1s), 1.0f, disp};
    float Xj[4];
    act_h(tij, qij, Xi, Xj);
    const float P0 = Xj[0], P1 = Xj[1], P2 = Xj[2], h = Xj[3];
    const bool ok = !(P2 < 0.25f);
    const float rn = sqrtf(P0 * P0 + P1 * P1 + P2 * P2);
    const float rb_ = P2 + k1 * rn;
    const float dm = ok ? 1.0f / rb_ : 0.0f;
    const float iden = ok ? 1.0f / (rb_ * rb_ * rn) : 0.0f;
    // projection gradients g[c] = d(x_c)/dP
    float g[2][3];
    g[0][0] = fx * (rb_ * rn - k1 * P0 * P0) * iden;
    g[0][1] = -fx * k1 * P0 * P1 * iden;
    g[0][2] = -fx * P0 * (k1 * P2 + rn) * iden;
    g[1][0] = -fy * k1 * P0 * P1 * iden;
    g[1][1] = fy * (rb_ * rn - k1 * P1 * P1) * iden;
    g[1][2] = -fy * P1 * (k1 * P2 + rn) * iden;
    const float xu = fx * P0 * dm + cx, xv = fy * P1 * dm + cy;
    float wu = ok ? 0.001f * wu_in : 0.0f;
    float wv = ok ? 0.001f * wv_in : 0.0f;
    if (rb.kind != 0) {
        wu *= robust_weight(rb, tu - xu);
        wv *= robust_weight(rb, tv - xv);
    }
    L.Jf[0] = 0.0f;
    L.Jf[1] = 0.0f;
    L.r[0] = kResidual ? tu - xu : 0.0f;
    L.r[1] = kResidual ? tv - xv : 0.0f;
#pragma unroll
    for (int ch = 0; ch < 2; ch++) {
        const float* gc = g[ch];
        L.Jj[ch][0] = h * gc[0];
        L.Jj[ch][1] = h * gc[1];
        L.Jj[ch][2] = h * gc[2];
        L.Jj[ch][3] = P1 * gc[2] - P2 * gc[1];
        L.Jj[ch][4] = P2 * gc[0] - P0 * gc[2];
        L.Jj[ch][5] = P0 * gc[1] - P1 * gc[0];
        L.Jz[ch] = gc[0] * tij[0] + gc[1] * tij[1] + gc[2] * tij[2];
        adj_t(tij, qij, L.Jj[ch], L.Ji[ch]);
#pragma unroll
        for (int n = 0; n < 6; n++) L.Ji[ch][n] = -L.Ji[ch][n];
    }
    L.we[0] = wu;
    L.we[1] = wv;
    L.wd[0] = wu * act;
    L.wd[1] = wv * act;
    L.w[0] = stereo ? 0.0f : wu;
    L.w[1] = stereo ? 0.0f : wv;
}

template <bool kIntr, bool kResidual>
__device__ __forceinline__ void linearize(const float* tij, const float* qij, bool stereo, float fx, float fy,
                                          float cx, float cy, float u, float v, float disp, float wu_in, float wv_in,
                                          float tu, float tv, float act, float iscale, PixelLin& L,
                                          const RobustSpec rb = RobustSpec{}, const SrcIntr si = SrcIntr{}) {
    if (rb.cam == 1) {
        linearize_mei<kResidual>(tij, qij, stereo, fx, fy, cx, cy, u, v, disp, wu_in, wv_in, tu, tv, act, L, rb, si);
        return;
    }
    // (the focal derivative below assumes one camera: the rig solve has no intrinsics block)
    float Xi[4] = {si.on ? (u - si.cx) / si.fx : (u - cx) / fx, si.on ? (v - si.cy) / si.fy : (v - cy) / fy, 1.0f,
                   disp};
    float Xj[4];
    act_h(tij, qij, Xi, Xj);
    const float x = Xj[0], y = Xj[1], h = Xj[3];
    const bool ok = !(Xj[2] < 0.25f);
    const float d = ok ? 1.0f / Xj[2] : 0.0f;
    const float d2 = d * d;
    float wu = ok ? 0.001f * wu_in : 0.0f;
    float wv = ok ? 0.001f * wv_in : 0.0f;
    if (rb.kind != 0) {  // needs the residual even where the caller does not
        wu *= robust_weight(rb, tu - (fx * d * x + cx));
        wv *= robust_weight(rb, tv - (fy * d * y + cy));
    }
    if (kIntr) {
        float dXi[4] = {-Xi[0] / fx, -Xi[1] / fy, 0.0f, 0.0f};
        float dXj[4];
        act_h(tij, qij, dXi, dXj);
        L.Jf[0] = iscale * (fx * d * dXj[0] - fx * x * d2 * dXj[2] + x * d);
        L.Jf[1] = iscale * (fy * d * dXj[1] - fy * y * d2 * dXj[2] + y * d);
    } else {
        L.Jf[0] = 0.0f;
        L.Jf[1] = 0.0f;
    }
    if (kResidual) {
        L.r[0] = tu - (fx * d * x + cx);
        L.r[1] = tv - (fy * d * y + cy);
    } else {
        L.r[0] = 0.0f;
        L.r[1] = 0.0f;
    }
    // x channel
    L.Jj[0][0] = fx * (h * d);
    L.Jj[0][1] = 0.0f;
    L.Jj[0][2] = fx * (-x * h * d2);
    L.Jj[0][3] = fx * (-x * y * d2);
    L.Jj[0][4] = fx * (1.0f + x * x * d2);
    L.Jj[0][5] = fx * (-y * d);
    L.Jz[0] = fx * (tij[0] * d - tij[2] * (x * d2));
    // y channel
    L.Jj[1][0] = 0.0f;
    L.Jj[1][1] = fy * (h * d);
    L.Jj[1][2] = fy * (-y * h * d2);
    L.Jj[1][3] = fy * (-1.0f - y * y * d2);
    L.Jj[1][4] = fy * (x * y * d2);
    L.Jj[1][5] = fy * (x * d);
    L.Jz[1] = fy * (tij[1] * d - tij[2] * (y * d2));
#pragma unroll
    for (int ch = 0; ch < 2; ch++) {
        adj_t(tij, qij, L.Jj[ch], L.Ji[ch]);
#pragma unroll
        for (int n = 0; n < 6; n++) L.Ji[ch][n] = -L.Ji[ch][n];
    }
    L.we[0] = wu;
    L.we[1] = wv;
    L.wd[0] = wu * act;
    L.wd[1] = wv * act;
    L.w[0] = stereo ? 0.0f : wu;
    L.w[1] = stereo ? 0.0f : wv;
}

}  // namespace vipe
