// Lie-group algebra on small register arrays (SO3, RxSO3, SE3, Sim3; float or
// double), shared by the lietorch kernels (lie.cu) and the Sim3 bundle
// adjustment (ba.cu).  Storage and tangent conventions are lietorch's: SO3
// [qx qy qz qw], RxSO3 [qx qy qz qw s], SE3 [tx ty tz qx qy qz qw], Sim3
// [tx ty tz qx qy qz qw s]; tangents SO3 [phi], RxSO3 [phi sigma], SE3
// [tau phi], Sim3 [tau phi sigma].  Loading an element normalises its quaternion.
#pragma once

#include "common.cuh"

#include <math.h>

namespace vipe {
namespace lie {

constexpr double kEps = 1e-6;
constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------- small matrices

template <typename S, int R, int C>
struct Mat {
    S m[R][C];
    __device__ S& operator()(int r, int c) { return m[r][c]; }
    __device__ const S& operator()(int r, int c) const { return m[r][c]; }
};

template <typename S, int R, int C>
__device__ __forceinline__ Mat<S, R, C> zeros() {
    Mat<S, R, C> z;
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
        for (int c = 0; c < C; c++) z.m[r][c] = S(0);
    return z;
}

template <typename S, int N>
__device__ __forceinline__ Mat<S, N, N> eye() {
    Mat<S, N, N> z = zeros<S, N, N>();
#pragma unroll
    for (int r = 0; r < N; r++) z.m[r][r] = S(1);
    return z;
}

template <typename S, int R, int K, int C>
__device__ __forceinline__ Mat<S, R, C> mm(const Mat<S, R, K>& a, const Mat<S, K, C>& b) {
    Mat<S, R, C> o;
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
        for (int c = 0; c < C; c++) {
            S s = S(0);
#pragma unroll
            for (int k = 0; k < K; k++) s += a.m[r][k] * b.m[k][c];
            o.m[r][c] = s;
        }
    return o;
}

template <typename S, int R, int C>
__device__ __forceinline__ void mv(const Mat<S, R, C>& a, const S* x, S* y) {
#pragma unroll
    for (int r = 0; r < R; r++) {
        S s = S(0);
#pragma unroll
        for (int c = 0; c < C; c++) s += a.m[r][c] * x[c];
        y[r] = s;
    }
}

// row vector times matrix: y = x^T A
template <typename S, int R, int C>
__device__ __forceinline__ void vm(const S* x, const Mat<S, R, C>& a, S* y) {
#pragma unroll
    for (int c = 0; c < C; c++) {
        S s = S(0);
#pragma unroll
        for (int r = 0; r < R; r++) s += x[r] * a.m[r][c];
        y[c] = s;
    }
}

template <typename S, int R, int C>
__device__ __forceinline__ Mat<S, R, C> add(const Mat<S, R, C>& a, const Mat<S, R, C>& b, S sb = S(1)) {
    Mat<S, R, C> o;
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
        for (int c = 0; c < C; c++) o.m[r][c] = a.m[r][c] + sb * b.m[r][c];
    return o;
}

template <typename S>
__device__ __forceinline__ Mat<S, 3, 3> hat(const S* v) {
    Mat<S, 3, 3> h;
    h.m[0][0] = S(0); h.m[0][1] = -v[2]; h.m[0][2] = v[1];
    h.m[1][0] = v[2]; h.m[1][1] = S(0); h.m[1][2] = -v[0];
    h.m[2][0] = -v[1]; h.m[2][1] = v[0]; h.m[2][2] = S(0);
    return h;
}

template <typename S, int N>
__device__ __forceinline__ void set_block(Mat<S, N, N>& M, int r0, int c0, const Mat<S, 3, 3>& B, S s = S(1)) {
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) M.m[r0 + r][c0 + c] = s * B.m[r][c];
}

// ---------------------------------------------------------------- quaternions

template <typename S>
struct Quat {
    S x, y, z, w;
};

template <typename S>
__device__ __forceinline__ Quat<S> qnormalize(Quat<S> q) {
    const S n = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return {q.x / n, q.y / n, q.z / n, q.w / n};
}

template <typename S>
__device__ __forceinline__ Quat<S> qmul(const Quat<S>& a, const Quat<S>& b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
            a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}

template <typename S>
__device__ __forceinline__ void qrot(const Quat<S>& q, const S* p, S* o) {
    const S u0 = S(2) * (q.y * p[2] - q.z * p[1]);
    const S u1 = S(2) * (q.z * p[0] - q.x * p[2]);
    const S u2 = S(2) * (q.x * p[1] - q.y * p[0]);
    o[0] = p[0] + q.w * u0 + (q.y * u2 - q.z * u1);
    o[1] = p[1] + q.w * u1 + (q.z * u0 - q.x * u2);
    o[2] = p[2] + q.w * u2 + (q.x * u1 - q.y * u0);
}

template <typename S>
__device__ __forceinline__ Mat<S, 3, 3> qmat(const Quat<S>& q) {
    Mat<S, 3, 3> R;
    const S xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const S xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
    const S wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    R.m[0][0] = S(1) - S(2) * (yy + zz); R.m[0][1] = S(2) * (xy - wz); R.m[0][2] = S(2) * (xz + wy);
    R.m[1][0] = S(2) * (xy + wz); R.m[1][1] = S(1) - S(2) * (xx + zz); R.m[1][2] = S(2) * (yz - wx);
    R.m[2][0] = S(2) * (xz - wy); R.m[2][1] = S(2) * (yz + wx); R.m[2][2] = S(1) - S(2) * (xx + yy);
    return R;
}

template <typename S>
__device__ __forceinline__ Quat<S> so3_exp_q(const S* phi) {
    const S t2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
    const S t = sqrt(t2);
    S im, re;
    if (t < S(kEps)) {
        const S t4 = t2 * t2;
        im = S(0.5) - S(1.0 / 48.0) * t2 + S(1.0 / 3840.0) * t4;
        re = S(1) - S(1.0 / 8.0) * t2 + S(1.0 / 384.0) * t4;
    } else {
        im = sin(S(0.5) * t) / t;
        re = cos(S(0.5) * t);
    }
    return qnormalize(Quat<S>{im * phi[0], im * phi[1], im * phi[2], re});
}

// atan-based logarithm of a unit quaternion
template <typename S>
__device__ __forceinline__ void so3_log(const Quat<S>& q, S* phi) {
    const S n2 = q.x * q.x + q.y * q.y + q.z * q.z;
    const S w = q.w;
    S f;
    if (n2 < S(kEps * kEps)) {
        f = S(2) / w - S(2.0 / 3.0) * n2 / (w * w * w);
    } else {
        const S n = sqrt(n2);
        if (fabs(w) < S(kEps))
            f = (w > S(0) ? S(kPi) : -S(kPi)) / n;
        else
            f = S(2) * atan(n / w) / n;
    }
    phi[0] = f * q.x;
    phi[1] = f * q.y;
    phi[2] = f * q.z;
}

template <typename S>
__device__ __forceinline__ Mat<S, 3, 3> so3_left_jac(const S* phi) {
    const Mat<S, 3, 3> P = hat(phi);
    const Mat<S, 3, 3> P2 = mm(P, P);
    const S t2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
    const S t = sqrt(t2);
    const S c1 = (t < S(kEps)) ? S(1.0 / 2.0) - S(1.0 / 24.0) * t2 : (S(1) - cos(t)) / t2;
    const S c2 = (t < S(kEps)) ? S(1.0 / 6.0) - S(1.0 / 120.0) * t2 : (t - sin(t)) / (t2 * t);
    return add(add(eye<S, 3>(), P, c1), P2, c2);
}

template <typename S>
__device__ __forceinline__ Mat<S, 3, 3> so3_left_jac_inv(const S* phi) {
    const Mat<S, 3, 3> P = hat(phi);
    const Mat<S, 3, 3> P2 = mm(P, P);
    const S t2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
    const S t = sqrt(t2);
    const S ht = S(0.5) * t;
    const S c2 = (t < S(kEps)) ? S(1.0 / 12.0) : (S(1) - t * cos(ht) / (S(2) * sin(ht))) / (t * t);
    return add(add(eye<S, 3>(), P, S(-0.5)), P2, c2);
}

// 4x4 projector block of the unit quaternion (shared by all groups)
template <typename S, int N>
__device__ __forceinline__ void quat_projector(const Quat<S>& q, Mat<S, N, N>& J, int o) {
    const S v[3] = {-q.x, -q.y, -q.z};
    const Mat<S, 3, 3> H = hat(v);
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) J.m[o + r][o + c] = S(0.5) * ((r == c ? q.w : S(0)) + H.m[r][c]);
#pragma unroll
    for (int c = 0; c < 3; c++) J.m[o + 3][o + c] = S(0.5) * v[c];
}

// ---------------------------------------------------------------- groups

template <typename S>
struct SO3 {
    static constexpr int N = 4, K = 3;
    Quat<S> q;
    __device__ static SO3 load(const S* d) { return {qnormalize(Quat<S>{d[0], d[1], d[2], d[3]})}; }
    __device__ void store(S* d) const { d[0] = q.x; d[1] = q.y; d[2] = q.z; d[3] = q.w; }
    __device__ static SO3 Exp(const S* a) { return {so3_exp_q(a)}; }
    __device__ void Log(S* a) const { so3_log(q, a); }
    __device__ SO3 inv() const { return {Quat<S>{-q.x, -q.y, -q.z, q.w}}; }
    __device__ SO3 operator*(const SO3& o) const { return {qnormalize(qmul(q, o.q))}; }
    __device__ void act(const S* p, S* o) const { qrot(q, p, o); }
    __device__ void act4(const S* p, S* o) const { qrot(q, p, o); o[3] = p[3]; }
    __device__ Mat<S, K, K> Adj() const { return qmat(q); }
    __device__ static Mat<S, K, K> adj(const S* a) { return hat(a); }
    __device__ Mat<S, 4, 4> mat4() const {
        Mat<S, 4, 4> T = eye<S, 4>();
        const Mat<S, 3, 3> R = qmat(q);
        set_block(T, 0, 0, R);
        return T;
    }
    __device__ Mat<S, 3, 3> mat3() const { return qmat(q); }
    __device__ Mat<S, N, N> projector() const {
        Mat<S, N, N> J = zeros<S, N, N>();
        quat_projector(q, J, 0);
        return J;
    }
    __device__ static Mat<S, K, K> left_jac(const S* a) { return so3_left_jac(a); }
    __device__ static Mat<S, K, K> left_jac_inv(const S* a) { return so3_left_jac_inv(a); }
    __device__ static Mat<S, 3, K> act_jac(const S* p) {
        const S m[3] = {-p[0], -p[1], -p[2]};
        return hat(m);
    }
    __device__ static Mat<S, 4, K> act4_jac(const S* p) {
        Mat<S, 4, K> J = zeros<S, 4, K>();
        const S m[3] = {-p[0], -p[1], -p[2]};
        const Mat<S, 3, 3> H = hat(m);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) J.m[r][c] = H.m[r][c];
        return J;
    }
};

template <typename S>
struct RxSO3 {
    static constexpr int N = 5, K = 4;
    Quat<S> q;
    S s;
    __device__ static RxSO3 load(const S* d) { return {qnormalize(Quat<S>{d[0], d[1], d[2], d[3]}), d[4]}; }
    __device__ void store(S* d) const { d[0] = q.x; d[1] = q.y; d[2] = q.z; d[3] = q.w; d[4] = s; }
    __device__ static RxSO3 Exp(const S* a) { return {so3_exp_q(a), exp(a[3])}; }
    __device__ void Log(S* a) const {
        so3_log(q, a);
        a[3] = log(s);
    }
    __device__ RxSO3 inv() const { return {Quat<S>{-q.x, -q.y, -q.z, q.w}, S(1) / s}; }
    __device__ RxSO3 operator*(const RxSO3& o) const { return {qnormalize(qmul(q, o.q)), s * o.s}; }
    __device__ void act(const S* p, S* o) const {
        qrot(q, p, o);
        o[0] *= s; o[1] *= s; o[2] *= s;
    }
    __device__ void act4(const S* p, S* o) const { act(p, o); o[3] = p[3]; }
    __device__ Mat<S, K, K> Adj() const {
        Mat<S, K, K> A = eye<S, K>();
        set_block(A, 0, 0, qmat(q));
        return A;
    }
    __device__ static Mat<S, K, K> adj(const S* a) {
        Mat<S, K, K> A = zeros<S, K, K>();
        set_block(A, 0, 0, hat(a));
        return A;
    }
    __device__ Mat<S, 3, 3> mat3() const {
        Mat<S, 3, 3> R = qmat(q);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) R.m[r][c] *= s;
        return R;
    }
    __device__ Mat<S, 4, 4> mat4() const {
        Mat<S, 4, 4> T = eye<S, 4>();
        set_block(T, 0, 0, mat3());
        return T;
    }
    __device__ Mat<S, N, N> projector() const {
        Mat<S, N, N> J = zeros<S, N, N>();
        quat_projector(q, J, 0);
        J.m[4][3] = s;
        return J;
    }
    __device__ static Mat<S, K, K> left_jac(const S* a) {
        Mat<S, K, K> J = eye<S, K>();
        set_block(J, 0, 0, so3_left_jac(a));
        return J;
    }
    __device__ static Mat<S, K, K> left_jac_inv(const S* a) {
        Mat<S, K, K> J = eye<S, K>();
        set_block(J, 0, 0, so3_left_jac_inv(a));
        return J;
    }
    __device__ static Mat<S, 3, K> act_jac(const S* p) {
        Mat<S, 3, K> J;
        const S m[3] = {-p[0], -p[1], -p[2]};
        const Mat<S, 3, 3> H = hat(m);
#pragma unroll
        for (int r = 0; r < 3; r++) {
#pragma unroll
            for (int c = 0; c < 3; c++) J.m[r][c] = H.m[r][c];
            J.m[r][3] = p[r];
        }
        return J;
    }
    __device__ static Mat<S, 4, K> act4_jac(const S* p) {
        Mat<S, 4, K> J = zeros<S, 4, K>();
        const S m[3] = {-p[0], -p[1], -p[2]};
        const Mat<S, 3, 3> H = hat(m);
#pragma unroll
        for (int r = 0; r < 3; r++) {
#pragma unroll
            for (int c = 0; c < 3; c++) J.m[r][c] = H.m[r][c];
            J.m[r][3] = p[r];
        }
        return J;
    }
    // W(phi, sigma): translation map of the Sim3 exponential (left Jacobian of
    // the scaled rotation acting on translations), closed form by cases of
    // small rotation / small scale.
    __device__ static Mat<S, 3, 3> calcW(const S* a) {
        const S sig = a[3];
        const S th = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        const Mat<S, 3, 3> P = hat(a);
        const Mat<S, 3, 3> P2 = mm(P, P);
        const S sc = exp(sig);
        S A, B, C;
        if (fabs(sig) < S(kEps)) {
            C = S(1);
            if (fabs(th) < S(kEps)) {
                A = S(0.5);
                B = S(1.0 / 6.0);
            } else {
                const S t2 = th * th;
                A = (S(1) - cos(th)) / t2;
                B = (th - sin(th)) / (t2 * th);
            }
        } else {
            C = (sc - S(1)) / sig;
            if (fabs(th) < S(kEps)) {
                const S s2 = sig * sig;
                A = ((sig - S(1)) * sc + S(1)) / s2;
                B = (sc * S(0.5) * s2 + sc - S(1) - sig * sc) / (s2 * sig);
            } else {
                const S t2 = th * th;
                const S sa = sc * sin(th);
                const S sb = sc * cos(th);
                const S cc = t2 + sig * sig;
                A = (sa * sig + (S(1) - sb) * th) / (th * cc);
                B = (C - ((sb - S(1)) * sig + sa * th) / cc) / t2;
            }
        }
        return add(add(add(zeros<S, 3, 3>(), P, A), P2, B), eye<S, 3>(), C);
    }
};

template <typename S>
struct SE3 {
    static constexpr int N = 7, K = 6;
    SO3<S> r;
    S t[3];
    __device__ static SE3 load(const S* d) {
        SE3 g;
        g.t[0] = d[0]; g.t[1] = d[1]; g.t[2] = d[2];
        g.r = SO3<S>::load(d + 3);
        return g;
    }
    __device__ void store(S* d) const {
        d[0] = t[0]; d[1] = t[1]; d[2] = t[2];
        r.store(d + 3);
    }
    __device__ static SE3 Exp(const S* a) {
        SE3 g;
        g.r = SO3<S>::Exp(a + 3);
        mv(so3_left_jac(a + 3), a, g.t);
        return g;
    }
    __device__ void Log(S* a) const {
        r.Log(a + 3);
        mv(so3_left_jac_inv(a + 3), t, a);
    }
    __device__ SE3 inv() const {
        SE3 g;
        g.r = r.inv();
        S o[3];
        g.r.act(t, o);
        g.t[0] = -o[0]; g.t[1] = -o[1]; g.t[2] = -o[2];
        return g;
    }
    __device__ SE3 operator*(const SE3& o) const {
        SE3 g;
        g.r = r * o.r;
        S p[3];
        r.act(o.t, p);
        g.t[0] = t[0] + p[0]; g.t[1] = t[1] + p[1]; g.t[2] = t[2] + p[2];
        return g;
    }
    __device__ void act(const S* p, S* o) const {
        r.act(p, o);
        o[0] += t[0]; o[1] += t[1]; o[2] += t[2];
    }
    __device__ void act4(const S* p, S* o) const {
        r.act(p, o);
        o[0] += t[0] * p[3]; o[1] += t[1] * p[3]; o[2] += t[2] * p[3];
        o[3] = p[3];
    }
    __device__ Mat<S, K, K> Adj() const {
        const Mat<S, 3, 3> R = r.mat3();
        const Mat<S, 3, 3> TR = mm(hat(t), R);
        Mat<S, K, K> A = zeros<S, K, K>();
        set_block(A, 0, 0, R);
        set_block(A, 0, 3, TR);
        set_block(A, 3, 3, R);
        return A;
    }
    __device__ static Mat<S, K, K> adj(const S* a) {
        Mat<S, K, K> A = zeros<S, K, K>();
        const Mat<S, 3, 3> P = hat(a + 3), T = hat(a);
        set_block(A, 0, 0, P);
        set_block(A, 0, 3, T);
        set_block(A, 3, 3, P);
        return A;
    }
    __device__ Mat<S, 3, 3> mat3() const { return r.mat3(); }
    __device__ Mat<S, 4, 4> mat4() const {
        Mat<S, 4, 4> T = eye<S, 4>();
        set_block(T, 0, 0, r.mat3());
        T.m[0][3] = t[0]; T.m[1][3] = t[1]; T.m[2][3] = t[2];
        return T;
    }
    __device__ Mat<S, N, N> projector() const {
        Mat<S, N, N> J = zeros<S, N, N>();
        const S m[3] = {-t[0], -t[1], -t[2]};
        set_block(J, 0, 0, eye<S, 3>());
        set_block(J, 0, 3, hat(m));
        quat_projector(r.q, J, 3);
        return J;
    }
    // Q block of the SE3 left Jacobian
    __device__ static Mat<S, 3, 3> calcQ(const S* a) {
        const Mat<S, 3, 3> T = hat(a), P = hat(a + 3);
        const S th = sqrt(a[3] * a[3] + a[4] * a[4] + a[5] * a[5]);
        const S t2 = th * th, t4 = t2 * t2;
        const S c1 = (th < S(kEps)) ? S(1.0 / 6.0) - S(1.0 / 120.0) * t2 : (th - sin(th)) / (t2 * th);
        const S c2 = (th < S(kEps)) ? S(1.0 / 24.0) - S(1.0 / 720.0) * t2 : (t2 + S(2) * cos(th) - S(2)) / (S(2) * t4);
        const S c3 = (th < S(kEps)) ? S(1.0 / 120.0) - S(1.0 / 2520.0) * t2
                                    : (S(2) * th - S(3) * sin(th) + th * cos(th)) / (S(2) * t4 * th);
        const Mat<S, 3, 3> PT = mm(P, T), TP = mm(T, P), PTP = mm(PT, P), PPT = mm(P, PT), TPP = mm(TP, P);
        const Mat<S, 3, 3> PTPP = mm(PTP, P), PPTP = mm(P, PTP);
        Mat<S, 3, 3> Q;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                Q.m[i][j] = S(0.5) * T.m[i][j] + c1 * (PT.m[i][j] + TP.m[i][j] + PTP.m[i][j]) +
                            c2 * (PPT.m[i][j] + TPP.m[i][j] - S(3) * PTP.m[i][j]) +
                            c3 * (PTPP.m[i][j] + PPTP.m[i][j]);
        return Q;
    }
    __device__ static Mat<S, K, K> left_jac(const S* a) {
        const Mat<S, 3, 3> J = so3_left_jac(a + 3);
        Mat<S, K, K> O = zeros<S, K, K>();
        set_block(O, 0, 0, J);
        set_block(O, 0, 3, calcQ(a));
        set_block(O, 3, 3, J);
        return O;
    }
    __device__ static Mat<S, K, K> left_jac_inv(const S* a) {
        const Mat<S, 3, 3> Ji = so3_left_jac_inv(a + 3);
        const Mat<S, 3, 3> Q = calcQ(a);
        const Mat<S, 3, 3> M = mm(mm(Ji, Q), Ji);
        Mat<S, K, K> O = zeros<S, K, K>();
        set_block(O, 0, 0, Ji);
        set_block(O, 0, 3, M, S(-1));
        set_block(O, 3, 3, Ji);
        return O;
    }
    __device__ static Mat<S, 3, K> act_jac(const S* p) {
        Mat<S, 3, K> J;
        const S m[3] = {-p[0], -p[1], -p[2]};
        const Mat<S, 3, 3> H = hat(m);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                J.m[r][c] = (r == c) ? S(1) : S(0);
                J.m[r][3 + c] = H.m[r][c];
            }
        return J;
    }
    __device__ static Mat<S, 4, K> act4_jac(const S* p) {
        Mat<S, 4, K> J = zeros<S, 4, K>();
        const S m[3] = {-p[0], -p[1], -p[2]};
        const Mat<S, 3, 3> H = hat(m);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                J.m[r][c] = (r == c) ? p[3] : S(0);
                J.m[r][3 + c] = H.m[r][c];
            }
        return J;
    }
};

template <typename S>
struct Sim3 {
    static constexpr int N = 8, K = 7;
    RxSO3<S> r;
    S t[3];
    __device__ static Sim3 load(const S* d) {
        Sim3 g;
        g.t[0] = d[0]; g.t[1] = d[1]; g.t[2] = d[2];
        g.r = RxSO3<S>::load(d + 3);
        return g;
    }
    __device__ void store(S* d) const {
        d[0] = t[0]; d[1] = t[1]; d[2] = t[2];
        r.store(d + 3);
    }
    __device__ static Sim3 Exp(const S* a) {
        Sim3 g;
        g.r = RxSO3<S>::Exp(a + 3);
        mv(RxSO3<S>::calcW(a + 3), a, g.t);
        return g;
    }
    __device__ void Log(S* a) const {
        r.Log(a + 3);
        const Mat<S, 3, 3> W = RxSO3<S>::calcW(a + 3);
        // solve W tau = t (3x3 inverse by cofactors)
        const S c00 = W.m[1][1] * W.m[2][2] - W.m[1][2] * W.m[2][1];
        const S c01 = W.m[1][2] * W.m[2][0] - W.m[1][0] * W.m[2][2];
        const S c02 = W.m[1][0] * W.m[2][1] - W.m[1][1] * W.m[2][0];
        const S det = W.m[0][0] * c00 + W.m[0][1] * c01 + W.m[0][2] * c02;
        Mat<S, 3, 3> Wi;
        Wi.m[0][0] = c00 / det;
        Wi.m[1][0] = c01 / det;
        Wi.m[2][0] = c02 / det;
        Wi.m[0][1] = (W.m[0][2] * W.m[2][1] - W.m[0][1] * W.m[2][2]) / det;
        Wi.m[1][1] = (W.m[0][0] * W.m[2][2] - W.m[0][2] * W.m[2][0]) / det;
        Wi.m[2][1] = (W.m[0][1] * W.m[2][0] - W.m[0][0] * W.m[2][1]) / det;
        Wi.m[0][2] = (W.m[0][1] * W.m[1][2] - W.m[0][2] * W.m[1][1]) / det;
        Wi.m[1][2] = (W.m[0][2] * W.m[1][0] - W.m[0][0] * W.m[1][2]) / det;
        Wi.m[2][2] = (W.m[0][0] * W.m[1][1] - W.m[0][1] * W.m[1][0]) / det;
        mv(Wi, t, a);
    }
    __device__ Sim3 inv() const {
        Sim3 g;
        g.r = r.inv();
        S o[3];
        g.r.act(t, o);
        g.t[0] = -o[0]; g.t[1] = -o[1]; g.t[2] = -o[2];
        return g;
    }
    __device__ Sim3 operator*(const Sim3& o) const {
        Sim3 g;
        g.r = r * o.r;
        S p[3];
        r.act(o.t, p);
        g.t[0] = t[0] + p[0]; g.t[1] = t[1] + p[1]; g.t[2] = t[2] + p[2];
        return g;
    }
    __device__ void act(const S* p, S* o) const {
        r.act(p, o);
        o[0] += t[0]; o[1] += t[1]; o[2] += t[2];
    }
    __device__ void act4(const S* p, S* o) const {
        r.act(p, o);
        o[0] += p[3] * t[0]; o[1] += p[3] * t[1]; o[2] += p[3] * t[2];
        o[3] = p[3];
    }
    __device__ Mat<S, K, K> Adj() const {
        Mat<S, K, K> A = eye<S, K>();
        const Mat<S, 3, 3> R = qmat(r.q);
        set_block(A, 0, 0, r.mat3());
        set_block(A, 0, 3, mm(hat(t), R));
        A.m[0][6] = -t[0]; A.m[1][6] = -t[1]; A.m[2][6] = -t[2];
        set_block(A, 3, 3, R);
        return A;
    }
    __device__ static Mat<S, K, K> adj(const S* a) {
        Mat<S, K, K> A = zeros<S, K, K>();
        const Mat<S, 3, 3> P = hat(a + 3), T = hat(a);
        set_block(A, 0, 0, add(P, eye<S, 3>(), a[6]));
        set_block(A, 0, 3, T);
        A.m[0][6] = -a[0]; A.m[1][6] = -a[1]; A.m[2][6] = -a[2];
        set_block(A, 3, 3, P);
        return A;
    }
    __device__ Mat<S, 3, 3> mat3() const { return r.mat3(); }
    __device__ Mat<S, 4, 4> mat4() const {
        Mat<S, 4, 4> T = eye<S, 4>();
        set_block(T, 0, 0, r.mat3());
        T.m[0][3] = t[0]; T.m[1][3] = t[1]; T.m[2][3] = t[2];
        return T;
    }
    __device__ Mat<S, N, N> projector() const {
        Mat<S, N, N> J = zeros<S, N, N>();
        const S m[3] = {-t[0], -t[1], -t[2]};
        set_block(J, 0, 0, eye<S, 3>());
        set_block(J, 0, 3, hat(m));
        J.m[0][6] = t[0]; J.m[1][6] = t[1]; J.m[2][6] = t[2];
        quat_projector(r.q, J, 3);
        J.m[7][6] = r.s;
        return J;
    }
    // left Jacobian as the ad-series truncated after the fourth power
    __device__ static Mat<S, K, K> left_jac(const S* a) {
        const Mat<S, K, K> X = adj(a);
        const Mat<S, K, K> X2 = mm(X, X);
        const Mat<S, K, K> X3 = mm(X, X2);
        const Mat<S, K, K> X4 = mm(X2, X2);
        Mat<S, K, K> O = eye<S, K>();
        O = add(O, X, S(1.0 / 2.0));
        O = add(O, X2, S(1.0 / 6.0));
        O = add(O, X3, S(1.0 / 24.0));
        O = add(O, X4, S(1.0 / 120.0));
        return O;
    }
    __device__ static Mat<S, K, K> left_jac_inv(const S* a) {
        const Mat<S, K, K> X = adj(a);
        const Mat<S, K, K> X2 = mm(X, X);
        const Mat<S, K, K> X4 = mm(X2, X2);
        Mat<S, K, K> O = eye<S, K>();
        O = add(O, X, S(-1.0 / 2.0));
        O = add(O, X2, S(1.0 / 12.0));
        O = add(O, X4, S(-1.0 / 720.0));
        return O;
    }
    __device__ static Mat<S, 3, K> act_jac(const S* p) {
        Mat<S, 3, K> J;
        const S m[3] = {-p[0], -p[1], -p[2]};
        const Mat<S, 3, 3> H = hat(m);
#pragma unroll
        for (int r = 0; r < 3; r++) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                J.m[r][c] = (r == c) ? S(1) : S(0);
                J.m[r][3 + c] = H.m[r][c];
            }
            J.m[r][6] = p[r];
        }
        return J;
    }
    __device__ static Mat<S, 4, K> act4_jac(const S* p) {
        Mat<S, 4, K> J = zeros<S, 4, K>();
        const S m[3] = {-p[0], -p[1], -p[2]};
        const Mat<S, 3, 3> H = hat(m);
#pragma unroll
        for (int r = 0; r < 3; r++) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                J.m[r][c] = (r == c) ? p[3] : S(0);
                J.m[r][3 + c] = H.m[r][c];
            }
            J.m[r][6] = p[r];
        }
        return J;
    }
};

// ---------------------------------------------------------------- kernels

#define LIE_LOOP(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)blockDim.x * gridDim.x)

enum Op {
    kExp, kExpB, kLog, kLogB, kInv, kInvB, kMul, kMulB, kAdj, kAdjB, kAdjT, kAdjTB, kAct, kActB, kAct4, kAct4B,
    kMatrix, kProj, kJinv
};

}  // namespace lie
}  // namespace vipe
