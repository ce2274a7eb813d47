// Hand-written adjoint of the dense bundle adjustment (no counterpart in the
// reference, which has no BA backward: vipe csrc/slam_ext/slam.cpp binds only
// forward entry points).
//
// The forward LM step at state x_k = (poses T, inverse depths d) is
//   y   = v - E Q w_z,      S' = B - E Q E^T + D,     S' dxi = y,
//   dz  = Q (w_z - E~^T dxi)                 (E~: E without pose t0's rows,
//                                             the reference's back-substitution,
//                                             geom_kernels.cu:1186)
//   T  <- Exp(dxi) T,   d <- d + dz,
// with B, v, E, C = 1/Q, w_z sums over edge pixels of the reprojection
// Jacobians (geom_kernels.cu:178-524) and D = ep + lm diag(S) the LM damping.
// Going backwards through the iterations (states re-read from the forward's
// tape, Jacobians recomputed, never stored):
//
//   g_dxi = J_l(dxi)^T g_T,   g_T <- Ad(Exp dxi)^T g_T          (retraction)
//   a     = Q g_dz                                               (g_dz = g_d)
//   lam   = S'^-1 (g_dxi - E~ a)          (the same reduced system, re-solved)
//   mu    = Q E^T lam,  dzf = Q (w_z - E^T dxi),  L = lm lam o dxi (damping)
//   g_wz  = a - mu,     g_C = mu dzf - a dz - Q^2 sum_a L_a E_a^2,
//   g_E   = -dzf lam + mu dxi - a dxi~ + 2 Q L o E,
//   g_v   = lam,        g_B = -lam dxi^T - diag(L)
//
// Every remaining dependence is a sum over (edge, pixel) of a scalar phi of the
// Jacobian rows J_c, the depth Jacobian Jz_c and the residual r_c, with the
// adjoint quantities held fixed; its gradient gives the targets and weights
// directly, and with respect to the two poses and the pixel's depth it needs the
// derivatives of Jacobian-vector products J.v.  Those are taken exactly: the
// transformed point is X' = Tij X with X = (x, y, 1, d); a left perturbation
// s A of the target pose (s B of the source pose) moves it by Ps = A X'
// (-Tij B X), and J.v along a tangent v = (v_i, v_j) is grad f . (v_j X' -
// Tij v_i X).  Their mixed derivative splits, for every direction v, into
//   Ps . (h_v + grad f x v_j,phi) + e_phi . [target: -(Y_v x grad f); source: R^T (Y_v x grad f)]
// with Y_v = R (v_i,tau d + v_i,phi x X3) and h_v from the projection's second
// derivative.  So per edge the pixels only accumulate G0 = sum g X^T (3x4) and
// one 3-vector for the rotation dofs, contracted with Ps per pose direction
// once per edge; the per-pixel directions of the damping terms fit the same form.
//
// Sim3 (D = 7, tangent [tau, phi, sigma], X' = s R X3 + t d): the generator of sigma moves P by
// sigma P (target pose) or -s R sigma X3 (source pose), so the directions gain
// Pt_v += v_j,sigma P and Y_v = s R (v_i,tau W + v_i,phi x X3 + v_i,sigma X3), the Ps
// coefficient gains v_j,sigma grad f, and the scale dofs take one more per-edge moment,
// os = sum Y_v . grad f (target: -os, source: +os), beside G0 and the rotation vector (whose
// source rows use the pure rotation R of s R).  Every kernel below is written for D = 6 and 7.

// Precision: the per-pixel work is FP32 like the forward; the re-solve and every
// pose-level sum are FP64.

#include "ba_internal.cuh"
#include "se3_device.cuh"

namespace vipe {
namespace ba {

constexpr int kAdjThreads = 256;
constexpr int kAdjMaxDeg = 64;       // edges leaving one depth frame

// ---------------------------------------------------------------- small helpers

__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// v <- ad(xi)^T v.  SE3, xi = (tau, phi): (-phi x v_tau, -tau x v_tau - phi x v_phi).
// Sim3, xi = (tau, phi, sigma), ad(xi) = [[phi x + sigma I, tau x, -tau], [0, phi x, 0], [0, 0, 0]]:
// (-phi x v_tau + sigma v_tau, -tau x v_tau - phi x v_phi, -tau . v_tau).
template <int D>
__device__ __forceinline__ void adT_apply(const double* xi, double* v) {
    if constexpr (D == 7) {
        const double vs = -(xi[0] * v[0] + xi[1] * v[1] + xi[2] * v[2]);
        double a[3], b[3], c[3];
        cross3(xi + 3, v, a);
        cross3(xi, v, b);
        cross3(xi + 3, v + 3, c);
        for (int n = 0; n < 3; n++) {
            v[3 + n] = -b[n] - c[n];
            v[n] = -a[n] + xi[6] * v[n];
        }
        v[6] = vs;
        return;
    }
    double a[3], b[3], c[3];
    cross3(xi + 3, v, a);
    cross3(xi, v, b);
    cross3(xi + 3, v + 3, c);
    for (int n = 0; n < 3; n++) {
        v[n] = -a[n];
        v[3 + n] = -b[n] - c[n];
    }
}

// 4x4 homogeneous matrices (row-major, double)
struct M4 {
    double m[16];
};

__device__ __forceinline__ M4 mzero() {
    M4 z;
    for (int q = 0; q < 16; q++) z.m[q] = 0.0;
    return z;
}

__device__ __forceinline__ M4 mmul(const M4& a, const M4& b) {
    M4 c;
    for (int r = 0; r < 4; r++)
        for (int k = 0; k < 4; k++) {
            double s = 0.0;
            for (int j = 0; j < 4; j++) s += a.m[4 * r + j] * b.m[4 * j + k];
            c.m[4 * r + k] = s;
        }
    return c;
}

__device__ __forceinline__ M4 madd(const M4& a, const M4& b, double sb) {
    M4 c;
    for (int q = 0; q < 16; q++) c.m[q] = a.m[q] + sb * b.m[q];
    return c;
}

// se3 generator of xi = (tau, phi): [[phi x, tau], [0, 0]]
__device__ __forceinline__ M4 hat(const double* xi) {
    M4 h = mzero();
    h.m[1] = -xi[5];
    h.m[2] = xi[4];
    h.m[4] = xi[5];
    h.m[6] = -xi[3];
    h.m[8] = -xi[4];
    h.m[9] = xi[3];
    h.m[3] = xi[0];
    h.m[7] = xi[1];
    h.m[11] = xi[2];
    return h;
}

__device__ __forceinline__ void quat_to_rot(const double* q, double* R) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    R[0] = 1 - 2 * (y * y + z * z);
    R[1] = 2 * (x * y - w * z);
    R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);
    R[4] = 1 - 2 * (x * x + z * z);
    R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);
    R[7] = 2 * (y * z + w * x);
    R[8] = 1 - 2 * (x * x + y * y);
}

// Tij = Tj Ti^-1 as a 4x4 [s R | t] (SE3: s = 1; stereo edges: the fixed baseline (-0.1, 0, 0))
template <int D>
__device__ M4 edge_matrix(const float* poses, int a, int b) {
    float tij[3], qij[4], sij = 1.f;
    if constexpr (D == 6) {
        edge_pose(poses, a, b, tij, qij);
    } else {
        EdgeTf T;
        edge_tf<7>(poses, a, b, T);
        for (int n = 0; n < 3; n++) tij[n] = T.t[n];
        for (int n = 0; n < 4; n++) qij[n] = T.q[n];
        sij = T.s;
    }
    const double q[4] = {qij[0], qij[1], qij[2], qij[3]};
    double R[9];
    quat_to_rot(q, R);
    M4 T;
    for (int r = 0; r < 3; r++) {
        for (int c = 0; c < 3; c++) T.m[4 * r + c] = (D == 6) ? R[3 * r + c] : (double)sij * R[3 * r + c];
        T.m[4 * r + 3] = tij[r];
    }
    T.m[12] = T.m[13] = T.m[14] = 0.0;
    T.m[15] = 1.0;
    return T;
}

// the edge's 2D-vector [source pose, target pose] of a window-pose field (zero
// for poses outside the window; drop_t0 also zeroes pose t0)
template <int D, typename Tin>
__device__ __forceinline__ void edge_dir(const Tin* field, int ia, int ib, int t0, int P, bool drop_t0, double* v) {
    for (int n = 0; n < 2 * D; n++) v[n] = 0.0;
    const int la = ia - t0, lb = ib - t0;
    if (la >= 0 && la < P && !(drop_t0 && la == 0))
        for (int n = 0; n < D; n++) v[n] = (double)field[D * la + n];
    if (lb >= 0 && lb < P && !(drop_t0 && lb == 0))
        for (int n = 0; n < D; n++) v[D + n] = (double)field[D * lb + n];
}

// y = Ad(Tij) x in FP64 from the edge's 4x4 [s R | t] (s recovered as |column 0|):
// SE3 [[R, [t]x R], [0, R]];  Sim3 [[s R, [t]x R, -t], [0, R, 0], [0, 0, 1]]
template <int D>
__device__ __forceinline__ void ad_apply_m4(const M4& T, const double* x, double* y) {
    const double s = (D == 6) ? 1.0 : sqrt(T.m[0] * T.m[0] + T.m[4] * T.m[4] + T.m[8] * T.m[8]);
    double rt[3], rp[3];
    for (int r = 0; r < 3; r++) {
        rt[r] = T.m[4 * r] * x[0] + T.m[4 * r + 1] * x[1] + T.m[4 * r + 2] * x[2];  // s R x_tau
        rp[r] = (T.m[4 * r] * x[3] + T.m[4 * r + 1] * x[4] + T.m[4 * r + 2] * x[5]) / s;  // R x_phi
    }
    const double t[3] = {T.m[3], T.m[7], T.m[11]};
    double tx[3];
    cross3(t, rp, tx);
    for (int r = 0; r < 3; r++) {
        y[r] = rt[r] + tx[r];
        y[3 + r] = rp[r];
    }
    if constexpr (D == 7) {
        for (int r = 0; r < 3; r++) y[r] -= t[r] * x[6];
        y[6] = x[6];
    }
}

// row r of the 3x4 matrix M times X = (x, y, 1, d)
__device__ __forceinline__ float mrow(const float* M, int r, const float* X) {
    return M[4 * r] * X[0] + M[4 * r + 1] * X[1] + M[4 * r + 2] + M[4 * r + 3] * X[3];
}

// ---------------------------------------------------------------- kernels

// gT <- incoming pose gradients (left tangent, lietorch layout: SE3 (N, 7) with [6] unused,
// Sim3 (N, 8) with [7] unused)
__global__ void ba_adj_init_kernel(BAPtrs base, Batch B) {
    BA_BIND(B, base);
    const int D = d.dof;
    for (int q = threadIdx.x; q < d.N * D; q += blockDim.x)
        w.adj_gT[q] = (double)io.g_poses[(q / D) * (D + 1) + q % D];
}

// retraction T' = Exp(dxi) T:  g_dxi = J_l(dxi)^T g_T',  g_T = Ad(Exp dxi)^T g_T'
// with J_l = sum ad^n/(n+1)!, Ad(Exp) = sum ad^n/n! (series in FP64).
template <int D>
__global__ void ba_adj_prep_kernel(BAPtrs base, Batch B) {
    BA_BIND(B, base);
    if (w.status[0]) return;
    for (int a = threadIdx.x; a < d.P; a += blockDim.x) {
        double xi[D], term[D], adacc[D], jl[D];
        for (int n = 0; n < D; n++) xi[n] = (double)io.dx[D * a + n];
        double* g = w.adj_gT + (size_t)(d.t0 + a) * D;
        for (int n = 0; n < D; n++) {
            term[n] = g[n];
            adacc[n] = g[n];
            jl[n] = g[n];
        }
        double c = 1.0;  // 1/k!
        for (int k = 1; k <= 30; k++) {
            adT_apply<D>(xi, term);
            c /= k;
            double mx = 0.0;
            for (int n = 0; n < D; n++) {
                adacc[n] += c * term[n];
                jl[n] += c / (k + 1) * term[n];
                mx = fmax(mx, fabs(term[n]));
            }
            if (mx * c < 1e-30) break;
        }
        for (int n = 0; n < D; n++) {
            w.adj_rhs[D * a + n] = jl[n];
            g[n] = adacc[n];
        }
    }
}

// per (depth frame, pixel chunk): first the per-pixel Q = 1/C and w of the
// forward step (read from the tape, where the forward frame kernel recorded
// them, and stored for ba_adj_frame_b_kernel), then for each edge leaving the
// frame the 12 sums  sum_p a_p act wd_c Jz_c [Ji_c, Jj_c],  a_p = Q_p g_d(p).
// 6 CTAs per SM (40 registers): latency-bound, 8.3 vs 9.0 ms per 256-clip step at 4
// Sim3 target-pose rows of one pixel (tau: d grad f, phi: P x grad f, sigma: grad f . P) with
// the forward's mask and weight scale: acc += a act wd Jz Jj per channel
__device__ __forceinline__ void sim3_target_sums(const EdgeTf& T, float fx, float fy, float cx, float cy, float u,
                                                 float v, float disp, float w0, float w1, float act, float a,
                                                 float* acc) {
    const float X3[3] = {(u - cx) / fx, (v - cy) / fy, 1.0f};
    float RX[3];
    qrot(T.q, X3, RX);
    const float P[3] = {T.s * RX[0] + T.t[0] * disp, T.s * RX[1] + T.t[1] * disp, T.s * RX[2] + T.t[2] * disp};
    if (P[2] < 0.25f) return;
    const float iz = 1.0f / P[2];
    const float wc[2] = {0.001f * w0, 0.001f * w1};
#pragma unroll
    for (int ch = 0; ch < 2; ch++) {
        const float g[3] = {ch == 0 ? fx * iz : 0.f, ch == 0 ? 0.f : fy * iz,
                            ch == 0 ? -fx * P[0] * iz * iz : -fy * P[1] * iz * iz};
        const float jz = g[0] * T.t[0] + g[1] * T.t[1] + g[2] * T.t[2];
        const float c = a * act * (wc[ch] * act) * jz;
        acc[0] += c * disp * g[0];
        acc[1] += c * disp * g[1];
        acc[2] += c * disp * g[2];
        acc[3] += c * (P[1] * g[2] - P[2] * g[1]);
        acc[4] += c * (P[2] * g[0] - P[0] * g[2]);
        acc[5] += c * (P[0] * g[1] - P[1] * g[0]);
        acc[6] += c * (g[0] * P[0] + g[1] * P[1] + g[2] * P[2]);
    }
}

// o = Ad(Tij)^T y (a target-pose row pulled back to the source pose, up to sign):
// SE3 (R^T y_tau, R^T (y_phi + y_tau x t)); Sim3 adds s to the first and -t . y_tau + y_sigma
template <int D>
__device__ __forceinline__ void adT_tf(const EdgeTf& T, const float* y, float* o) {
    const float qc[4] = {-T.q[0], -T.q[1], -T.q[2], T.q[3]};
    const float yt[3] = {y[0], y[1], y[2]};
    const float u[3] = {y[3] + (y[1] * T.t[2] - y[2] * T.t[1]), y[4] + (y[2] * T.t[0] - y[0] * T.t[2]),
                        y[5] + (y[0] * T.t[1] - y[1] * T.t[0])};
    qrot(qc, yt, o);
    qrot(qc, u, o + 3);
    if constexpr (D == 7) {
        o[0] *= T.s;
        o[1] *= T.s;
        o[2] *= T.s;
        o[6] = y[6] - (T.t[0] * y[0] + T.t[1] * y[1] + T.t[2] * y[2]);
    }
}

template <int D>
__global__ void __launch_bounds__(kAdjThreads, 6) ba_adj_frame_a_kernel(BAPtrs base, Batch B, float alpha) {
    BA_BIND(B, base);
    if (w.status[0]) return;
    __shared__ float red[kAdjThreads / 32][12];
    __shared__ float pa[kAdjMaxChunk];
    const int s = local_ % d.K, c = local_ / d.K, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int HW = d.HW, W = d.W;
    const int k = w.kx[s];
    const float act = io.depth_active[k];
    const float fx = io.intr[0], fy = io.intr[1], cx = io.intr[2], cy = io.intr[3];
    const int p0 = c * d.chunk_f, p1 = min(HW, p0 + d.chunk_f);
    if (d.chunk_f > kAdjMaxChunk) {
        if (tid == 0) atomicOr(w.status, VIPE_ERR_CAPACITY);
        return;
    }
    const int eb = w.fe_ptr[s], ee = w.fe_ptr[s + 1];
    // (Q, w) of the forward step, as its frame kernel recorded them in the tape
    const float2* qt = tape_qw(io.ftape, d);
    for (int p = p0 + tid; p < p1; p += kAdjThreads) {
        const float2 qw2 = qt[(size_t)s * HW + p];
        float* qw = w.qwf + ((size_t)s * HW + p) * 3;
        qw[0] = qw2.x;
        qw[1] = qw2.y;
        pa[p - p0] = qw2.x * io.g_disps[(size_t)k * HW + p];
    }
    __syncthreads();
    for (int q = eb; q < ee; q++) {
        const int e = w.fe_list[q];
        const int b = (int)io.jj[e];
        EdgeTf Tf;
        edge_tf<D>(io.poses, k, b, Tf);
        // source rows are -Ad^T(Tij) of the target rows, so only the target-pose sums
        // are accumulated per pixel; the source half follows once per edge
        float acc[D];
#pragma unroll
        for (int n = 0; n < D; n++) acc[n] = 0.f;
        if (act != 0.f) {
            const float* wp = io.weights + (size_t)e * 2 * HW;
            for (int p = p0 + tid; p < p1; p += kAdjThreads) {
                const float u = (float)(p % W), v = (float)(p / W);
                const float disp = io.disps[(size_t)k * HW + p];
                const float a = pa[p - p0];
                if constexpr (D == 6) {
                    PixelLin L;
                    linearize<false, false>(Tf.t, Tf.q, k == b, fx, fy, cx, cy, u, v, disp, __ldg(wp + p),
                                            __ldg(wp + HW + p), 0.f, 0.f, act, 1.f, L);
#pragma unroll
                    for (int ch = 0; ch < 2; ch++) {
                        const float g = a * act * L.wd[ch] * L.Jz[ch];
#pragma unroll
                        for (int n = 0; n < 6; n++) acc[n] += g * L.Jj[ch][n];
                    }
                } else {
                    sim3_target_sums(Tf, fx, fy, cx, cy, u, v, disp, __ldg(wp + p), __ldg(wp + HW + p), act, a, acc);
                }
            }
        }
#pragma unroll
        for (int n = 0; n < D; n++) {
            const float sv = warp_sum(acc[n]);
            if (lane == 0) red[warp][n] = sv;
        }
        __syncthreads();
        if (tid == 0) {
            float sj[D], si[D];
            for (int n = 0; n < D; n++) {
                float sv = 0.f;
                for (int r = 0; r < kAdjThreads / 32; r++) sv += red[r][n];
                sj[n] = sv;
            }
            adT_tf<D>(Tf, sj, si);
            float* o = w.adj_aslot + ((size_t)e * d.CF + c) * 2 * D;
            for (int n = 0; n < D; n++) {
                o[n] = -si[n];
                o[D + n] = sj[n];
            }
        }
        __syncthreads();
    }
}

// rhs = g_dxi - E~ a per window pose (pose t0 keeps g_dxi: E~ has no rows for it)
__global__ void ba_adj_rhs_kernel(BAPtrs base, Batch B) {
    BA_BIND(B, base);
    if (w.status[0]) return;
    const int D = d.dof;
    for (int q = threadIdx.x; q < D * d.P; q += blockDim.x) {
        const int a = q / D, n = q % D;
        if (a == 0) continue;
        double sub = 0.0;
        for (int r = w.pe_ptr[a]; r < w.pe_ptr[a + 1]; r++) {
            const int ent = w.pe_list[r];
            const int e = ent >> 2, fl = ent & 3;
            for (int c = 0; c < d.CF; c++) {
                const float* src = w.adj_aslot + ((size_t)e * d.CF + c) * 2 * D;
                if (fl & 1) sub += (double)src[n];
                if (fl & 2) sub += (double)src[D + n];
            }
        }
        w.adj_rhs[q] -= sub;
    }
}

// Jacobian rows of one pixel of one edge from the edge's 3x4 transform M0 =
// [s R | t] (SE3: s = 1; same values as the reference formulas, geom_kernels.cu:338-350):
//   target pose:  tau_n: grad f . e_n W        phi_n: e_n . (P x grad f)     (Sim3 sigma: grad f . P)
//   source pose:  tau_n: -W (M^T grad f)_n     phi_n: -e_n . (X3 x M^T grad f) (Sim3 sigma: -X3 . M^T grad f)
// with P = M0 X, W = d, grad f the projection gradient on P, M the 3x3 part of M0.
template <int D>
struct PixJ {
    float P[3];
    float iz;
    float gf[2][3];
    float rg[2][3];     // M^T grad f per channel
    float x0, x1, w;    // the pixel's ray (x0, x1, 1) and inverse depth
    float jz[2];
};

// element n of channel ch's Jacobian row [source D | target D], formed from the stored
// gradient (the rows are cheap to re-form; holding all 4D of them costs registers)
template <int D>
__device__ __forceinline__ float jrow(const PixJ<D>& o, int ch, int n) {
    const float* g = o.gf[ch];
    const float* rg = o.rg[ch];
    if (n < D) {
        switch (n) {
            case 0: return -o.w * rg[0];
            case 1: return -o.w * rg[1];
            case 2: return -o.w * rg[2];
            case 3: return -(o.x1 * rg[2] - rg[1]);
            case 4: return -(rg[0] - o.x0 * rg[2]);
            case 5: return -(o.x0 * rg[1] - o.x1 * rg[0]);
            default: return -(o.x0 * rg[0] + o.x1 * rg[1] + rg[2]);  // Sim3 scale
        }
    }
    switch (n - D) {
        case 0: return g[0] * o.w;
        case 1: return g[1] * o.w;
        case 2: return g[2] * o.w;
        case 3: return o.P[1] * g[2] - o.P[2] * g[1];
        case 4: return o.P[2] * g[0] - o.P[0] * g[2];
        case 5: return o.P[0] * g[1] - o.P[1] * g[0];
        default: return g[0] * o.P[0] + g[1] * o.P[1] + g[2] * o.P[2];  // Sim3 scale
    }
}

template <int D>
__device__ __forceinline__ bool pix_jac(const float* M0, const float* X, float fx, float fy, PixJ<D>& o) {
#pragma unroll
    for (int r = 0; r < 3; r++) o.P[r] = mrow(M0, r, X);
    if (o.P[2] < 0.25f) return false;  // the forward's MIN_DEPTH mask
    const float iz = 1.f / o.P[2];
    o.iz = iz;
    o.gf[0][0] = fx * iz; o.gf[0][1] = 0.f; o.gf[0][2] = -fx * o.P[0] * iz * iz;
    o.gf[1][0] = 0.f; o.gf[1][1] = fy * iz; o.gf[1][2] = -fy * o.P[1] * iz * iz;
    o.x0 = X[0];
    o.x1 = X[1];
    o.w = X[3];
#pragma unroll
    for (int ch = 0; ch < 2; ch++) {
        const float* g = o.gf[ch];
#pragma unroll
        for (int n = 0; n < 3; n++) o.rg[ch][n] = M0[n] * g[0] + M0[4 + n] * g[1] + M0[8 + n] * g[2];
        o.jz[ch] = g[0] * M0[3] + g[1] * M0[7] + g[2] * M0[11];
    }
    return true;
}

__device__ __forceinline__ void cross3f(const float* a, const float* b, float* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// One tangent direction v = [v_i | v_j] (2D) at one pixel: z = v_i,tau W + v_i,phi x X3 (+ v_i,sigma X3),
// Y = M z, Pt = M^t_v X = v_j,tau W + v_j,phi x P (+ v_j,sigma P) - Y, and dPt/dW.
struct DirPix {
    float Y[3], Pt[3], dPt[3];
};

template <int D>
__device__ __forceinline__ void dir_pix(const float* M0, const float* X, const float* P, const float* v, DirPix& o) {
    const float W = X[3];
    float z[3], c[3];
    const float X3[3] = {X[0], X[1], 1.f};
    cross3f(v + 3, X3, c);
#pragma unroll
    for (int n = 0; n < 3; n++) z[n] = v[n] * W + c[n];
    if constexpr (D == 7) {
#pragma unroll
        for (int n = 0; n < 3; n++) z[n] += v[6] * X3[n];
    }
#pragma unroll
    for (int r = 0; r < 3; r++) o.Y[r] = M0[4 * r] * z[0] + M0[4 * r + 1] * z[1] + M0[4 * r + 2] * z[2];
    const float* vj = v + D;
    float cp[3];
    cross3f(vj + 3, P, cp);
#pragma unroll
    for (int r = 0; r < 3; r++) o.Pt[r] = vj[r] * W + cp[r] - o.Y[r];
    // d/dW: v_j,tau + v_j,phi x t (+ v_j,sigma t) - M v_i,tau
    const float t[3] = {M0[3], M0[7], M0[11]};
    float ct[3];
    cross3f(vj + 3, t, ct);
#pragma unroll
    for (int r = 0; r < 3; r++)
        o.dPt[r] = vj[r] + ct[r] - (M0[4 * r] * v[0] + M0[4 * r + 1] * v[1] + M0[4 * r + 2] * v[2]);
    if constexpr (D == 7) {
#pragma unroll
        for (int r = 0; r < 3; r++) {
            o.Pt[r] += vj[6] * P[r];
            o.dPt[r] += vj[6] * t[r];
        }
    }
}

// Mixed second derivative along direction v with coefficient cd, channel ch:
//   f^{s v}_c = grad f . (M^{sv}_k X) + Ps_k . h,  h = (-f iz^2 Zt, 0, f iz^2 Xt - 2 iz f^v)  (u; v: rows 1, 2)
// and, for pose directions k, grad f . (M^{sv}_k X) = Ps_k . (grad f x v_j,phi + v_j,sigma grad f)
// + e_k,phi . [target: -(Y x grad f); source: R^T (Y x grad f)]
// + e_k,sigma [target: -Y . grad f; source: Y . grad f]  (Sim3).
// Adds to g0h (Ps coefficient valid for every s-direction), g0x (pose-only Ps
// coefficient), om (rotation-dof vector), os (scale-dof scalar) and returns the depth
// s-direction value grad f . dPt/dW (the h part for depth is g0h . t, added by the caller).
template <int D>
__device__ __forceinline__ float mixed(const PixJ<D>& J, int ch, float fxy, const float* v, const DirPix& Dp, float fv,
                                       float cd, float* g0h, float* g0x, float* om, float* os) {
    const float* g = J.gf[ch];
    const float iz = J.iz, iz2 = iz * iz;
    g0h[ch] += cd * (-fxy * iz2 * Dp.Pt[2]);
    g0h[2] += cd * (fxy * iz2 * Dp.Pt[ch] - 2.f * iz * fv);
    float gx[3];
    cross3f(g, v + D + 3, gx);
    float yg[3];
    cross3f(Dp.Y, g, yg);
#pragma unroll
    for (int r = 0; r < 3; r++) {
        g0x[r] += cd * gx[r];
        om[r] += cd * yg[r];
    }
    if constexpr (D == 7) {
        const float sj = v[13];
#pragma unroll
        for (int r = 0; r < 3; r++) g0x[r] += cd * sj * g[r];
        *os += cd * (Dp.Y[0] * g[0] + Dp.Y[1] * g[1] + Dp.Y[2] * g[2]);
    }
    return cd * (g[0] * Dp.dPt[0] + g[1] * Dp.dPt[1] + g[2] * Dp.dPt[2]);
}

// n consecutive per-edge constants (16-byte aligned shared memory) into registers
// with 16-byte loads
template <int n>
__device__ __forceinline__ void lds_row(const float* p, float* out) {
#pragma unroll
    for (int k = 0; k < n; k += 4) {
        const float4 v = *reinterpret_cast<const float4*>(p + k);
        out[k] = v.x;
        if (k + 1 < n) out[k + 1] = v.y;
        if (k + 2 < n) out[k + 2] = v.z;
        if (k + 3 < n) out[k + 3] = v.w;
    }
}

// 0 that the compiler cannot see through: adding it to a loop's shared-memory
// address keeps the loads inside the loop (not hoisted into registers)
__device__ __forceinline__ int opaque_zero() {
    int z;
    asm volatile("mov.u32 %0, 0;" : "=r"(z));
    return z;
}

// per-pixel floats kept in shared memory by ba_adj_frame_b_kernel: a, dzf, mu, gwz, gC, gd, disp, Q, Es[D]
__host__ __device__ constexpr int kPixF(int D) { return 8 + D; }
// per-edge floats: M0 [0, 12), the directions lam, dxi, dxi~ (2D each) from kOffDir, the damping
// weights lm lam dxi of the edge's two poses (2D) at kOffDmp, the three directions in target form
// (D each) from kOffTf; rows padded to 16 bytes for vector reads (SE3 78 used of 80, Sim3 89 of 92)
// (every 2D block starts on a 16-byte boundary: SE3 M0 | 3 x 12 | 12 | 3 x 6 in 80 floats, Sim3
// M0 | 3 x 16 | 16 | 3 x 7 in 100)
__host__ __device__ constexpr int kStride2(int D) { return (2 * D + 3) / 4 * 4; }
__host__ __device__ constexpr int kOffDir(int D) { return 12; }
__host__ __device__ constexpr int kOffDmp(int D) { return 12 + 3 * kStride2(D); }
__host__ __device__ constexpr int kOffTf(int D) { return kOffDmp(D) + kStride2(D); }
__host__ __device__ constexpr int kEdgeF(int D) { return (kOffTf(D) + 3 * D + 3) / 4 * 4; }
__host__ __device__ constexpr int kMom(int D) { return D == 7 ? 16 : 15; }  // G0, om (, os)

// per (depth frame, pixel chunk): the per-pixel adjoint quantities, then the
// gradient of phi (with the exact derivative of the LM damping) for every edge
// leaving the frame.  Dynamic shared memory: kPixF(D) floats per pixel.
template <int D>
__global__ void __launch_bounds__(kAdjThreads, 2) ba_adj_frame_b_kernel(BAPtrs base, Batch B, float alpha, float lm,
                                                                          int first) {
    constexpr int D2 = 2 * D, S2 = kStride2(D), OD = kOffDir(D), OM = kOffDmp(D), OT = kOffTf(D), NM = kMom(D);
    BA_BIND(B, base);
    if (w.status[0]) return;
    extern __shared__ float pix[];  // [kPixF(D)][chunk]: a, dzf, mu, gwz, gC, gd, disp, Q, Es[D]
    __shared__ __align__(16) float Esh[kAdjMaxDeg][kEdgeF(D)];
    __shared__ int grp[kAdjMaxDeg];  // -1: unique target; else index of the first edge with the same target
    __shared__ float red[kAdjThreads / 32][16];
    __shared__ int any_dup;
    const int s = local_ % d.K, c = local_ / d.K, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int HW = d.HW, W = d.W, t0 = d.t0, P = d.P;
    const int k = w.kx[s];
    const float act = io.depth_active[k];
    const float fx = io.intr[0], fy = io.intr[1], cx = io.intr[2], cy = io.intr[3];
    const int p0 = c * d.chunk_f, p1 = min(HW, p0 + d.chunk_f), np_ = p1 - p0;
    const int eb = w.fe_ptr[s], ee = w.fe_ptr[s + 1];
    const int deg = ee - eb;
    if (deg > kAdjMaxDeg || d.chunk_f > kAdjMaxChunk) {
        if (tid == 0) atomicOr(w.status, VIPE_ERR_CAPACITY);
        return;
    }
    const int CH = d.chunk_f;
    float* pa = pix;
    float* pdzf = pix + CH;
    float* pmu = pix + 2 * CH;
    float* pgwz = pix + 3 * CH;
    float* pgC = pix + 4 * CH;
    float* pgd = pix + 5 * CH;
    float* pdisp = pix + 6 * CH;
    float* pQ = pix + 7 * CH;
    float* pEs = pix + 8 * CH;  // D x CH: the frame's own-pose slot of E at each pixel
    const bool self_in = k >= t0 && k < t0 + P;

    // per-edge data (offsets above)
    if (tid == 0) any_dup = 0;
    __syncthreads();
    for (int q = warp; q < deg; q += kAdjThreads / 32) {
        const int e = w.fe_list[eb + q];
        const int b = (int)io.jj[e];
        float* Eq = Esh[q];
        if (lane < 3) {
            const M4 T = edge_matrix<D>(io.poses, k, b);
            for (int col = 0; col < 4; col++) Eq[4 * lane + col] = (float)T.m[4 * lane + col];
        } else if (lane < 6) {
            const int dir = lane - 3;
            double v[D2];
            if (dir == 0)
                edge_dir<D>(w.adj_lam, k, b, t0, P, false, v);
            else
                edge_dir<D>(io.dx, k, b, t0, P, dir == 2, v);
            for (int n = 0; n < D2; n++) Eq[OD + S2 * dir + n] = (float)v[n];
        } else if (lane == 6) {
            double vl[D2], vd[D2];
            edge_dir<D>(w.adj_lam, k, b, t0, P, false, vl);
            edge_dir<D>(io.dx, k, b, t0, P, false, vd);
            for (int n = 0; n < D2; n++) Eq[OM + n] = (float)((double)lm * vl[n] * vd[n]);
        } else if (lane >= 8 && lane < 11) {
            // J . v = Jj . (v_j - Ad(Tij) v_i) (source rows are -Ad^T of the target rows):
            // the three directions as one D-vector each
            const int dir = lane - 8;
            double v[D2], av[D];
            if (dir == 0)
                edge_dir<D>(w.adj_lam, k, b, t0, P, false, v);
            else
                edge_dir<D>(io.dx, k, b, t0, P, dir == 2, v);
            const M4 T = edge_matrix<D>(io.poses, k, b);
            ad_apply_m4<D>(T, v, av);
            for (int n = 0; n < D; n++) Eq[OT + D * dir + n] = (float)(v[D + n] - av[n]);
        } else if (lane == 7) {
            int g = -1;
            if (b != k)
                for (int q2 = 0; q2 < deg; q2++) {
                    if (q2 == q) continue;
                    if ((int)io.jj[w.fe_list[eb + q2]] == b) {
                        g = q2 < q ? q2 : q;
                        for (int q3 = 0; q3 < q2 && q3 < q; q3++)
                            if ((int)io.jj[w.fe_list[eb + q3]] == b) g = min(g, q3);
                        break;
                    }
                }
            grp[q] = g;
            if (g >= 0) atomicOr(&any_dup, 1);
        }
    }
    __syncthreads();
    const bool dup = any_dup != 0;

    // target-slot E contribution of edge q at a pixel (sum over channels)
    auto tvec = [&](int q, const float* X, int p, float* out) {
        const int e = w.fe_list[eb + q];
        PixJ<D> J;
#pragma unroll
        for (int n = 0; n < D; n++) out[n] = 0.f;
        if (!pix_jac<D>(Esh[q], X, fx, fy, J)) return;
        const float* wp = io.weights + (size_t)e * 2 * HW;
        const float wc[2] = {0.001f * __ldg(wp + p), 0.001f * __ldg(wp + HW + p)};
#pragma unroll
        for (int ch = 0; ch < 2; ch++) {
            const float g = act * act * wc[ch] * J.jz[ch];
#pragma unroll
            for (int n = 0; n < D; n++) out[n] += g * jrow<D>(J, ch, D + n);
        }
    };

    // ---- per-pixel adjoint quantities
    for (int i = tid; i < np_; i += kAdjThreads) {
        const int p = p0 + i;
        const float u = (float)(p % W), v = (float)(p / W);
        const float disp = io.disps[(size_t)k * HW + p];
        const float X[4] = {(u - cx) / fx, (v - cy) / fy, 1.f, disp};
        float eD = 0.f, eDt = 0.f, eL = 0.f, dampC = 0.f;
        float Es[D];
#pragma unroll
        for (int n = 0; n < D; n++) Es[n] = 0.f;
        if (act != 0.f) {
            for (int q = 0; q < deg; q++) {
                const int e = w.fe_list[eb + q];
                const bool stereo = (int)io.jj[e] == k;
                const float* Eq = Esh[q];
                PixJ<D> J;
                if (!pix_jac<D>(Eq, X, fx, fy, J)) continue;
                const float* wp = io.weights + (size_t)e * 2 * HW;
                const float wc[2] = {0.001f * __ldg(wp + p), 0.001f * __ldg(wp + HW + p)};
                float tv[D];
#pragma unroll
                for (int n = 0; n < D; n++) tv[n] = 0.f;
#pragma unroll
                for (int ch = 0; ch < 2; ch++) {
                    const float g = act * act * wc[ch] * J.jz[ch];
                    float jl = 0.f, jd = 0.f, jdt = 0.f;
#pragma unroll
                    for (int n = 0; n < D; n++) {
                        const float jn = jrow<D>(J, ch, D + n);
                        jl += jn * Eq[OT + n];
                        jd += jn * Eq[OT + D + n];
                        jdt += jn * Eq[OT + 2 * D + n];
                    }
                    eL += g * jl;
                    eD += g * jd;
                    eDt += g * jdt;
#pragma unroll
                    for (int n = 0; n < D; n++) {
                        Es[n] += g * jrow<D>(J, ch, n);
                        if (stereo) Es[n] += g * jrow<D>(J, ch, D + n);
                        else tv[n] += g * jrow<D>(J, ch, D + n);
                    }
                }
                if (!stereo && grp[q] < 0)
#pragma unroll
                    for (int n = 0; n < D; n++) dampC += Eq[OM + D + n] * tv[n] * tv[n];
            }
            if (dup) {  // targets shared by several edges: the slot holds their sum
                for (int q = 0; q < deg; q++) {
                    if (grp[q] != q) continue;
                    float sum[D], tv[D];
                    for (int n = 0; n < D; n++) sum[n] = 0.f;
                    for (int q2 = q; q2 < deg; q2++)
                        if (grp[q2] == q) {
                            tvec(q2, X, p, tv);
                            for (int n = 0; n < D; n++) sum[n] += tv[n];
                        }
                    for (int n = 0; n < D; n++) dampC += Esh[q][OM + D + n] * sum[n] * sum[n];
                }
            }
            if (self_in && deg > 0) {
                // lm lam dxi of the frame's own pose: the source half of any edge's damping weights
#pragma unroll
                for (int n = 0; n < D; n++) dampC += Esh[0][OM + n] * Es[n] * Es[n];
            }
        }
        const float* qw = w.qwf + ((size_t)s * HW + p) * 3;
        const float Q = qw[0], wz = qw[1];
        const float a = Q * io.g_disps[(size_t)k * HW + p];
        const float dzf = Q * (wz - eD);
        const float dz = Q * (wz - eDt);
        const float mu = Q * eL;
        const float gwz = a - mu;
        const float gC = mu * dzf - a * dz - Q * Q * dampC;
        const float dsens = io.disps_sens[(size_t)k * HW + p];
        const float msk = (dsens > 0.f ? 1.f : 0.f) * act;
        io.g_eta[(size_t)s * HW + p] += act * gC;
        io.g_dsens[(size_t)k * HW + p] += act * msk * alpha * gwz;
        pa[i] = a;
        pdzf[i] = dzf;
        pmu[i] = mu;
        pgwz[i] = gwz;
        pgC[i] = gC;
        pgd[i] = -act * msk * alpha * gwz;
        pdisp[i] = disp;
        pQ[i] = Q;
#pragma unroll
        for (int n = 0; n < D; n++) pEs[n * CH + i] = Es[n];
    }
    __syncthreads();

    // ---- per edge: phi gradients
    for (int q = 0; q < deg; q++) {
        const int e = w.fe_list[eb + q];
        const int b = (int)io.jj[e];
        const bool stereo = k == b;
        // read through a volatile view: every use reloads from shared memory instead of
        // the compiler hoisting the edge's 60 constants into registers for the pixel loop
        // (which spilled the loop's own state)
        const volatile float* Eq = Esh[q];
        const float* Eqc = Esh[q];
        const float* tp = io.targets + (size_t)e * 2 * HW;
        const float* wp = io.weights + (size_t)e * 2 * HW;
        float* gtp = io.g_targets + (size_t)e * 2 * HW;
        float* gwp = io.g_weights + (size_t)e * 2 * HW;
        float mom[NM];  // G0 (3x4), the rotation-dof vector (and the scale-dof scalar)
#pragma unroll
        for (int m = 0; m < NM; m++) mom[m] = 0.f;
        for (int i = tid; i < np_; i += kAdjThreads) {
            const float* Eqv = Esh[q] + opaque_zero();  // per-pixel re-reads, see opaque_zero
            const int p = p0 + i;
            const float u = (float)(p % W), v = (float)(p / W);
            const float X[4] = {(u - cx) / fx, (v - cy) / fy, 1.f, pdisp[i]};
            // Sim3: this pixel's targets, weights and (after the first iteration) the gradients so
            // far are issued before the Jacobian so that their latency hides under it (74 vs 81
            // ms per 256-clip step), and the read-once targets and the gradients go through L2
            // with the streaming (evict-first) hint, which keeps the weights the two passes share
            // and the spilled registers resident (68.2 vs 72.8 ms); the SE3 form keeps plain
            // accesses at their uses (the earlier loads cost it spills, the hints 1.5 %)
            constexpr bool kHoist = D == 7;
            float tg0 = 0.f, tg1 = 0.f, wg0 = 0.f, wg1 = 0.f;
            float ogt0 = 0.f, ogt1 = 0.f, ogw0 = 0.f, ogw1 = 0.f;
            if constexpr (kHoist) {
                tg0 = __ldcs(tp + p);
                tg1 = __ldcs(tp + HW + p);
                wg0 = __ldg(wp + p);
                wg1 = __ldg(wp + HW + p);
                if (!first) {
                    ogt0 = __ldcs(gtp + p);
                    ogt1 = __ldcs(gtp + HW + p);
                    ogw0 = __ldcs(gwp + p);
                    ogw1 = __ldcs(gwp + HW + p);
                }
            }
            PixJ<D> J;
            if (!pix_jac<D>(Eqc, X, fx, fy, J)) {  // invalid pixel: zero weight, no gradient
                if (first) {
                    gtp[p] = 0.f;
                    gtp[HW + p] = 0.f;
                    gwp[p] = 0.f;
                    gwp[HW + p] = 0.f;
                }
                continue;
            }
            const float iz = J.iz, iz2 = iz * iz;
            const float a = pa[i], dzf = pdzf[i], mu = pmu[i], gwz = pgwz[i], gC = pgC[i], Q = pQ[i];
            if constexpr (!kHoist) {
                tg0 = __ldg(tp + p);
                tg1 = __ldg(tp + HW + p);
                wg0 = __ldg(wp + p);
                wg1 = __ldg(wp + HW + p);
            }
            const float rr[2] = {tg0 - (fx * J.P[0] * iz + cx), tg1 - (fy * J.P[1] * iz + cy)};
            const float wc[2] = {0.001f * wg0, 0.001f * wg1};
            // the per-pixel damping direction beta (slot E values of this edge's two poses)
            float beta[D2];
            {
                float tv[D];
                if (!stereo) {
                    if (grp[q] < 0) {
#pragma unroll
                        for (int n = 0; n < D; n++) {
                            tv[n] = 0.f;
#pragma unroll
                            for (int ch = 0; ch < 2; ch++) tv[n] += act * act * wc[ch] * J.jz[ch] * jrow<D>(J, ch, D + n);
                        }
                    } else {
                        float t2[D];
                        for (int n = 0; n < D; n++) tv[n] = 0.f;
                        for (int q2 = grp[q]; q2 < deg; q2++)
                            if (grp[q2] == grp[q]) {
                                tvec(q2, X, p, t2);
                                for (int n = 0; n < D; n++) tv[n] += t2[n];
                            }
                    }
                }
                float dmp[D2];  // damping weights lm lam dxi of the edge's two poses
                lds_row<D2>(Eqv + OM, dmp);
#pragma unroll
                for (int n = 0; n < D; n++) {
                    const float es = pEs[n * CH + i];
                    beta[n] = 2.f * Q * dmp[n] * es;
                    beta[D + n] = 2.f * Q * dmp[D + n] * (stereo ? es : tv[n]);
                }
            }
            float g0h[3] = {0.f, 0.f, 0.f}, g0x[3] = {0.f, 0.f, 0.f}, om[3] = {0.f, 0.f, 0.f}, g4[3] = {0.f, 0.f, 0.f};
            float os = 0.f;
            float gdp = 0.f;
#pragma unroll
            for (int ch = 0; ch < 2; ch++) {
                const float* g = J.gf[ch];
                const float fxy = ch == 0 ? fx : fy;
                // J . v for the edge's directions lam, dxi, dxi~, beta and the damping sum lm lam dxi J^2
                float ft[3] = {0.f, 0.f, 0.f}, fb = 0.f, fg = 0.f;
                {
                    float wv[3 * D];
                    lds_row<3 * D>(Eqv + OT, wv);
#pragma unroll
                    for (int n = 0; n < D; n++) {
                        const float jn = jrow<D>(J, ch, D + n);
                        ft[0] += jn * wv[n];
                        ft[1] += jn * wv[D + n];
                        ft[2] += jn * wv[2 * D + n];
                    }
                }
                {
                    float dmp[D2];
                    lds_row<D2>(Eqv + OM, dmp);
#pragma unroll
                    for (int n = 0; n < D2; n++) {
                        const float jn = jrow<D>(J, ch, n);
                        fb += jn * beta[n];
                        fg += dmp[n] * jn * jn;
                    }
                }
                const float fjz = J.jz[ch];
                const float wpc = stereo ? 0.f : wc[ch];
                const float A = act * act * wc[ch];
                const float G3 = -dzf * ft[0] + mu * ft[1] - a * ft[2];
                const float c0 = -wpc * ft[0] - A * gwz * fjz;
                const float c1 = wpc * (rr[ch] - ft[1]) - A * fjz * dzf;
                const float c2 = -wpc * ft[0] + A * fjz * mu;
                const float c3 = -A * fjz * a;
                const float c4 = A * (gwz * rr[ch] + 2.f * gC * fjz + G3 + fb);
                const float cB = -2.f * wpc;  // along gamma = lm lam dxi o J
                const float cE = A * fjz;     // along beta
                // the first backward iteration writes (the buffers are not cleared beforehand)
                const size_t pc = (size_t)ch * HW + p;
                const float ogt = kHoist ? (ch == 0 ? ogt0 : ogt1) : (first ? 0.f : gtp[pc]);
                const float ogw = kHoist ? (ch == 0 ? ogw0 : ogw1) : (first ? 0.f : gwp[pc]);
                const float ngt = ogt + wpc * ft[0] + A * gwz * fjz;
                if constexpr (kHoist)
                    __stcs(gtp + pc, ngt);
                else
                    gtp[pc] = ngt;
                const float ngw = ogw +
                          0.001f * ((stereo ? 0.f : ft[0] * (rr[ch] - ft[1]) - fg) +
                                    act * act * (gwz * fjz * rr[ch] + gC * fjz * fjz + fjz * (G3 + fb)));
                if constexpr (kHoist)
                    __stcs(gwp + pc, ngw);
                else
                    gwp[pc] = ngw;
                // first derivatives (s part) and the depth t-direction (column 3 of G0)
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    g0h[r] += c0 * g[r];
                    g4[r] += c4 * g[r];
                }
                g0h[ch] += c4 * (-fxy * iz2 * Eq[11]);
                g0h[2] += c4 * (fxy * iz2 * Eq[4 * ch + 3] - 2.f * iz * fjz);
                // every tangent direction enters linearly: one combined direction
                float ud[D2];
                {
                    float dv[D2];
                    lds_row<D2>(Eqv + OM, dv);
#pragma unroll
                    for (int n = 0; n < D2; n++) ud[n] = cE * beta[n] + cB * dv[n] * jrow<D>(J, ch, n);
                    lds_row<D2>(Eqv + OD, dv);
#pragma unroll
                    for (int n = 0; n < D2; n++) ud[n] += c1 * dv[n];
                    lds_row<D2>(Eqv + OD + S2, dv);
#pragma unroll
                    for (int n = 0; n < D2; n++) ud[n] += c2 * dv[n];
                    lds_row<D2>(Eqv + OD + 2 * S2, dv);
#pragma unroll
                    for (int n = 0; n < D2; n++) ud[n] += c3 * dv[n];
                }
                // J . ud from the dot products above (ud is their linear combination)
                const float fu = c1 * ft[0] + c2 * ft[1] + c3 * ft[2] + cE * fb + cB * fg;
                DirPix Dp;
                dir_pix<D>(Eqc, X, J.P, ud, Dp);
                gdp += mixed<D>(J, ch, fxy, ud, Dp, fu, 1.f, g0h, g0x, om, &os);
            }
            // depth s-direction of this pixel: Ps = t (column 3 of M0)
            gdp += g0h[0] * Eq[3] + g0h[1] * Eq[7] + g0h[2] * Eq[11];
            pgd[i] += gdp;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const float gr = g0h[r] + g0x[r];
                mom[4 * r + 0] += gr * X[0];
                mom[4 * r + 1] += gr * X[1];
                mom[4 * r + 2] += gr;
                mom[4 * r + 3] += gr * X[3] + g4[r];
                mom[12 + r] += om[r];
            }
            if constexpr (D == 7) mom[15] += os;
        }
#pragma unroll
        for (int m = 0; m < NM; m++) {
            const float sv = warp_sum(mom[m]);
            if (lane == 0) red[warp][m] = sv;
        }
        __syncthreads();
        if (tid < NM) {
            float sv = 0.f;
            for (int r = 0; r < kAdjThreads / 32; r++) sv += red[r][tid];
            w.adj_gpart[((size_t)e * d.CF + c) * kAdjAcc + tid] = stereo ? 0.f : sv;
        }
        __syncthreads();
    }
    // ---- pass-through plus this iteration's depth gradient
    for (int i = tid; i < np_; i += kAdjThreads) io.g_disps[(size_t)k * HW + p0 + i] += pgd[i];
}

// per edge: the 2D pose gradients from the moments: <M^s_k, G0> plus, for the
// rotation dofs, -om (target pose) or R^T om (source pose), and for the Sim3 scale dof
// -os (target) or +os (source)
// (k < D: source pose i, M^s = -T hat(e_k); k >= D: target pose j, M^s = hat(e_{k-D}) T,
// hat of a Sim3 tangent [tau, phi, sigma] = [[phi x + sigma I, tau], [0, 0]])
template <int D>
__global__ void ba_adj_edge_reduce_kernel(BAPtrs base, Batch B) {
    BA_BIND(B, base);
    if (w.status[0]) return;
    constexpr int NM = kMom(D);
    __shared__ double G[16];
    const int e = local_, tid = threadIdx.x;
    for (int m = tid; m < NM; m += blockDim.x) {
        double sv = 0.0;
        for (int c = 0; c < d.CF; c++) sv += (double)w.adj_gpart[((size_t)e * d.CF + c) * kAdjAcc + m];
        G[m] = sv;
    }
    __syncthreads();
    if (tid >= 2 * D) return;
    const int ia = (int)io.ii[e], ib = (int)io.jj[e];
    double out = 0.0;
    if (ia != ib) {
        const M4 T = edge_matrix<D>(io.poses, ia, ib);
        const bool src = tid < D;
        const int n = tid % D;
        M4 H = mzero();
        if (n < 6) {
            double unit[6] = {0, 0, 0, 0, 0, 0};
            unit[n] = 1.0;
            H = hat(unit);
        } else {
            H.m[0] = H.m[5] = H.m[10] = 1.0;  // the scale generator diag(1, 1, 1, 0)
        }
        const M4 Ms = src ? madd(mzero(), mmul(T, H), -1.0) : mmul(H, T);
        for (int r = 0; r < 3; r++)
            for (int col = 0; col < 4; col++) out += Ms.m[4 * r + col] * G[4 * r + col];
        if (n >= 3 && n < 6) {
            if (src) {
                // R^T om with R the rotation of Tij (the 3x3 block of T is s R)
                const double sc = (D == 6) ? 1.0 : sqrt(T.m[0] * T.m[0] + T.m[4] * T.m[4] + T.m[8] * T.m[8]);
                out += (T.m[0 * 4 + (n - 3)] * G[12] + T.m[1 * 4 + (n - 3)] * G[13] + T.m[2 * 4 + (n - 3)] * G[14]) / sc;
            } else {
                out -= G[12 + n - 3];
            }
        } else if (n == 6) {
            out += src ? G[15] : -G[15];
        }
    }
    w.adj_gedge[(size_t)e * 2 * D + tid] = out;
}

// gT[f] += per-edge pose gradients (every frame of the graph, fixed ones too);
// one warp per frame, edges in index order, fixed reduction order.
template <int D>
__global__ void ba_adj_pose_kernel(BAPtrs base, Batch B) {
    BA_BIND(B, base);
    if (w.status[0]) return;
    const int lane = threadIdx.x & 31;
    for (int f = threadIdx.x >> 5; f < d.N; f += blockDim.x >> 5) {
        double acc[D];
        for (int n = 0; n < D; n++) acc[n] = 0.0;
        for (int e = lane; e < d.E; e += 32) {
            const int ia = (int)io.ii[e], ib = (int)io.jj[e];
            if (ia == f)
                for (int n = 0; n < D; n++) acc[n] += w.adj_gedge[(size_t)e * 2 * D + n];
            if (ib == f)
                for (int n = 0; n < D; n++) acc[n] += w.adj_gedge[(size_t)e * 2 * D + D + n];
        }
        for (int n = 0; n < D; n++) {
            const double sv = warp_sum(acc[n]);
            if (lane == 0) w.adj_gT[(size_t)f * D + n] += sv;
        }
    }
}

__global__ void ba_adj_finish_kernel(BAPtrs base, Batch B) {
    BA_BIND(B, base);
    const int D = d.dof;
    for (int q = threadIdx.x; q < d.N * (D + 1); q += blockDim.x) {
        const int f = q / (D + 1), n = q % (D + 1);
        io.g_poses[q] = n < D ? (float)w.adj_gT[(size_t)f * D + n] : 0.f;
    }
}

__global__ void ba_adj_status_kernel(BAPtrs base, Batch B) {
    BA_BIND(B, base);
    if (w.status[0] && io.status) atomicOr(io.status, w.status[0]);
}

}  // namespace ba
}  // namespace vipe

using namespace vipe;
using namespace vipe::ba;

extern "C" int vipe_slam_ba_batch_backward(const vipe_ba_batch_plan* plan, const float* tape_poses,
                                           const float* tape_disps, const double* tape_factor, const float* tape_dx,
                                           const float* intrinsics, const float* disps_sens, const float* targets,
                                           const float* weights, const float* eta, const int64_t* ii,
                                           const int64_t* jj, const float* depth_active, int iterations, float lm,
                                           float ep, float alpha, float* grad_poses, float* grad_disps,
                                           float* grad_targets, float* grad_weights, float* grad_eta,
                                           float* grad_disps_sens, int32_t* dev_status, void* stream) {
    (void)ep;  // the damping's constant part has no derivative; only lm enters the adjoint
    if (!plan) return VIPE_ERR_ARG;
    if (!plan->d_table) {
        set_last_error("vipe_slam_ba_batch_backward: plan is not bound to a workspace");
        return VIPE_ERR_WORKSPACE;
    }
    if (!plan->adjoint) {
        set_last_error("vipe_slam_ba_batch_backward: plan was created without the adjoint buffers");
        return VIPE_ERR_ARG;
    }
    if (iterations < 0 || !tape_poses || !tape_disps || !tape_factor || !tape_dx || !intrinsics || !disps_sens ||
        !eta || !depth_active || !grad_poses || !grad_disps || !grad_eta || !grad_disps_sens)
        return VIPE_ERR_ARG;
    if (plan->edges > 0 && (!targets || !weights || !ii || !jj || !grad_targets || !grad_weights))
        return VIPE_ERR_ARG;
    size_t smem_b = 0;
    const int dof = plan->geo.dof;
    const int pixf = kPixF(dof);
    for (const auto& gd : plan->gds) smem_b = std::max(smem_b, (size_t)pixf * gd.d.chunk_f * sizeof(float));
    if (smem_b > (size_t)pixf * kAdjMaxChunk * sizeof(float)) {
        set_last_error("vipe_slam_ba_batch_backward: pixel chunk beyond 1536 (use more frame_chunks)");
        return VIPE_ERR_CAPACITY;
    }
    cudaStream_t st = as_stream(stream);
    const Geometry& geo = plan->geo;
    const long HW = (long)plan->ht * plan->wd;
    const int G = geo.G;
    const Batch per_graph{plan->d_table, nullptr, G};
    // with iterations the first backward iteration writes every target / weight gradient
    if (plan->edges > 0 && iterations == 0) {
        VIPE_CUDA_TRY(cudaMemsetAsync(grad_targets, 0, sizeof(float) * plan->edges * 2 * HW, st));
        VIPE_CUDA_TRY(cudaMemsetAsync(grad_weights, 0, sizeof(float) * plan->edges * 2 * HW, st));
    }
    VIPE_CUDA_TRY(cudaMemsetAsync(grad_eta, 0, sizeof(float) * plan->kx * HW, st));
    VIPE_CUDA_TRY(cudaMemsetAsync(grad_disps_sens, 0, sizeof(float) * plan->frames * HW, st));
    if (dof == 7)
        VIPE_CUDA_TRY(cudaFuncSetAttribute(ba_adj_frame_b_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(pixf * kAdjMaxChunk * sizeof(float))));
    else
        VIPE_CUDA_TRY(cudaFuncSetAttribute(ba_adj_frame_b_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(pixf * kAdjMaxChunk * sizeof(float))));
    BAPtrs base{const_cast<float*>(tape_poses), const_cast<float*>(tape_disps), const_cast<float*>(intrinsics),
                disps_sens, targets, weights, eta, ii, jj, depth_active, const_cast<float*>(tape_dx), nullptr,
                nullptr, dev_status, 0, 1, grad_poses, grad_disps, grad_targets, grad_weights, grad_eta,
                grad_disps_sens, const_cast<double*>(tape_factor)};
    int rc = launch_index(geo, plan->d_table, base, nullptr, st);
    if (rc != VIPE_OK) return rc;
    ba_adj_init_kernel<<<G, 256, 0, st>>>(base, per_graph);
    VIPE_LAUNCH_CHECK();
    auto grid = [&](int k) { return (unsigned)geo.off[k][G]; };
    const Batch frames{plan->d_table, plan->d_off + (size_t)kOffFrame * (G + 1), G};
    const Batch edges{plan->d_table, plan->d_off + (size_t)kOffEdgeRed * (G + 1), G};
    for (int itr = iterations - 1; itr >= 0; itr--) {
        base.poses = const_cast<float*>(tape_poses) + (size_t)itr * plan->frames * (dof + 1);
        base.disps = const_cast<float*>(tape_disps) + (size_t)itr * plan->frames * HW;
        base.dx = const_cast<float*>(tape_dx) + (size_t)itr * plan->poses * dof;
        base.ftape = const_cast<double*>(tape_factor) + (size_t)itr * plan->ftape_stride;
        {
            VIPE_PROF("ba_adj_prep", st);
            if (dof == 7)
                ba_adj_prep_kernel<7><<<G, 128, 0, st>>>(base, per_graph);
            else
                ba_adj_prep_kernel<6><<<G, 128, 0, st>>>(base, per_graph);
        }
        VIPE_LAUNCH_CHECK();
        if (grid(kOffFrame) > 0) {
            VIPE_PROF("ba_adj_frame_a", st);
            if (dof == 7)
                ba_adj_frame_a_kernel<7><<<grid(kOffFrame), kAdjThreads, 0, st>>>(base, frames, alpha);
            else
                ba_adj_frame_a_kernel<6><<<grid(kOffFrame), kAdjThreads, 0, st>>>(base, frames, alpha);
        }
        VIPE_LAUNCH_CHECK();
        {
            VIPE_PROF("ba_adj_rhs", st);
            ba_adj_rhs_kernel<<<G, 256, 0, st>>>(base, per_graph);
        }
        VIPE_LAUNCH_CHECK();
        if ((rc = launch_chol_resolve(geo, plan->d_table, base, st)) != VIPE_OK) return rc;
        if (grid(kOffFrame) > 0) {
            VIPE_PROF("ba_adj_frame_b", st);
            auto fb = dof == 7 ? ba_adj_frame_b_kernel<7> : ba_adj_frame_b_kernel<6>;
            fb<<<grid(kOffFrame), kAdjThreads, smem_b, st>>>(base, frames, alpha, lm,
                                                                                 itr == iterations - 1 ? 1 : 0);
        }
        VIPE_LAUNCH_CHECK();
        if (grid(kOffEdgeRed) > 0) {
            VIPE_PROF("ba_adj_edge_reduce", st);
            if (dof == 7)
                ba_adj_edge_reduce_kernel<7><<<grid(kOffEdgeRed), 32, 0, st>>>(base, edges);
            else
                ba_adj_edge_reduce_kernel<6><<<grid(kOffEdgeRed), 32, 0, st>>>(base, edges);
        }
        VIPE_LAUNCH_CHECK();
        {
            VIPE_PROF("ba_adj_pose", st);
            if (dof == 7)
                ba_adj_pose_kernel<7><<<G, 256, 0, st>>>(base, per_graph);
            else
                ba_adj_pose_kernel<6><<<G, 256, 0, st>>>(base, per_graph);
        }
        VIPE_LAUNCH_CHECK();
    }
    ba_adj_finish_kernel<<<G, 256, 0, st>>>(base, per_graph);
    VIPE_LAUNCH_CHECK();
    if (dev_status) {
        ba_adj_status_kernel<<<G, 1, 0, st>>>(base, per_graph);
        VIPE_LAUNCH_CHECK();
    }
    return VIPE_OK;
}
