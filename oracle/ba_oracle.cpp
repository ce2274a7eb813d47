// CPU oracle for the dense bundle adjustment of the DROID-style SLAM backend.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product path loads this file: it is
// compiled by oracle/Makefile into oracle/_build/libvipe_oracle.so and called by
// tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the
// checker.  It restates, in plain C++, the algorithm of the reference's fused BA
// (vipe: csrc/slam_ext/geom_kernels.cu) so that the CUDA path can be compared
// against it on the same inputs:
//
//   * per-edge reprojection, Jacobians and the 12x12 pose block
//       geom_kernels.cu:178-524 (projective_transform_kernel), incl. the 0.001
//       weight scale (:311-312), MIN_DEPTH = 0.25 (:33,307-312), the stereo rule
//       ii == jj (:231-241, :359, :407) and the focal-length terms (:314-332)
//   * row gathers "accum"                       geom_kernels.cu:1043-1089
//   * Schur complement pair enumeration          geom_kernels.cu:1426-1509
//   * focal-length augmented system              geom_kernels.cu:1511-1624
//   * LM damping  diag += ep + lm * diag         geom_kernels.cu:1269-1288, :1389-1417
//   * LM loop (C, w, Q, E rows, EvT quirk, retraction order)
//                                               geom_kernels.cu:1626-1824
//   * SE3 exp / retraction                       geom_kernels.cu:69-177, :974-1023
//
// The sparse Cholesky (Eigen 3.4 SimplicialLLT, not available here) is replaced by
// a dense LL^T in double; the factorisation is unique for an SPD matrix, so the
// solution agrees to rounding.  On a non-positive pivot dx = 0, as the reference
// does on solver failure (geom_kernels.cu:1283-1285).
//
// Scalar type S selects the arithmetic: S = float follows the reference's FP32
// device arithmetic; S = double is the all-FP64 oracle.  Assembly and the solve
// are always double, as in the reference host code.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// Number of host threads the oracle may use (set by oracle_set_threads).
int g_threads = 1;
int g_backsub_all_rows = 0;  // see oracle_set_backsub_all_rows

// Robust kernel of the reference's generic solver (vipe/slam/ba/kernel.py:40-153), applied as
// w <- w * kernel(r) per flow channel (terms.py:73-75); see oracle_set_robust.
int g_rb_kind = 0;
double g_rb_c = 1.0;
std::vector<double> g_rb_mu;

// Camera model of the frames (oracle_set_camera): 0 pinhole, 1 MEI with distortion g_k1
// (vipe/utils/cameras.py:220-330).
int g_cam = 0;
double g_k1 = 0.0;

// MEI unprojection of the normalised pinhole coordinates in X[0], X[1] (in place):
// r2 = u^2 + v^2, q = sqrt(1 + (1 - k1^2) r2), s = (k1 + q) / (1 + r2), X = u s / (s - k1)
template <typename S>
void mei_unproject(S k1, S* X) {
    const S u = X[0], v = X[1], r2 = u * u + v * v;
    const S q = std::sqrt(S(1) + (S(1) - k1 * k1) * r2);
    const S f = (k1 + q) / (S(1) + r2);
    X[0] = u * f / (f - k1);
    X[1] = v * f / (f - k1);
}

template <typename S>
S robust_weight(int kind, S c, S mu, S r) {
    if (kind == 1) {  // Huber
        const S a = std::fabs(r);
        return a <= c ? S(1) : c / std::max(a, S(1e-8));
    }
    if (kind == 2) {  // Tukey
        const S t = std::max(S(1) - (r / c) * (r / c), S(0));
        return t * t;
    }
    if (kind == 3) {  // GNC-TLS at scalar mu; mu = inf is the hard indicator
        const S r2 = r * r, c2 = c * c;
        if (!(mu < S(INFINITY))) return r2 < c2 ? S(1) : S(0);
        if (r2 < (mu / (mu + S(1))) * c2) return S(1);
        if (r2 <= ((mu + S(1)) / mu) * c2)
            return std::max(std::sqrt(c2 * mu * (mu + S(1)) / std::max(r2, S(1e-12))) - mu, S(0));
        return S(0);
    }
    return S(1);
}

// Static-chunked parallel for over [0, n) on g_threads std::threads (the
// toolchain here ships no OpenMP runtime).
template <typename F>
void parallel_for(long n, F&& f) {
    const int T = std::max(1, std::min<int>(g_threads, (int)std::max<long>(1, n)));
    if (T == 1) {
        for (long i = 0; i < n; i++) f(i);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++)
        pool.emplace_back([&, t] {
            for (long i = t; i < n; i += T) f(i);
        });
    for (auto& th : pool) th.join();
}

constexpr double kMinDepth = 0.25;

// rotate X by unit quaternion q (q = x,y,z,w)
template <typename S>
inline void rotate(const S* q, const S* X, S* Y) {
    S uv0 = S(2) * (q[1] * X[2] - q[2] * X[1]);
    S uv1 = S(2) * (q[2] * X[0] - q[0] * X[2]);
    S uv2 = S(2) * (q[0] * X[1] - q[1] * X[0]);
    Y[0] = X[0] + q[3] * uv0 + (q[1] * uv2 - q[2] * uv1);
    Y[1] = X[1] + q[3] * uv1 + (q[2] * uv0 - q[0] * uv2);
    Y[2] = X[2] + q[3] * uv2 + (q[0] * uv1 - q[1] * uv0);
}

// homogeneous point action of (t, q): Y = [R X + t*w, w]
template <typename S>
inline void act_h(const S* t, const S* q, const S* X, S* Y) {
    rotate(q, X, Y);
    Y[3] = X[3];
    Y[0] += X[3] * t[0];
    Y[1] += X[3] * t[1];
    Y[2] += X[3] * t[2];
}

// adjoint-transpose style map used for the source-pose Jacobian
// (geom_kernels.cu:88-102): Y = Ad(T)^T X with T = (t, q)
template <typename S>
inline void adj_t(const S* t, const S* q, const S* X, S* Y) {
    S qi[4] = {-q[0], -q[1], -q[2], q[3]};
    rotate(qi, X, Y);
    rotate(qi, X + 3, Y + 3);
    S u[3] = {t[2] * X[1] - t[1] * X[2], t[0] * X[2] - t[2] * X[0], t[1] * X[0] - t[0] * X[1]};
    S v[3];
    rotate(qi, u, v);
    Y[3] += v[0];
    Y[4] += v[1];
    Y[5] += v[2];
}

// relative pose Tij = Tj * Ti^-1 (geom_kernels.cu:104-114)
template <typename S>
inline void relative(const S* ti, const S* qi, const S* tj, const S* qj, S* tij, S* qij) {
    qij[0] = -qj[3] * qi[0] + qj[0] * qi[3] - qj[1] * qi[2] + qj[2] * qi[1];
    qij[1] = -qj[3] * qi[1] + qj[1] * qi[3] - qj[2] * qi[0] + qj[0] * qi[2];
    qij[2] = -qj[3] * qi[2] + qj[2] * qi[3] - qj[0] * qi[1] + qj[1] * qi[0];
    qij[3] = qj[3] * qi[3] + qj[0] * qi[0] + qj[1] * qi[1] + qj[2] * qi[2];
    S r[3];
    rotate(qij, ti, r);
    tij[0] = tj[0] - r[0];
    tij[1] = tj[1] - r[1];
    tij[2] = tj[2] - r[2];
}

// SE3 exponential, tangent order (tau, phi) (geom_kernels.cu:116-177)
template <typename S>
inline void se3_exp(const S* xi, S* t, S* q) {
    const S* phi = xi + 3;
    S th2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
    S th = std::sqrt(th2);
    S imag, real;
    if (th2 < S(1e-8)) {
        imag = S(0.5) - S(1.0 / 48.0) * th2 + S(1.0 / 3840.0) * th2 * th2;
        real = S(1) - S(1.0 / 8.0) * th2 + S(1.0 / 384.0) * th2 * th2;
    } else {
        imag = std::sin(S(0.5) * th) / th;
        real = std::cos(S(0.5) * th);
    }
    q[0] = imag * phi[0];
    q[1] = imag * phi[1];
    q[2] = imag * phi[2];
    q[3] = real;
    t[0] = xi[0];
    t[1] = xi[1];
    t[2] = xi[2];
    if (th > S(1e-4)) {
        S tau[3] = {xi[0], xi[1], xi[2]};
        S c1[3] = {phi[1] * tau[2] - phi[2] * tau[1], phi[2] * tau[0] - phi[0] * tau[2],
                   phi[0] * tau[1] - phi[1] * tau[0]};
        S c2[3] = {phi[1] * c1[2] - phi[2] * c1[1], phi[2] * c1[0] - phi[0] * c1[2],
                   phi[0] * c1[1] - phi[1] * c1[0]};
        S a = (S(1) - std::cos(th)) / th2;
        S b = (th - std::sin(th)) / (th * th2);
        for (int k = 0; k < 3; k++) t[k] += a * c1[k] + b * c2[k];
    }
}

// left retraction T <- Exp(xi) * T (geom_kernels.cu:974-1023)
template <typename S>
inline void retract(const S* xi, S* pose) {
    S dt[3], dq[4];
    se3_exp(xi, dt, dq);
    const S* q = pose + 3;
    S q1[4];
    q1[0] = dq[3] * q[0] + dq[0] * q[3] + dq[1] * q[2] - dq[2] * q[1];
    q1[1] = dq[3] * q[1] + dq[1] * q[3] + dq[2] * q[0] - dq[0] * q[2];
    q1[2] = dq[3] * q[2] + dq[2] * q[3] + dq[0] * q[1] - dq[1] * q[0];
    q1[3] = dq[3] * q[3] - dq[0] * q[0] - dq[1] * q[1] - dq[2] * q[2];
    S t1[3];
    rotate(dq, pose, t1);
    for (int k = 0; k < 3; k++) pose[k] = t1[k] + dt[k];
    for (int k = 0; k < 4; k++) pose[3 + k] = q1[k];
}

// Dense LL^T solve in place; returns false on a non-positive pivot.
bool cholesky_solve(std::vector<double>& A, std::vector<double>& b, int n) {
    for (int j = 0; j < n; j++) {
        double d = A[(size_t)j * n + j];
        for (int k = 0; k < j; k++) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        if (!(d > 0.0)) return false;
        d = std::sqrt(d);
        A[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; i++) {
            double s = A[(size_t)i * n + j];
            for (int k = 0; k < j; k++) s -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = s / d;
        }
    }
    for (int i = 0; i < n; i++) {
        double s = b[i];
        for (int k = 0; k < i; k++) s -= A[(size_t)i * n + k] * b[k];
        b[i] = s / A[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int k = i + 1; k < n; k++) s -= A[(size_t)k * n + i] * b[k];
        b[i] = s / A[(size_t)i * n + i];
    }
    return true;
}

struct Index {
    std::vector<int64_t> kx;      // sorted unique of cat(arange(t0,t1), ii)
    std::vector<int64_t> ii_exp;  // cat(arange(t0,t1), ii)
    std::vector<int64_t> jj_exp;  // cat(arange(t0,t1), jj)
    std::vector<int64_t> kk_exp;  // position of ii_exp in kx
};

Index build_index(const int64_t* ii, const int64_t* jj, int E, int t0, int t1) {
    Index ix;
    for (int t = t0; t < t1; t++) {
        ix.ii_exp.push_back(t);
        ix.jj_exp.push_back(t);
    }
    for (int e = 0; e < E; e++) {
        ix.ii_exp.push_back(ii[e]);
        ix.jj_exp.push_back(jj[e]);
    }
    ix.kx = ix.ii_exp;
    std::sort(ix.kx.begin(), ix.kx.end());
    ix.kx.erase(std::unique(ix.kx.begin(), ix.kx.end()), ix.kx.end());
    for (int64_t v : ix.ii_exp)
        ix.kk_exp.push_back(std::lower_bound(ix.kx.begin(), ix.kx.end(), v) - ix.kx.begin());
    return ix;
}

// Schur pair enumeration, in the order of geom_kernels.cu:1440-1468:
// for pose i, pose j, row k of i, row l of j sharing a depth frame.
void schur_pairs(const Index& ix, int t0, int t1, std::vector<int64_t>& pi, std::vector<int64_t>& pj,
                 std::vector<int64_t>& trip) {
    const int P = t1 - t0;
    std::vector<std::vector<int64_t>> graph(P), index(P);
    for (size_t n = 0; n < ix.jj_exp.size(); n++) {
        int64_t j = ix.jj_exp[n];
        if (j >= t0 && j < t1) {
            graph[j - t0].push_back(ix.kk_exp[n]);
            index[j - t0].push_back((int64_t)n);
        }
    }
    for (int i = 0; i < P; i++)
        for (int j = 0; j < P; j++)
            for (size_t k = 0; k < graph[i].size(); k++)
                for (size_t l = 0; l < graph[j].size(); l++)
                    if (graph[i][k] == graph[j][l]) {
                        pi.push_back(i);
                        pj.push_back(j);
                        trip.push_back(index[i][k]);
                        trip.push_back(index[j][l]);
                        trip.push_back(graph[i][k]);
                    }
}

template <typename S>
struct EdgeTerms {
    S H[12][12];  // full symmetric 12x12 of [Ji Jj]^T W [Ji Jj]
    S v[12];      // [vi; vj]
    S F[12];      // [fi; fj] focal coupling
    S hf, vf, energy;
};

template <typename S>
int run_ba(double* poses_io, double* disps_io, double* intr_io, const double* disps_sens, const double* targets,
           const double* weights, const double* eta, const int64_t* ii, const int64_t* jj,
           const double* depth_active, int N, int H, int W, int E, int nkx, int t0, int t1, int iters, double lm,
           double ep, int motion_only, double alpha, int opt_intr, double intr_lm, double intr_ep,
           double intr_scale, int compute_energy, double* dx_out, double* dz_out, double* energy_out) {
    const int HW = H * W;
    const int P = t1 - t0;
    if (P <= 0 || t0 < 0 || t1 > N) return 1;
    for (int e = 0; e < E; e++)
        if (ii[e] < 0 || ii[e] >= N || jj[e] < 0 || jj[e] >= N) return 2;

    Index ix = build_index(ii, jj, E, t0, t1);
    const int K = (int)ix.kx.size();
    if (K != nkx) return 3;
    const int R = (int)ix.ii_exp.size();  // rows of E = P + E

    std::vector<S> poses(poses_io, poses_io + (size_t)N * 7);
    std::vector<S> disps(disps_io, disps_io + (size_t)N * HW);
    S intr[4] = {S(intr_io[0]), S(intr_io[1]), S(intr_io[2]), S(intr_io[3])};

    std::vector<EdgeTerms<S>> terms(E);
    std::vector<S> Eii((size_t)E * 6 * HW), Eij((size_t)E * 6 * HW), Cii((size_t)E * HW), bz((size_t)E * HW),
        Efi((size_t)E * HW);
    std::vector<double> dx_d((size_t)P * 6, 0.0);
    std::vector<S> dz((size_t)K * HW, S(0));
    double df = 0.0;

    std::vector<int64_t> spi, spj, strip;
    if (!motion_only) schur_pairs(ix, t0, t1, spi, spj, strip);

    for (int itr = 0; itr < iters; itr++) {
        const S fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
        // ---------------- per-edge linearisation ----------------
        parallel_for(E, [&](long e) {
            const int a = (int)ii[e], b = (int)jj[e];
            const S act = S(depth_active[a]);
            S tij[3], qij[4];
            if (a == b) {
                tij[0] = S(-0.1); tij[1] = 0; tij[2] = 0;
                qij[0] = 0; qij[1] = 0; qij[2] = 0; qij[3] = 1;
            } else {
                relative(&poses[a * 7], &poses[a * 7 + 3], &poses[b * 7], &poses[b * 7 + 3], tij, qij);
            }
            EdgeTerms<S>& T = terms[e];
            std::memset(&T, 0, sizeof(T));
            for (int p = 0; p < HW; p++) {
                const int r = p / W, c = p % W;
                S Xi[4] = {(S(c) - cx) / fx, (S(r) - cy) / fy, S(1), disps[(size_t)a * HW + p]};
                if (g_cam == 1) mei_unproject(S(g_k1), Xi);
                S Xj[4];
                act_h(tij, qij, Xi, Xj);
                const S x = Xj[0], y = Xj[1], h = Xj[3];
                const bool ok = !(Xj[2] < S(kMinDepth));
                const S d = ok ? S(1) / Xj[2] : S(0);
                const S d2 = d * d;
                // MEI: projection (pu, pv) and its gradients gm[c] in Xj (rows of the camera's Jp)
                S pu = fx * d * x + cx, pv = fy * d * y + cy, gm[2][3] = {{0, 0, 0}, {0, 0, 0}};
                if (g_cam == 1) {
                    const S k1 = S(g_k1), rn = std::sqrt(x * x + y * y + Xj[2] * Xj[2]), rb = Xj[2] + k1 * rn;
                    const S dm = ok ? S(1) / rb : S(0), iden = ok ? S(1) / (rb * rb * rn) : S(0);
                    pu = fx * x * dm + cx;
                    pv = fy * y * dm + cy;
                    gm[0][0] = fx * (rb * rn - k1 * x * x) * iden;
                    gm[0][1] = -fx * k1 * x * y * iden;
                    gm[0][2] = -fx * x * (k1 * Xj[2] + rn) * iden;
                    gm[1][0] = -fy * k1 * x * y * iden;
                    gm[1][1] = fy * (rb * rn - k1 * y * y) * iden;
                    gm[1][2] = -fy * y * (k1 * Xj[2] + rn) * iden;
                }
                S wu = ok ? S(0.001) * S(weights[(((size_t)e * 2 + 0) * HW) + p]) : S(0);
                S wv = ok ? S(0.001) * S(weights[(((size_t)e * 2 + 1) * HW) + p]) : S(0);
                S Jfu = 0, Jfv = 0;
                if (opt_intr) {
                    S dXi[4] = {-Xi[0] / fx, -Xi[1] / fy, 0, 0};
                    S dXj[4];
                    act_h(tij, qij, dXi, dXj);
                    Jfu = S(intr_scale) * (fx * d * dXj[0] - fx * x * d2 * dXj[2] + x * d);
                    Jfv = S(intr_scale) * (fy * d * dXj[1] - fy * y * d2 * dXj[2] + y * d);
                }
                const S ru = S(targets[(((size_t)e * 2 + 0) * HW) + p]) - pu;
                const S rv = S(targets[(((size_t)e * 2 + 1) * HW) + p]) - pv;
                if (g_rb_kind != 0) {
                    const S mu = S(g_rb_mu.empty() ? 1.0 : g_rb_mu[std::min<size_t>(itr, g_rb_mu.size() - 1)]);
                    wu *= robust_weight(g_rb_kind, S(g_rb_c), mu, ru);
                    wv *= robust_weight(g_rb_kind, S(g_rb_c), mu, rv);
                }
                T.energy += wu * ru * ru + wv * rv * rv;
                for (int ch = 0; ch < 2; ch++) {
                    S J[12];
                    S* Ji = J;
                    S* Jj = J + 6;
                    S Jz, w, res, Jf;
                    if (ch == 0) {
                        Jj[0] = fx * (h * d); Jj[1] = 0; Jj[2] = fx * (-x * h * d2);
                        Jj[3] = fx * (-x * y * d2); Jj[4] = fx * (1 + x * x * d2); Jj[5] = fx * (-y * d);
                        Jz = fx * (tij[0] * d - tij[2] * (x * d2));
                        w = wu; res = ru; Jf = Jfu;
                    } else {
                        Jj[0] = 0; Jj[1] = fy * (h * d); Jj[2] = fy * (-y * h * d2);
                        Jj[3] = fy * (-1 - y * y * d2); Jj[4] = fy * (x * y * d2); Jj[5] = fy * (x * d);
                        Jz = fy * (tij[1] * d - tij[2] * (y * d2));
                        w = wv; res = rv; Jf = Jfv;
                    }
                    if (g_cam == 1) {  // any central camera: (h g, P x g) and g . t from its gradient g
                        const S* gc = gm[ch];
                        Jj[0] = h * gc[0]; Jj[1] = h * gc[1]; Jj[2] = h * gc[2];
                        Jj[3] = y * gc[2] - Xj[2] * gc[1];
                        Jj[4] = Xj[2] * gc[0] - x * gc[2];
                        Jj[5] = x * gc[1] - y * gc[0];
                        Jz = gc[0] * tij[0] + gc[1] * tij[1] + gc[2] * tij[2];
                    }
                    const S wd = w * act;
                    const size_t q = (size_t)e * HW + p;
                    if (ch == 0) { Cii[q] = 0; bz[q] = 0; Efi[q] = 0; }
                    Cii[q] += wd * Jz * Jz;
                    bz[q] += wd * res * Jz;
                    if (opt_intr) Efi[q] += wd * Jz * Jf;
                    if (a == b) w = 0;
                    adj_t(tij, qij, Jj, Ji);
                    for (int n = 0; n < 6; n++) Ji[n] = -Ji[n];
                    for (int n = 0; n < 12; n++)
                        for (int m = 0; m <= n; m++) T.H[n][m] += w * J[n] * J[m];
                    for (int n = 0; n < 6; n++) {
                        T.v[n] += w * res * Ji[n];
                        T.v[6 + n] += w * res * Jj[n];
                        if (opt_intr) {
                            T.F[n] += w * Ji[n] * Jf;
                            T.F[6 + n] += w * Jj[n] * Jf;
                        }
                        const size_t o = ((size_t)e * 6 + n) * HW + p;
                        if (ch == 0) { Eii[o] = 0; Eij[o] = 0; }
                        Eii[o] += wd * Jz * Ji[n];
                        Eij[o] += wd * Jz * Jj[n];
                    }
                    if (opt_intr) {
                        T.hf += w * Jf * Jf;
                        T.vf += w * res * Jf;
                    }
                }
            }
            for (int n = 0; n < 12; n++)
                for (int m = n + 1; m < 12; m++) T.H[n][m] = T.H[m][n];
        });

        // ---------------- pose system (double) ----------------
        const int dim = 6 * P + (opt_intr ? 1 : 0);
        std::vector<double> A((size_t)dim * dim, 0.0), bvec(dim, 0.0);
        auto in_range = [&](int64_t f) { return f >= t0 && f < t1; };
        for (int e = 0; e < E; e++) {
            const EdgeTerms<S>& T = terms[e];
            const int64_t fr[2] = {ii[e], jj[e]};
            for (int u = 0; u < 2; u++)
                for (int v = 0; v < 2; v++) {
                    if (!in_range(fr[u]) || !in_range(fr[v])) continue;
                    const int pu = (int)(fr[u] - t0), pv = (int)(fr[v] - t0);
                    for (int r = 0; r < 6; r++)
                        for (int c = 0; c < 6; c++)
                            A[(size_t)(6 * pu + r) * dim + 6 * pv + c] += (double)T.H[6 * u + r][6 * v + c];
                }
            for (int u = 0; u < 2; u++) {
                if (!in_range(fr[u])) continue;
                const int pu = (int)(fr[u] - t0);
                for (int r = 0; r < 6; r++) bvec[6 * pu + r] += (double)T.v[6 * u + r];
                if (opt_intr)
                    for (int r = 0; r < 6; r++) {
                        A[(size_t)(6 * pu + r) * dim + 6 * P] += (double)T.F[6 * u + r];
                        A[(size_t)(6 * P) * dim + 6 * pu + r] += (double)T.F[6 * u + r];
                    }
            }
        }
        if (opt_intr) {
            S hsum = 0, vsum = 0;
            for (int e = 0; e < E; e++) { hsum += terms[e].hf; vsum += terms[e].vf; }
            A[(size_t)(6 * P) * dim + 6 * P] += (double)hsum;
            bvec[6 * P] += (double)vsum;
        }

        // energy (before the update)
        std::vector<S> act(K), msk((size_t)K * HW);
        for (int k = 0; k < K; k++) act[k] = S(depth_active[ix.kx[k]]);
        if (!motion_only)
            for (int k = 0; k < K; k++)
                for (int p = 0; p < HW; p++)
                    msk[(size_t)k * HW + p] = (disps_sens[(size_t)ix.kx[k] * HW + p] > 0 ? S(1) : S(0)) * act[k];
        if (compute_energy) {
            S en = 0;
            for (int e = 0; e < E; e++) en += terms[e].energy;
            if (!motion_only)
                for (int k = 0; k < K; k++)
                    for (int p = 0; p < HW; p++) {
                        S dd = disps[(size_t)ix.kx[k] * HW + p] - S(disps_sens[(size_t)ix.kx[k] * HW + p]);
                        en += msk[(size_t)k * HW + p] * S(alpha) * dd * dd;
                    }
            energy_out[itr] = (double)en;
        }

        if (!motion_only) {
            // gather rows onto depth frames (accum)
            std::vector<S> C((size_t)K * HW), w((size_t)K * HW), Ef((size_t)K * HW, S(0));
            std::vector<S> Csum((size_t)K * HW, S(0)), bsum((size_t)K * HW, S(0)), Efsum((size_t)K * HW, S(0));
            for (int e = 0; e < E; e++) {
                const int k = (int)ix.kk_exp[P + e];
                for (int p = 0; p < HW; p++) {
                    Csum[(size_t)k * HW + p] += Cii[(size_t)e * HW + p];
                    bsum[(size_t)k * HW + p] += bz[(size_t)e * HW + p];
                    Efsum[(size_t)k * HW + p] += Efi[(size_t)e * HW + p];
                }
            }
            for (int k = 0; k < K; k++)
                for (int p = 0; p < HW; p++) {
                    const size_t q = (size_t)k * HW + p;
                    const S m = msk[q];
                    C[q] = act[k] * (Csum[q] + S(eta[q]) + m * S(alpha)) + (S(1) - act[k]);
                    const S dd = disps[(size_t)ix.kx[k] * HW + p] - S(disps_sens[(size_t)ix.kx[k] * HW + p]);
                    w[q] = act[k] * (bsum[q] - m * S(alpha) * dd);
                    if (opt_intr) Ef[q] = Efsum[q] * act[k];
                }
            std::vector<S> Q((size_t)K * HW);
            for (size_t q = 0; q < Q.size(); q++) Q[q] = S(1) / C[q];

            // E rows: first P rows accumulate Eii over edges with ii == t; then Eij
            std::vector<S> Erow((size_t)R * 6 * HW, S(0));
            for (int e = 0; e < E; e++) {
                const int64_t a = ii[e];
                if (in_range(a)) {
                    S* dst = &Erow[(size_t)(a - t0) * 6 * HW];
                    const S* src = &Eii[(size_t)e * 6 * HW];
                    for (int q = 0; q < 6 * HW; q++) dst[q] += src[q];
                }
                std::memcpy(&Erow[(size_t)(P + e) * 6 * HW], &Eij[(size_t)e * 6 * HW], sizeof(S) * 6 * HW);
            }
            for (int r = 0; r < R; r++) {
                const S ra = S(depth_active[ix.ii_exp[r]]);
                for (int q = 0; q < 6 * HW; q++) Erow[(size_t)r * 6 * HW + q] *= ra;
            }

            // S = E Q E^T over the enumerated pairs, v = E Q w
            const size_t npairs = spi.size();
            std::vector<double> Sblk(npairs * 36);
            parallel_for((long)npairs, [&](long n) {
                const S* Ea = &Erow[(size_t)strip[3 * n + 0] * 6 * HW];
                const S* Eb = &Erow[(size_t)strip[3 * n + 1] * 6 * HW];
                const S* q = &Q[(size_t)strip[3 * n + 2] * HW];
                for (int r = 0; r < 6; r++)
                    for (int c = 0; c < 6; c++) {
                        S s = 0;
                        for (int p = 0; p < HW; p++) s += Ea[r * HW + p] * q[p] * Eb[c * HW + p];
                        Sblk[n * 36 + r * 6 + c] = (double)s;
                    }
            });
            for (size_t n = 0; n < npairs; n++)
                for (int r = 0; r < 6; r++)
                    for (int c = 0; c < 6; c++)
                        A[(size_t)(6 * spi[n] + r) * dim + 6 * spj[n] + c] -= Sblk[n * 36 + r * 6 + c];
            for (int r = 0; r < R; r++) {
                const int64_t pj = ix.jj_exp[r];
                if (!in_range(pj)) continue;
                const int k = (int)ix.kk_exp[r];
                for (int n = 0; n < 6; n++) {
                    S s = 0;
                    for (int p = 0; p < HW; p++)
                        s += Q[(size_t)k * HW + p] * w[(size_t)k * HW + p] * Erow[((size_t)r * 6 + n) * HW + p];
                    bvec[6 * (pj - t0) + n] -= (double)s;
                }
            }
            if (opt_intr) {
                for (int r = 0; r < R; r++) {
                    const int64_t pj = ix.jj_exp[r];
                    if (!in_range(pj)) continue;
                    const int k = (int)ix.kk_exp[r];
                    for (int n = 0; n < 6; n++) {
                        S s = 0;
                        for (int p = 0; p < HW; p++)
                            s += Erow[((size_t)r * 6 + n) * HW + p] * (Q[(size_t)k * HW + p] * Ef[(size_t)k * HW + p]);
                        A[(size_t)(6 * (pj - t0) + n) * dim + 6 * P] -= (double)s;
                        A[(size_t)(6 * P) * dim + 6 * (pj - t0) + n] -= (double)s;
                    }
                }
                S sff = 0, sfw = 0;
                for (size_t q = 0; q < Q.size(); q++) {
                    sff += Ef[q] * Q[q] * Ef[q];
                    sfw += Ef[q] * Q[q] * w[q];
                }
                A[(size_t)(6 * P) * dim + 6 * P] -= (double)sff;
                bvec[6 * P] -= (double)sfw;
            }

            // damped solve
            for (int i = 0; i < dim; i++) {
                const bool sc = i >= 6 * P;
                const double l = sc ? (double)(float)intr_lm : (double)(float)lm;
                const double e0 = sc ? (double)(float)intr_ep : (double)(float)ep;
                A[(size_t)i * dim + i] += e0 + l * A[(size_t)i * dim + i];
            }
            std::vector<double> x = bvec;
            if (!cholesky_solve(A, x, dim)) std::fill(x.begin(), x.end(), 0.0);
            for (int i = 0; i < 6 * P; i++) dx_d[i] = (double)(S)x[i];
            df = opt_intr ? x[6 * P] : 0.0;

            // back substitution dz = Q (w - sum_rows E^T dx) (rows of pose t0 skipped)
            std::vector<S> dwsum((size_t)K * HW, S(0));
            for (int r = 0; r < R; r++) {
                const int64_t pr = ix.jj_exp[r] - t0;
                if (pr < (g_backsub_all_rows ? 0 : 1) || pr >= P) continue;
                const int k = (int)ix.kk_exp[r];
                for (int p = 0; p < HW; p++) {
                    S s = 0;
                    for (int n = 0; n < 6; n++) s += Erow[((size_t)r * 6 + n) * HW + p] * S(dx_d[pr * 6 + n]);
                    dwsum[(size_t)k * HW + p] += s;
                }
            }
            for (size_t q = 0; q < dz.size(); q++) {
                dz[q] = Q[q] * (w[q] - dwsum[q]);
                if (opt_intr) dz[q] = dz[q] - Q[q] * Ef[q] * S(df);
            }
            for (int t = 0; t < P; t++) {
                S xi[6];
                for (int n = 0; n < 6; n++) xi[n] = S(dx_d[t * 6 + n]);
                retract(xi, &poses[(size_t)(t0 + t) * 7]);
            }
            if (opt_intr) {
                intr[0] += S(df * intr_scale);
                intr[1] += S(df * intr_scale);
            }
            for (int k = 0; k < K; k++)
                for (int p = 0; p < HW; p++) disps[(size_t)ix.kx[k] * HW + p] += dz[(size_t)k * HW + p];
        } else {
            for (int i = 0; i < dim; i++) {
                const bool sc = i >= 6 * P;
                const double l = sc ? (double)(float)intr_lm : (double)(float)lm;
                const double e0 = sc ? (double)(float)intr_ep : (double)(float)ep;
                A[(size_t)i * dim + i] += e0 + l * A[(size_t)i * dim + i];
            }
            std::vector<double> x = bvec;
            if (!cholesky_solve(A, x, dim)) std::fill(x.begin(), x.end(), 0.0);
            for (int i = 0; i < 6 * P; i++) dx_d[i] = (double)(S)x[i];
            df = opt_intr ? x[6 * P] : 0.0;
            for (int t = 0; t < P; t++) {
                S xi[6];
                for (int n = 0; n < 6; n++) xi[n] = S(dx_d[t * 6 + n]);
                retract(xi, &poses[(size_t)(t0 + t) * 7]);
            }
            if (opt_intr) {
                intr[0] += S(df * intr_scale);
                intr[1] += S(df * intr_scale);
            }
        }
    }

    for (size_t n = 0; n < poses.size(); n++) poses_io[n] = (double)poses[n];
    for (size_t n = 0; n < disps.size(); n++) disps_io[n] = (double)disps[n];
    for (int n = 0; n < 4; n++) intr_io[n] = (double)intr[n];
    for (int n = 0; n < 6 * P; n++) dx_out[n] = dx_d[n];
    if (dz_out && !motion_only)
        for (size_t n = 0; n < dz.size(); n++) dz_out[n] = (double)dz[n];
    return 0;
}

}  // namespace

extern "C" {

void oracle_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

// Full LM bundle adjustment (restatement of ba_cuda_impl).  All buffers are
// host double arrays in the reference's layouts; poses/disps/intrinsics are
// updated in place.  use_fp64 = 0 runs FP32 arithmetic, 1 runs all-FP64.
int oracle_ba(int use_fp64, double* poses, double* disps, double* intrinsics, const double* disps_sens,
              const double* targets, const double* weights, const double* eta, const int64_t* ii,
              const int64_t* jj, const double* depth_active, int N, int H, int W, int E, int nkx, int t0, int t1,
              int iters, double lm, double ep, int motion_only, double alpha, int opt_intr, double intr_lm,
              double intr_ep, double intr_scale, int compute_energy, double* dx_out, double* dz_out,
              double* energy_out) {
    if (use_fp64)
        return run_ba<double>(poses, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active, N,
                              H, W, E, nkx, t0, t1, iters, lm, ep, motion_only, alpha, opt_intr, intr_lm, intr_ep,
                              intr_scale, compute_energy, dx_out, dz_out, energy_out);
    return run_ba<float>(poses, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active, N, H, W,
                         E, nkx, t0, t1, iters, lm, ep, motion_only, alpha, opt_intr, intr_lm, intr_ep, intr_scale,
                         compute_energy, dx_out, dz_out, energy_out);
}

// Index construction of ba_cuda_impl: kx (sorted unique depth frames) and
// kk_exp (inverse map of cat(arange(t0,t1), ii)).  Returns |kx|; arrays must
// hold at least (t1 - t0 + E) entries.
int oracle_ba_index(const int64_t* ii, const int64_t* jj, int E, int t0, int t1, int64_t* kx_out,
                    int64_t* kk_out) {
    Index ix = build_index(ii, jj, E, t0, t1);
    for (size_t n = 0; n < ix.kx.size(); n++) kx_out[n] = ix.kx[n];
    for (size_t n = 0; n < ix.kk_exp.size(); n++) kk_out[n] = ix.kk_exp[n];
    return (int)ix.kx.size();
}

// Schur pair list of schur_block (geom_kernels.cu:1440-1468).  With out
// pointers NULL returns the pair count only.
long oracle_schur_pairs(const int64_t* ii, const int64_t* jj, int E, int t0, int t1, int64_t* pi_out,
                        int64_t* pj_out, int64_t* trip_out) {
    Index ix = build_index(ii, jj, E, t0, t1);
    std::vector<int64_t> pi, pj, trip;
    schur_pairs(ix, t0, t1, pi, pj, trip);
    if (pi_out) {
        std::memcpy(pi_out, pi.data(), pi.size() * sizeof(int64_t));
        std::memcpy(pj_out, pj.data(), pj.size() * sizeof(int64_t));
        std::memcpy(trip_out, trip.data(), trip.size() * sizeof(int64_t));
    }
    return (long)pi.size();
}

// CSR of accum_cuda(data, ix = ii, jx = kx) (geom_kernels.cu:1043-1089): for each
// depth frame kx[s], the rows (edges) whose ii equals it, taken in argsort(ii)
// order (a stable sort here: ascending edge index within a frame).  Returns the
// number of depth frames; ptr_out (K+1), idx_out (E).
int oracle_accum_csr(const int64_t* ii, const int64_t* jj, int E, int t0, int t1, int64_t* ptr_out,
                     int64_t* idx_out) {
    Index ix = build_index(ii, jj, E, t0, t1);
    std::vector<int64_t> order(E);
    for (int e = 0; e < E; e++) order[e] = e;
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return ii[a] < ii[b]; });
    size_t i = 0;
    int64_t n = 0;
    ptr_out[0] = 0;
    for (size_t j = 0; j < ix.kx.size(); j++) {
        while (i < order.size() && ii[order[i]] <= ix.kx[j]) {
            if (ii[order[i]] == ix.kx[j]) idx_out[n++] = order[i];
            i++;
        }
        ptr_out[j + 1] = n;
    }
    return (int)ix.kx.size();
}

// Back-substitution rows: the reference's EvT6x1_kernel skips the rows whose
// target pose is t0 (`idx <= 0`, geom_kernels.cu:1186), although pose t0 is
// optimised.  all_rows = 1 restores them (the generic solver's Schur
// back-substitution, vipe/slam/ba/solver.py:183-186, has no such skip); the
// default 0 is the fused kernel's behaviour.
void oracle_set_backsub_all_rows(int all_rows) { g_backsub_all_rows = all_rows ? 1 : 0; }

void oracle_set_camera(int camera_model, double k1) {
    g_cam = camera_model;
    g_k1 = k1;
}

// kind 0 none, 1 Huber, 2 Tukey, 3 GNC-TLS; mu[i] is the GNC mu of iteration i (n entries)
void oracle_set_robust(int kind, double c, const double* mu, int n) {
    g_rb_kind = kind;
    g_rb_c = c;
    g_rb_mu.assign(mu, mu + (mu ? n : 0));
}

}  // extern "C"
