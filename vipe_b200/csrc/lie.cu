// Lie-group kernels: SO3, RxSO3, SE3, Sim3 (float / double) — drop-in for the
// reference's lietorch_ext (vipe csrc/lietorch_ext/lietorch.cpp:306-336,
// kernels lietorch_gpu.cu:24-298, group math so3.h / rxso3.h / se3.h / sim3.h).
//
// Storage (as in the reference): SO3 [qx qy qz qw], RxSO3 [qx qy qz qw s],
// SE3 [tx ty tz qx qy qz qw], Sim3 [tx ty tz qx qy qz qw s]; tangents
// SO3 [phi], RxSO3 [phi sigma], SE3 [tau phi], Sim3 [tau phi sigma].  Loading an
// element normalises its quaternion, as the reference's constructors do.
//
// The group algebra is written here on small register arrays (no Eigen):
// closed-form exponential/logarithm (atan-based SO3 log), adjoint matrices,
// left Jacobians (SE3 via the Q block, Sim3 via its truncated series), the
// RxSO3 "W" matrix of the Sim3 exponential, point actions and their Jacobians.
// Gradients with respect to group elements use row stride N with the first K
// entries meaningful (reference convention, lietorch_gpu.cu:37-98).
//
// One thread per group element, grid-stride; the ops are elementwise and
// memory-bound: bytes per element = (inputs + outputs) * sizeof(scalar).

#include "lie_group.cuh"

namespace vipe {
namespace lie {

template <typename G, typename S>
__global__ void lie_kernel(int op, int64_t n, const S* __restrict__ in0, const S* __restrict__ in1,
                           const S* __restrict__ in2, S* __restrict__ out0, S* __restrict__ out1) {
    constexpr int N = G::N, K = G::K;
    LIE_LOOP(i, n) {
        switch (op) {
            case kExp: {
                G::Exp(in0 + i * K).store(out0 + i * N);
                break;
            }
            case kExpB: {  // in0 grad (stride N), in1 a
                const Mat<S, K, K> J = G::left_jac(in1 + i * K);
                vm(in0 + i * N, J, out0 + i * K);
                break;
            }
            case kLog: {
                G::load(in0 + i * N).Log(out0 + i * K);
                break;
            }
            case kLogB: {  // in0 grad (stride K), in1 X -> dX (stride N)
                S a[K];
                G::load(in1 + i * N).Log(a);
                const Mat<S, K, K> J = G::left_jac_inv(a);
                S g[K];
                vm(in0 + i * K, J, g);
#pragma unroll
                for (int k = 0; k < N; k++) out0[i * N + k] = k < K ? g[k] : S(0);
                break;
            }
            case kInv: {
                G::load(in0 + i * N).inv().store(out0 + i * N);
                break;
            }
            case kInvB: {  // in0 grad (stride N), in1 X
                const Mat<S, K, K> A = G::load(in1 + i * N).inv().Adj();
                S g[K];
                vm(in0 + i * N, A, g);
#pragma unroll
                for (int k = 0; k < N; k++) out0[i * N + k] = k < K ? -g[k] : S(0);
                break;
            }
            case kMul: {
                (G::load(in0 + i * N) * G::load(in1 + i * N)).store(out0 + i * N);
                break;
            }
            case kMulB: {  // in0 grad (stride N), in1 X, in2 Y
                const Mat<S, K, K> A = G::load(in1 + i * N).Adj();
                S g[K];
                vm(in0 + i * N, A, g);
#pragma unroll
                for (int k = 0; k < N; k++) {
                    out0[i * N + k] = k < K ? in0[i * N + k] : S(0);
                    out1[i * N + k] = k < K ? g[k] : S(0);
                }
                break;
            }
            case kAdj: {
                mv(G::load(in0 + i * N).Adj(), in1 + i * K, out0 + i * K);
                break;
            }
            case kAdjB: {  // in0 db (stride K), in1 X, in2 a -> dX (stride N), da
                const Mat<S, K, K> A = G::load(in1 + i * N).Adj();
                S b[K], gx[K];
                mv(A, in2 + i * K, b);
                vm(in0 + i * K, A, out1 + i * K);
                vm(in0 + i * K, G::adj(b), gx);
#pragma unroll
                for (int k = 0; k < N; k++) out0[i * N + k] = k < K ? -gx[k] : S(0);
                break;
            }
            case kAdjT: {
                const Mat<S, K, K> A = G::load(in0 + i * N).Adj();
                vm(in1 + i * K, A, out0 + i * K);  // A^T a
                break;
            }
            case kAdjTB: {  // in0 db (stride K), in1 X, in2 a -> dX (stride N), da
                const Mat<S, K, K> A = G::load(in1 + i * N).Adj();
                S c[K], gx[K];
                mv(A, in0 + i * K, c);
#pragma unroll
                for (int k = 0; k < K; k++) out1[i * K + k] = c[k];
                vm(in2 + i * K, G::adj(c), gx);
#pragma unroll
                for (int k = 0; k < N; k++) out0[i * N + k] = k < K ? -gx[k] : S(0);
                break;
            }
            case kAct: {
                G::load(in0 + i * N).act(in1 + i * 3, out0 + i * 3);
                break;
            }
            case kActB: {  // in0 dq (stride 3), in1 X, in2 p -> dX (stride N), dp
                const G X = G::load(in1 + i * N);
                S q[3], gx[K];
                X.act(in2 + i * 3, q);
                vm(in0 + i * 3, X.mat3(), out1 + i * 3);
                vm(in0 + i * 3, G::act_jac(q), gx);
#pragma unroll
                for (int k = 0; k < N; k++) out0[i * N + k] = k < K ? gx[k] : S(0);
                break;
            }
            case kAct4: {
                G::load(in0 + i * N).act4(in1 + i * 4, out0 + i * 4);
                break;
            }
            case kAct4B: {  // in0 dq (stride 4), in1 X, in2 p -> dX (stride N), dp
                const G X = G::load(in1 + i * N);
                S q[4], gx[K];
                X.act4(in2 + i * 4, q);
                vm(in0 + i * 4, X.mat4(), out1 + i * 4);
                vm(in0 + i * 4, G::act4_jac(q), gx);
#pragma unroll
                for (int k = 0; k < N; k++) out0[i * N + k] = k < K ? gx[k] : S(0);
                break;
            }
            case kMatrix: {
                const Mat<S, 4, 4> T = G::load(in0 + i * N).mat4();
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int c = 0; c < 4; c++) out0[i * 16 + r * 4 + c] = T.m[r][c];
                break;
            }
            case kProj: {
                const Mat<S, N, N> J = G::load(in0 + i * N).projector();
#pragma unroll
                for (int r = 0; r < N; r++)
#pragma unroll
                    for (int c = 0; c < N; c++) out0[i * N * N + r * N + c] = J.m[r][c];
                break;
            }
            case kJinv: {
                S a[K];
                G::load(in0 + i * N).Log(a);
                mv(G::left_jac_inv(a), in1 + i * K, out0 + i * K);
                break;
            }
            default:
                break;
        }
    }
}

template <typename S>
int launch_typed(int group, int op, int64_t n, const void* a, const void* b, const void* c, void* o0, void* o1,
                 cudaStream_t st) {
    if (n <= 0) return VIPE_OK;
    const int threads = 256;
    const int64_t want = (n + threads - 1) / threads;
    const int blocks = (int)(want < 148 * 32 ? want : 148 * 32);
    const S* i0 = static_cast<const S*>(a);
    const S* i1 = static_cast<const S*>(b);
    const S* i2 = static_cast<const S*>(c);
    S* q0 = static_cast<S*>(o0);
    S* q1 = static_cast<S*>(o1);
    VIPE_PROF("lie", st);
    switch (group) {
        case 1: lie_kernel<SO3<S>, S><<<blocks, threads, 0, st>>>(op, n, i0, i1, i2, q0, q1); break;
        case 2: lie_kernel<RxSO3<S>, S><<<blocks, threads, 0, st>>>(op, n, i0, i1, i2, q0, q1); break;
        case 3: lie_kernel<SE3<S>, S><<<blocks, threads, 0, st>>>(op, n, i0, i1, i2, q0, q1); break;
        case 4: lie_kernel<Sim3<S>, S><<<blocks, threads, 0, st>>>(op, n, i0, i1, i2, q0, q1); break;
        default: return VIPE_ERR_GROUP;
    }
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

int launch(int group, int dtype, int op, int64_t n, const void* a, const void* b, const void* c, void* o0, void* o1,
           void* stream) {
    if (group < 1 || group > 4) return VIPE_ERR_GROUP;
    if (n < 0) return VIPE_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    if (dtype == VIPE_F32) return launch_typed<float>(group, op, n, a, b, c, o0, o1, st);
    if (dtype == VIPE_F64) return launch_typed<double>(group, op, n, a, b, c, o0, o1, st);
    return VIPE_ERR_DTYPE;
}

}  // namespace lie
}  // namespace vipe

using vipe::lie::launch;
namespace L = vipe::lie;

extern "C" {
int vipe_lie_expm(int g, int dt, int64_t b, const void* a, void* X, void* s) {
    return launch(g, dt, L::kExp, b, a, nullptr, nullptr, X, nullptr, s);
}
int vipe_lie_expm_backward(int g, int dt, int64_t b, const void* grad, const void* a, void* da, void* s) {
    return launch(g, dt, L::kExpB, b, grad, a, nullptr, da, nullptr, s);
}
int vipe_lie_logm(int g, int dt, int64_t b, const void* X, void* a, void* s) {
    return launch(g, dt, L::kLog, b, X, nullptr, nullptr, a, nullptr, s);
}
int vipe_lie_logm_backward(int g, int dt, int64_t b, const void* grad, const void* X, void* dX, void* s) {
    return launch(g, dt, L::kLogB, b, grad, X, nullptr, dX, nullptr, s);
}
int vipe_lie_inv(int g, int dt, int64_t b, const void* X, void* Y, void* s) {
    return launch(g, dt, L::kInv, b, X, nullptr, nullptr, Y, nullptr, s);
}
int vipe_lie_inv_backward(int g, int dt, int64_t b, const void* grad, const void* X, void* dX, void* s) {
    return launch(g, dt, L::kInvB, b, grad, X, nullptr, dX, nullptr, s);
}
int vipe_lie_mul(int g, int dt, int64_t b, const void* X, const void* Y, void* Z, void* s) {
    return launch(g, dt, L::kMul, b, X, Y, nullptr, Z, nullptr, s);
}
int vipe_lie_mul_backward(int g, int dt, int64_t b, const void* grad, const void* X, const void* Y, void* dX,
                          void* dY, void* s) {
    return launch(g, dt, L::kMulB, b, grad, X, Y, dX, dY, s);
}
int vipe_lie_adj(int g, int dt, int64_t b, const void* X, const void* a, void* out, void* s) {
    return launch(g, dt, L::kAdj, b, X, a, nullptr, out, nullptr, s);
}
int vipe_lie_adj_backward(int g, int dt, int64_t b, const void* grad, const void* X, const void* a, void* dX,
                          void* da, void* s) {
    return launch(g, dt, L::kAdjB, b, grad, X, a, dX, da, s);
}
int vipe_lie_adjT(int g, int dt, int64_t b, const void* X, const void* a, void* out, void* s) {
    return launch(g, dt, L::kAdjT, b, X, a, nullptr, out, nullptr, s);
}
int vipe_lie_adjT_backward(int g, int dt, int64_t b, const void* grad, const void* X, const void* a, void* dX,
                           void* da, void* s) {
    return launch(g, dt, L::kAdjTB, b, grad, X, a, dX, da, s);
}
int vipe_lie_act(int g, int dt, int64_t b, const void* X, const void* p, void* q, void* s) {
    return launch(g, dt, L::kAct, b, X, p, nullptr, q, nullptr, s);
}
int vipe_lie_act_backward(int g, int dt, int64_t b, const void* grad, const void* X, const void* p, void* dX,
                          void* dp, void* s) {
    return launch(g, dt, L::kActB, b, grad, X, p, dX, dp, s);
}
int vipe_lie_act4(int g, int dt, int64_t b, const void* X, const void* p, void* q, void* s) {
    return launch(g, dt, L::kAct4, b, X, p, nullptr, q, nullptr, s);
}
int vipe_lie_act4_backward(int g, int dt, int64_t b, const void* grad, const void* X, const void* p, void* dX,
                           void* dp, void* s) {
    return launch(g, dt, L::kAct4B, b, grad, X, p, dX, dp, s);
}
int vipe_lie_as_matrix(int g, int dt, int64_t b, const void* X, void* T, void* s) {
    return launch(g, dt, L::kMatrix, b, X, nullptr, nullptr, T, nullptr, s);
}
int vipe_lie_projector(int g, int dt, int64_t b, const void* X, void* P, void* s) {
    return launch(g, dt, L::kProj, b, X, nullptr, nullptr, P, nullptr, s);
}
int vipe_lie_Jinv(int g, int dt, int64_t b, const void* X, const void* a, void* out, void* s) {
    return launch(g, dt, L::kJinv, b, X, a, nullptr, out, nullptr, s);
}
}
