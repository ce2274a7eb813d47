// Proximity-edge construction of the factor graph on the GPU.
//
// Reference: FactorGraph.add_proximity_factors, vipe/slam/components/factor_graph.py:409-486,
// after the candidate distances d (from slam_ext.frame_distance) are computed.  There the
// host walks every existing edge to suppress a diamond of candidates, filters, appends the
// neighbourhood edges, argsorts d and greedily accepts candidates in a Python loop with one
// .item() synchronisation per candidate.  Here one CTA does all of it:
//   1. the suppression state is a bitmask of the (t - t0) x (t - t1) candidates in shared
//      memory (up to 1.7 M candidates: t = 1024 with t0 = t1 = 0 fits);
//   2. existing edges (active then inactive) mark their diamonds
//      |di| + |dj| <= max(min(|i - j| - 2, nms), 0) in parallel;
//   3. the neighbourhood edges are written in the reference's order (i ascending; (i, i) first
//      under cross_view; (i, j), (j, i) for j in [max(i - rad - 1, 0), i)) and mark their cells;
//   4. the candidates still alive with i - rad >= j and not d > thresh are compacted in index
//      order and sorted by distance with a stable LSD radix sort (4-bit digits, per-warp ballot
//      ranks), so equal distances keep index order (numpy's stable argsort);
//   5. warp 0 scans them in order: a candidate whose cell is still clear is accepted, emitted
//      as (i, j), (j, i), and marks its diamond, until more than max_factors edges are out.
// Integer work, deterministic, no spin-waits (every loop is bounded by the candidate count).
#include "common.cuh"

#include <algorithm>

namespace vipe {
namespace {

constexpr int kEThreads = 1024;
constexpr long kMaxCandidates = 1700L * 1024;  // the bitmask (and 4.3 KB of tables) must fit 227 KB of smem

struct EdgeArgs {
    const float* d;
    const int64_t* ii_e;
    const int64_t* jj_e;
    int n_exist;
    int t0, t1, t, rad, nms, max_factors, cross_view;
    float thresh;
    uint32_t* keys[2];
    int* vals[2];
    int64_t* ii_out;
    int64_t* jj_out;
    int* n_out;
    int cap;
};

__device__ __forceinline__ uint32_t dist_key(float v) {
    // ascending float order as unsigned order; NaN last (argsort puts NaN at the end)
    if (v != v) return 0xffffffffu;
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ void mark(uint32_t* bits, const EdgeArgs& a, int i, int j) {
    const int nj = a.t - a.t1;
    if (i >= a.t0 && i < a.t && j >= a.t1 && j < a.t) {
        const long c = (long)(i - a.t0) * nj + (j - a.t1);
        atomicOr(&bits[c >> 5], 1u << (c & 31));
    }
}

__device__ __forceinline__ bool marked(const uint32_t* bits, long c) { return (bits[c >> 5] >> (c & 31)) & 1u; }

// the cells of edge (i, j)'s suppression diamond handled by lane `lane` of `nl` lanes
__device__ __forceinline__ void mark_diamond(uint32_t* bits, const EdgeArgs& a, int i, int j, int lane, int nl) {
    const int r = max(min(abs(i - j) - 2, a.nms), 0);
    const int side = 2 * a.nms + 1;
    for (int q = lane; q < side * side; q += nl) {
        const int di = q / side - a.nms, dj = q % side - a.nms;
        if (abs(di) + abs(dj) <= r) mark(bits, a, i + di, j + dj);
    }
}

__global__ void __launch_bounds__(kEThreads, 1) proximity_edges_kernel(EdgeArgs a) {
    extern __shared__ uint32_t bits[];
    __shared__ int hist[16], run[16], tile_tot[16];
    __shared__ int wcnt[16][32], wpre[16][32];
    __shared__ int s_nv, s_all_one;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ni = a.t - a.t0, nj = a.t - a.t1;
    const long ncand = (long)ni * nj;
    const long nwords = (ncand + 31) >> 5;
    for (long w = tid; w < nwords; w += kEThreads) bits[w] = 0u;
    __syncthreads();
    // 2. existing edges: one warp per edge, lanes over the diamond
    for (int e = warp; e < a.n_exist; e += kEThreads / 32)
        mark_diamond(bits, a, (int)a.ii_e[e], (int)a.jj_e[e], lane, 32);
    // 3. neighbourhood edges, at their place in the reference's order
    for (int i = a.t0 + tid; i < a.t; i += kEThreads) {
        long pos = 0;  // edges emitted by frames t0 .. i-1
        for (int k = a.t0; k < i; k++) pos += (a.cross_view ? 1 : 0) + 2 * (k - max(k - a.rad - 1, 0));
        if (a.cross_view) {
            a.ii_out[pos] = i;
            a.jj_out[pos] = i;
            pos++;
            mark(bits, a, i, i);
        }
        for (int j = max(i - a.rad - 1, 0); j < i; j++) {
            a.ii_out[pos] = i;
            a.jj_out[pos] = j;
            a.ii_out[pos + 1] = j;
            a.jj_out[pos + 1] = i;
            pos += 2;
            mark(bits, a, i, j);
        }
    }
    __syncthreads();
    // 4a. compaction of the live candidates in index order
    if (tid == 0) s_nv = 0;
    __syncthreads();
    for (long base = 0; base < ncand; base += kEThreads) {
        const long k = base + tid;
        bool live = false;
        uint32_t key = 0;
        if (k < ncand) {
            const int i = a.t0 + (int)(k / nj), j = a.t1 + (int)(k % nj);
            const float dv = a.d[k];
            live = !(i - a.rad < j) && !(dv > a.thresh) && !marked(bits, k);
            key = dist_key(dv);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, live);
        if (lane == 0) wcnt[0][warp] = __popc(bal);
        __syncthreads();
        if (warp == 0) {
            const int v = wcnt[0][lane];
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            wpre[0][lane] = incl - v;
            if (lane == 31) tile_tot[0] = incl;
        }
        __syncthreads();
        if (live) {
            const int dst = s_nv + wpre[0][warp] + __popc(bal & ((1u << lane) - 1u));
            a.keys[0][dst] = key;
            a.vals[0][dst] = (int)k;
        }
        __syncthreads();
        if (tid == 0) s_nv += tile_tot[0];
        __syncthreads();
    }
    const int nv = s_nv;
    // 4b. stable LSD radix sort of (key, index), 4-bit digits
    int src = 0;
    for (int shift = 0; shift < 32; shift += 4) {
        if (tid < 16) hist[tid] = 0;
        __syncthreads();
        for (int k = tid; k < nv; k += kEThreads) atomicAdd(&hist[(a.keys[src][k] >> shift) & 15u], 1);
        __syncthreads();
        if (tid == 0) {
            s_all_one = 0;
            int acc = 0;
            for (int q = 0; q < 16; q++) {
                if (hist[q] == nv) s_all_one = 1;
                run[q] = acc;
                acc += hist[q];
            }
        }
        __syncthreads();
        if (s_all_one) continue;  // every key has the same digit: the order stands
        const int dst = src ^ 1;
        for (int base = 0; base < nv; base += kEThreads) {
            const int k = base + tid;
            const bool valid = k < nv;
            const uint32_t key = valid ? a.keys[src][k] : 0u;
            const int val = valid ? a.vals[src][k] : 0;
            const int dig = valid ? (int)((key >> shift) & 15u) : 16;
            int rank = 0;
            for (int dv = 0; dv < 16; dv++) {
                const unsigned bal = __ballot_sync(0xffffffffu, dig == dv);
                if (lane == 0) wcnt[dv][warp] = __popc(bal);
                if (dig == dv) rank = __popc(bal & ((1u << lane) - 1u));
            }
            __syncthreads();
            if (warp < 16) {
                const int v = wcnt[warp][lane];
                int incl = v;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                wpre[warp][lane] = incl - v;
                if (lane == 31) tile_tot[warp] = incl;
            }
            __syncthreads();
            if (valid) {
                const int o = run[dig] + wpre[dig][warp] + rank;
                a.keys[dst][o] = key;
                a.vals[dst][o] = val;
            }
            __syncthreads();
            if (tid < 16) run[tid] += tile_tot[tid];
            __syncthreads();
        }
        src = dst;
    }
    // 5. greedy scan by warp 0
    if (warp != 0) return;
    long nb = 0;
    for (int k = a.t0; k < a.t; k++) nb += (a.cross_view ? 1 : 0) + 2 * (k - max(k - a.rad - 1, 0));
    long count = nb;
    bool done = false;
    for (int base = 0; base < nv && !done; base += 32) {
        const int mine = base + lane < nv ? a.vals[src][base + lane] : -1;
        const int m = min(32, nv - base);
        for (int q = 0; q < m; q++) {
            const int k = __shfl_sync(0xffffffffu, mine, q);
            if (marked(bits, k)) continue;  // suppressed by an accepted edge (uniform across the warp)
            if (count > a.max_factors) {
                done = true;
                break;
            }
            const int i = a.t0 + k / nj, j = a.t1 + k % nj;
            if (lane == 0) {
                a.ii_out[count] = i;
                a.jj_out[count] = j;
                a.ii_out[count + 1] = j;
                a.jj_out[count + 1] = i;
            }
            count += 2;
            mark_diamond(bits, a, i, j, lane, 32);
            __syncwarp();
        }
    }
    if (lane == 0) *a.n_out = (int)count;
}

}  // namespace
}  // namespace vipe

using namespace vipe;

extern "C" size_t vipe_slam_proximity_edges_workspace_size(int t0, int t1, int t) {
    if (t1 < 0 || t0 < t1 || t <= t0) return 0;
    const long n = (long)(t - t0) * (t - t1);
    return (size_t)n * 2 * (sizeof(uint32_t) + sizeof(int)) + 256;
}

extern "C" long vipe_slam_proximity_edges_capacity(int t0, int t1, int t, int rad, int max_factors, int cross_view) {
    if (t1 < 0 || t0 < t1 || t <= t0 || rad < 0) return 0;
    long nb = 0;
    for (int k = t0; k < t; k++) nb += (cross_view ? 1 : 0) + 2 * (k - std::max(k - rad - 1, 0));
    return std::max(nb, (long)max_factors + 2);
}

extern "C" int vipe_slam_proximity_edges(const float* d, const int64_t* ii_exist, const int64_t* jj_exist,
                                         int num_exist, int t0, int t1, int t, int rad, int nms, float thresh,
                                         int max_factors, int cross_view, int64_t* ii_out, int64_t* jj_out,
                                         int out_cap, int* num_out, void* workspace, size_t workspace_bytes,
                                         void* stream) {
    if (t1 < 0 || t0 < t1 || t <= t0 || rad < 0 || nms < 0 || num_exist < 0 || max_factors < 0) return VIPE_ERR_ARG;
    if (!d || !ii_out || !jj_out || !num_out || (num_exist > 0 && (!ii_exist || !jj_exist))) return VIPE_ERR_ARG;
    const long ncand = (long)(t - t0) * (t - t1);
    if (ncand > kMaxCandidates) {
        set_last_error("proximity edges: more than 1.7 M candidate pairs (t - t0) x (t - t1)");
        return VIPE_ERR_CAPACITY;
    }
    if ((long)out_cap < vipe_slam_proximity_edges_capacity(t0, t1, t, rad, max_factors, cross_view))
        return VIPE_ERR_ARG;
    const size_t need = vipe_slam_proximity_edges_workspace_size(t0, t1, t);
    if (!workspace || workspace_bytes < need) return VIPE_ERR_WORKSPACE;
    EdgeArgs a{};
    a.d = d;
    a.ii_e = ii_exist;
    a.jj_e = jj_exist;
    a.n_exist = num_exist;
    a.t0 = t0; a.t1 = t1; a.t = t; a.rad = rad; a.nms = nms;
    a.max_factors = max_factors;
    a.cross_view = cross_view ? 1 : 0;
    a.thresh = thresh;
    char* ws = static_cast<char*>(workspace);
    a.keys[0] = reinterpret_cast<uint32_t*>(ws);
    a.keys[1] = a.keys[0] + ncand;
    a.vals[0] = reinterpret_cast<int*>(a.keys[1] + ncand);
    a.vals[1] = a.vals[0] + ncand;
    a.ii_out = ii_out;
    a.jj_out = jj_out;
    a.n_out = num_out;
    a.cap = out_cap;
    const size_t smem = (size_t)((ncand + 31) >> 5) * sizeof(uint32_t);
    cudaStream_t st = as_stream(stream);
    VIPE_CUDA_TRY(cudaFuncSetAttribute(proximity_edges_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)std::max<size_t>(smem, 4)));
    VIPE_PROF("proximity_edges", st);
    proximity_edges_kernel<<<1, kEThreads, smem, st>>>(a);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}
