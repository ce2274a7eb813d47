// Internals shared by the bundle-adjustment translation units (ba.cu: index
// build, linearisation, assembly, Cholesky, update; ba_adjoint.cu: the
// hand-written adjoint).  Not part of the C ABI.
#pragma once

#include "common.cuh"
#include "lie_group.cuh"
#include "se3_device.cuh"

#include <algorithm>
#include <vector>

namespace vipe {
namespace ba {

constexpr int kMaxSlots = 31;          // window poses coupled to one depth frame that the tensor-core
                                       // frame kernel takes (SE3; Sim3: 27): 2 x (accumulator
                                       // columns) <= 512; a single graph's wider frames take the
                                       // wide-frame kernel, a batch refuses them
constexpr int kMaxPoses = 1024;        // t1 - t0 of a single graph (the index kernel's pose bitmask);
                                       // batches: 6P+1 unknowns must fit the staged Cholesky panel
constexpr int kWideTile = 64;          // output block of the wide-frame Gram product
constexpr int kWideGroup = 8;          // wide frames staged and multiplied together
constexpr int kNT = 105;               // per-edge terms, see term layout below
constexpr int kEdgeThreads = 256;
constexpr int kFrameThreads = 128;     // one pixel per thread; 32-pixel blocks per warp
constexpr int kIndexThreads = 1024;
constexpr int kEdgeCache = 64;        // edges of a depth frame whose per-edge constants a CTA caches
constexpr int kAdjMaxChunk = 1536;    // pixels of one (frame, chunk) block of the adjoint frame kernels
// the plan's pixel chunk for adjoint plans: SE3 1536; Sim3 1024, so that the second adjoint frame
// kernel's per-pixel arrays (one more float per pixel) and 100-float edge rows leave room for
// two CTAs per SM
__host__ __device__ constexpr int adj_plan_chunk(int dof) { return dof == 7 ? 1024 : kAdjMaxChunk; }

// per-edge term layout
//   [0,78)   upper triangle (row-major, n >= m) of the 12x12 block [Ji Jj]^T W [Ji Jj]
//   [78,84)  vi     [84,90) vj     [90,96) fi    [96,102) fj
//   102 hf   103 vf   104 flow energy
constexpr int kTV = 78, kTF = 90, kTHF = 102, kTVF = 103, kTEN = 104;

__host__ __device__ inline int tri12(int r, int c) { return r >= c ? r * (r + 1) / 2 + c : c * (c + 1) / 2 + r; }

struct Dims {
    int N, H, W, HW, E, K, t0, t1, P, dim;
    int kx0, kx1;      // frames [kx0, kx1) join kx with the edges' sources (= [t0, t1) except for
                       // a rig solve that optimises the rig, whose pose window spans every frame)
    int CHe, chunk_e;  // edge kernel pixel chunks
    int CF, chunk_f;   // frame kernel pixel chunks
    long tile_cap;     // capacity of frame SYRK tiles (tensor-core frames, per pixel chunk)
    long wtile_cap;    // capacity of wide-frame Gram tiles (summed over pixel chunks)
    int adj;           // 1: the workspace also holds the adjoint buffers
    int dof;           // pose tangent size: 6 (SE3) or 7 (Sim3)
    int wide;          // 1: depth frames may couple more than max_slots window poses (single SE3
                       // graphs with P > max_slots): those frames take the wide-frame kernel
};

// Per-edge term layouts for pose tangent size `dof`:
//   chunk partials (ne_of):  Hjj upper triangle (dof(dof+1)/2), vj, fj, hf, vf, energy
//   FP64 terms (nt_of):      upper triangle of the (2 dof)^2 block [Ji Jj]^T W [Ji Jj],
//                            [vi; vj], [fi; fj], hf, vf, energy
__host__ __device__ inline int ne_of(int dof) { return dof * (dof + 1) / 2 + 2 * dof + 3; }
__host__ __device__ inline int tri_of(int dof) { return (2 * dof) * (2 * dof + 1) / 2; }
__host__ __device__ inline int nt_of(int dof) { return tri_of(dof) + 4 * dof + 3; }
__host__ __device__ inline int tv_of(int dof) { return tri_of(dof); }
__host__ __device__ inline int tf_of(int dof) { return tri_of(dof) + 2 * dof; }
__host__ __device__ inline int thf_of(int dof) { return tri_of(dof) + 4 * dof; }
__host__ __device__ inline int max_slots(int dof) { return dof == 6 ? kMaxSlots : 27; }
constexpr int kMaxNE = 45;  // ne_of(7)

struct Work {
    int* status;   // [0] error code
    int* meta;     // [0] nkx [1] sum_m [2] sum_tiles [3] max_m
    int* flag;
    int* rank;
    int* kx;
    int* fe_ptr;
    int* fe_list;
    int* edge_slot;
    int* fp_ptr;
    int* fp_list;
    int* self_slot;
    int* ftile_off;
    int* pe_ptr;
    int* pe_list;
    int* pf_ptr;
    int* pf_list;
    float* epart;    // E * CHe * kNT
    double* eterm;   // E * kNT
    float* spart;    // tile_cap * CF * 16
    float* fen;      // K * CF
    float* qwf;      // K * HW * 3
    double* Hm;      // dim * dim
    double* bv;      // dim
    double* df;      // 1
    double* linv;    // inverse diagonal blocks of the Cholesky factor
    double* yv;      // dim: forward-substitution result of the multi-launch Cholesky
    int* wide_list;  // K: depth rows whose slot count exceeds max_slots (wide frames), ascending
    float* ebuf;     // kWideGroup x (dof * P + 3) x chunk_f: wide frames' scaled rows e_p over one pixel chunk
    int* wtile_off;  // K + 1: first Gram tile of each wide frame in wtile
    float* wtile;    // wtile_cap x 16: wide frames' upper-triangle 4 x 4 Gram tiles, all chunks summed
    // adjoint (carved only when Dims::adj)
    double* adj_gT;    // N * dof running left-tangent gradient of every pose
    double* adj_rhs;   // dim     g_dxi, then g_dxi - E~ Q g_dz
    double* adj_lam;   // dim     lambda = S'^-1 rhs
    float* adj_aslot;  // E * CF * 2 dof  per (edge, pixel chunk): sum a act wd Jz [Ji, Jj]
    float* adj_gpart;  // E * CF * kAdjAcc  per (edge, pixel chunk) pose-gradient moments
    double* adj_gedge; // E * 2 dof  per-edge pose gradient [source pose, target pose]
};

constexpr int kAdjAcc = 48;  // 4 moment matrices of 3 x 4 per edge

__host__ __device__ inline int npt_of(int m, int dof = 6) {
    int nt = (dof * m + 2 + 3) / 4;
    return nt * (nt + 1) / 2;
}

// slots (window poses) a depth frame of graph d may couple: the tensor-core frame kernel's
// limit, or any number up to the window for graphs that take the wide-frame kernel
__host__ __device__ inline int slot_cap(const Dims& d) { return d.wide ? d.P : max_slots(d.dof); }

// rows of the wide-frame staging buffer: one frame's entries at most, plus one row of
// per-pixel depth-prior energies
__host__ __device__ inline long wide_rows(const Dims& d) { return d.wide ? (long)d.dof * d.P + 3 : 0; }

// che / cf: pixel-chunk counts of the per-edge and per-frame kernels; 0 picks
// them so that one graph alone launches about two CTAs per SM.  single: a graph
// solved on its own (not in a batch), which may hold wide frames.
inline Dims make_dims(int N, int H, int W, int E, int K, int t0, int t1, int che = 0, int cf = 0, int dof = 6,
                      bool single = false) {
    Dims d;
    d.N = N; d.H = H; d.W = W; d.HW = H * W; d.E = E; d.K = K; d.t0 = t0; d.t1 = t1;
    d.kx0 = t0; d.kx1 = t1;
    d.P = t1 - t0;
    d.dof = dof;
    d.dim = dof * d.P + 1;
    const int target = 2 * 148;
    if (che <= 0) che = E > 0 ? (target + E - 1) / E : 1;
    che = std::max(1, std::min(che, std::max(1, d.HW / 1024)));
    d.chunk_e = (d.HW + che - 1) / che;
    d.CHe = (d.HW + d.chunk_e - 1) / d.chunk_e;
    if (cf <= 0) cf = K > 0 ? (target + K - 1) / K : 1;
    cf = std::max(1, std::min(cf, 8));
    int chunk = (d.HW + cf - 1) / cf;
    chunk = ((chunk + 255) / 256) * 256;
    d.chunk_f = chunk;
    d.CF = (d.HW + chunk - 1) / chunk;
    d.wide = (single && dof == 6 && d.P > max_slots(dof)) ? 1 : 0;
    // Upper bound of sum over frames of npt(m_s): slots are <= M per frame and
    // sum_s m_s <= E + K.  npt(m) <= (a m + 3.25)^2 / 2, a = dof / 4.
    auto tiles_bound = [&](int M) {
        M = std::max(1, std::min(M, d.P));
        const double a = dof / 4.0;
        const double b1 = (double)K * npt_of(M, dof);
        const double b2 = (a * M + 3.25) / 2.0 * (a * (double)(E + K) + 3.25 * K);
        return (long)std::min(b1, b2) + K + 1;
    };
    d.tile_cap = tiles_bound(max_slots(dof));
    d.wtile_cap = d.wide ? tiles_bound(d.P) : 1;
    d.adj = 0;
    return d;
}

template <typename C>
inline void carve(C& c, const Dims& d, Work* w) {
    const size_t N = d.N, E = d.E, K = d.K, P = d.P;
    auto take_i = [&](int*& dst, size_t n) {
        auto p = c.template take<int>(n);
        if (w) dst = (int*)p;
    };
    int* dummy;
    take_i(w ? w->status : dummy, 4);
    take_i(w ? w->meta : dummy, 8);
    take_i(w ? w->flag : dummy, N);
    take_i(w ? w->rank : dummy, N);
    take_i(w ? w->kx : dummy, N);
    take_i(w ? w->fe_ptr : dummy, K + 1);
    take_i(w ? w->fe_list : dummy, E + 1);
    take_i(w ? w->edge_slot : dummy, E + 1);
    take_i(w ? w->fp_ptr : dummy, K + 1);
    take_i(w ? w->fp_list : dummy, E + K + 1);
    take_i(w ? w->self_slot : dummy, K + 1);
    take_i(w ? w->ftile_off : dummy, K + 1);
    take_i(w ? w->pe_ptr : dummy, P + 1);
    take_i(w ? w->pe_list : dummy, 2 * E + 1);
    take_i(w ? w->pf_ptr : dummy, P + 1);
    take_i(w ? w->pf_list : dummy, E + K + 1);
    auto pf = c.template take<float>((size_t)std::max<size_t>(1, E) * d.CHe * ne_of(d.dof));
    auto pd = c.template take<double>((size_t)std::max<size_t>(1, E) * nt_of(d.dof));
    auto ps = c.template take<float>((size_t)d.tile_cap * d.CF * 16);
    auto pen = c.template take<float>(K * d.CF + 1);
    auto pq = c.template take<float>(K * (size_t)d.HW * 3);
    auto pH = c.template take<double>((size_t)d.dim * d.dim);
    auto pb = c.template take<double>((size_t)d.dim);
    auto pdf = c.template take<double>(4);
    auto pli = c.template take<double>((size_t)((d.dim + 31) / 32) * 32 * 32);
    auto pyv = c.template take<double>((size_t)d.dim);
    auto pwl = c.template take<int>(K + 1);
    auto peb = c.template take<float>(d.wide ? (size_t)kWideGroup * wide_rows(d) * d.chunk_f : 1);
    auto pwo = c.template take<int>(K + 1);
    auto pwt = c.template take<float>((size_t)d.wtile_cap * 16);
    if (w) {
        w->epart = (float*)pf;
        w->eterm = (double*)pd;
        w->spart = (float*)ps;
        w->fen = (float*)pen;
        w->qwf = (float*)pq;
        w->Hm = (double*)pH;
        w->bv = (double*)pb;
        w->df = (double*)pdf;
        w->linv = (double*)pli;
        w->yv = (double*)pyv;
        w->wide_list = (int*)pwl;
        w->ebuf = (float*)peb;
        w->wtile_off = (int*)pwo;
        w->wtile = (float*)pwt;
        w->adj_gT = nullptr;
        w->adj_rhs = w->adj_lam = nullptr;
        w->adj_aslot = w->adj_gpart = nullptr;
        w->adj_gedge = nullptr;
    }
    if (d.adj) {
        const size_t D = d.dof;
        auto g1 = c.template take<double>(N * D);
        auto g2 = c.template take<double>((size_t)d.dim);
        auto g3 = c.template take<double>((size_t)d.dim);
        auto g4 = c.template take<float>((size_t)std::max<size_t>(1, E) * d.CF * 2 * D);
        auto g5 = c.template take<float>((size_t)std::max<size_t>(1, E) * d.CF * kAdjAcc);
        auto g6 = c.template take<double>((size_t)std::max<size_t>(1, E) * 2 * D);
        if (w) {
            w->adj_gT = (double*)g1;
            w->adj_rhs = (double*)g2;
            w->adj_lam = (double*)g3;
            w->adj_aslot = (float*)g4;
            w->adj_gpart = (float*)g5;
            w->adj_gedge = (double*)g6;
        }
    }
}

// ---------------------------------------------------------------- graph table
//
// Every kernel runs over a table of graphs.  A single solve is a table of one;
// a batch places many clips' graphs side by side: inputs are concatenated
// along their leading axis (frames, edges, depth rows, window poses) and each
// graph's descriptor holds its sizes, its carve of the workspace and its
// offsets into the concatenated tensors.  Edge indices stay local to their
// graph.  A launch over the batch is one flat grid: per kernel, boff[g] is the
// first block of graph g (boff[G] = total), found by binary search.

struct BAPtrs {
    float* poses;              // (frames, 7)
    float* disps;              // (frames, H, W)
    float* intr;               // (graphs, 4)
    const float* disps_sens;   // (frames, H, W)
    const float* targets;      // (edges, 2, H, W)
    const float* weights;      // (edges, 2, H, W)
    const float* eta;          // (depth rows, H, W)
    const int64_t* ii;         // (edges,) local frame index
    const int64_t* jj;
    const float* depth_active; // (frames,)
    float* dx;                 // (window poses, 6)
    float* dz;                 // (depth rows, H*W)
    float* energy;             // (graphs, energy_stride)
    int32_t* status;           // device status word(s): graph g uses status[g * status_stride]
    int energy_stride;
    int status_stride;
    // adjoint inputs/outputs (frames/edges/depth rows concatenated like the inputs)
    float* g_poses;    // (frames, 7) in: d loss / d poses_out; out: d loss / d poses_in (left tangent, [6] = 0)
    float* g_disps;    // (frames, H, W) in: d loss / d disps_out; out: d loss / d disps_in
    float* g_targets;  // (edges, 2, H, W) out (accumulated)
    float* g_weights;  // (edges, 2, H, W) out (accumulated)
    float* g_eta;      // (depth rows, H, W) out (accumulated)
    float* g_dsens;    // (frames, H, W) out (accumulated)
    double* ftape;     // one iteration of the tape record (graph slots at ftape_off): factor, (Q, w)
    RobustSpec rb;     // robust reweighting of the flow residuals (kind 0: none)
    int exact_backsub; // 1: the depth back-substitution keeps the rows of pose t0 (the generic
                       // solver's Schur back-substitution); 0: skips them like the reference's
                       // fused kernel (geom_kernels.cu:1186)
};

// factor tape slot of one graph: the Cholesky factor (dim x dim, lower
// triangle used), the inverse diagonal blocks, and the failure flag ...
__host__ __device__ inline long factor_slot_doubles(const Dims& d) {
    return (long)d.dim * d.dim + (long)((d.dim + 31) / 32) * 32 * 32 + 2;
}
// ... followed by the depth elimination's per-pixel (Q, w) of every depth row,
// (K, HW) float pairs, as the forward frame kernel formed them
__host__ __device__ inline long tape_slot_doubles(const Dims& d) { return factor_slot_doubles(d) + (long)d.K * d.HW; }
__device__ __forceinline__ float2* tape_qw(double* slot, const Dims& d) {
    return reinterpret_cast<float2*>(slot + factor_slot_doubles(d));
}

struct GraphDesc {
    Dims d;
    Work w;
    long frame_off, edge_off, kx_off, pose_off;
    long ftape_off;  // doubles: this graph's slot in one iteration of the factor tape
    int g;
};

struct Batch {
    const GraphDesc* gds;  // device table
    const int* boff;       // per-kernel block offsets, or nullptr (see locate)
    int G;
    const int* order = nullptr;  // per-graph grids: block slot b runs graph order[b] (else graph b)
    int blocks_per_graph = 1;    // per-graph grids: consecutive blocks of one graph (a cluster)
};

// Graph of this block.  With boff: flat grid over all graphs.  Without: a
// single graph (G == 1, local = blockIdx.x) or blocks_per_graph consecutive
// blocks per graph (slot = blockIdx.x / blocks_per_graph, in `order` when given).
__device__ __forceinline__ int locate(const Batch& B, int& local) {
    if (B.boff == nullptr) {
        if (B.G == 1) {
            local = blockIdx.x;
            return 0;
        }
        const int slot = (int)blockIdx.x / B.blocks_per_graph;
        local = (int)blockIdx.x % B.blocks_per_graph;
        return B.order ? __ldg(B.order + slot) : slot;
    }
    const int x = blockIdx.x;
    int lo = 0, hi = B.G;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(B.boff + mid) <= x) lo = mid; else hi = mid;
    }
    local = x - __ldg(B.boff + lo);
    return lo;
}

__device__ __forceinline__ BAPtrs rebase(const BAPtrs& b, const GraphDesc& g) {
    const long HW = g.d.HW;
    BAPtrs p;
    p.poses = b.poses + g.frame_off * (g.d.dof + 1);
    p.disps = b.disps + g.frame_off * HW;
    p.intr = b.intr + (long)g.g * 4;
    p.disps_sens = b.disps_sens + g.frame_off * HW;
    p.targets = b.targets ? b.targets + g.edge_off * 2 * HW : nullptr;
    p.weights = b.weights ? b.weights + g.edge_off * 2 * HW : nullptr;
    p.eta = b.eta + g.kx_off * HW;
    p.ii = b.ii ? b.ii + g.edge_off : nullptr;
    p.jj = b.jj ? b.jj + g.edge_off : nullptr;
    p.depth_active = b.depth_active + g.frame_off;
    p.dx = b.dx + g.pose_off * g.d.dof;
    p.dz = b.dz ? b.dz + g.kx_off * HW : nullptr;
    p.energy = b.energy ? b.energy + (long)g.g * b.energy_stride : nullptr;
    p.status = b.status ? b.status + (long)g.g * b.status_stride : nullptr;
    p.energy_stride = b.energy_stride;
    p.status_stride = b.status_stride;
    p.g_poses = b.g_poses ? b.g_poses + g.frame_off * (g.d.dof + 1) : nullptr;
    p.g_disps = b.g_disps ? b.g_disps + g.frame_off * HW : nullptr;
    p.g_targets = b.g_targets ? b.g_targets + g.edge_off * 2 * HW : nullptr;
    p.g_weights = b.g_weights ? b.g_weights + g.edge_off * 2 * HW : nullptr;
    p.g_eta = b.g_eta ? b.g_eta + g.kx_off * HW : nullptr;
    p.g_dsens = b.g_dsens ? b.g_dsens + g.frame_off * HW : nullptr;
    p.ftape = b.ftape ? b.ftape + g.ftape_off : nullptr;
    p.rb = b.rb;
    p.exact_backsub = b.exact_backsub;
    return p;
}

// binds d, w, P (rebased pointers) and local_ (block index within the graph)
#define BA_BIND(B, base)                                \
    int local_;                                         \
    const int g_ = locate(B, local_);                   \
    const GraphDesc* __restrict__ gd_ = (B).gds + g_;   \
    const Dims d = gd_->d;                              \
    const Work w = gd_->w;                              \
    const BAPtrs io = rebase(base, *gd_);                \
    (void)io;                                           \
    (void)d;

struct EdgeArgs {
    const float* poses;
    const float* disps;
    const float* intr;
    const float* targets;
    const float* weights;
    const int64_t* ii;
    const int64_t* jj;
    float iscale;
};

// Per-pixel accumulation needs only the target-pose block: the source-pose
// Jacobian of every pixel is Ji = -M Jj with M = Ad^T(Tij) constant per edge
// (the adjoint pull-back used by the reference, geom_kernels.cu:88-102), so
//   Hii = M Hjj M^T,  Hij = -M Hjj,  vi = -M vj,  fi = -M fj.
// Chunk partial layout (kNE floats): [0,21) Hjj upper triangle (n >= m),
// [21,27) vj, [27,33) fj, 33 hf, 34 vf, 35 flow energy.
constexpr int kNE = 36;

__host__ __device__ inline int tri6(int r, int c) { return r >= c ? r * (r + 1) / 2 + c : c * (c + 1) / 2 + r; }

struct FrameArgs {
    const float* poses;
    const float* disps;
    const float* disps_sens;
    const float* intr;
    const float* targets;
    const float* weights;
    const float* eta;
    const float* depth_active;
    const int64_t* jj;
    float alpha;
    float iscale;
};

constexpr int kCholThreads = 256;
constexpr int kNB = 32;
constexpr int kPanelRows = 768;  // systems up to 768 unknowns stage their panel in shared memory

__host__ __device__ inline int chol_ldr(int dim) {
    // transposed panel row length: >= max(dim, 32) + 4 (tiles read up to 3 rows
    // past the last panel row, which are zero-filled), == 2 (mod 4) doubles so
    // that 16-byte row-pair loads stay aligned
    int r = (dim < kNB ? kNB : dim) + 4;
    r = (r + 3) & ~3;
    return r + 2;
}

// Launch geometry of a table of graphs: per kernel, the flat block count of
// each graph and their running offsets (uploaded as Batch::boff for batches).
enum { kOffEdge = 0, kOffEdgeRed, kOffFrame, kOffPairs, kOffRhs, kOffRetr, kNumOff };

struct Geometry {
    int G = 0;
    int dof = 6;
    std::vector<int> off[kNumOff];  // G + 1 entries each
    size_t chol_smem = 0;
    int chol_cluster = 1;  // CTAs (one cluster) per graph in the Cholesky launch
    bool any_edges = false;
    bool chol_big = false;  // a single graph whose reduced system exceeds the staged panel:
                            // multi-launch blocked Cholesky
    bool wide = false;      // a single graph that may hold wide frames
    int dim = 0;            // reduced-system size of a single graph
};

inline void fill_geometry(const std::vector<Dims>& dims, Geometry& geo) {
    geo.G = (int)dims.size();
    for (int k = 0; k < kNumOff; k++) geo.off[k].assign(geo.G + 1, 0);
    for (int g = 0; g < geo.G; g++) {
        const Dims& d = dims[g];
        const long npairs = (long)d.P * (d.P + 1) / 2;
        const int cnt[kNumOff] = {d.E * d.CHe, d.E, d.K * d.CF, (int)ceil_div(npairs, 8), (int)ceil_div(d.P + 1, 8),
                                  (int)ceil_div(d.P, 128)};
        for (int k = 0; k < kNumOff; k++) geo.off[k][g + 1] = geo.off[k][g] + cnt[k];
        geo.chol_big = dims.size() == 1 && d.dim > kPanelRows;
        if (!geo.chol_big) geo.chol_smem = std::max(geo.chol_smem, (size_t)chol_ldr(d.dim) * kNB * sizeof(double));
        // a single large reduced system splits its trailing updates over a cluster of
        // CTAs (batches already fill the GPU with one CTA per graph)
        geo.chol_cluster = dims.size() == 1 ? (d.dim >= 256 ? 8 : (d.dim >= 128 ? 4 : 1)) : 1;
        geo.wide = dims.size() == 1 && d.wide;
        geo.dim = d.dim;
        geo.any_edges |= d.E > 0;
        geo.dof = d.dof;
    }
}

struct SolveArgs {
    int iterations;
    float lm, ep, alpha;
    int motion_only, intr;
    float ilm, iep, iscale;
    int compute_energy;
    const float* mu_sched = nullptr;  // host: the robust kernel's mu at each iteration (GNC), or none
};

// ---------------------------------------------------------------- relative pose of an edge
// SE3 (D = 6, poses (N, 7)) or Sim3 (D = 7, poses (N, 8) [t q s]): Tij = Tj Ti^-1; ii == jj is a
// stereo edge with the fixed baseline (-0.1, 0, 0)

struct EdgeTf {
    float t[3], q[4], s;
};

template <int D>
__device__ __forceinline__ void edge_tf(const float* poses, int a, int b, EdgeTf& T) {
    if (D == 6) {
        edge_pose(poses, a, b, T.t, T.q);
        T.s = 1.f;
    } else if (a == b) {
        T.t[0] = -0.1f; T.t[1] = 0.f; T.t[2] = 0.f;
        T.q[0] = 0.f; T.q[1] = 0.f; T.q[2] = 0.f; T.q[3] = 1.f;
        T.s = 1.f;
    } else {
        float pi[8], pj[8];
#pragma unroll
        for (int n = 0; n < 8; n++) {
            pi[n] = __ldg(poses + 8 * a + n);
            pj[n] = __ldg(poses + 8 * b + n);
        }
        const lie::Sim3<float> G = lie::Sim3<float>::load(pj) * lie::Sim3<float>::load(pi).inv();
        T.t[0] = G.t[0]; T.t[1] = G.t[1]; T.t[2] = G.t[2];
        T.q[0] = G.r.q.x; T.q[1] = G.r.q.y; T.q[2] = G.r.q.z; T.q[3] = G.r.q.w;
        T.s = G.r.s;
    }
}

// y = Ad(Tij) x for a tangent x of the source pose: the source-pose Jacobian rows
// are -Ad^T(Tij) times the target-pose rows, so Ji . x = -Jj . (Ad x).
//   SE3:  Ad = [[R, [t]x R], [0, R]];   Sim3: Ad = [[s R, [t]x R, -t], [0, R, 0], [0, 0, 1]]
template <int D>
__device__ __forceinline__ void edge_ad_apply(const EdgeTf& T, const float* x, float* y) {
    float rt[3], rp[3];
    qrot(T.q, x, rt);
    qrot(T.q, x + 3, rp);
    y[0] = T.s * rt[0] + (T.t[1] * rp[2] - T.t[2] * rp[1]);
    y[1] = T.s * rt[1] + (T.t[2] * rp[0] - T.t[0] * rp[2]);
    y[2] = T.s * rt[2] + (T.t[0] * rp[1] - T.t[1] * rp[0]);
    y[3] = rp[0];
    y[4] = rp[1];
    y[5] = rp[2];
    if constexpr (D == 7) {
        y[0] -= T.t[0] * x[6];
        y[1] -= T.t[1] * x[6];
        y[2] -= T.t[2] * x[6];
        y[6] = x[6];
    }
}

// host launchers implemented in ba.cu
int check_dims(int num_frames, int ht, int wd, int num_edges, int num_kx, int t0, int t1);
int ensure_attributes();
int launch_index(const Geometry& geo, const GraphDesc* d_table, const BAPtrs& base, const GraphDesc* init,
                 cudaStream_t st);
// one LM step's linearisation, assembly and (solve) factorised solve (dx = Delta xi) at
// the state held by base.poses / base.disps; nothing is updated
int launch_linearize_solve(const Geometry& geo, const GraphDesc* d_table, const int* d_off, const BAPtrs& base,
                           const SolveArgs& a, int itr, cudaStream_t st, bool solve = true);
// the damped reduced solve alone (Hm, bv of every graph -> dx)
int launch_cholesky(const Geometry& geo, const GraphDesc* d_table, const int* d_off, const BAPtrs& base,
                    const SolveArgs& a, cudaStream_t st);
// adj_lam = S'^-1 adj_rhs per graph, with the factor recorded in base.ftape
int launch_chol_resolve(const Geometry& geo, const GraphDesc* d_table, const BAPtrs& base, cudaStream_t st);

}  // namespace ba
}  // namespace vipe

// Host-side plan of a batch of graphs (opaque to C callers).
struct vipe_ba_batch_plan {
    int G = 0;
    int adjoint = 0;
    std::vector<vipe::ba::GraphDesc> gds;  // Work pointers valid once bound
    vipe::ba::Geometry geo;
    size_t bytes = 0;
    long frames = 0, edges = 0, kx = 0, poses = 0;
    long ftape_stride = 0;  // doubles of one iteration of the factor tape
    int ht = 0, wd = 0;
    void* ws = nullptr;  // workspace the table was uploaded to
    vipe::ba::GraphDesc* d_table = nullptr;
    int* d_off = nullptr;
    std::vector<int> off_host;  // kNumOff x (G + 1), the image of d_off
};
