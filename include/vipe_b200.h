/*
 * vipe_b200 — C ABI of the B200 (sm_100a) implementation of ViPE's DROID-style
 * SLAM backend hot path: dense bundle adjustment (slam_ext), correlation
 * build/lookup (droid_net_ext) and the lietorch group kernels (lietorch_ext).
 *
 * Conventions for every entry point:
 *   - all tensor arguments are raw DEVICE pointers to contiguous row-major
 *     buffers in the layouts of the reference extension (shapes given per
 *     function); integer index tensors are int64 like the reference's `long`;
 *   - work is enqueued on `stream` (a cudaStream_t passed as void*); nothing
 *     synchronises the stream unless the comment says so;
 *   - the return value is a vipe_status (0 = success).  Host-side argument
 *     errors are detected before any launch; device-side findings (bad
 *     indices, solver failure) are written to the optional `dev_status` word
 *     (int32 in device memory) and read by the caller when it wants them;
 *   - buffers named *_out are written completely; buffers named *_io are
 *     updated in place (as the reference mutates poses/disps/intrinsics).
 *
 * The library holds no torch types: the Python package vipe_b200.ext mirrors
 * the reference's pybind modules on top of this ABI.
 */
#ifndef VIPE_B200_H
#define VIPE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum vipe_status {
    VIPE_OK = 0,
    VIPE_ERR_ARG = 1,          /* bad shape / size / null pointer             */
    VIPE_ERR_INDEX = 2,        /* edge index outside [0, num_frames)          */
    VIPE_ERR_RANGE = 3,        /* empty or invalid optimisation window t0..t1 */
    VIPE_ERR_KX_MISMATCH = 4,  /* eta rows != |unique(cat(arange(t0,t1),ii))| */
    VIPE_ERR_WORKSPACE = 5,    /* workspace smaller than required             */
    VIPE_ERR_CAPACITY = 6,     /* graph exceeds a documented kernel limit     */
    VIPE_ERR_CUDA = 7,         /* a CUDA runtime call failed                  */
    VIPE_ERR_DTYPE = 8,        /* unsupported element type                    */
    VIPE_ERR_GROUP = 9,        /* unsupported Lie group id                    */
    VIPE_ERR_DEVICE_WAIT = 10, /* a kernel's bounded wait on its tensor-core   */
                               /* work expired; the call's outputs are invalid */
    VIPE_WARN_SOLVER = 16      /* (dev_status only) Cholesky failed: dx = 0   */
};

/* element types for dtype-generic entry points */
enum vipe_dtype { VIPE_F32 = 0, VIPE_F64 = 1, VIPE_F16 = 2, VIPE_BF16 = 3 };

/* Human-readable message for a status code (static storage). */
const char* vipe_status_string(int status);

/* Last CUDA error text seen by the library on this thread ("" if none). */
const char* vipe_last_error(void);

/* Launch profiler (no counterpart in the reference).  While enabled, each
 * kernel launch of the library is bracketed by CUDA events on its stream.
 * vipe_profile_collect synchronises those events, writes per-kernel-name total
 * milliseconds and launch counts (names: NUL-terminated, `name_stride` bytes
 * apart) and clears the record; returns the number of kernel names. */
void vipe_profile_enable(int on);
int vipe_profile_collect(char* names, int name_stride, float* total_ms, int* launches, int max_kernels);

/* HBM write-bandwidth probe (no counterpart in the reference; a measurement
 * helper for write-bound kernels' rooflines): writes `bytes` (a multiple of 16,
 * 16-byte aligned `dst`) with 16-byte stores, one per thread, over a grid that
 * covers the buffer once.  Time it with events on `stream`. */
int vipe_hbm_write_probe(void* dst, size_t bytes, void* stream);

/* =====================================================================
 * slam_ext — dense bundle adjustment and geometry helpers
 * ===================================================================== */

/* Bytes of device workspace needed by vipe_slam_ba_extended for a graph of
 * `num_edges` edges over `num_frames` frames of ht x wd depth maps, depth-row
 * count `num_kx` (= eta.shape[0]) and window [t0, t1). */
size_t vipe_slam_ba_workspace_size(int num_frames, int ht, int wd, int num_edges, int num_kx, int t0, int t1);

/* Replaces slam_ext.ba_extended (reference: csrc/slam_ext/slam.cpp:46-51,
 * implementation csrc/slam_ext/geom_kernels.cu:1626-1847).
 *   poses_io      (num_frames, 7) f32  [tx ty tz qx qy qz qw], updated in place
 *   disps_io      (num_frames, ht, wd) f32, updated in place
 *   intrinsics_io (4,) f32 [fx fy cx cy], fx/fy updated when optimize_intrinsics
 *   disps_sens    (num_frames, ht, wd) f32
 *   targets, weights (num_edges, 2, ht, wd) f32
 *   eta           (num_kx, ht, wd) f32
 *   ii, jj        (num_edges,) int64
 *   depth_active  (num_frames,) f32
 * Outputs (last LM iteration, as the reference returns them):
 *   dx_out     (t1-t0, 6) f32
 *   dz_out     (num_kx, ht*wd) f32, untouched when motion_only
 *   energy_out (iterations,) f32 when compute_energy, else may be NULL
 * workspace: device buffer of vipe_slam_ba_workspace_size() bytes.
 * dev_status: optional device int32; receives VIPE_ERR_INDEX /
 *   VIPE_ERR_KX_MISMATCH / VIPE_ERR_CAPACITY found on the device (the call then
 *   leaves poses/disps untouched) or VIPE_WARN_SOLVER (dx = 0, as the reference
 *   does on Cholesky failure).
 * Capacity (VIPE_ERR_CAPACITY): t1 - t0 <= 1024 window poses (ViPE's keyframe
 *   buffer: the backend's global BA over every keyframe).  Any number of window
 *   poses may be coupled to one depth frame: frames coupled to more than 31 take
 *   a wide-frame kernel instead of the tensor-core one, and reduced systems of
 *   more than 768 unknowns a multi-launch blocked Cholesky.  The workspace grows
 *   with the window (vipe_slam_ba_workspace_size). */
int vipe_slam_ba_extended(float* poses_io, float* disps_io, float* intrinsics_io, const float* disps_sens,
                          const float* targets, const float* weights, const float* eta, const int64_t* ii,
                          const int64_t* jj, const float* depth_active, int num_frames, int ht, int wd,
                          int num_edges, int num_kx, int t0, int t1, int iterations, float lm, float ep,
                          int motion_only, float alpha, int optimize_intrinsics, float intrinsics_lm,
                          float intrinsics_ep, float intrinsics_scale, int compute_energy, float* dx_out,
                          float* dz_out, float* energy_out, void* workspace, size_t workspace_bytes,
                          int32_t* dev_status, void* stream);

/* Fused BA with the generic solver's robust kernels (no counterpart in the reference's
 * fused path, which refuses robust kernels, vipe/slam/components/buffer.py:531-547; the
 * semantics are those of its generic solver, vipe/slam/ba/kernel.py:40-162 and
 * terms.py:73-75).  Arguments of vipe_slam_ba_extended plus:
 *   robust_kind 0 none, 1 Huber (w = 1 if |r| <= c else c/|r|), 2 Tukey
 *     (w = max(1 - (r/c)^2, 0)^2), 3 GNC-TLS (w at scalar mu per kernel.py:97-153);
 *     each flow channel's weight is multiplied by w(r) of its residual at the linearisation
 *     point;
 *   robust_threshold c > 0 (kinds 1-3);
 *   mu_schedule (HOST array of `iterations` floats, kind 3 only): mu of each LM iteration,
 *     +inf for the hard TLS indicator (see the generic solver's schedule, buffer.py:686-695).
 * The depth back-substitution keeps the rows of pose t0 (the generic solver's Schur
 * back-substitution; vipe_slam_ba_extended skips them like the reference's fused kernel). */
int vipe_slam_ba_extended_robust(float* poses_io, float* disps_io, float* intrinsics_io, const float* disps_sens,
                                 const float* targets, const float* weights, const float* eta, const int64_t* ii,
                                 const int64_t* jj, const float* depth_active, int num_frames, int ht, int wd,
                                 int num_edges, int num_kx, int t0, int t1, int iterations, float lm, float ep,
                                 int motion_only, float alpha, int optimize_intrinsics, float intrinsics_lm,
                                 float intrinsics_ep, float intrinsics_scale, int compute_energy, float* dx_out,
                                 float* dz_out, float* energy_out, int robust_kind, float robust_threshold,
                                 const float* mu_schedule, void* workspace, size_t workspace_bytes,
                                 int32_t* dev_status, void* stream);

/* vipe_slam_ba_extended_robust with the frames' camera model (the reference's fused path takes
 * single-view pinhole buffers only, buffer.py:387-388; its generic solver projects through
 * vipe/slam/maths/geom.py:187-298 with any CameraType):
 *   camera_model 0 pinhole, 1 MEI (unified model, vipe/utils/cameras.py:220-330) with
 *     distortion = k1 in [0, 1]; intrinsics_io holds fx, fy, cx, cy at the flow resolution as
 *     for pinhole.  MEI refuses optimize_intrinsics (VIPE_ERR_ARG). */
int vipe_slam_ba_extended_generic(float* poses_io, float* disps_io, float* intrinsics_io, const float* disps_sens,
                                  const float* targets, const float* weights, const float* eta, const int64_t* ii,
                                  const int64_t* jj, const float* depth_active, int num_frames, int ht, int wd,
                                  int num_edges, int num_kx, int t0, int t1, int iterations, float lm, float ep,
                                  int motion_only, float alpha, int optimize_intrinsics, float intrinsics_lm,
                                  float intrinsics_ep, float intrinsics_scale, int compute_energy, float* dx_out,
                                  float* dz_out, float* energy_out, int robust_kind, float robust_threshold,
                                  const float* mu_schedule, int camera_model, float distortion, void* workspace,
                                  size_t workspace_bytes, int32_t* dev_status, void* stream);

/* Multi-view rigs in the fused BA: the generic solver's terms with rig extrinsics
 * (vipe/slam/ba/terms.py:98-262, vipe/slam/maths/geom.py:187-298: each term projects depth frame
 * d_i = p_i * n_views + q_i into frame (p_j, q_j) through R_qj^-1 G_pj G_pi^-1 R_qi); the
 * reference's fused path refuses n_views > 1 and non-identity rigs (buffer.py:387-404).
 *   poses_io (num_keyframes, 7) keyframe poses G (updated in the window [t0, t1));
 *   rig (n_views, 7) extrinsics R_q (cam-to-central, [tx ty tz qx qy qz qw]); fixed, or with
 *     optimize_rig_rotation the rotations of views 1..n_views-1 are optimised and written back
 *     (the generic solver's rig group: 6-DoF rig steps, minus the pose Jacobians, damping
 *     rig_lm * diag + rig_ep, view 0 fixed, only the rotation of a step applied,
 *     buffer.py:668-673 and retractor.py:34-38; every (keyframe, view) is then an unknown of
 *     the virtual solve, so num_keyframes * n_views <= 1024);
 *   disps_io, disps_sens (num_keyframes * n_views, ht, wd), depth_active (num_keyframes * n_views);
 *   ii, jj: source and target depth-frame indices (k * n_views + q) of the num_edges terms,
 *     ii != jj; eta (num_kx, ht*wd) over kx = unique(arange(t0 n_views, t1 n_views) ++ ii);
 *   intrinsics (n_views, 4): fx fy cx cy of each view at the flow resolution (fixed): a term
 *     unprojects with its source view's row and projects with its target view's (the generic
 *     solver's per-view intrinsics, terms.py:175-206);
 *   dx_out (t1 - t0, 6) keyframe steps; dz_out (num_kx, ht*wd); energy_out (iterations) or NULL;
 *   robust kernel, mu schedule and camera model as vipe_slam_ba_extended_generic; with the MEI
 *     camera view_distortion (device, n_views floats in [0, 1], or NULL for `distortion` in
 *     every view) gives each view its k1, used as its intrinsics rows are;
 * Generic-solver back-substitution (rows of pose t0 kept).  Limits: n_views * (t1 - t0) <= 1024.
 * Workspace: vipe_slam_ba_rig_workspace_size. */
size_t vipe_slam_ba_rig_workspace_size(int num_keyframes, int n_views, int ht, int wd, int num_edges, int num_kx,
                                       int t0, int t1, int optimize_rig_rotation);
int vipe_slam_ba_rig(float* poses_io, float* rig, int n_views, float* disps_io, const float* intrinsics,
                     const float* disps_sens, const float* targets, const float* weights, const float* eta,
                     const int64_t* ii, const int64_t* jj, const float* depth_active, int num_keyframes, int ht,
                     int wd, int num_edges, int num_kx, int t0, int t1, int iterations, float lm, float ep,
                     int motion_only, float alpha, int compute_energy, float* dx_out, float* dz_out,
                     float* energy_out, int robust_kind, float robust_threshold, const float* mu_schedule,
                     int camera_model, float distortion, const float* view_distortion, int optimize_rig_rotation,
                     float rig_lm, float rig_ep, void* workspace, size_t workspace_bytes, int32_t* dev_status,
                     void* stream);

/* Replaces slam_ext.ba (reference: csrc/slam_ext/slam.cpp:42-45,
 * geom_kernels.cu:1826-1834): ba_extended with depth_active = 1, no focal
 * optimisation and no energy.  depth_active_scratch: device f32 buffer of
 * num_frames entries that the call fills with ones. */
int vipe_slam_ba(float* poses_io, float* disps_io, float* intrinsics_io, const float* disps_sens, const float* targets,
                 const float* weights, const float* eta, const int64_t* ii, const int64_t* jj, int num_frames, int ht,
                 int wd, int num_edges, int num_kx, int t0, int t1, int iterations, float lm, float ep,
                 int motion_only, float alpha, float* depth_active_scratch, float* dx_out, float* dz_out,
                 void* workspace, size_t workspace_bytes, int32_t* dev_status, void* stream);

/* Bundle adjustment for callers that cannot allocate device memory.  No
 * counterpart in the reference (its ba_cuda_impl allocates through ATen).
 * Hosts that forbid allocation after start-up, or bindings (cgo, JNI, plain C)
 * whose runtime has no CUDA allocator, cannot provide the workspace that
 * vipe_slam_ba_extended takes.  This entry point runs the same solve, with the
 * same arguments minus workspace/workspace_bytes, on a scratch array compiled
 * into the library: VIPE_BA_NOALLOC_SCRATCH_BYTES (32 MiB) of device memory on
 * every GPU that loads the library, held until the process exits.  It calls no
 * cudaMalloc/cudaFree.
 *   - Graphs whose vipe_slam_ba_workspace_size() exceeds the scratch are
 *     rejected with VIPE_ERR_CAPACITY before any launch (vipe_last_error()
 *     names both sizes).  A 64-keyframe 48x64 graph with 628 edges needs
 *     about 24 MiB.
 *   - The first call on a device looks up the scratch's device address there
 *     (cudaGetSymbolAddress, which loads the library's module on that device);
 *     make that first call before any stream capture.  The address is kept for
 *     the life of the process, so the device must not be reset
 *     (cudaDeviceReset) between calls.
 *   - Invalid sizes give the same status codes as vipe_slam_ba_extended.
 *   - Every call on a device shares the one array and the next call overwrites
 *     it: calls whose work overlaps on the GPU (different streams, or
 *     concurrent host threads) race and must be serialised by the caller. */
#define VIPE_BA_NOALLOC_SCRATCH_BYTES (32u << 20)
int vipe_slam_ba_extended_noalloc(float* poses_io, float* disps_io, float* intrinsics_io, const float* disps_sens,
                                  const float* targets, const float* weights, const float* eta, const int64_t* ii,
                                  const int64_t* jj, const float* depth_active, int num_frames, int ht, int wd,
                                  int num_edges, int num_kx, int t0, int t1, int iterations, float lm, float ep,
                                  int motion_only, float alpha, int optimize_intrinsics, float intrinsics_lm,
                                  float intrinsics_ep, float intrinsics_scale, int compute_energy, float* dx_out,
                                  float* dz_out, float* energy_out, int32_t* dev_status, void* stream);

/* Batched bundle adjustment: many clips' graphs solved together, each phase of
 * the LM step one launch over all graphs.  No counterpart in the reference,
 * whose ba_cuda_impl (csrc/slam_ext/geom_kernels.cu:1626-1824) solves one graph
 * per call; per graph the arithmetic is that of vipe_slam_ba_extended.
 *
 * Layout: graph g has num_frames[g] frames, num_edges[g] edges, num_kx[g]
 * depth rows and window [t0[g], t1[g]); every tensor of the single-graph call
 * is concatenated over the graphs along its leading axis, in graph order:
 *   poses (sum frames, 7), disps / disps_sens (sum frames, ht, wd),
 *   depth_active (sum frames), targets / weights (sum edges, 2, ht, wd),
 *   ii / jj (sum edges) int64 holding frame indices LOCAL to their graph,
 *   eta (sum kx, ht, wd), intrinsics (num_graphs, 4),
 *   dx_out (sum (t1-t0), 6), dz_out (sum kx, ht*wd),
 *   energy_out (num_graphs, iterations), dev_status (num_graphs) int32.
 * The plan is host-side; bind uploads its graph table into a device workspace
 * of vipe_slam_ba_batch_workspace_size() bytes (synchronises `stream`).
 * vipe_slam_ba_batch_solve then only enqueues kernels (no allocation, copy or
 * synchronisation), so it may be captured into a CUDA graph.
 * edge_chunks / frame_chunks: pixel chunks per edge / per depth frame for the
 * linearisation kernels (0 = chosen from the batch size).  with_adjoint: also
 * reserve the buffers of vipe_slam_ba_batch_backward.
 * group_id: 3 = SE3 (poses (.., 7), dx (.., 6)), or 4 = Sim3: poses (.., 8)
 * [tx ty tz qx qy qz qw s], dx (.., 7) [tau phi sigma], the same residuals,
 * weights, masks and solver with 7x7 pose blocks and retraction
 * T <- Exp(dx) T in Sim3 (no counterpart in the reference, whose fused BA is
 * SE3-only); window sizes up to 109 poses; no focal-length optimisation and no
 * adjoint for Sim3.
 * tape_poses, tape_disps, tape_factor, tape_dx (optional, all or none): the
 * record the backward pass reads — per iteration the state entering it,
 * (iterations, sum frames, 7) and (iterations, sum frames, ht, wd), the
 * factorised reduced system with the depth elimination's per-pixel (Q, w),
 * (iterations, totals_out[4]) doubles, and the pose step,
 * (iterations, sum (t1-t0), 6). */
typedef struct vipe_ba_batch_plan vipe_ba_batch_plan;
int vipe_slam_ba_batch_plan_create(int num_graphs, const int* num_frames, const int* num_edges, const int* num_kx,
                                   const int* t0, const int* t1, int ht, int wd, int edge_chunks, int frame_chunks,
                                   int group_id, int with_adjoint, vipe_ba_batch_plan** plan_out);
size_t vipe_slam_ba_batch_workspace_size(const vipe_ba_batch_plan* plan);
/* totals_out[5] = {sum frames, sum edges, sum kx, sum (t1-t0), doubles of one
 * iteration of the tape_factor record} */
int vipe_slam_ba_batch_totals(const vipe_ba_batch_plan* plan, int64_t* totals_out);
int vipe_slam_ba_batch_bind(vipe_ba_batch_plan* plan, void* workspace, size_t workspace_bytes, void* stream);
int vipe_slam_ba_batch_solve(const vipe_ba_batch_plan* plan, float* poses_io, float* disps_io, float* intrinsics_io,
                             const float* disps_sens, const float* targets, const float* weights, const float* eta,
                             const int64_t* ii, const int64_t* jj, const float* depth_active, int iterations,
                             float lm, float ep, int motion_only, float alpha, int optimize_intrinsics,
                             float intrinsics_lm, float intrinsics_ep, float intrinsics_scale, int compute_energy,
                             float* dx_out, float* dz_out, float* energy_out, int32_t* dev_status,
                             float* tape_poses, float* tape_disps, double* tape_factor, float* tape_dx,
                             void* stream);
void vipe_slam_ba_batch_plan_destroy(vipe_ba_batch_plan* plan);

/* Adjoint of vipe_slam_ba_batch_solve (no counterpart in the reference, which
 * has no BA backward).  Given the forward's tape and the gradients of a loss
 * with respect to the solve's outputs, writes the gradients with respect to its
 * inputs; the plan must have been created with_adjoint.  Every LM step is
 * differentiated exactly, with its linear solve differentiated implicitly (the
 * same damped reduced system re-solved with the incoming gradients), the LM
 * damping ep + lm*diag(S) included; Jacobians are recomputed from the tape
 * and the factorised reduced system and per-pixel (Q, w) are read back from it.
 * Not covered: motion_only and optimize_intrinsics solves.
 *   grad_poses (sum frames, 7): in, d loss / d poses_out as left-tangent
 *     gradients in columns 0..5 (lietorch's layout for group gradients,
 *     csrc/lietorch_ext/lietorch_gpu.cu:85-98); out, d loss / d poses_in, same
 *     layout, column 6 = 0;
 *   grad_disps (sum frames, ht, wd): in, d loss / d disps_out; out, d loss / d disps_in;
 *   grad_targets, grad_weights (sum edges, 2, ht, wd), grad_eta (sum kx, ht, wd),
 *   grad_disps_sens (sum frames, ht, wd): out.  dev_status as in the solve; the
 *   gradients of a graph whose status holds an error code are undefined. */
int vipe_slam_ba_batch_backward(const vipe_ba_batch_plan* plan, const float* tape_poses, const float* tape_disps,
                                const double* tape_factor, const float* tape_dx, const float* intrinsics,
                                const float* disps_sens, const float* targets, const float* weights, const float* eta,
                                const int64_t* ii, const int64_t* jj, const float* depth_active, int iterations,
                                float lm, float ep, float alpha, float* grad_poses, float* grad_disps,
                                float* grad_targets, float* grad_weights, float* grad_eta, float* grad_disps_sens,
                                int32_t* dev_status, void* stream);

/* Debug view of the device-built graph index (bit-exact tests against the
 * reference's host-side index: _unique/kk_exp geom_kernels.cu:1649-1656, the
 * accum CSR :1043-1089, the Schur pair enumeration :1440-1468).  Runs only the
 * index construction of vipe_slam_ba_extended into `workspace` and copies:
 *   kx_out (num_kx) int64 — sorted unique depth frames
 *   kk_out (t1-t0+num_edges) int64 — inverse map of cat(arange(t0,t1), ii)
 *   pair_out: up to pair_cap (a, b) pose pairs (int32, local ids) that receive
 *   a Schur block, sorted; *num_pairs gets the count.
 *   csr_ptr_out (num_kx+1), csr_idx_out (num_edges) int64, optional (both or
 *   neither): the device's per-depth-row edge lists — the edges whose source
 *   frame is kx[s], ascending — i.e. the CSR of the reference's
 *   accum_cuda(., ii, kx) (geom_kernels.cu:1766-1785).
 * Synchronises `stream`. */
int vipe_slam_ba_index_debug(const int64_t* ii, const int64_t* jj, int num_frames, int num_edges, int num_kx, int t0,
                             int t1, int64_t* kx_out, int64_t* kk_out, int32_t* pair_out, int pair_cap,
                             int* num_pairs, int64_t* csr_ptr_out, int64_t* csr_idx_out, void* workspace,
                             size_t workspace_bytes, void* stream);

/* Replaces slam_ext.frame_distance (reference: geom_kernels.cu:613-768,
 * 1849-1877).  poses (num_poses,7), disps (num_disps,ht,wd), intrinsics
 * (num_views,4), pi,pj (pose rows), qi,qj (intrinsics rows), di (disp rows)
 * (num,) int64 -> dist_out (num,) f32.  A pair with an index outside its
 * tensor gets NaN (the reference reads out of bounds). */
int vipe_slam_frame_distance(const float* poses, const float* disps, const float* intrinsics, const int64_t* pi,
                             const int64_t* pj, const int64_t* qi, const int64_t* qj, const int64_t* di, int num,
                             int num_poses, int num_disps, int num_views, int ht, int wd, float beta, float* dist_out,
                             void* stream);

/* Replaces slam_ext.projmap (reference: geom_kernels.cu:526-611, 1879-1903).
 * poses (num_frames,7), disps (num_frames,ht,wd), ii,jj (num,) int64
 * -> coords_out (num,ht,wd,3) f32 (third channel 0), valid_out (num,ht,wd,1);
 * NaN for an edge with an index outside [0, num_frames). */
int vipe_slam_projmap(const float* poses, const float* disps, const float* intrinsics, const int64_t* ii,
                      const int64_t* jj, int num, int num_frames, int ht, int wd, float* coords_out, float* valid_out,
                      void* stream);

/* Replaces slam_ext.depth_filter (reference: geom_kernels.cu:770-885,
 * 1905-1929).  ix (num,) int64, thresh (num,) f32 -> counter_out (num,ht,wd). */
int vipe_slam_depth_filter(const float* poses, const float* disps, const float* intrinsics, const int64_t* ix,
                           const float* thresh, int num_frames, int num, int ht, int wd, float* counter_out,
                           void* stream);

/* Replaces slam_ext.iproj (reference: geom_kernels.cu:887-953, 1931-1950).
 * -> points_out (num_frames,ht,wd,3) f32. */
int vipe_slam_iproj(const float* poses, const float* disps, const float* intrinsics, int num_frames, int ht, int wd,
                    float* points_out, void* stream);

/* Proximity-edge construction of the factor graph (reference: the host loops of
 * FactorGraph.add_proximity_factors, vipe/slam/components/factor_graph.py:431-486),
 * given the candidate distances.  Candidates are (i, j), i in [t0, t), j in [t1, t),
 * row-major: d ((t-t0) x (t-t1)) f32, e.g. slam_ext.frame_distance of every pair.
 * ii_exist, jj_exist (num_exist) int64: the graph's active then inactive edges.
 * Emits into ii_out / jj_out (int64, out_cap >= vipe_slam_proximity_edges_capacity())
 * exactly the reference's edge list, in its order: the neighbourhood edges, then the
 * greedy NMS over candidates in ascending distance (ties in index order), and writes
 * the count to *num_out (device int32).  One CTA; up to 1.7 M candidates (t = 1024,
 * t0 = t1 = 0); workspace of vipe_slam_proximity_edges_workspace_size() bytes. */
size_t vipe_slam_proximity_edges_workspace_size(int t0, int t1, int t);
long vipe_slam_proximity_edges_capacity(int t0, int t1, int t, int rad, int max_factors, int cross_view);
int vipe_slam_proximity_edges(const float* d, const int64_t* ii_exist, const int64_t* jj_exist, int num_exist, int t0,
                              int t1, int t, int rad, int nms, float thresh, int max_factors, int cross_view,
                              int64_t* ii_out, int64_t* jj_out, int out_cap, int* num_out, void* workspace,
                              size_t workspace_bytes, void* stream);

/* =====================================================================
 * lietorch_ext — group kernels.  group_id: 1 SO3, 2 RxSO3, 3 SE3, 4 Sim3
 * (reference dispatch: csrc/lietorch_ext/dispatch.h:17-50).  dtype VIPE_F32 or
 * VIPE_F64.  `batch` group elements; embedding size N, tangent size K per group
 * (SO3 4/3, RxSO3 5/4, SE3 7/6, Sim3 8/7).  Gradients with respect to group
 * elements are stored with row stride N (first K entries used), as in the
 * reference (csrc/lietorch_ext/lietorch_gpu.cu:85-98).
 * Bindings replaced: csrc/lietorch_ext/lietorch.cpp:306-336.
 * ===================================================================== */
int vipe_lie_expm(int group_id, int dtype, int64_t batch, const void* a, void* X_out, void* stream);
int vipe_lie_expm_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* a, void* da_out,
                           void* stream);
int vipe_lie_logm(int group_id, int dtype, int64_t batch, const void* X, void* a_out, void* stream);
int vipe_lie_logm_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* X, void* dX_out,
                           void* stream);
int vipe_lie_inv(int group_id, int dtype, int64_t batch, const void* X, void* Y_out, void* stream);
int vipe_lie_inv_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* X, void* dX_out,
                          void* stream);
int vipe_lie_mul(int group_id, int dtype, int64_t batch, const void* X, const void* Y, void* Z_out, void* stream);
int vipe_lie_mul_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* X, const void* Y,
                          void* dX_out, void* dY_out, void* stream);
int vipe_lie_adj(int group_id, int dtype, int64_t batch, const void* X, const void* a, void* b_out, void* stream);
int vipe_lie_adj_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* X, const void* a,
                          void* dX_out, void* da_out, void* stream);
int vipe_lie_adjT(int group_id, int dtype, int64_t batch, const void* X, const void* a, void* b_out, void* stream);
int vipe_lie_adjT_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* X, const void* a,
                           void* dX_out, void* da_out, void* stream);
int vipe_lie_act(int group_id, int dtype, int64_t batch, const void* X, const void* p, void* q_out, void* stream);
int vipe_lie_act_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* X, const void* p,
                          void* dX_out, void* dp_out, void* stream);
int vipe_lie_act4(int group_id, int dtype, int64_t batch, const void* X, const void* p, void* q_out, void* stream);
int vipe_lie_act4_backward(int group_id, int dtype, int64_t batch, const void* grad, const void* X, const void* p,
                           void* dX_out, void* dp_out, void* stream);
int vipe_lie_as_matrix(int group_id, int dtype, int64_t batch, const void* X, void* T_out, void* stream);
int vipe_lie_projector(int group_id, int dtype, int64_t batch, const void* X, void* P_out, void* stream);
int vipe_lie_Jinv(int group_id, int dtype, int64_t batch, const void* X, const void* a, void* b_out, void* stream);

/* =====================================================================
 * droid_net_ext — correlation lookup and build
 * Bindings replaced: csrc/droid_net_ext/droid.cpp:75-81.
 * ===================================================================== */

/* corr_index_forward (correlation_kernels.cu:22-66,115-136).
 * volume (B, h1, w1, h2, w2) dtype, coords (B, 2, h1, w1) f32
 * -> corr_out (B, 2r+1, 2r+1, h1, w1) dtype (x-offset major). */
int vipe_corr_index_forward(int dtype, const void* volume, const float* coords, int B, int h1, int w1, int h2, int w2,
                            int radius, void* corr_out, void* stream);

/* corr_index_backward (correlation_kernels.cu:68-113,138-158).
 * -> volume_grad_out (B, h1, w1, h2, w2) dtype (written completely). */
int vipe_corr_index_backward(int dtype, const float* coords, const void* corr_grad, int B, int h1, int w1, int h2,
                             int w2, int radius, void* volume_grad_out, void* stream);

/* Coordinate gradient of corr_index_forward (no reference counterpart: the
 * reference's CorrSampler.backward returns no coordinate gradient,
 * vipe/slam/networks/droid_net.py:40-45).  The exact derivative of the bilinear
 * weights inside each cell, contracted with corr_grad (B, 2r+1, 2r+1, h1, w1)
 * dtype -> coords_grad_out (B, 2, h1, w1) f32 (written completely). */
int vipe_corr_index_coords_backward(int dtype, const void* volume, const float* coords, const void* corr_grad, int B,
                                    int h1, int w1, int h2, int w2, int radius, float* coords_grad_out, void* stream);

/* altcorr_forward (altcorr_kernel.cu:26-138,368-392).
 * fmap1 (B,H1,W1,C), fmap2 (B,H2,W2,C) dtype, coords (B,S,H1,W1,2) f32
 * -> corr_out (B,S,(2r+1)^2,H1,W1) dtype. */
int vipe_altcorr_forward(int dtype, const void* fmap1, const void* fmap2, const float* coords, int B, int S, int H1,
                         int W1, int H2, int W2, int C, int radius, void* corr_out, void* stream);

/* altcorr_backward (altcorr_kernel.cu:242-366,426-455), f32 only.
 * -> fmap1_grad_out, fmap2_grad_out (shapes of the fmaps), coords_grad_out
 * (B,S,H1,W1,2): the reference returns zeros there; this library writes the
 * exact derivative of the bilinear lookup when `exact_coords_grad` is 1 and
 * zeros otherwise. */
int vipe_altcorr_backward(const float* fmap1, const float* fmap2, const float* coords, const float* corr_grad, int B,
                          int S, int H1, int W1, int H2, int W2, int C, int radius, int exact_coords_grad,
                          float* fmap1_grad_out, float* fmap2_grad_out, float* coords_grad_out, void* stream);

/* altcorr_index_forward (altcorr_kernel.cu:140-240,394-424).
 * fmap1 (B,Nf,H,W,C) dtype (level 0), fmap2 levels l=0..L-1 each
 * (B,Nf,H>>l... floor sizes H2[l],W2[l],C), coords (B,M,H,W,2) f32,
 * ii, jj (M,) int64 -> corr_out (B,M,L*(2r+1)^2,H,W) f32. */
int vipe_altcorr_index_forward(int dtype, const void* fmap1, const void* const* fmap2_levels, const int* H2,
                               const int* W2, int num_levels, const float* coords, const int64_t* ii,
                               const int64_t* jj, int B, int Nf, int M, int H, int W, int C, int radius,
                               float* corr_out, void* stream);

/* Adjoint of altcorr_index_forward (no reference counterpart: the reference
 * binds only the forward, droid.cpp:75-81).  corr_grad (B, M, L*(2r+1)^2, H, W)
 * f32 -> fmap1_grad_out (B, Nf, H, W, C) f32, level_grads_out[l]
 * (B, Nf, H2[l], W2[l], C) f32 (all zeroed here, then accumulated with
 * atomics: edges sharing a frame add into the same rows) and, when not NULL,
 * coords_grad_out (B, M, H, W, 2) f32: the exact derivative of the bilinear
 * weights summed over levels (level l scaled by 2^-l) if exact_coords_grad,
 * zeros otherwise.  dtype VIPE_F32, VIPE_F16 or VIPE_BF16 (the maps). */
int vipe_altcorr_index_backward(int dtype, const void* fmap1, const void* const* fmap2_levels, const int* H2,
                                const int* W2, int num_levels, const float* coords, const int64_t* ii,
                                const int64_t* jj, const float* corr_grad, int B, int Nf, int M, int H, int W, int C,
                                int radius, int exact_coords_grad, float* fmap1_grad_out,
                                float* const* level_grads_out, float* coords_grad_out, void* stream);

/* Channels-last feature pyramid of AltCorrBlock (reference: eager torch,
 * vipe/slam/networks/droid_net.py:130-142): level l of fmaps / 4 average-pooled
 * l times (2x2, floor sizes), each level rounded to the element type before the
 * next pools it, FP32 window sums in avg_pool2d's order — bit-identical to the
 * reference's levels.  fmaps (num, C, H, W); level_out[l] (num, H>>l, W>>l, C),
 * 16-byte aligned; dtype VIPE_F32, VIPE_F16 or VIPE_BF16; 1 <= num_levels <= 4;
 * C a multiple of 8 (16-bit) or 4 (FP32), at most 256. */
int vipe_corr_pyramid_nhwc(int dtype, const void* fmaps, int num, int C, int H, int W, int num_levels,
                           void* const* level_out, void* stream);

/* Adjoint of vipe_corr_pyramid_nhwc (the reference differentiates the eager ops
 * through torch autograd): level_grads[l] (num, H>>l, W>>l, C) FP32 ->
 * fmaps_grad_out (num, C, H, W) in dtype, written completely (FP32 sums, one
 * rounding). */
int vipe_corr_pyramid_nhwc_backward(int dtype, const float* const* level_grads, int num, int C, int H, int W,
                                    int num_levels, void* fmaps_grad_out, void* stream);

/* =====================================================================
 * corr_ext — spatial correlation sampler of the AOT tracker's attention
 * Bindings replaced: csrc/corr_ext/correlation_sampler.cpp:82-85 (forward,
 * backward; kernels csrc/corr_ext/correlation_cuda_kernel.cu).
 * ===================================================================== */

/* out (num, patchH, patchW, oH, oW), oH = (H + 2 padH - ((kH-1) dilationH + 1)) / dH + 1
 * (oW likewise): sum over channels and kernel taps of input1[y1][x1] * input2[y1 + s][x1 + t],
 * y1 = oh dH - padH + i dilationH, s = ph dilation_patchH - dilation_patchH (patchH-1) / 2,
 * terms outside either map skipped (the reference GPU forward's convention).  input1,
 * input2 (num, C, H, W); dtype VIPE_F32, VIPE_F64, VIPE_F16 or VIPE_BF16 (FP32
 * accumulation, FP64 for VIPE_F64). */
int vipe_corr_sample_forward(int dtype, const void* input1, const void* input2, int num, int C, int H, int W, int kH,
                             int kW, int patchH, int patchW, int padH, int padW, int dilationH, int dilationW,
                             int dilation_patchH, int dilation_patchW, int dH, int dW, void* out, void* stream);

/* Adjoint of vipe_corr_sample_forward: grad_output (num, patchH, patchW, oH, oW) ->
 * grad_input1_out, grad_input2_out (num, C, H, W), written completely (gathers, no atomics). */
int vipe_corr_sample_backward(int dtype, const void* input1, const void* input2, const void* grad_output, int num,
                              int C, int H, int W, int kH, int kW, int patchH, int patchW, int padH, int padW,
                              int dilationH, int dilationW, int dilation_patchH, int dilation_patchW, int dH, int dW,
                              void* grad_input1_out, void* grad_input2_out, void* stream);

/* CorrBlock lookup fused with the first layer of the update operator's corr_encoder
 * (reference: droid_net.py:94-102 then UpdateModule.corr_encoder[0:2], :455-460):
 * out[b][o][p] = ReLU(bias[o] + sum_k weight[o][k] corr[b][k][p]) with corr the 196-channel
 * radius-3 lookup of the 4-level pyramid at coords / 2^l (channel l*49 + i*7 + j, i the x
 * offset).  levels[l] (B, H, W, H>>l, W>>l), coords (B, 2, H, W) f32, weight (128, 196) and
 * out (B, 128, H, W) in dtype (VIPE_F16 or VIPE_BF16), bias (128) f32 or NULL.  tcgen05
 * tensor cores; the lookup never leaves the chip.  dev_status (device int32): nonzero if a
 * bounded wait expired. */
int vipe_corr_encoder_lookup(int dtype, const void* const* levels, int num_levels, const float* coords, int B, int H,
                             int W, const void* weight, const float* bias, void* out, int32_t* dev_status,
                             void* stream);

/* All-pairs correlation volume with its average-pooled pyramid — the build of
 * CorrBlock (vipe/slam/networks/droid_net.py:56-69,94-102): for each of the
 * `num` pairs, level l holds avg_pool^l((fmap1/4)^T (fmap2/4)) over the target
 * (h2, w2) axes.  fmap1, fmap2 (num, C, ht, wd) in `in_dtype` (VIPE_F16 or
 * VIPE_BF16), C % 16 == 0.  level_out[l] (num, ht, wd, ht>>l, wd>>l) in
 * `out_dtype` (VIPE_F32, VIPE_F16 or VIPE_BF16).  ht, wd divisible by
 * 2^(num_levels-1).  Uses tcgen05 tensor cores with TMEM accumulators.
 * The first int32 of `workspace` becomes nonzero if a bounded wait inside the
 * kernel expired (the output is then incomplete). */
size_t vipe_corr_volume_workspace_size(int num, int C, int ht, int wd);

/* Adjoint of vipe_corr_volume_build (the reference differentiates torch.matmul and
 * avg_pool2d with autograd, droid_net.py:56-69,94-102): level_grads[l] (num, ht*wd,
 * ht>>l, wd>>l) in grad_dtype (VIPE_F16, VIPE_BF16 or VIPE_F32) ->
 * fmap1_grad_out = (1/16) fmap2 Gt^T and fmap2_grad_out = (1/16) fmap1 Gt, (num, C, ht,
 * wd) FP32 (either may be NULL), Gt = sum_l unpool_l(G_l) / 4^l formed on the fly.
 * fmap1, fmap2 (num, C, ht, wd) in map_dtype (VIPE_F16 / VIPE_BF16: the operands the
 * forward multiplied).  tcgen05 tensor cores: kind::f16 for 16-bit gradients, kind::tf32
 * with a hi + lo split of Gt for FP32 gradients.  C <= 128, ht*wd a multiple of 128, wd of
 * 8, ht and wd of 2^(num_levels-1).  16-bit maps and gradients of one type with wd a
 * multiple of 64 take a TMA-fed warp-specialised kernel (G_0 tiles loaded by TMA, the pooled
 * levels added in shared memory); other shapes form Gt in the producer warps.  dev_status
 * (device int32): set nonzero if a bounded wait expired (the gradients are then incomplete). */
int vipe_corr_volume_backward(int map_dtype, int grad_dtype, const void* fmap1, const void* fmap2,
                              const void* const* level_grads, int num, int C, int ht, int wd, int num_levels,
                              float* fmap1_grad_out, float* fmap2_grad_out, int32_t* dev_status, void* stream);
/* Test hook: on != 0 sends every vipe_corr_volume_backward call through the producer-formed
 * kernel (so the two kernels can be held to each other on the same shapes). */
void vipe_corr_volume_backward_force_generic(int on);
int vipe_corr_volume_build(int in_dtype, int out_dtype, const void* fmap1, const void* fmap2, int num, int C, int ht,
                           int wd, int num_levels, void* const* level_out, void* workspace, size_t workspace_bytes,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VIPE_B200_H */
