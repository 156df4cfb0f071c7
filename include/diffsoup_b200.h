/*
 * diffsoup_b200.h -- C ABI of libdiffsoup_b200.so, the B200 (sm_100a)
 * implementation of DiffSoup's differentiable rasterize-and-shade path.
 *
 * Conventions
 *  - Every entry point returns DS_OK (0) or an error status; ds_last_error()
 *    returns the message of the last failure on the calling thread.  No entry
 *    point exits the process.
 *  - Pointers are device pointers unless the parameter name ends in _host.
 *    Tensors are dense, C-contiguous, with the layouts of the reference
 *    (kenji-tojo/diffsoup python/diffsoup): pos [B,V,4] f32 clip space,
 *    tri [T,3] i32, rast [B,H,W,4] f32 = (b0, b1, z_ndc, tri_id+1), 0 = empty.
 *  - Work is enqueued on `stream` (a cudaStream_t).  Entry points documented
 *    as "host-synchronising" read a count back, like the reference's launcher
 *    does; all others never block the host and can be captured in a CUDA graph.
 *  - Outputs that accumulate must be zeroed by the caller, as in the reference
 *    (python/diffsoup/rasterize.py:171,177,271, multires.py:238,305).
 *  - Temporary device memory comes from the caller as (workspace, bytes);
 *    the matching *_workspace_size() function gives the required size.
 */
#ifndef DIFFSOUP_B200_H
#define DIFFSOUP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* ds_stream_t; /* cudaStream_t */

enum {
    DS_OK = 0,
    DS_ERR_ARG = 1,         /* shape / argument mismatch (reference: std::runtime_error) */
    DS_ERR_CUDA = 2,        /* CUDA runtime error (reference: CUDA_CHECK -> exit(1)) */
    DS_ERR_WORKSPACE = 3,   /* workspace smaller than *_workspace_size() */
    DS_ERR_OVERFLOW = 4,    /* a count exceeds the 32-bit range of the reference's layout */
};

/* Bits of the device status word written by the tiled kernels. */
enum {
    DS_STATUS_LIST_OVERFLOW = 1, /* tile lists exceeded capacity; affected tiles ran the exhaustive path */
    DS_STATUS_RECORD_FALLBACK = 2, /* some blocks' fragment records did not fit; they were re-enumerated */
    DS_STATUS_SPLIT_LIMIT = 4, /* ds_split_soup_count: a face's split tree exceeded its limits (see there) */
    DS_STATUS_MMA_TIMEOUT = 8, /* a tensor-core stage of the training step's shading did not complete within its
                                  bounded wait; the step's outputs are not valid */
};

const char* ds_last_error(void);
const char* ds_version(void);

/* ===================================================================== */
/*  Reference operator mirror: one entry point per `_core` function.      */
/* ===================================================================== */

/* replaces _core.compute_triangle_rects (src/main.cpp:30-48,
 * src/cuda/rasterize.cu:43-168).  rects [B*T,4] = (h0, h_len, w0, w_len),
 * prefix [B*T] inclusive sum of h_len*w_len.  Host-synchronising: writes the
 * total (the reference's return value) to *num_frags_host. */
size_t ds_compute_triangle_rects_workspace(int B, int T);
int ds_compute_triangle_rects(int H, int W, int B, int V, const float* pos, int T, const int* tri, int* rects,
                              int* prefix, int* num_frags_host, void* workspace, size_t workspace_bytes,
                              ds_stream_t stream);

/* replaces _core.compute_fragments (src/main.cpp:50-76, rasterize.cu:208-305).
 * frag_pix [num_frags,3] must be pre-filled with -1 (rasterize.py:69). */
int ds_compute_fragments(int H, int W, int B, int V, const float* pos, int T, const int* tri, const int* prefix,
                         const int* rects, int num_frags, int* frag_pix, float* frag_attrs, ds_stream_t stream);

/* replaces _core.filter_valid_fragments (src/main.cpp:96-108,
 * rasterize.cu:402-487).  Order preserving (the reference's block order is
 * not).  Host-synchronising: writes the valid count to *count_host. */
size_t ds_filter_valid_fragments_workspace(int num_frags);
int ds_filter_valid_fragments(int num_frags, const int* frag_pix, const float* frag_attrs, int* frag_pix_out,
                              float* frag_attrs_out, int* count_host, void* workspace, size_t workspace_bytes,
                              ds_stream_t stream);

/* replaces _core.depth_test (src/main.cpp:78-94, rasterize.cu:307-400).
 * Writes the winning fragment of every covered pixel into rast (others are
 * left untouched; the caller zeroes rast). */
size_t ds_depth_test_workspace(int B, int H, int W);
int ds_depth_test(int B, int H, int W, int num_frags, const int* frag_pix, const float* frag_attrs,
                  const float* frag_alpha, const float* alpha_thresh, float* rast, void* workspace,
                  size_t workspace_bytes, ds_stream_t stream);

/* No counterpart in the reference: the depth test of ds_depth_test for
 * callers that cannot allocate device memory (an embedding application that
 * owns all device memory, a fixed memory budget, or a loop that cannot pay for
 * cudaMalloc/cudaFree).  It allocates nothing: its 8-byte-per-pixel depth
 * keys live in a fixed __device__ buffer of this library, so B*H*W is limited
 * to 2^21 pixels (larger batches return DS_ERR_ARG).  All calls on a device
 * share that buffer (each clears what it uses); calls whose GPU work overlaps
 * race on it.  The first call on each device looks up the buffer's address
 * (cudaGetSymbolAddress); make it before any stream capture.  That address is
 * cached for the device's context: do not use this entry point across a
 * cudaDeviceReset.  Fragments outside the batch are skipped. */
int ds_depth_test_noalloc(int B, int H, int W, int num_frags, const int* frag_pix, const float* frag_attrs,
                          const float* frag_alpha, const float* alpha_thresh, float* rast, ds_stream_t stream);

/* replaces _core.backward_edge_grad (src/main.cpp:112-130, rasterize.cu:653-921).
 * grad_pos [B,V,4] accumulates. */
int ds_backward_edge_grad(int B, int H, int W, int C, const float* color, const float* grad_color,
                          const float* rast, int V, const float* pos, float* grad_pos, const int* tri,
                          ds_stream_t stream);

/* replaces _core.backward_opacity_aux_loss (src/main.cpp:134-154,
 * rasterize.cu:923-992).  grad_frag_alpha accumulates. */
int ds_backward_opacity_aux_loss(int B, int H, int W, int C, const float* color, const float* target,
                                 const float* rast, int num_frags, const int* frag_pix, const float* frag_attrs,
                                 const float* frag_alpha, float* grad_frag_alpha, ds_stream_t stream);

/* replaces _core.encode_view_dir_sh2 (src/main.cpp:158-170, encoding.cu:89-130). */
int ds_encode_view_dir_sh2(int B, int H, int W, const float* rast, const float* inv_mvp, float* encoding,
                           ds_stream_t stream);

/* replaces _core.multires_triangle_alpha (src/main.cpp:174-191, multires.cu:130-176).
 * S must equal the lattice size of levels [min_level, max_level]. */
int ds_multires_triangle_alpha(int num_frags, const float* frag_attrs, int min_level, int max_level, int S,
                               const float* alpha_src, float* frag_alpha, ds_stream_t stream);

/* replaces _core.backward_multires_triangle_alpha (src/main.cpp:193-210,
 * multires.cu:178-222).  grad_alpha_src [T,S] accumulates. */
int ds_backward_multires_triangle_alpha(int num_frags, const float* frag_attrs, int min_level, int max_level,
                                        int S, float* grad_alpha_src, const float* grad_frag_alpha,
                                        ds_stream_t stream);

/* replaces _core.multires_triangle_color (src/main.cpp:212-232, multires.cu:224-266).
 * out [B,H,W,C] accumulates (the reference zero-initialises it). */
int ds_multires_triangle_color(int B, int H, int W, const float* rast, int min_level, int max_level, int S, int C,
                               const float* features, float* out, ds_stream_t stream);

/* replaces _core.backward_multires_triangle_color (src/main.cpp:234-254,
 * multires.cu:268-311).  grad_features [T,S,C] accumulates. */
int ds_backward_multires_triangle_color(int B, int H, int W, const float* rast, int min_level, int max_level,
                                        int S, int C, float* grad_features, const float* grad_out,
                                        ds_stream_t stream);

/* replaces _core.accumulate_to_level_forward (src/main.cpp:258-280,
 * multires.cu:329-389).  out [T,S_target,C] is overwritten. */
int ds_accumulate_to_level_forward(int T, int min_level, int max_level, int target_level, int S, int S_target,
                                   int C, const float* features, float* out, ds_stream_t stream);

/* replaces _core.accumulate_to_level_backward (src/main.cpp:282-304,
 * multires.cu:393-450).  grad_features [T,S,C] accumulates. */
int ds_accumulate_to_level_backward(int T, int min_level, int max_level, int target_level, int S, int S_target,
                                    int C, float* grad_features, const float* grad_out, ds_stream_t stream);

/* ===================================================================== */
/*  B200 path: screen-tile binning, tiled rasterizer, tiled aux gradient  */
/* ===================================================================== */

/* One view of a batch.  Views may differ in resolution; their pixels are
 * packed one after another in the rast/colour buffers (pix_offset), and their
 * 16x16 screen tiles are numbered consecutively (tile_base). */
typedef struct {
    int32_t H, W;
    int32_t tiles_x, tiles_y;
    int64_t pix_offset; /* first pixel of this view in the packed buffers */
    int32_t tile_base;  /* first tile of this view */
    int32_t pad;
} ds_view_desc;

#define DS_TILE 16

/* Fills desc_host[b] for views of the given heights and widths; returns the
 * total tile count and writes the total pixel count to *num_pixels_host. */
int ds_make_view_table(int B, const int* H_host, const int* W_host, ds_view_desc* desc_host,
                       int64_t* num_pixels_host);

/* Bytes of workspace for binning B*T triangles into num_tiles tiles with room
 * for list_capacity (triangle, tile) entries. */
size_t ds_tiles_workspace_size(int B, int T, int num_tiles, int64_t list_capacity);

/* Screen-tile binning (replaces compute_triangle_rects + compute_fragments +
 * filter_valid_fragments of rasterize.py:40-76): per (view, triangle) rect of
 * rasterize.cu:43-137, then per-tile triangle lists.  Never host-synchronising;
 * lists that would exceed list_capacity set DS_STATUS_LIST_OVERFLOW in
 * *status (device int) and those tiles fall back to testing every triangle of
 * their view, so results stay exact. */
int ds_tiles_bin(int B, const ds_view_desc* views, int num_tiles, int V, const float* pos, int T, const int* tri,
                 void* workspace, size_t workspace_bytes, int64_t list_capacity, int* status, ds_stream_t stream);

/* Tiled forward rasterizer with stochastic opacity (replaces
 * rasterize_multires_triangle_alpha, python/diffsoup/multires.py:52-102:
 * multires_triangle_alpha + threshold + depth_test).  Uses the bins of the
 * preceding ds_tiles_bin on the same workspace.  alpha_src [T,S] at `level`.
 * Threshold: thr_mode 0 = constant thr_const (0.5 is stochastic=False);
 * thr_mode 1 = Philox-4x32-10 uniform keyed by (seed, iteration, view,
 * pixel, triangle) with rng = device uint64[2] {seed, iteration}.
 * Writes every pixel of rast (zeros where empty). */
int ds_tiles_rasterize(int B, const ds_view_desc* views, int num_tiles, int V, const float* pos, int T,
                       const int* tri, int level, int S, const float* alpha_src, int thr_mode, float thr_const,
                       const uint64_t* rng, float* rast, void* workspace, size_t workspace_bytes,
                       int64_t list_capacity, ds_stream_t stream);

/* Tiled opacity auxiliary gradient (replaces the forward of
 * _OpacityAuxLossFn, python/diffsoup/rasterize.py:147-190: fragments +
 * multires_triangle_alpha + backward_opacity_aux_loss +
 * backward_multires_triangle_alpha).  Recomputes the fragments tile by tile
 * from the bins.  color/target [pixels, C]; grad_alpha_src [T,S] accumulates
 * scale * dL/dalpha_src. */
int ds_tiles_opacity_aux(int B, const ds_view_desc* views, int num_tiles, int V, const float* pos, int T,
                         const int* tri, int level, int S, const float* alpha_src, int C, const float* color,
                         const float* target, const float* rast, float scale, float* grad_alpha_src,
                         void* workspace, size_t workspace_bytes, int64_t list_capacity, ds_stream_t stream);

/* ===================================================================== */
/*  Batched training step                                                 */
/* ===================================================================== */

/* One training step of examples/02_synthetic.py:354-388 with an MSE
 * photometric loss, for B views at once:
 *   alpha = sigmoid(accumulate_to_level(min..max -> max, alpha_src))
 *   feat  = sigmoid(accumulate_to_level(min..max -> max, feat_src))
 *   pos   = project(verts, mvp)                                (utils.py:412-426)
 *   rast  = rasterize_multires_triangle_alpha(pos, tri, max, alpha, stochastic)
 *   x     = [multires_triangle_color(rast, feat), enc(rast, inv_mvp)]
 *           enc = the 3-D view direction, or encode_view_dir_sh2 (9
 *           coefficients, examples/02_synthetic.py:364) with view_enc = 1
 *   color = mask ? ColorMLP(x) : 1;  loss = mean((color - target)^2)
 *           + opacity_aux_loss(...) + edge_grad(...)   (zero-valued hooks)
 * and the gradients of loss with respect to verts, feat_src, alpha_src and
 * the MLP parameters (overwritten, not accumulated).  The MLP runs on the
 * BF16 tensor cores with FP32 accumulation (see `precision`).  Built shading
 * MLPs (features + encoding -> hidden layers -> 3): the reference's own model
 * 7 + SH2 -> 16 -> 16 -> 3 (examples/02_synthetic.py:289-306), 8 + direction
 * -> 16 -> 3 and 16 + direction -> 64 -> 64 -> 3; others return DS_ERR_ARG.
 * Never host-synchronising; capturable in a CUDA graph.  With stochastic
 * opacity, rng = device uint64[2] {seed, iteration} and the iteration is
 * incremented on the device at the end of the step. */
typedef struct {
    int32_t B, T, V;         /* views, triangles, vertices */
    int32_t C;               /* feature channels */
    int32_t min_level, max_level;
    int32_t hidden, n_layers;/* shading MLP: (C+enc) -> hidden x n_layers -> 3 */
    int32_t stochastic;      /* 1: Philox threshold per (view, pixel, triangle); 0: thr_const */
    float thr_const;
    /* Fragment records per pixel reserved in the workspace (plus one chunk
     * of 256 per rasterizer warp).  The rasterizer keeps every fragment in
     * front of each pixel's surface there, and the opacity auxiliary gradient
     * reads them back; blocks that do not fit are re-enumerated (same
     * result, status bit DS_STATUS_RECORD_FALLBACK).  0 re-enumerates every
     * block.  2 covers the benchmark scenes. */
    float frag_records;
    /* Shading precision.  0: features gathered as BF16, MLP operands BF16
     * (one mma per product).  1: split BF16 -- fp32 features, every MLP
     * operand as bf16 hi + bf16 lo and each product hi*hi + hi*lo + lo*hi on
     * the BF16 tensor cores (FP32 accumulation), gradients within ~1e-5 of
     * FP64 instead of the ~5e-3 that BF16 inputs alone cause. */
    int32_t precision;
    /* Pixel block of one rasterizer warp (8 per 16x16 tile): 0 = 8x4,
     * 1 = 16x2, 2 = 4x8.  Same results; the fastest depends on the scene
     * (diffsoup_b200.step.TrainStep.autotune times them). */
    int32_t block_shape;
    /* View encoding appended to the features: 0 = the 3-D view direction
     * (3 inputs), 1 = its SH2 coefficients (9 inputs, encoding.cu:56-118). */
    int32_t view_enc;
    /* Target images: 0 = fp32 [pixels,3]; 1 = 8-bit [pixels,3] (the
     * reference's datasets are 8-bit images), read as value / 255. */
    int32_t target_u8;
    /* Shading kernel of the 16 + direction -> 64 -> 64 -> 3 MLP in BF16
     * precision: 0 = warp-level tensor-core products (mma.sync) with operand
     * tiles in shared memory; 1 = tcgen05.mma on 128-pixel tiles with the
     * accumulators (and the weight gradients of the whole launch) in tensor
     * memory.  Other MLPs and split precision ignore it. */
    int32_t shade_mode;
} ds_step_config;

/* Packed MLP parameter layout (fp32): W0[hidden][C+3] b0[hidden]
 * (Wl[hidden][hidden] bl[hidden]) x (n_layers-1) Wout[3][hidden] bout[3],
 * i.e. torch.nn.Linear weights in ColorMLP order. */
int ds_mlp_param_count(int C, int hidden, int n_layers);

/* The same count for a step's MLP: W0 has C+3 or C+9 columns (view_enc). */
int ds_step_mlp_param_count(const ds_step_config* cfg);

size_t ds_train_step_workspace_size(const ds_step_config* cfg, int num_tiles, int64_t num_pixels,
                                    int64_t list_capacity);

/* Profiling hook: while set, ds_train_step records events[i] (cudaEvent_t)
 * on its stream at the phase boundaries start | prep | bin | raster | shade |
 * aux | edge | end (n <= 8; n = 0 disables). */
int ds_train_step_set_events(void* const* events, int n);

/* Byte offsets inside the train-step workspace of its intermediates, for
 * inspection after a step: [0] pos [B,V,4] f32, [1] opacity [T,S_max] f32,
 * [2] features [T,S_max,Cp] f32 (Cp = C rounded up to a multiple of 8,
 * padding channels zero), [3] features bf16 [T,S_max,Cp], [4] rast [pixels,4],
 * [5] colour [pixels,3], [6] dL/dcolour [pixels,3], [7] |c - target| summed
 * [pixels], [8] dL/dpos [B,V,4] f64, [9] dL/dopacity, [10] dL/dfeatures [T,S_max,Cp],
 * [11] fragment records int32 [capacity,4] {pixel, triangle | visible << 31,
 * b0 bits, b1 bits}, [12] record count of each 256-record chunk int32,
 * [13] int32 {records reserved, blocks re-enumerated}, [14] ids of the
 * re-enumerated 8x4 blocks (tile * 8 + block) int32; [15] holds the record
 * capacity itself.  offsets has room for 16 entries. */
int ds_train_step_layout(const ds_step_config* cfg, int num_tiles, int64_t num_pixels, int64_t list_capacity,
                         int64_t* offsets);

/* verts [V,3], tri [T,3], mvp/inv_mvp [B,4,4], feat_src [T,S,C],
 * alpha_src [T,S], target [pixels,3] fp32 or uint8 (cfg->target_u8; views
 * packed by ds_view_desc),
 * loss [1]; grad_* match their parameters.  rast_out [pixels,4] and
 * color_out [pixels,3] are optional (NULL: kept in the workspace). */
int ds_train_step(const ds_step_config* cfg, const ds_view_desc* views, int num_tiles, int64_t num_pixels,
                  const float* verts, const int* tri, const float* mvp, const float* inv_mvp, const float* feat_src,
                  const float* alpha_src, const float* mlp_params, const void* target, uint64_t* rng, float* loss,
                  float* grad_verts, float* grad_feat_src, float* grad_alpha_src, float* grad_mlp_params,
                  float* rast_out, float* color_out, void* workspace, size_t workspace_bytes, int64_t list_capacity,
                  int* status, ds_stream_t stream);

/* 3-D view direction per covered pixel (compute_view_direction of
 * src/cuda/encoding.cu:28-53, which the reference does not export): enc [B,H,W,3]. */
int ds_encode_view_dir(int B, int H, int W, const float* rast, const float* inv_mvp, float* encoding,
                       ds_stream_t stream);

/* Pixels per triangle of an ID buffer: counts[id] += number of pixels of
 * rast [num_pixels,4] whose rast[..,3] == id + 1 (count_triangle_ids,
 * python/diffsoup/rasterize.py:348-366, computed there with torch.bincount).
 * counts [num_tris] int64 accumulates (the caller zeroes it).  An ID at or
 * above num_tris is not counted and sets *status |= 1 (status may be NULL);
 * the reference asserts on that case.  Not host-synchronising. */
int ds_count_triangle_ids(int64_t num_pixels, const float* rast, int num_tris, int64_t* counts, int* status,
                          ds_stream_t stream);

/* ===================================================================== */
/*  Optimiser updates                                                     */
/* ===================================================================== */

/* Adam as torch.optim.Adam computes it (examples/02_synthetic.py:310-315
 * uses it for features, opacities and the MLP): for the n elements of param,
 * with t = *step + 1,
 *   exp_avg    <- exp_avg + (1 - beta1) (grad - exp_avg)
 *   exp_avg_sq <- beta2 exp_avg_sq + (1 - beta2) grad^2
 *   param      <- param - lr / (1 - beta1^t) * exp_avg
 *                         / (sqrt(exp_avg_sq) / sqrt(1 - beta2^t) + eps)
 * then *step <- t.  step is a device int32 (the state's step count), so the
 * update captures into a CUDA graph.  The hyperparameters are doubles, as
 * torch's Python scalars are (1 - beta is formed before rounding to FP32).
 * Not host-synchronising. */
int ds_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, double lr,
                 double beta1, double beta2, double eps, int* step, ds_stream_t stream);

/* replaces VectorAdam.step (python/diffsoup/optimize.py:36-68) for one
 * parameter of `rows` vectors of `dim` components (vertex positions: dim 3):
 * with t = *step + 1, per row
 *   g1 <- beta1 g1 + (1 - beta1) grad          g1 [rows, dim]
 *   g2 <- beta2 g2 + (1 - beta2) |grad|^2      g2 [rows, 1]
 *   param <- param - lr (g1 / (1 - beta1^t)) / (sqrt(g2 / (1 - beta2^t)) + 1e-8)
 * then *step <- t (device int32).  Not host-synchronising. */
int ds_vector_adam_step(float* param, const float* grad, float* g1, float* g2, int64_t rows, int dim, double lr,
                        double beta1, double beta2, int* step, ds_stream_t stream);

/* Clip-space positions pos [B,V,4] = mvp[b] . (verts[v], 1) with mvp [B,4,4]
 * row-major (project_vertices, examples/utils.py:412-426; the training step
 * projects with the same kernel).  pos 16-byte aligned. */
int ds_project_vertices(int B, int V, const float* verts, const float* mvp, float* pos, ds_stream_t stream);

/* ===================================================================== */
/*  Soup subdivision (resampling): longest-edge splits under a threshold  */
/* ===================================================================== */

/* replaces _core.split_triangle_soup (src/main.cpp:308-340, src/remesh.cpp)
 * with mode 0 and _core.split_triangle_soup_clip (src/main.cpp:342-388,
 * src/remesh_clip.cpp) with mode 1.  A face is bisected at its longest edge
 * (squared length in world units, mode 0; in mode 1 in NDC with x scaled by
 * aspect_wh = W/H, edges with an end outside the NDC cube ignored, faces
 * with valid[t] <= 0 never split); both halves continue.  num_splits < 0
 * (the reference's `*_until` functions, which training calls,
 * examples/utils.py:540): split while the longest edge is at least tau
 * (mode 0) or 2 tau (mode 1: tau is the reference's tau_ratio in image
 * heights); tau <= 0 splits nothing.  num_splits > 0: the num_splits longest
 * splits of all faces, as the reference's queue pops them, stopping early at
 * the threshold when tau > 0; splits of exactly equal length at the cut-off
 * are taken in face order (the reference's heap takes them in an unspecified
 * order).  num_splits == 0: nothing.  mvp_host: row-major 4x4 in host memory
 * (mode 1; NULL in mode 0).
 *
 * Two calls on one workspace.  ds_split_soup_count writes split_offsets [M+1]
 * (int64, device): the exclusive offsets of each face's splits and their
 * total, which it also returns in *total_splits_host; host-synchronising (a
 * split budget runs a search of counting passes), like the reference's
 * binding returning its arrays.  A face whose split tree would exceed 2^20
 * splits or a depth of 40, or a pass above 2^27 splits, sets
 * DS_STATUS_SPLIT_LIMIT in *status (device int); do not emit then.
 * ds_split_soup_emit follows the plan the count call left in the workspace
 * and writes, for S = total splits: out_verts [N+3S,3] (the inputs, then per
 * split the two copies of the split point and the copy of the opposite
 * vertex), out_faces [M+S,3], out_map [M+S] (input face of each output face)
 * and out_flag [M+S] (1 for faces never split), the reference's four outputs.
 * The same triangles as the reference, bit for bit; new vertices and faces
 * are numbered per input face in depth-first order (the reference's follow its
 * global queue order). */
size_t ds_split_soup_workspace_size(int M);
int ds_split_soup_count(int mode, const float* mvp_host, float aspect_wh, float tau, int num_splits, int N,
                        const float* verts, int M, const int* faces, const int* valid, int64_t* split_offsets,
                        int64_t* total_splits_host, void* workspace, size_t workspace_bytes, int* status,
                        ds_stream_t stream);
int ds_split_soup_emit(int mode, const float* mvp_host, float aspect_wh, int N, const float* verts, int M,
                       const int* faces, const int64_t* split_offsets, int64_t total_splits, const void* workspace,
                       float* out_verts, int* out_faces, int* out_map, int* out_flag, int* status,
                       ds_stream_t stream);

/* ===================================================================== */
/*  Inference render: the viewer's deferred shading without a window      */
/* ===================================================================== */

/* The LUT is the viewer's pair of RGBA8 textures (viewer/src/viewer.cpp:
 * 549-554, packed by examples/05_benchmark_fps.py:56-80 and :315-317):
 * texel t = face * S + lattice index at `level` (S = texels per face),
 * lut0[t] = 255 * (f0, f1, f2, f3), lut1[t] = 255 * (f4, f5, f6, opacity),
 * num_texels >= T * S (the texture may be padded).  mlp_params packs
 * W1 [16,16], b1 [16], W2 [16,16], b2 [16], W3 [3,16], b3 [3] (torch Linear
 * layout [out, in]; 595 floats). */

/* Opacity channel as FP32 for the geometry pass: alpha[t] = lut1[t].a / 255
 * for t < num_texels (the texture fetch of viewer.cpp:228, UNORM8 decode). */
int ds_render_lut_opacity(int64_t num_texels, const unsigned char* lut1, float* alpha, ds_stream_t stream);

/* Post pass of viewer.cpp:241-341 over a G-buffer gbuf [num_pixels,4] in the
 * rasterizer's layout (b0, b1, z/w, triangle id + 1; id 0 = empty): LUT
 * interpolation at the fragment's lattice cell (viewer.cpp:197-230), view
 * direction through inv_mvp [B,16] at the pixel centre, SH2 encoding, MLP
 * 16 -> 16 -> 16 -> 3 and mix(A.rgb, mlp, A.a); empty pixels take the
 * background.  Writes rgb [num_pixels,3] FP32 and/or rgba8 [num_pixels,4]
 * (either may be NULL, not both). */
int ds_render_deferred(int B, const ds_view_desc* views, int64_t num_pixels, const float* gbuf, int level,
                       const unsigned char* lut0, const unsigned char* lut1, int64_t num_texels,
                       const float* inv_mvp, const float* mlp_params, float bg_r, float bg_g, float bg_b,
                       float* rgb, unsigned char* rgba8, ds_stream_t stream);

/* Bytes of workspace for ds_render_frame. */
size_t ds_render_workspace_size(int B, int V, int T, int num_tiles, int64_t list_capacity);

/* One frame of the viewer (replaces Viewer::launch_benchmark's render_one,
 * viewer/src/viewer.cpp:861-909, and Viewer::render, :663-720) for B views:
 * projection of verts [V,3] by mvp [B,4,4] row-major, screen-tile binning,
 * the geometry pass (nearest fragment whose LUT opacity alpha [T,S] -- from
 * ds_render_lut_opacity -- is at least 0.5; triangle ID buffer into gbuf)
 * and the post pass of ds_render_deferred.  Never host-synchronising and
 * capturable in a CUDA graph; a bin list overflow sets DS_STATUS_LIST_OVERFLOW
 * in *status and stays exact (ds_tiles_bin). */
int ds_render_frame(int B, const ds_view_desc* views, int num_tiles, int64_t num_pixels, int V, const float* verts,
                    int T, const int* faces, const float* mvp, const float* inv_mvp, int level,
                    const unsigned char* lut0, const unsigned char* lut1, int64_t num_texels, const float* alpha,
                    const float* mlp_params, float bg_r, float bg_g, float bg_b, float* gbuf, float* rgb,
                    unsigned char* rgba8, void* workspace, size_t workspace_bytes, int64_t list_capacity,
                    int* status, ds_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* DIFFSOUP_B200_H */
