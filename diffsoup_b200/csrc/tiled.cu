// diffsoup_b200/csrc/tiled.cu -- screen-tile binning, tiled forward
// rasterizer and tiled opacity auxiliary gradient.
//
// The reference enumerates one fragment per bbox pixel into global memory,
// compacts it, and resolves depth with 64-bit atomics
// (src/cuda/rasterize.cu:139-400).  Here each (view, triangle) is binned into
// the 16x16 screen tiles its rect (rasterize.cu:43-137) overlaps; one CTA per
// tile stages the tile's triangle records in shared memory, each warp skips
// the triangles whose rect misses its 8x4 pixel block, and every thread
// resolves its own pixel's depth test in registers.  No fragment list, no
// global atomics, one coalesced 16-byte store per pixel.
//
// Results equal the reference's: coverage, barycentrics and depth use its
// FP32 arithmetic, the depth key is bits(z+2) with ties broken by the lower
// triangle index (its fragment order), and the opacity test is applied
// before the depth comparison exactly as depth_test_kernel does.
#include "edge_math.cuh"
#include "scan.cuh"

namespace dsb {

// Per (view, triangle) record: clip vertices and the pixel rect
// [y0, y1) x [x0, x1) (empty when y1 <= y0).
struct __align__(16) TriRec {
    float4 p0, p1, p2;
    int4 rect;  // y0, y1, x0, x1
};
static_assert(sizeof(TriRec) == 64, "TriRec layout");

constexpr int kTileThreads = 256;  // one pixel per thread of a 16x16 tile
constexpr int kAuxSmemS = 160;     // per-warp shared accumulator for lattices up to level 4

struct TileWs {
    TriRec* recs;
    int* counts;
    int64_t* offsets;  // [num_tiles + 1] exclusive prefix of counts
    int* cursor;
    int* list;
    int* work;  // persistent-kernel tile queue counters [2]
    void* scan;
};

static inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

static TileWs carve(void* ws, int B, int T, int num_tiles, int64_t capacity, size_t* total) {
    char* p = reinterpret_cast<char*>(ws);
    TileWs w;
    size_t o = 0;
    w.recs = reinterpret_cast<TriRec*>(p + o); o += al256((size_t)B * T * sizeof(TriRec));
    w.counts = reinterpret_cast<int*>(p + o); o += al256((size_t)num_tiles * sizeof(int));
    w.offsets = reinterpret_cast<int64_t*>(p + o); o += al256((size_t)(num_tiles + 1) * sizeof(int64_t));
    w.cursor = reinterpret_cast<int*>(p + o); o += al256((size_t)num_tiles * sizeof(int));
    w.work = reinterpret_cast<int*>(p + o); o += 256;
    w.scan = p + o; o += al256(scan_workspace_bytes(num_tiles));
    w.list = reinterpret_cast<int*>(p + o); o += al256((size_t)capacity * sizeof(int));
    if (total) *total = o;
    return w;
}

__device__ __forceinline__ int find_view(const ds_view_desc* __restrict__ views, int B, int tile) {
    int lo = 0, hi = B - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&views[mid].tile_base) <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Tile range of a rect; false when the rect is empty.
__device__ __forceinline__ bool rect_tiles(const int4 r, int& tx0, int& tx1, int& ty0, int& ty1) {
    if (r.y <= r.x || r.w <= r.z) return false;
    tx0 = r.z / DS_TILE; tx1 = (r.w - 1) / DS_TILE;
    ty0 = r.x / DS_TILE; ty1 = (r.y - 1) / DS_TILE;
    return true;
}

// Pass 1: records and per-tile counts.
__global__ void __launch_bounds__(kThreads) bin_setup_kernel(int B, const ds_view_desc* __restrict__ views, int V,
                                                             const float* __restrict__ pos, int T,
                                                             const int* __restrict__ tri, TriRec* __restrict__ recs,
                                                             int* __restrict__ counts) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * T) return;
    const int b = (int)(i / T), t = (int)(i % T);
    const ds_view_desc vd = views[b];
    const float* P = pos + (size_t)b * V * 4;
    TriRec r;
    r.p0 = load_vertex(P, __ldg(tri + t * 3 + 0));
    r.p1 = load_vertex(P, __ldg(tri + t * 3 + 1));
    r.p2 = load_vertex(P, __ldg(tri + t * 3 + 2));
    int h0, hl, w0, wl;
    triangle_rect(vd.H, vd.W, r.p0, r.p1, r.p2, h0, hl, w0, wl);
    r.rect = make_int4(h0, h0 + hl, w0, w0 + wl);
    recs[i] = r;
    int tx0, tx1, ty0, ty1;
    if (!rect_tiles(r.rect, tx0, tx1, ty0, ty1)) return;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) atomicAdd(counts + vd.tile_base + ty * vd.tiles_x + tx, 1);
}

// Pass 2: scatter record indices into the per-tile lists.
__global__ void __launch_bounds__(kThreads) bin_fill_kernel(int B, const ds_view_desc* __restrict__ views, int T,
                                                            const TriRec* __restrict__ recs,
                                                            const int64_t* __restrict__ offsets,
                                                            int* __restrict__ cursor, int* __restrict__ list,
                                                            int64_t capacity, int* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * T) return;
    const int b = (int)(i / T);
    const ds_view_desc vd = views[b];
    const int4 rc = recs[i].rect;
    int tx0, tx1, ty0, ty1;
    if (!rect_tiles(rc, tx0, tx1, ty0, ty1)) return;
    bool over = false;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const int tile = vd.tile_base + ty * vd.tiles_x + tx;
            const int64_t at = offsets[tile] + atomicAdd(cursor + tile, 1);
            if (at < capacity) list[at] = (int)i; else over = true;
        }
    if (over) atomicOr(status, DS_STATUS_LIST_OVERFLOW);
}

struct TileGeom {
    int b, px, py, H, W;
    int64_t pix;  // packed pixel index
    bool valid;
    int wx0, wy0;  // this warp's 8x4 block origin
    int64_t begin, end;  // entry range in the list, or [b*T, b*T+T) records when exhaustive
    bool exhaustive;
};

__device__ __forceinline__ TileGeom tile_geometry(int tile, int B, const ds_view_desc* __restrict__ views, int T,
                                                  const int64_t* __restrict__ offsets, int64_t capacity) {
    TileGeom g;
    g.b = find_view(views, B, tile);
    const ds_view_desc vd = views[g.b];
    const int tl = tile - vd.tile_base;
    const int tx = tl % vd.tiles_x, ty = tl / vd.tiles_x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    g.wx0 = tx * DS_TILE + (warp & 1) * 8;
    g.wy0 = ty * DS_TILE + (warp >> 1) * 4;
    g.px = g.wx0 + (lane & 7);
    g.py = g.wy0 + (lane >> 3);
    g.H = vd.H; g.W = vd.W;
    g.valid = g.px < vd.W && g.py < vd.H;
    g.pix = vd.pix_offset + (int64_t)g.py * vd.W + g.px;
    g.begin = offsets[tile];
    g.end = offsets[tile + 1];
    g.exhaustive = g.end > capacity;
    if (g.exhaustive) { g.begin = (int64_t)g.b * T; g.end = g.begin + T; }
    return g;
}

__device__ __forceinline__ bool warp_overlaps(const int4 r, int wx0, int wy0) {
    return r.x < wy0 + 4 && r.y > wy0 && r.z < wx0 + 8 && r.w > wx0;
}

__device__ __forceinline__ int next_tile(int* work, int* s_tile) {
    __syncthreads();
    if (threadIdx.x == 0) *s_tile = atomicAdd(work, 1);
    __syncthreads();
    return *s_tile;
}

// Forward: depth test with stochastic opacity, one CTA per tile (persistent).
__global__ void __launch_bounds__(kTileThreads) raster_kernel(int B, const ds_view_desc* __restrict__ views,
                                                              int num_tiles, int T, const TriRec* __restrict__ recs,
                                                              const int64_t* __restrict__ offsets,
                                                              const int* __restrict__ list, int64_t capacity,
                                                              int level, int S, const float* __restrict__ alpha_src,
                                                              int thr_mode, float thr_const,
                                                              const uint64_t* __restrict__ rng, int* work,
                                                              float* __restrict__ rast) {
    __shared__ TriRec s_rec[kTileThreads];
    __shared__ int s_tri[kTileThreads];
    __shared__ int s_tile;
    uint64_t seed = 0;
    uint32_t iter = 0;
    if (thr_mode == 1) { seed = rng[0]; iter = (uint32_t)rng[1]; }
    for (int tile = next_tile(work, &s_tile); tile < num_tiles; tile = next_tile(work, &s_tile)) {
        const TileGeom g = tile_geometry(tile, B, views, T, offsets, capacity);
        const float ndc_x = pix_ndc(g.px, g.W), ndc_y = pix_ndc(g.py, g.H);
        const uint32_t pixel_id = (uint32_t)(g.py * g.W + g.px);
        unsigned long long best = ~0ull;
        float bb0 = 0.f, bb1 = 0.f, bz = 0.f;
        for (int64_t c0 = g.begin; c0 < g.end; c0 += kTileThreads) {
            const int n = (int)min((int64_t)kTileThreads, g.end - c0);
            __syncthreads();
            if ((int)threadIdx.x < n) {
                const int64_t e = c0 + threadIdx.x;
                const int ri = g.exhaustive ? (int)e : __ldg(list + e);
                s_rec[threadIdx.x] = recs[ri];
                s_tri[threadIdx.x] = ri - g.b * T;
            }
            __syncthreads();
            for (int j = 0; j < n; ++j) {
                const int4 r = s_rec[j].rect;
                if (!warp_overlaps(r, g.wx0, g.wy0)) continue;  // warp-uniform
                if (!g.valid || g.px < r.z || g.px >= r.w || g.py < r.x || g.py >= r.y) continue;
                float b0, b1, depth;
                if (!fragment_at(ndc_y, ndc_x, s_rec[j].p0, s_rec[j].p1, s_rec[j].p2, b0, b1, depth)) continue;
                if (depth <= -1.f) continue;
                const uint32_t t = (uint32_t)s_tri[j];
                const unsigned long long key = depth_key(depth, t);
                if (key >= best) continue;
                const float alpha = interp_scalar(b0, b1, level, level, alpha_src + (size_t)t * S);
                const float thr = thr_mode == 1 ? philox_uniform(seed, iter, (uint32_t)g.b, pixel_id, t) : thr_const;
                if (alpha < thr) continue;
                best = key; bb0 = b0; bb1 = b1; bz = depth;
            }
        }
        if (g.valid) {
            float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
            if (best != ~0ull) o = make_float4(bb0, bb1, bz, (float)((uint32_t)(best & 0xffffffffu) + 1u));
            reinterpret_cast<float4*>(rast)[g.pix] = o;
        }
    }
}

// Opacity auxiliary gradient: re-enumerates each tile's fragments and
// scatters dL/dalpha through the lattice adjoint.  All lanes of a warp work
// on the same triangle at a time, so contributions are summed per warp in
// shared memory and flushed with one global atomic per touched sample.
__global__ void __launch_bounds__(kTileThreads) aux_kernel(int B, const ds_view_desc* __restrict__ views,
                                                           int num_tiles, int T, const TriRec* __restrict__ recs,
                                                           const int64_t* __restrict__ offsets,
                                                           const int* __restrict__ list, int64_t capacity, int level,
                                                           int S, const float* __restrict__ alpha_src, int C,
                                                           const float* __restrict__ color,
                                                           const float* __restrict__ target,
                                                           const float* __restrict__ rast, float scale, int* work,
                                                           float* __restrict__ grad_alpha_src) {
    __shared__ TriRec s_rec[kTileThreads];
    __shared__ int s_tri[kTileThreads];
    __shared__ float s_acc[kTileThreads / 32][kAuxSmemS];
    __shared__ int s_tile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool use_smem = S <= kAuxSmemS;
    if (use_smem)
        for (int k = lane; k < S; k += 32) s_acc[warp][k] = 0.f;
    for (int tile = next_tile(work, &s_tile); tile < num_tiles; tile = next_tile(work, &s_tile)) {
        const TileGeom g = tile_geometry(tile, B, views, T, offsets, capacity);
        const float ndc_x = pix_ndc(g.px, g.W), ndc_y = pix_ndc(g.py, g.H);
        int tp = -1;
        float zp = 0.f, loss = 0.f;
        if (g.valid) {
            const float4 rp = reinterpret_cast<const float4*>(rast)[g.pix];
            tp = (int)rp.w - 1;
            zp = rp.z;
            if (target != nullptr) {
                for (int c = 0; c < C; ++c) loss += fabsf(color[g.pix * C + c] - target[g.pix * C + c]);
            } else {
                loss = color[g.pix];  // caller passes the per-pixel sum |c - target| directly
            }
        }
        for (int64_t c0 = g.begin; c0 < g.end; c0 += kTileThreads) {
            const int n = (int)min((int64_t)kTileThreads, g.end - c0);
            __syncthreads();
            if ((int)threadIdx.x < n) {
                const int64_t e = c0 + threadIdx.x;
                const int ri = g.exhaustive ? (int)e : __ldg(list + e);
                s_rec[threadIdx.x] = recs[ri];
                s_tri[threadIdx.x] = ri - g.b * T;
            }
            __syncthreads();
            for (int j = 0; j < n; ++j) {
                const int4 r = s_rec[j].rect;
                if (!warp_overlaps(r, g.wx0, g.wy0)) continue;  // warp-uniform
                const int t = s_tri[j];
                bool hit = g.valid && g.px >= r.z && g.px < r.w && g.py >= r.x && g.py < r.y;
                float b0 = 0.f, b1 = 0.f, depth = 0.f;
                if (hit) hit = fragment_at(ndc_y, ndc_x, s_rec[j].p0, s_rec[j].p1, s_rec[j].p2, b0, b1, depth);
                if (hit && tp >= 0 && depth > zp) hit = false;
                uint32_t idx[3] = {0, 0, 0};
                float gw[3] = {0.f, 0.f, 0.f};
                if (hit) {
                    const float* as = alpha_src + (size_t)t * S;
                    const float alpha = interp_scalar(b0, b1, level, level, as);
                    const float ga = aux_alpha_grad(loss, alpha, tp >= 0 && t == tp) * scale;
                    float w[3];
                    lattice_cell(b0, b1, level, idx, w);
                    gw[0] = ga * w[0]; gw[1] = ga * w[1]; gw[2] = ga * w[2];
                }
                if (use_smem) {
                    if (!__any_sync(0xffffffffu, hit)) continue;
                    if (hit) {
#pragma unroll
                        for (int k = 0; k < 3; ++k) atomicAdd(&s_acc[warp][idx[k]], gw[k]);
                    }
                    __syncwarp();
                    float* dst = grad_alpha_src + (size_t)t * S;
                    for (int k = lane; k < S; k += 32) {
                        const float v = s_acc[warp][k];
                        if (v != 0.f) { atomicAdd(dst + k, v); s_acc[warp][k] = 0.f; }
                    }
                    __syncwarp();
                } else if (hit) {
                    float* dst = grad_alpha_src + (size_t)t * S;
#pragma unroll
                    for (int k = 0; k < 3; ++k) atomicAdd(dst + idx[k], gw[k]);
                }
            }
        }
    }
}

}  // namespace dsb

using namespace dsb;

extern "C" {

size_t ds_tiles_workspace_size(int B, int T, int num_tiles, int64_t list_capacity) {
    size_t total = 0;
    carve(nullptr, B, T, num_tiles, list_capacity, &total);
    return total;
}

static int check_tiles_args(int B, const ds_view_desc* views, int num_tiles, int V, const float* pos, int T,
                            size_t ws_bytes, int64_t capacity) {
    DS_CHECK_ARG(B >= 0 && num_tiles >= 0 && V >= 0 && T >= 0 && capacity >= 0, "tiles: bad sizes");
    DS_CHECK_ARG((int64_t)B * T <= 0x7fffffff, "tiles: B*T exceeds int32");
    DS_CHECK_ARG(capacity <= 0x7fffffff, "tiles: list capacity exceeds int32");
    DS_CHECK_ARG(B == 0 || views != nullptr, "tiles: null view table");
    DS_CHECK_ARG(((uintptr_t)pos & 15) == 0, "tiles: pos not 16-byte aligned");
    if (ws_bytes < ds_tiles_workspace_size(B, T, num_tiles, capacity))
        return set_error(DS_ERR_WORKSPACE, "tiles: workspace too small (%zu < %zu)", ws_bytes,
                         ds_tiles_workspace_size(B, T, num_tiles, capacity));
    return DS_OK;
}

int ds_tiles_bin(int B, const ds_view_desc* views, int num_tiles, int V, const float* pos, int T, const int* tri,
                 void* workspace, size_t workspace_bytes, int64_t list_capacity, int* status, ds_stream_t stream) {
    int rc = check_tiles_args(B, views, num_tiles, V, pos, T, workspace_bytes, list_capacity);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    TileWs w = carve(workspace, B, T, num_tiles, list_capacity, nullptr);
    DS_CUDA(cudaMemsetAsync(w.counts, 0, (size_t)num_tiles * sizeof(int), st));
    DS_CUDA(cudaMemsetAsync(w.cursor, 0, (size_t)num_tiles * sizeof(int), st));
    const int64_t n = (int64_t)B * T;
    if (n > 0) bin_setup_kernel<<<blocks_for(n), kThreads, 0, st>>>(B, views, V, pos, T, tri, w.recs, w.counts);
    int64_t* total_dev = nullptr;
    rc = device_scan<int, int64_t>(w.counts, num_tiles, w.offsets, false, w.scan, st, &total_dev);
    if (rc) return rc;
    // offsets[num_tiles] = total number of entries
    DS_CUDA(cudaMemcpyAsync(w.offsets + num_tiles, total_dev, sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    if (n > 0)
        bin_fill_kernel<<<blocks_for(n), kThreads, 0, st>>>(B, views, T, w.recs, w.offsets, w.cursor, w.list,
                                                            list_capacity, status);
    return check_launch("tiles_bin");
}

static unsigned tile_grid(int num_tiles) {
    const int per_sm = 4;  // 256-thread CTAs, ~17 KB shared each
    return (unsigned)max(1, min(num_tiles, kSMs * per_sm));
}

int ds_tiles_rasterize(int B, const ds_view_desc* views, int num_tiles, int V, const float* pos, int T,
                       const int* tri, int level, int S, const float* alpha_src, int thr_mode, float thr_const,
                       const uint64_t* rng, float* rast, void* workspace, size_t workspace_bytes,
                       int64_t list_capacity, ds_stream_t stream) {
    (void)tri;
    int rc = check_tiles_args(B, views, num_tiles, V, pos, T, workspace_bytes, list_capacity);
    if (rc) return rc;
    DS_CHECK_ARG(level >= 0 && level <= 12 && (uint32_t)S == feats_at_level(level), "Invalid feature size.");
    DS_CHECK_ARG(thr_mode == 0 || (thr_mode == 1 && rng != nullptr), "tiles_rasterize: bad threshold mode");
    DS_CHECK_ARG(((uintptr_t)rast & 15) == 0, "tiles_rasterize: rast not 16-byte aligned");
    if (num_tiles == 0) return DS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    TileWs w = carve(workspace, B, T, num_tiles, list_capacity, nullptr);
    DS_CUDA(cudaMemsetAsync(w.work, 0, sizeof(int), st));
    raster_kernel<<<tile_grid(num_tiles), kTileThreads, 0, st>>>(B, views, num_tiles, T, w.recs, w.offsets, w.list,
                                                                 list_capacity, level, S, alpha_src, thr_mode,
                                                                 thr_const, rng, w.work, rast);
    return check_launch("tiles_rasterize");
}

int ds_tiles_opacity_aux(int B, const ds_view_desc* views, int num_tiles, int V, const float* pos, int T,
                         const int* tri, int level, int S, const float* alpha_src, int C, const float* color,
                         const float* target, const float* rast, float scale, float* grad_alpha_src,
                         void* workspace, size_t workspace_bytes, int64_t list_capacity, ds_stream_t stream) {
    (void)tri;
    int rc = check_tiles_args(B, views, num_tiles, V, pos, T, workspace_bytes, list_capacity);
    if (rc) return rc;
    DS_CHECK_ARG(level >= 0 && level <= 12 && (uint32_t)S == feats_at_level(level), "Invalid feature size.");
    DS_CHECK_ARG(C > 0, "tiles_opacity_aux: C must be positive");
    DS_CHECK_ARG(target != nullptr || C == 1, "tiles_opacity_aux: without a target, color holds one value per pixel");
    DS_CHECK_ARG(((uintptr_t)rast & 15) == 0, "tiles_opacity_aux: rast not 16-byte aligned");
    if (num_tiles == 0) return DS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    TileWs w = carve(workspace, B, T, num_tiles, list_capacity, nullptr);
    DS_CUDA(cudaMemsetAsync(w.work + 1, 0, sizeof(int), st));
    aux_kernel<<<tile_grid(num_tiles), kTileThreads, 0, st>>>(B, views, num_tiles, T, w.recs, w.offsets, w.list,
                                                              list_capacity, level, S, alpha_src, C, color, target,
                                                              rast, scale, w.work + 1, grad_alpha_src);
    return check_launch("tiles_opacity_aux");
}

}  // extern "C"
