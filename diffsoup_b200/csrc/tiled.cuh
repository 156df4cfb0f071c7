// diffsoup_b200/csrc/tiled.cuh -- internal interface of the tiled rasterizer
// used by the training step (csrc/step.cu).
#pragma once

#include "common.cuh"

namespace dsb {

// Per (view, triangle): the pixel rect [y0, y1) x [x0, x1) (empty when
// y1 <= y0) and bounds [zlo, zhi] on the NDC depth of every fragment the
// triangle can produce.  With every w > 0 (the rect test culls the rest), a
// fragment's depth z/w is a convex combination of the vertices' z_i/w_i, so
// [min, max] of those bound it; the bounds are widened by the rounding of the
// fragment arithmetic.
struct __align__(16) TriBox {
    short y0, y1, x0, x1;
    float zlo, zhi;
};
static_assert(sizeof(TriBox) == 16, "TriBox layout");

// Per (view, triangle): the clip-space vertices, and their NDC x, y
// (x_k / w_k, y_k / w_k: a = (x0, y0, x1, y1), b = (x2, y2, m_lo, m_hi) with
// m the binning pass's 64-bit mask of the tiles the triangle may cover).
struct __align__(16) TriVerts {
    float4 p0, p1, p2;
};

struct __align__(16) TriNdc {
    float4 a, b;
};

// The per-(view, triangle) tables the binning pass leaves in the tiles
// workspace, indexed view * T + triangle.
struct TileTables {
    const TriBox* boxes;
    const TriVerts* verts;
    const TriNdc* ndc;
    const int64_t* offsets;  // [num_tiles + 1] list ranges: a tile whose range is empty has no covered pixel
};

TileTables tiles_tables(void* workspace, int B, int T, int num_tiles, int64_t list_capacity);

// Fragment record store.  The forward rasterizer can keep, per pixel, every
// fragment in front of (or level with) the visible surface -- exactly the
// fragments the opacity auxiliary gradient visits (rasterize.cu:950) -- so
// that the backward pass reads them instead of re-enumerating the tiles.
// Records are 16 bytes {pixel, triangle | visible << 31, b0, b1}, written in
// chunks of kRecChunk that warps reserve with one atomic each; chunk_fill
// holds each chunk's record count.  Blocks whose records do not fit (more
// than the per-warp buffer, or the store is full) are listed in `fallback`
// and re-enumerated by the backward pass.
constexpr int kRecChunk = 256;

struct RecordStore {
    int4* rec;         // [capacity]
    int* chunk_fill;   // [capacity / kRecChunk]
    int* counters;     // [0] records reserved, [1] fallback blocks; zeroed before the rasterizer
    int* fallback;     // [num_tiles * 8] block ids
    int64_t capacity;  // multiple of kRecChunk
};

// Pixel blocks of the tiled kernels: a warp takes 32 pixels of a 16x16 tile,
// 2^bwl wide and 32 / 2^bwl high (bwl 3: 8x4, the default; 4: 16x2; 2: 4x8).
// The rasterizer and the opacity pass of one step must use the same shape
// (re-enumerated blocks are named by block index).
constexpr int kDefaultBlockShape = 3;

// Rasterizer of ds_tiles_rasterize; records fragments when rs != nullptr.
int tiles_rasterize_impl(int B, const ds_view_desc* views, int num_tiles, int T, int level, int S,
                         const float* alpha_src, int thr_mode, float thr_const, const uint64_t* rng, float* rast,
                         void* workspace, int64_t list_capacity, const RecordStore* rs, cudaStream_t st, int bwl);

// Opacity auxiliary gradient with a per-pixel loss l1 [pixels]: from the
// records plus the fallback blocks when rs != nullptr, else by
// re-enumerating every block.
int tiles_aux_impl(int B, const ds_view_desc* views, int num_tiles, int T, int level, int S, const float* alpha_src,
                   const float* l1, const float* rast, float scale, float* grad_alpha_src, void* workspace,
                   int64_t list_capacity, const RecordStore* rs, cudaStream_t st, int bwl);


}  // namespace dsb
