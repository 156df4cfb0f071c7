// diffsoup_b200/csrc/tiled.cu -- screen-tile binning, tiled forward
// rasterizer and tiled opacity auxiliary gradient.
//
// The reference enumerates one fragment per bbox pixel into global memory,
// compacts it, and resolves depth with 64-bit atomics
// (src/cuda/rasterize.cu:139-400).  Here each (view, triangle) is binned into
// the 16x16 screen tiles its rect (rasterize.cu:43-137) overlaps, and each
// tile's list is sorted by the triangles' near-depth bound.  A work item is
// one 8x4 pixel block of a tile, owned by one warp: the warp filters the
// tile's triangle boxes 32 at a time (rect overlap, depth bound), stages the
// survivors' vertices in its own shared memory, and every lane resolves its
// pixel's depth test in registers.  Warps never wait for each other: no
// fragment list, no CTA barrier, no global atomics, one 16-byte store per
// pixel.
//
// Results equal the reference's: coverage, barycentrics and depth use its
// FP32 arithmetic, the depth key is bits(z+2) with ties broken by the lower
// triangle index (its fragment order), and the opacity test is applied
// before the depth comparison exactly as depth_test_kernel does.
#include "edge_math.cuh"
#include "scan.cuh"
#include "tiled.cuh"

namespace dsb {

constexpr int kWarpsPerCta = 8;
constexpr int kBlocksPerTile = 8;  // 32-pixel blocks of a 16x16 tile, one warp each
static_assert(DS_TILE == 16, "the block decode of block_geometry assumes 16x16 tiles");
constexpr int kSortMax = 512;      // longest tile list sorted by depth
constexpr int kSortWarps = 8;      // warps (tiles) per CTA of the sort pass

// One entry of a tile's list: the (view, triangle) record's pixel rect and
// near depth bound, and the record index -- what the rasterizer's staging
// and the sort by depth read, without a second, dependent load.
struct __align__(16) ListEntry {
    short y0, y1, x0, x1;
    float zlo;
    int ri;
};
static_assert(sizeof(ListEntry) == 16, "ListEntry layout");
constexpr int kAuxSmemS = 160;     // per-warp shared accumulator for lattices up to level 4

struct TileWs {
    TriBox* boxes;
    TriVerts* verts;
    TriNdc* ndc;
    TriEdges* edges;
    int* counts;
    int64_t* offsets;  // [num_tiles + 1] exclusive prefix of counts
    int* cursor;
    int* sorted;       // per tile: 1 when its list is ordered by zlo
    ListEntry* list;
    ListEntry* fill;   // the fill pass's unsorted lists (same offsets)
    int* work;         // persistent-kernel work counters [2]
    void* scan;
};

static inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

static TileWs carve(void* ws, int B, int T, int num_tiles, int64_t capacity, size_t* total) {
    char* p = reinterpret_cast<char*>(ws);
    TileWs w;
    size_t o = 0;
    w.boxes = reinterpret_cast<TriBox*>(p + o); o += al256((size_t)B * T * sizeof(TriBox));
    w.verts = reinterpret_cast<TriVerts*>(p + o); o += al256((size_t)B * T * sizeof(TriVerts));
    w.ndc = reinterpret_cast<TriNdc*>(p + o); o += al256((size_t)B * T * sizeof(TriNdc));
    w.edges = reinterpret_cast<TriEdges*>(p + o); o += al256((size_t)B * T * sizeof(TriEdges));
    w.counts = reinterpret_cast<int*>(p + o); o += al256((size_t)num_tiles * sizeof(int));
    w.offsets = reinterpret_cast<int64_t*>(p + o); o += al256((size_t)(num_tiles + 1) * sizeof(int64_t));
    w.cursor = reinterpret_cast<int*>(p + o); o += al256((size_t)num_tiles * sizeof(int));
    w.sorted = reinterpret_cast<int*>(p + o); o += al256((size_t)num_tiles * sizeof(int));
    w.work = reinterpret_cast<int*>(p + o); o += 256;
    w.scan = p + o; o += al256(scan_workspace_bytes(num_tiles));
    w.list = reinterpret_cast<ListEntry*>(p + o); o += al256((size_t)capacity * sizeof(ListEntry));
    w.fill = reinterpret_cast<ListEntry*>(p + o); o += al256((size_t)capacity * sizeof(ListEntry));
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

// Tile range of a box; false when its rect is empty.
__device__ __forceinline__ bool box_tiles(const TriBox& r, int& tx0, int& tx1, int& ty0, int& ty1) {
    if (r.y1 <= r.y0 || r.x1 <= r.x0) return false;
    tx0 = r.x0 / DS_TILE; tx1 = (r.x1 - 1) / DS_TILE;
    ty0 = r.y0 / DS_TILE; ty1 = (r.y1 - 1) / DS_TILE;
    return true;
}

// False only when no pixel centre of the tile can be covered by the
// triangle (the conservative test of block_surely_outside over the tile's
// 16x16 pixel centres).
__device__ __forceinline__ bool tile_may_cover(const TriVerts& v, const ds_view_desc& vd, int tx, int ty) {
    const int x = tx * DS_TILE, y = ty * DS_TILE;
    return !block_surely_outside(v.p0, v.p1, v.p2, pix_ndc(x, vd.W), pix_ndc(x + DS_TILE - 1, vd.W), pix_ndc(y, vd.H),
                                 pix_ndc(y + DS_TILE - 1, vd.H));
}

// The items of a warp, 32 at a time: lane j owns n_j consecutive items and
// f(valid, owner, k) is called by every lane for one item each pass (k-th
// item of lane `owner`; valid is false for the lanes past the last item).
// Every lane must call this (f may shuffle).
template <class F>
__device__ __forceinline__ void warp_items(int n, F&& f) {
    const int lane = threadIdx.x & 31;
    int excl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, excl, o);
        if (lane >= o) excl += v;
    }
    const int total = __shfl_sync(0xffffffffu, excl, 31);
    excl -= n;  // first item of this lane
    for (int base = 0; base < total; base += 32) {
        const int slot = base + lane;
        int owner = 0;  // the last lane whose first item is at or before slot
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int e = __shfl_sync(0xffffffffu, excl, owner + step);
            if (e <= slot) owner += step;
        }
        const int k = slot - __shfl_sync(0xffffffffu, excl, owner);
        f(slot < total, owner, k);
    }
}

// Pass 1: boxes, vertices, depth bounds, edge records and per-tile counts.
// The (triangle, tile) pairs of a warp's 32 triangles are tested 32 at a
// time (warp_items), so lanes do not wait on the lane with the largest rect.
__global__ void __launch_bounds__(kThreads) bin_setup_kernel(int B, const ds_view_desc* __restrict__ views, int V,
                                                             const float* __restrict__ pos, int T,
                                                             const int* __restrict__ tri, TriBox* __restrict__ boxes,
                                                             TriVerts* __restrict__ verts, TriNdc* __restrict__ ndc,
                                                             TriEdges* __restrict__ edges, int* __restrict__ counts) {
    __shared__ unsigned long long s_mask[kThreads];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < (int64_t)B * T;
    const int b = live ? (int)(i / T) : 0, t = live ? (int)(i % T) : 0;
    const ds_view_desc vd = views[b];
    TriVerts v;
    TriBox r;
    r.y0 = r.y1 = r.x0 = r.x1 = 0;
    r.zlo = r.zhi = 0.f;
    int tx0 = 0, tx1 = -1, ty0 = 0, ty1 = -1;
    if (live) {
        const float* P = pos + (size_t)b * V * 4;
        v.p0 = load_vertex(P, __ldg(tri + t * 3 + 0));
        v.p1 = load_vertex(P, __ldg(tri + t * 3 + 1));
        v.p2 = load_vertex(P, __ldg(tri + t * 3 + 2));
        int h0, hl, w0, wl;
        triangle_rect(vd.H, vd.W, v.p0, v.p1, v.p2, h0, hl, w0, wl);
        r.y0 = (short)h0; r.y1 = (short)(h0 + hl); r.x0 = (short)w0; r.x1 = (short)(w0 + wl);
        // depth bounds (only used when the rect is non-empty, i.e. every w > 0)
        const float d0 = v.p0.z / v.p0.w, d1 = v.p1.z / v.p1.w, d2 = v.p2.z / v.p2.w;
        const float mz = fmaxf(fmaxf(fabsf(v.p0.z), fabsf(v.p1.z)), fabsf(v.p2.z));
        const float mw = fminf(fminf(v.p0.w, v.p1.w), v.p2.w);
        const float margin = 1e-5f + 4e-6f * (mz / mw + fmaxf(fmaxf(fabsf(d0), fabsf(d1)), fabsf(d2)));
        r.zlo = fminf(fminf(d0, d1), d2) - margin;
        r.zhi = fmaxf(fmaxf(d0, d1), d2) + margin;
        if (!(r.zlo == r.zlo && r.zhi == r.zhi)) { r.zlo = -INFINITY; r.zhi = INFINITY; }  // NaN: no bounds
        boxes[i] = r;
        verts[i] = v;
        if (!box_tiles(r, tx0, tx1, ty0, ty1)) { tx1 = tx0 - 1; ty1 = ty0 - 1; }
    } else {
        v.p0 = v.p1 = v.p2 = make_float4(0.f, 0.f, 0.f, 1.f);
    }
    // tiles the triangle may cover; for rects of at most 64 tiles their bit
    // mask (row-major over the rect) rides in the NDC record's spare lanes
    const int ntx = tx1 - tx0 + 1, nty = ty1 - ty0 + 1;
    const int ntiles = ntx > 0 && nty > 0 ? ntx * nty : 0;
    s_mask[threadIdx.x] = 0ull;
    __syncwarp();
    const int wbase = threadIdx.x & ~31;
    warp_items(ntiles, [&](bool valid, int owner, int k) {
        float4 q[3];
        const float4 mine[3] = {v.p0, v.p1, v.p2};
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            q[j].x = __shfl_sync(0xffffffffu, mine[j].x, owner);
            q[j].y = __shfl_sync(0xffffffffu, mine[j].y, owner);
            q[j].z = __shfl_sync(0xffffffffu, mine[j].z, owner);
            q[j].w = __shfl_sync(0xffffffffu, mine[j].w, owner);
        }
        const int otx0 = __shfl_sync(0xffffffffu, tx0, owner), oty0 = __shfl_sync(0xffffffffu, ty0, owner);
        const int ontx = __shfl_sync(0xffffffffu, ntx, owner), ont = __shfl_sync(0xffffffffu, ntiles, owner);
        const int ob = __shfl_sync(0xffffffffu, b, owner);
        if (!valid) return;
        const ds_view_desc ovd = views[ob];
        const int ty = oty0 + k / ontx, tx = otx0 + k % ontx;
        TriVerts ov;
        ov.p0 = q[0]; ov.p1 = q[1]; ov.p2 = q[2];
        if (tile_may_cover(ov, ovd, tx, ty)) {
            atomicAdd(counts + ovd.tile_base + ty * ovd.tiles_x + tx, 1);
            if (ont <= 64) atomicOr(&s_mask[wbase + owner], 1ull << k);
        }
    });
    __syncwarp();
    if (!live) return;
    const uint64_t m = ntiles <= 64 ? s_mask[threadIdx.x] : 0ull;
    TriEdges te;
#pragma unroll
    for (int k = 0; k < 3; ++k) te.e[k] = make_float4(0.f, 0.f, 1.f, 0.f);
    if (ntiles > 0)
        te = tri_edges_over_rect(v.p0, v.p1, v.p2, pix_ndc(r.x0, vd.W), pix_ndc(r.x1 - 1, vd.W), pix_ndc(r.y0, vd.H),
                                 pix_ndc(r.y1 - 1, vd.H));
    TriNdc q;
    q.a = make_float4(v.p0.x / v.p0.w, v.p0.y / v.p0.w, v.p1.x / v.p1.w, v.p1.y / v.p1.w);
    q.b = make_float4(v.p2.x / v.p2.w, v.p2.y / v.p2.w, __uint_as_float((uint32_t)m),
                      __uint_as_float((uint32_t)(m >> 32)));
    ndc[i] = q;
    edges[i] = te;
}

// Pass 2: scatter record indices into the per-tile lists: the tiles of the
// count pass's masks, distributed over the warp (warp_items), and for rects
// of more than 64 tiles the test itself, per triangle.
__global__ void __launch_bounds__(kThreads) bin_fill_kernel(int B, const ds_view_desc* __restrict__ views, int T,
                                                            const TriBox* __restrict__ boxes,
                                                            const TriVerts* __restrict__ verts,
                                                            const TriNdc* __restrict__ ndc,
                                                            const int64_t* __restrict__ offsets,
                                                            int* __restrict__ cursor, ListEntry* __restrict__ list,
                                                            int64_t capacity, int* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < (int64_t)B * T;
    const int b = live ? (int)(i / T) : 0;
    const ds_view_desc vd = views[b];
    int tx0 = 0, tx1 = -1, ty0 = 0, ty1 = -1;
    uint64_t m = 0;
    ListEntry le;
    le.y0 = le.y1 = le.x0 = le.x1 = 0;
    le.zlo = 0.f;
    le.ri = (int)i;
    if (live) {
        const TriBox rc = boxes[i];
        le.y0 = rc.y0; le.y1 = rc.y1; le.x0 = rc.x0; le.x1 = rc.x1;
        le.zlo = rc.zlo;
        if (box_tiles(rc, tx0, tx1, ty0, ty1)) {
            const float4 nb = ndc[i].b;
            m = (uint64_t)__float_as_uint(nb.z) | ((uint64_t)__float_as_uint(nb.w) << 32);
        } else {
            tx1 = tx0 - 1;
            ty1 = ty0 - 1;
        }
    }
    const int ntx = tx1 - tx0 + 1, nty = ty1 - ty0 + 1;
    const int ntiles = ntx > 0 && nty > 0 ? ntx * nty : 0;
    const bool small = ntiles <= 64;
    bool over = false;
    const uint32_t mlo = (uint32_t)m, mhi = (uint32_t)(m >> 32);
    const int4 lw = *reinterpret_cast<const int4*>(&le);
    warp_items(small ? __popcll(m) : 0, [&](bool valid, int owner, int k) {
        const uint32_t olo = __shfl_sync(0xffffffffu, mlo, owner), ohi = __shfl_sync(0xffffffffu, mhi, owner);
        const int4 ole = make_int4(__shfl_sync(0xffffffffu, lw.x, owner), __shfl_sync(0xffffffffu, lw.y, owner),
                                   __shfl_sync(0xffffffffu, lw.z, owner), __shfl_sync(0xffffffffu, lw.w, owner));
        const int otx0 = __shfl_sync(0xffffffffu, tx0, owner), oty0 = __shfl_sync(0xffffffffu, ty0, owner);
        const int ontx = __shfl_sync(0xffffffffu, ntx, owner), ob = __shfl_sync(0xffffffffu, b, owner);
        if (!valid) return;
        // the k-th tile of the owner's mask
        const int nlo = __popc(olo);
        const int bit = k < nlo ? (int)__fns(olo, 0, k + 1) : 32 + (int)__fns(ohi, 0, k - nlo + 1);
        const ds_view_desc ovd = views[ob];
        const int tile = ovd.tile_base + (oty0 + bit / ontx) * ovd.tiles_x + otx0 + bit % ontx;
        const int64_t at = offsets[tile] + atomicAdd(cursor + tile, 1);
        if (at < capacity) *reinterpret_cast<int4*>(list + at) = ole;
        else over = true;
    });
    if (live && !small) {  // large rects: the test itself
        for (int ty = ty0; ty <= ty1; ++ty)
            for (int tx = tx0; tx <= tx1; ++tx) {
                if (!tile_may_cover(verts[i], vd, tx, ty)) continue;
                const int tile = vd.tile_base + ty * vd.tiles_x + tx;
                const int64_t at = offsets[tile] + atomicAdd(cursor + tile, 1);
                if (at < capacity) list[at] = le; else over = true;
            }
    }
    if (over) atomicOr(status, DS_STATUS_LIST_OVERFLOW);
}

// Bitonic network over the R * 32 (key, position) pairs of a warp, element
// e = s * 32 + lane in register slot s, ascending.  Partners 32 or more apart
// sit in the same lane (a compare-exchange between two slots), nearer ones in
// the same slot of another lane (a shuffle).
template <int R>
__device__ __forceinline__ void warp_bitonic(float (&key)[R], int (&pos)[R], int lane) {
#pragma unroll
    for (int k = 2; k <= R * 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
#pragma unroll
                for (int s = 0; s < R; ++s) {
                    const int t = s ^ (j >> 5);
                    if (t > s) {
                        const bool up = ((s * 32 + lane) & k) == 0;  // the lower element keeps the smaller key
                        if ((key[s] > key[t]) == up && key[s] != key[t]) {
                            const float kk = key[s]; key[s] = key[t]; key[t] = kk;
                            const int pp = pos[s]; pos[s] = pos[t]; pos[t] = pp;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int s = 0; s < R; ++s) {
                    const float ok = __shfl_xor_sync(0xffffffffu, key[s], j);
                    const int op = __shfl_xor_sync(0xffffffffu, pos[s], j);
                    const bool up = ((s * 32 + lane) & k) == 0, lower = (lane & j) == 0;
                    const bool take = (lower == up) ? (ok < key[s]) : (ok > key[s]);
                    if (take) { key[s] = ok; pos[s] = op; }
                }
            }
        }
    }
}

// Sorts the n <= R * 32 entries of F by zlo into L (register network, one
// gather per entry).
template <int R>
__device__ __forceinline__ void sort_in_registers(const int4* __restrict__ F, int4* __restrict__ L, int n, int lane) {
    float key[R];
    int pos[R];
#pragma unroll
    for (int s = 0; s < R; ++s) {
        const int e = s * 32 + lane;
        key[s] = e < n ? fminf(__int_as_float(F[e].z), 3.0e38f) : INFINITY;  // real keys stay below the padding
        pos[s] = e;
    }
    warp_bitonic<R>(key, pos, lane);
#pragma unroll
    for (int s = 0; s < R; ++s) {
        const int e = s * 32 + lane;
        if (e < n) L[e] = F[pos[s]];
    }
}

// Pass 3: each tile's list ordered by zlo, from the fill pass's lists into
// the rasterizer's (warp per tile): the (key, position) pairs are sorted by a
// bitonic network in registers (up to 128 entries) or in shared memory (up to
// kSortMax), and each entry is then gathered once.  Longer lists are copied
// as they are and marked unsorted; lists cut by the capacity are not used.
__global__ void __launch_bounds__(kSortWarps * 32) sort_lists_kernel(int num_tiles,
                                                                     const int64_t* __restrict__ offsets,
                                                                     const ListEntry* __restrict__ fill,
                                                                     ListEntry* __restrict__ list, int64_t capacity,
                                                                     int* __restrict__ sorted) {
    __shared__ float s_key[kSortWarps][kSortMax];
    __shared__ short s_pos[kSortWarps][kSortMax];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kSortWarps + warp;
    if (tile >= num_tiles) return;
    const int64_t begin = offsets[tile], end = offsets[tile + 1];
    const int n = (int)(end - begin);
    if (end > capacity) {  // cut: the tile runs the exhaustive path
        if (lane == 0) sorted[tile] = 0;
        return;
    }
    const int4* F = reinterpret_cast<const int4*>(fill + begin);
    int4* L = reinterpret_cast<int4*>(list + begin);
    if (n > kSortMax) {
        for (int i = lane; i < n; i += 32) L[i] = F[i];
        if (lane == 0) sorted[tile] = 0;
        return;
    }
    if (n <= 32) {  // one entry per lane: bitonic network on (key, lane) in registers
        int4 ent = make_int4(0, 0, 0, 0);
        float key = INFINITY;
        int src = lane;
        if (lane < n) {
            ent = F[lane];
            key = fminf(__int_as_float(ent.z), 3.0e38f);  // real keys stay below the +inf padding
        }
        if (n > 1) {
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const float ok = __shfl_xor_sync(0xffffffffu, key, j);
                    const int os = __shfl_xor_sync(0xffffffffu, src, j);
                    // the lower lane of the pair keeps the smaller key in ascending runs
                    const bool up = (lane & k) == 0, lower = (lane & j) == 0;
                    const bool take = (lower == up) ? (ok < key) : (ok > key);
                    if (take) { key = ok; src = os; }
                }
            }
        }
        const int4 out = make_int4(__shfl_sync(0xffffffffu, ent.x, src), __shfl_sync(0xffffffffu, ent.y, src),
                                   __shfl_sync(0xffffffffu, ent.z, src), __shfl_sync(0xffffffffu, ent.w, src));
        if (lane < n) L[lane] = out;
        if (lane == 0) sorted[tile] = 1;
        return;
    }
    if (n <= 128) {
        if (n <= 64) sort_in_registers<2>(F, L, n, lane);
        else sort_in_registers<4>(F, L, n, lane);
        if (lane == 0) sorted[tile] = 1;
        return;
    }
    int size = 256;
    while (size < n) size <<= 1;
    float* key = s_key[warp];
    short* pos = s_pos[warp];
    for (int i = lane; i < size; i += 32) {
        key[i] = i < n ? fminf(__int_as_float(F[i].z), 3.0e38f) : INFINITY;  // real keys stay below the padding
        pos[i] = (short)i;
    }
    __syncwarp();
    for (int k = 2; k <= size; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < size; i += 32) {
                const int l = i ^ j;
                if (l > i) {
                    const float a = key[i], c = key[l];
                    const bool up = (i & k) == 0;
                    if ((a > c) == up && a != c) {
                        key[i] = c; key[l] = a;
                        const short t = pos[i]; pos[i] = pos[l]; pos[l] = t;
                    }
                }
            }
            __syncwarp();
        }
    }
    for (int i = lane; i < n; i += 32) L[i] = F[pos[i]];
    if (lane == 0) sorted[tile] = 1;
}

// Geometry of one work item (tile, 32-pixel block) for the calling lane.
// Blocks are 2^bwl pixels wide and 32 / 2^bwl high (bwl = 3: 8x4, 4: 16x2,
// 2: 4x8); a tile holds 8 of them, row-major, and lane l takes pixel
// (l mod width, l div width) of its block.
struct BlockGeom {
    int b, px, py, H, W;
    int64_t pix;          // packed pixel index
    bool valid;
    int wx0, wy0;         // block origin
    int bw, bh;           // block width and height
    int64_t begin, end;   // list range, or [b*T, b*T+T) records when exhaustive
    bool exhaustive, ordered;
};

__device__ __forceinline__ BlockGeom block_geometry(int item, int B, const ds_view_desc* __restrict__ views, int T,
                                                    const int64_t* __restrict__ offsets,
                                                    const int* __restrict__ sorted, int64_t capacity, int bwl) {
    BlockGeom g;
    const int tile = item / kBlocksPerTile, blk = item % kBlocksPerTile;
    g.b = find_view(views, B, tile);
    const ds_view_desc vd = views[g.b];
    const int tl = tile - vd.tile_base;
    const int tx = tl % vd.tiles_x, ty = tl / vd.tiles_x;
    const int lane = threadIdx.x & 31;
    g.bw = 1 << bwl;
    g.bh = 32 >> bwl;
    const int rl = 4 - bwl;  // log2 of the blocks per tile row (DS_TILE = 16)
    g.wx0 = tx * DS_TILE + ((blk & ((1 << rl) - 1)) << bwl);
    g.wy0 = ty * DS_TILE + (blk >> rl) * g.bh;
    g.px = g.wx0 + (lane & (g.bw - 1));
    g.py = g.wy0 + (lane >> bwl);
    g.H = vd.H; g.W = vd.W;
    g.valid = g.px < vd.W && g.py < vd.H;
    g.pix = vd.pix_offset + (int64_t)g.py * vd.W + g.px;
    g.begin = offsets[tile];
    g.end = offsets[tile + 1];
    g.exhaustive = g.end > capacity;
    g.ordered = !g.exhaustive && sorted[tile] != 0;
    if (g.exhaustive) { g.begin = (int64_t)g.b * T; g.end = g.begin + T; }
    return g;
}

__device__ __forceinline__ bool box_overlaps(const TriBox& r, const BlockGeom& g) {
    return r.y0 < g.wy0 + g.bh && r.y1 > g.wy0 && r.x0 < g.wx0 + g.bw && r.x1 > g.wx0;
}

__device__ __forceinline__ int warp_next(int* work) {
    int item = 0;
    if ((threadIdx.x & 31) == 0) item = atomicAdd(work, 1);
    return __shfl_sync(0xffffffffu, item, 0);
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Candidates of one group of up to 32 list entries staged in warp-private
// shared memory, in list order.
struct WarpStage {
    TriVerts v[32];
    TriBox box[32];
    int t[32];
    unsigned lanes[32];  // lanes of the block whose (valid) pixel lies inside the candidate's rect
};

// Lanes of the block whose pixel lies inside the pixel rect r (lane l =
// pixel (l mod bw, l div bw) of the block).
__device__ __forceinline__ unsigned rect_lanes(const TriBox& r, const BlockGeom& g) {
    const int cx0 = max((int)r.x0 - g.wx0, 0), cx1 = min((int)r.x1 - g.wx0, g.bw);
    const int cy0 = max((int)r.y0 - g.wy0, 0), cy1 = min((int)r.y1 - g.wy0, g.bh);
    if (cx0 >= cx1 || cy0 >= cy1) return 0u;
    const unsigned row = ((1u << cx1) - 1u) & ~((1u << cx0) - 1u);  // cx1 <= bw <= 16
    // one bit per block row, at the row's first lane: 0xffffffff / (2^bw - 1)
    const unsigned rows = g.bw == 8 ? 0x01010101u : (g.bw == 16 ? 0x00010001u : 0x11111111u);
    const int hi = cy1 * g.bw;  // <= 32
    const unsigned keep = (hi >= 32 ? ~0u : (1u << hi) - 1u) & ~((1u << (cy0 * g.bw)) - 1u);
    return row * (rows & keep);  // the row bits repeated on the kept rows (no carries)
}

// Loads entries [g0, g0+32) of the work item's range, keeps those whose box
// meets the block, whose depth bound passes `zcut` (zlo <= zcut) and whose
// edge record does not prove the block uncovered, stages them, and returns
// how many were staged.  *head_zlo receives the zlo of the group's first
// entry (the smallest, when the list is ordered).
__device__ __forceinline__ int stage_group(const BlockGeom& g, int64_t g0, const TriBox* __restrict__ boxes,
                                           const TriVerts* __restrict__ verts, const TriEdges* __restrict__ edges,
                                           const ListEntry* __restrict__ list, int T, float zcut, WarpStage& st,
                                           float* head_zlo) {
    const int lane = threadIdx.x & 31;
    const int64_t e = g0 + lane;
    const bool in = e < g.end;
    int ri = 0;
    TriBox bx;
    bx.y0 = bx.y1 = bx.x0 = bx.x1 = 0;
    bx.zlo = INFINITY; bx.zhi = INFINITY;
    if (in) {
        if (g.exhaustive) {
            ri = (int)e;
            bx = boxes[ri];
        } else {
            const int4 le = __ldg(reinterpret_cast<const int4*>(list + e));
            ri = le.w;
            bx.y0 = (short)(le.x & 0xffff); bx.y1 = (short)(le.x >> 16);
            bx.x0 = (short)(le.y & 0xffff); bx.x1 = (short)(le.y >> 16);
            bx.zlo = __int_as_float(le.z);
        }
    }
    *head_zlo = __shfl_sync(0xffffffffu, bx.zlo, 0);
    bool c = in && box_overlaps(bx, g) && bx.zlo <= zcut;
    if (c) {
        // pixel-centre extents of the block (clamped to the view)
        const float xa = pix_ndc(g.wx0, g.W), xb = pix_ndc(min(g.wx0 + g.bw - 1, g.W - 1), g.W);
        const float ya = pix_ndc(g.wy0, g.H), yb = pix_ndc(min(g.wy0 + g.bh - 1, g.H - 1), g.H);
        c = !edges_reject_block(edges[ri], xa, xb, ya, yb);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, c);
    const unsigned valid = __ballot_sync(0xffffffffu, g.valid);
    if (c) {
        const int k = __popc(mask & ((1u << lane) - 1u));
        st.v[k] = verts[ri];
        st.box[k] = bx;
        st.t[k] = ri - g.b * T;
        st.lanes[k] = rect_lanes(bx, g) & valid;
    }
    __syncwarp();
    return __popc(mask);
}

// Per-warp buffer of the fragment records of one 8x4 block (REC kernels).
constexpr int kRecCap = 192;

struct WarpRecs {
    int t[kRecCap];
    float b0[kRecCap], b1[kRecCap], z[kRecCap];
    unsigned char lane[kRecCap];
};

__device__ __forceinline__ void push_fallback(const RecordStore& rs, int item) {
    if ((threadIdx.x & 31) == 0) rs.fallback[atomicAdd(rs.counters + 1, 1)] = item;
}

// Writes the records of the finished block that lie in front of (or level
// with) each lane's final surface into the warp's chunk.  The chunk must
// hold all nrec of them (the kept count is not known before the pass), so a
// new one is reserved when it does not; `cid` = current chunk (-1: none,
// -2: the store is exhausted), `cfill` = records in it.  Record j's lane
// passes its pixel, surface depth and visible triangle by shuffle.
__device__ __forceinline__ void flush_records(const RecordStore& rs, const WarpRecs& R, int nrec, int item, uint32_t pix,
                                              unsigned long long best, float bz, int& cid, int& cfill) {
    const int lane = threadIdx.x & 31;
    if (nrec > kRecCap) {
        push_fallback(rs, item);
        return;
    }
    // the surface depth (+inf when empty) and the visible triangle as the backward pass reads it back from
    // rast (id + 1 stored as a float; -1 when empty)
    const float fz = best == ~0ull ? INFINITY : bz;
    const int ft = best == ~0ull ? -1 : (int)(float)((uint32_t)(best & 0xffffffffu) + 1u) - 1;
    if (cid == -1 || (cid >= 0 && cfill + nrec > kRecChunk)) {
        if (cid >= 0 && lane == 0) rs.chunk_fill[cid] = cfill;
        int base = 0;
        if (lane == 0) base = atomicAdd(rs.counters, kRecChunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        cid = (int64_t)base + kRecChunk <= rs.capacity ? base / kRecChunk : -2;
        cfill = 0;
    }
    if (cid == -2) {
        push_fallback(rs, item);
        return;
    }
    int4* out = rs.rec + (int64_t)cid * kRecChunk + cfill;
    const unsigned below = (1u << lane) - 1u;
    int at = 0;
    for (int j0 = 0; j0 < nrec; j0 += 32) {
        const int j = j0 + lane;
        const bool in = j < nrec;
        const int src = in ? (int)R.lane[j] : 0;
        const float sz = __shfl_sync(0xffffffffu, fz, src);
        const int stri = __shfl_sync(0xffffffffu, ft, src);
        const uint32_t p = __shfl_sync(0xffffffffu, pix, src);
        const bool keep = in && R.z[j] <= sz;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int t = R.t[j];
            const uint32_t tv = (uint32_t)t | (t == stri ? 0x80000000u : 0u);
            out[at + __popc(m & below)] = make_int4((int)p, (int)tv, __float_as_int(R.b0[j]), __float_as_int(R.b1[j]));
        }
        at += __popc(m);
    }
    cfill += at;
}

// Forward: depth test with stochastic opacity.  Each warp walks the
// triangles of its block front to back (the tile list is sorted by zlo) and
// stops once the next triangle's depth bound lies behind the winner of every
// lane: no later triangle can improve a key (the bound's margin keeps
// bits(z+2) strictly larger).  Within a triangle, the divisions run only when
// some lane survives the cheap edge-sign test.
//
// REC: also keeps every fragment whose depth key does not lie behind the
// lane's current winner.  Winner keys only decrease, and every fragment at
// or in front of a lane's final surface has zlo <= that depth <= the warp's
// bound at every point of the walk, so the walk meets and keeps all of them;
// at the end of the block those behind the final surface are dropped.
#ifndef DSB_RASTER_MIN_CTAS
#define DSB_RASTER_MIN_CTAS 4  // resident 8-warp CTAs per SM the register budget is sized for (64 registers)
#endif

template <bool REC>
__global__ void __launch_bounds__(kWarpsPerCta * 32, DSB_RASTER_MIN_CTAS) raster_kernel(
    int B, const ds_view_desc* __restrict__ views, int num_tiles, int T, const TriBox* __restrict__ boxes,
    const TriVerts* __restrict__ verts, const TriEdges* __restrict__ edges, const int64_t* __restrict__ offsets,
    const int* __restrict__ sorted, const ListEntry* __restrict__ list, int64_t capacity, int level, int S,
    const float* __restrict__ alpha_src, int thr_mode, float thr_const, const uint64_t* __restrict__ rng, int* work, float* __restrict__ rast,
    RecordStore rs, int bwl) {
    __shared__ WarpStage s_stage[kWarpsPerCta];
    __shared__ WarpRecs s_rec[REC ? kWarpsPerCta : 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpStage& st = s_stage[warp];
    WarpRecs& R = s_rec[REC ? warp : 0];
    uint64_t seed = 0;
    uint32_t iter = 0;
    if (thr_mode == 1) { seed = rng[0]; iter = (uint32_t)rng[1]; }
    int cid = -1, cfill = 0;  // REC: the warp's current record chunk
    const int items = num_tiles * kBlocksPerTile;
    for (int item = warp_next(work); item < items; item = warp_next(work)) {
        const BlockGeom g = block_geometry(item, B, views, T, offsets, sorted, capacity, bwl);
        if (g.begin >= g.end) {  // no candidate: background (a quarter to a third of the blocks)
            if (g.valid) reinterpret_cast<float4*>(rast)[g.pix] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const float ndc_x = pix_ndc(g.px, g.W), ndc_y = pix_ndc(g.py, g.H);
        const PhiloxPixel php = philox_pixel(seed, iter, (uint32_t)g.b, (uint32_t)(g.py * g.W + g.px));
        unsigned long long best = ~0ull;
        float bb0 = 0.f, bb1 = 0.f, bz = 0.f;
        float bz_cut = INFINITY;  // the winner's depth, +inf while the lane has none
        int nrec = 0;
        // max over the warp of the lanes' winning depth (+inf while a valid lane has none)
        float warp_far = warp_max(g.valid ? INFINITY : -INFINITY);
        bool all_won = false;  // every valid lane has a winner (before that, warp_far stays +inf)
        for (int64_t g0 = g.begin; g0 < g.end; g0 += 32) {
            float head;
            const int nc = stage_group(g, g0, boxes, verts, edges, list, T, warp_far, st, &head);
            if (g.ordered && head > warp_far) break;  // this group and all later ones lie behind
            for (int k = 0; k < nc; ++k) {
                if (st.box[k].zlo > warp_far) {
                    if (g.ordered) break;
                    continue;
                }
                const float4 p0 = st.v[k].p0, p1 = st.v[k].p1, p2 = st.v[k].p2;
                const TriBox r = st.box[k];
                // lanes inside the rect whose winner does not lie in front of the triangle: zlo's
                // margin exceeds the rounding of z + 2, so with zlo > bz every fragment's depth key
                // lies strictly behind the winner's (neither a winner nor a record)
                const bool near = ((st.lanes[k] >> lane) & 1u) && !(r.zlo > bz_cut);
                if (!__any_sync(0xffffffffu, near)) continue;  // warp-uniform
                float A0, A1, A2, A;
                edge_terms(ndc_y, ndc_x, p0, p1, p2, A0, A1, A2, A);
                const bool cand = near && !surely_outside(A0, A1, A2, A);
                if (!__any_sync(0xffffffffu, cand)) continue;  // warp-uniform
                bool improved = false, rec = false;
                float b0 = 0.f, b1 = 0.f, depth = 0.f;
                const uint32_t t = (uint32_t)st.t[k];
                if (cand) {
                    float z, w;
                    if (finish_coverage(A0, A1, A, p0, p1, p2, b0, b1, z, w)) {
                        depth = __fdiv_rn(z, w);
                        if (depth >= -1.f && depth <= 1.f) {
                            const unsigned long long key = depth_key(depth, t);
                            // keep it unless its depth key lies behind the current winner's: the
                            // winner's key only decreases, so nothing at or in front of the final
                            // surface is dropped (the winner's depth itself can grow within one
                            // bits(z+2) step when a lower triangle index takes a tie)
                            if (REC) rec = (key >> 32) <= (best >> 32);
                            if (depth > -1.f) {
                                if (key < best) {
                                    const float alpha = interp_level(b0, b1, level, alpha_src + (size_t)t * S);
                                    // Philox thresholds lie in [0, 1): an opacity of 1 passes without a draw
                                    const bool pass = thr_mode == 1
                                                          ? alpha >= 1.f || !(alpha < philox_uniform_tri(php, seed, t))
                                                          : !(alpha < thr_const);
                                    if (pass) {
                                        best = key; bb0 = b0; bb1 = b1; bz = depth; bz_cut = depth;
                                        improved = true;
                                    }
                                }
                            }
                        }
                    }
                }
                if (REC) {
                    const unsigned m = __ballot_sync(0xffffffffu, rec);
                    if (m) {
                        const int at = nrec + __popc(m & ((1u << lane) - 1u));
                        if (rec && at < kRecCap) {
                            R.t[at] = (int)t; R.b0[at] = b0; R.b1[at] = b1; R.z[at] = depth;
                            R.lane[at] = (unsigned char)lane;
                        }
                        nrec += __popc(m);
                    }
                }
                if (__any_sync(0xffffffffu, improved)) {
                    if (!all_won) all_won = __all_sync(0xffffffffu, !g.valid || best != ~0ull);
                    if (all_won) warp_far = warp_max(!g.valid ? -INFINITY : bz);
                }
            }
            __syncwarp();  // the stage is rewritten by the next group
        }
        if (g.valid) {
            float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
            if (best != ~0ull) o = make_float4(bb0, bb1, bz, (float)((uint32_t)(best & 0xffffffffu) + 1u));
            reinterpret_cast<float4*>(rast)[g.pix] = o;
        }
        if (REC && nrec > 0) {
            __syncwarp();
            flush_records(rs, R, nrec, item, (uint32_t)g.pix, best, bz, cid, cfill);
            __syncwarp();  // the buffer is rewritten by the next block
        }
    }
    if (REC && cid >= 0 && lane == 0) rs.chunk_fill[cid] = cfill;
}

// dL/dalpha of one fragment scattered through the lattice adjoint
// (rasterize.cu:951-970 followed by multires.cu:130-222).
__device__ __forceinline__ void aux_scatter(float b0, float b1, int level, int S, const float* __restrict__ alpha_src,
                                            int t, float loss, bool visible, float scale,
                                            float* __restrict__ grad_alpha_src) {
    const float alpha = interp_level(b0, b1, level, alpha_src + (size_t)t * S);
    const float ga = aux_alpha_grad(loss, alpha, visible) * scale;
    uint32_t idx[3];
    float w[3];
    lattice_cell(b0, b1, level, idx, w);
    float* dst = grad_alpha_src + (size_t)t * S;
#pragma unroll
    for (int q = 0; q < 3; ++q) atomicAdd(dst + idx[q], ga * w[q]);
}

// Opacity auxiliary gradient from the fragment records: one thread per
// record, blocks stride over the chunks.  A chunk holds whole 8x4 blocks in
// walk order, so neighbouring records often share a triangle and a lattice
// cell: runs of equal (triangle, cell) in a warp are summed with a segmented
// reduction before the global atomics.
__global__ void __launch_bounds__(kRecChunk) aux_records_kernel(RecordStore rs, int level, int S,
                                                               const float* __restrict__ alpha_src,
                                                               const float* __restrict__ l1, float scale,
                                                               float* __restrict__ grad_alpha_src) {
    const int lane = threadIdx.x & 31;
    const int64_t reserved = rs.counters[0];
    const int64_t nchunks = (reserved < rs.capacity ? reserved : rs.capacity) / kRecChunk;
    for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const bool valid = (int)threadIdx.x < rs.chunk_fill[c];
        int t = -1 - lane;
        uint32_t idx[3] = {0u, 0u, 0u};
        float g[3] = {0.f, 0.f, 0.f};
        if (valid) {
            const int4 r = rs.rec[c * kRecChunk + threadIdx.x];
            const uint32_t tv = (uint32_t)r.y;
            t = (int)(tv & 0x7fffffffu);
            const float b0 = __int_as_float(r.z), b1 = __int_as_float(r.w);
            float w[3];
            lattice_cell(b0, b1, (uint32_t)level, idx, w);
            // interp_scalar at one level (the same sum)
            const float* src = alpha_src + (size_t)t * S;
            float alpha = 0.f;
            alpha = madd(alpha, w[0], __ldg(src + idx[0]));
            alpha = madd(alpha, w[1], __ldg(src + idx[1]));
            alpha = madd(alpha, w[2], __ldg(src + idx[2]));
            const float ga = aux_alpha_grad(l1[(uint32_t)r.x], alpha, (tv >> 31) != 0) * scale;
#pragma unroll
            for (int q = 0; q < 3; ++q) g[q] = ga * w[q];
        }
        const int pt = __shfl_up_sync(0xffffffffu, t, 1);
        const uint32_t p0 = __shfl_up_sync(0xffffffffu, idx[0], 1), p1 = __shfl_up_sync(0xffffffffu, idx[1], 1),
                       p2 = __shfl_up_sync(0xffffffffu, idx[2], 1);
        const bool same = lane > 0 && pt == t && p0 == idx[0] && p1 == idx[1] && p2 == idx[2];
        const unsigned heads = __ballot_sync(0xffffffffu, !same);
        const int seg = __popc(heads & ((2u << lane) - 1u));
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int oseg = __shfl_down_sync(0xffffffffu, seg, o);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const float v = __shfl_down_sync(0xffffffffu, g[q], o);
                if (lane + o < 32 && oseg == seg) g[q] += v;
            }
        }
        if (valid && !same) {
            float* dst = grad_alpha_src + (size_t)t * S;
#pragma unroll
            for (int q = 0; q < 3; ++q) atomicAdd(dst + idx[q], g[q]);
        }
    }
}

// Opacity auxiliary gradient by re-enumeration: each block's fragments are
// recomputed and dL/dalpha is scattered through the lattice adjoint.
// Fragments behind the visible surface contribute nothing
// (rasterize.cu:950), so triangles whose depth bound lies behind every
// lane's surface are never staged.  All lanes of a warp work on the same
// triangle at a time, so contributions are summed per warp in shared memory
// and flushed with one global atomic per touched sample.  With item_list,
// only the blocks listed there (*item_count of them) are processed.
__global__ void __launch_bounds__(kWarpsPerCta * 32) aux_kernel(
    int B, const ds_view_desc* __restrict__ views, int num_tiles, int T, const TriBox* __restrict__ boxes,
    const TriVerts* __restrict__ verts, const TriEdges* __restrict__ edges, const int64_t* __restrict__ offsets,
    const int* __restrict__ sorted, const ListEntry* __restrict__ list, int64_t capacity, int level, int S,
    const float* __restrict__ alpha_src, int C,
    const float* __restrict__ color, const float* __restrict__ target, const float* __restrict__ rast, float scale,
    const int* __restrict__ item_list, const int* __restrict__ item_count, int* work,
    float* __restrict__ grad_alpha_src, int bwl) {
    __shared__ WarpStage s_stage[kWarpsPerCta];
    __shared__ float s_acc[kWarpsPerCta][kAuxSmemS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpStage& st = s_stage[warp];
    const bool use_smem = S <= kAuxSmemS;
    if (use_smem)
        for (int k = lane; k < S; k += 32) s_acc[warp][k] = 0.f;
    __syncwarp();
    const int items = item_list ? *item_count : num_tiles * kBlocksPerTile;
    for (int n = warp_next(work); n < items; n = warp_next(work)) {
        const int item = item_list ? item_list[n] : n;
        const BlockGeom g = block_geometry(item, B, views, T, offsets, sorted, capacity, bwl);
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
        // farthest surface of the block (+inf where a valid pixel is empty)
        const float warp_far = warp_max(!g.valid ? -INFINITY : (tp >= 0 ? zp : INFINITY));
        for (int64_t g0 = g.begin; g0 < g.end; g0 += 32) {
            float head;
            const int nc = stage_group(g, g0, boxes, verts, edges, list, T, warp_far, st, &head);
            if (g.ordered && head > warp_far) break;
            for (int k = 0; k < nc; ++k) {
                const TriBox r = st.box[k];
                const int t = st.t[k];
                const float4 p0 = st.v[k].p0, p1 = st.v[k].p1, p2 = st.v[k].p2;
                // lanes inside the rect whose surface does not lie in front of the triangle
                const bool near = ((st.lanes[k] >> lane) & 1u) && !(tp >= 0 && r.zlo > zp);
                if (!__any_sync(0xffffffffu, near)) continue;  // warp-uniform
                float A0, A1, A2, A;
                edge_terms(ndc_y, ndc_x, p0, p1, p2, A0, A1, A2, A);
                bool hit = near && !surely_outside(A0, A1, A2, A);
                if (!__any_sync(0xffffffffu, hit)) continue;  // warp-uniform
                float b0 = 0.f, b1 = 0.f;
                if (hit) {
                    float z, w;
                    hit = finish_coverage(A0, A1, A, p0, p1, p2, b0, b1, z, w);
                    if (hit) {
                        const float depth = __fdiv_rn(z, w);
                        hit = depth >= -1.f && depth <= 1.f && !(tp >= 0 && depth > zp);
                    }
                }
                if (!use_smem) {
                    if (hit) aux_scatter(b0, b1, level, S, alpha_src, t, loss, tp >= 0 && t == tp, scale,
                                         grad_alpha_src);
                    continue;
                }
                if (!__any_sync(0xffffffffu, hit)) continue;
                if (hit) {
                    const float alpha = interp_level(b0, b1, level, alpha_src + (size_t)t * S);
                    const float ga = aux_alpha_grad(loss, alpha, tp >= 0 && t == tp) * scale;
                    uint32_t idx[3];
                    float w[3];
                    lattice_cell(b0, b1, level, idx, w);
#pragma unroll
                    for (int q = 0; q < 3; ++q) atomicAdd(&s_acc[warp][idx[q]], ga * w[q]);
                }
                __syncwarp();
                float* dst = grad_alpha_src + (size_t)t * S;
                for (int q = lane; q < S; q += 32) {
                    const float v = s_acc[warp][q];
                    if (v != 0.f) { atomicAdd(dst + q, v); s_acc[warp][q] = 0.f; }
                }
                __syncwarp();
            }
            __syncwarp();
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
    DS_CHECK_ARG((int64_t)num_tiles * kBlocksPerTile <= 0x7fffffff, "tiles: too many tiles");
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
    // up to kScanOneMax tiles, one launch scans the counts, writes the total and clears the fill cursors
    const bool one_cta = num_tiles <= kScanOneMax;
    DS_CUDA(cudaMemsetAsync(w.counts, 0, (size_t)num_tiles * sizeof(int), st));
    if (!one_cta) DS_CUDA(cudaMemsetAsync(w.cursor, 0, (size_t)num_tiles * sizeof(int), st));
    const int64_t n = (int64_t)B * T;
    if (n > 0)
        bin_setup_kernel<<<blocks_for(n), kThreads, 0, st>>>(B, views, V, pos, T, tri, w.boxes, w.verts, w.ndc,
                                                              w.edges, w.counts);
    if (one_cta) {
        scan_one_cta_kernel<<<1, kScanOneThreads, 0, st>>>(w.counts, num_tiles, w.offsets, w.cursor);
    } else {
        int64_t* total_dev = nullptr;
        rc = device_scan<int, int64_t>(w.counts, num_tiles, w.offsets, false, w.scan, st, &total_dev);
        if (rc) return rc;
        // offsets[num_tiles] = total number of entries
        DS_CUDA(cudaMemcpyAsync(w.offsets + num_tiles, total_dev, sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    }
    if (n > 0)
        bin_fill_kernel<<<blocks_for(n), kThreads, 0, st>>>(B, views, T, w.boxes, w.verts, w.ndc, w.offsets, w.cursor,
                                                            w.fill,
                                                            list_capacity, status);
    if (num_tiles > 0)
        sort_lists_kernel<<<(unsigned)((num_tiles + kSortWarps - 1) / kSortWarps), kSortWarps * 32, 0, st>>>(
            num_tiles, w.offsets, w.fill, w.list, list_capacity, w.sorted);
    return check_launch("tiles_bin");
}

}  // extern "C"

namespace dsb {

// Persistent grid: as many 8-warp CTAs as fit on the SMs (queried once per
// kernel), capped by the number of blocks.
static unsigned block_grid(int num_tiles, const void* kernel, int& per_sm, size_t smem = 0) {
    if (per_sm == 0) {
        int n = 0;
        if (smem > 0) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kWarpsPerCta * 32, smem) != cudaSuccess || n < 1)
            n = 1;
        per_sm = n;
    }
    const int64_t warps = (int64_t)num_tiles * kBlocksPerTile;
    const int64_t ctas = (warps + kWarpsPerCta - 1) / kWarpsPerCta;
    const int64_t cap = (int64_t)sm_count() * per_sm;
    return (unsigned)(ctas < 1 ? 1 : (ctas < cap ? ctas : cap));
}

static int g_occ_raster = 0, g_occ_raster_rec = 0, g_occ_aux = 0;

int tiles_rasterize_impl(int B, const ds_view_desc* views, int num_tiles, int T, int level, int S,
                         const float* alpha_src, int thr_mode, float thr_const, const uint64_t* rng, float* rast,
                         void* workspace, int64_t list_capacity, const RecordStore* rs, cudaStream_t st, int bwl) {
    if (num_tiles == 0) return DS_OK;
    TileWs w = carve(workspace, B, T, num_tiles, list_capacity, nullptr);
    DS_CUDA(cudaMemsetAsync(w.work, 0, sizeof(int), st));
    if (rs != nullptr) {
        const void* k = reinterpret_cast<const void*>(&raster_kernel<true>);
        raster_kernel<true><<<block_grid(num_tiles, k, g_occ_raster_rec), kWarpsPerCta * 32, 0, st>>>(
            B, views, num_tiles, T, w.boxes, w.verts, w.edges, w.offsets, w.sorted, w.list, list_capacity, level, S,
            alpha_src, thr_mode, thr_const, rng, w.work, rast, *rs, bwl);
    } else {
        const void* k = reinterpret_cast<const void*>(&raster_kernel<false>);
        raster_kernel<false><<<block_grid(num_tiles, k, g_occ_raster), kWarpsPerCta * 32, 0, st>>>(
            B, views, num_tiles, T, w.boxes, w.verts, w.edges, w.offsets, w.sorted, w.list, list_capacity, level, S,
            alpha_src, thr_mode, thr_const, rng, w.work, rast, RecordStore{}, bwl);
    }
    return check_launch("tiles_rasterize");
}

static int aux_launch(int B, const ds_view_desc* views, int num_tiles, int T, int level, int S,
                      const float* alpha_src, int C, const float* color, const float* target, const float* rast,
                      float scale, float* grad_alpha_src, void* workspace, int64_t list_capacity,
                      const int* item_list, const int* item_count, cudaStream_t st, int bwl) {
    TileWs w = carve(workspace, B, T, num_tiles, list_capacity, nullptr);
    DS_CUDA(cudaMemsetAsync(w.work + 1, 0, sizeof(int), st));
    const void* k = reinterpret_cast<const void*>(&aux_kernel);
    aux_kernel<<<block_grid(num_tiles, k, g_occ_aux), kWarpsPerCta * 32, 0, st>>>(
        B, views, num_tiles, T, w.boxes, w.verts, w.edges, w.offsets, w.sorted, w.list, list_capacity, level, S,
        alpha_src, C,
        color, target, rast, scale, item_list, item_count, w.work + 1, grad_alpha_src, bwl);
    return check_launch("tiles_opacity_aux");
}

TileTables tiles_tables(void* workspace, int B, int T, int num_tiles, int64_t list_capacity) {
    const TileWs w = carve(workspace, B, T, num_tiles, list_capacity, nullptr);
    return TileTables{w.boxes, w.verts, w.ndc, w.offsets};
}

int tiles_aux_impl(int B, const ds_view_desc* views, int num_tiles, int T, int level, int S, const float* alpha_src,
                   const float* l1, const float* rast, float scale, float* grad_alpha_src, void* workspace,
                   int64_t list_capacity, const RecordStore* rs, cudaStream_t st, int bwl) {
    if (num_tiles == 0) return DS_OK;
    if (rs == nullptr)
        return aux_launch(B, views, num_tiles, T, level, S, alpha_src, 1, l1, nullptr, rast, scale, grad_alpha_src,
                          workspace, list_capacity, nullptr, nullptr, st, bwl);
    aux_records_kernel<<<sm_count() * 8, kRecChunk, 0, st>>>(*rs, level, S, alpha_src, l1, scale, grad_alpha_src);
    const int rc = check_launch("tiles_opacity_aux records");
    if (rc) return rc;
    return aux_launch(B, views, num_tiles, T, level, S, alpha_src, 1, l1, nullptr, rast, scale, grad_alpha_src,
                      workspace, list_capacity, rs->fallback, rs->counters + 1, st, bwl);
}

}  // namespace dsb

extern "C" {

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
    return tiles_rasterize_impl(B, views, num_tiles, T, level, S, alpha_src, thr_mode, thr_const, rng, rast,
                                workspace, list_capacity, nullptr, (cudaStream_t)stream, kDefaultBlockShape);
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
    return aux_launch(B, views, num_tiles, T, level, S, alpha_src, C, color, target, rast, scale, grad_alpha_src,
                      workspace, list_capacity, nullptr, nullptr, (cudaStream_t)stream, kDefaultBlockShape);
}

}  // extern "C"
