// diffsoup_b200/csrc/remesh.cu -- adaptive subdivision of the triangle soup
// (the resampling step of training, examples/utils.py:493-545), on the GPU.
//
// The reference splits on the CPU (src/remesh.cpp world-space lengths,
// src/remesh_clip.cpp screen-space lengths under one MVP) with a global
// priority queue: pop the longest edge, bisect its triangle, re-enqueue both
// halves, until the longest edge is below the threshold.  In a soup no two
// triangles share vertices, so a split only ever touches the descendants of
// one input face, and every face is split at its longest (considered) edge
// while that edge is at least the threshold: the queue's global order
// decides only the numbering of the new vertices and faces, not the geometry.
// Here each input face is one thread that walks its own split tree depth
// first, twice: a counting pass (the new faces of every family, scanned into
// offsets) and an emitting pass that writes the vertices and faces.
//
// Layout of the output, as the reference's (src/remesh.cpp:15-64): the N
// input vertices unchanged, then 3 vertices per split (the two copies of the
// split point and the copy of the opposite vertex); face slot t keeps the
// first child of every split of family t, and each split gives its second
// child a new slot after the M inputs.  New vertices and slots of a family are
// numbered in the depth-first order of its tree (the reference numbers them
// in global pop order), so the result equals the reference's up to that
// renumbering: the same set of triangles per family, bit for bit.
//
// Arithmetic follows the reference's host build (IEEE single precision, every
// product and sum rounded on its own, no FMA contraction).  A face whose
// longest edge ties with another takes the first in edge order (0,1), (1,2),
// (2,0); the reference's heap leaves such ties unordered.
#include <cstring>

#include "common.cuh"
#include "scan.cuh"

namespace dsb {

constexpr int kSplitThreads = 128;
constexpr int kSplitStack = 40;                 // pending second children along one path
constexpr int64_t kMaxFamilySplits = 1 << 20;   // per input face
constexpr int64_t kMaxTotalSplits = 1ll << 27;  // per call

struct SplitParams {
    int mode;      // 0 world (remesh.cpp), 1 clip (remesh_clip.cpp)
    float m[16];   // MVP, row-major (clip mode)
    float aspect;  // W / H (clip mode)
};

// Which edges a walk splits: those of squared length >= tau2 and, up to a
// per-face quota, those of exactly tie2 (a split budget's cut-off, below).
struct SplitPlan {
    float tau2, tie2;
};

struct SplitNode {
    float p[9];  // positions of the three corners
    int id[3];   // their vertex indices
    int slot;    // face slot
};

// ((m0 x + m1 y) + m2 z) + m3, each operation rounded (remesh_clip.cpp:19-29)
__device__ __forceinline__ float hom_row(const float* m, int r, const float* v) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4 * r + 0], v[0]), __fmul_rn(m[4 * r + 1], v[1])),
                               __fmul_rn(m[4 * r + 2], v[2])),
                     m[4 * r + 3]);
}

struct ClipPoint {
    float c[4];    // clip coordinates
    float n[3];    // NDC (0 where w <= 0)
    bool inside;   // w > 0 and inside the NDC cube
};

__device__ __forceinline__ ClipPoint clip_point(const SplitParams& P, const float* v) {
    ClipPoint q;
#pragma unroll
    for (int r = 0; r < 4; ++r) q.c[r] = hom_row(P.m, r, v);
    const bool wok = q.c[3] > 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) q.n[k] = wok ? __fdiv_rn(q.c[k], q.c[3]) : 0.f;
    q.inside = wok && q.n[0] >= -1.f && q.n[0] <= 1.f && q.n[1] >= -1.f && q.n[1] <= 1.f && q.n[2] >= -1.f &&
               q.n[2] <= 1.f;
    return q;
}

// Squared length of edge (A, B) in the metric: world (remesh.h:41-48) or
// image-height units, 0 when an end leaves the NDC cube (remesh_clip.cpp:33-78).
// a, b: the ends' clip points (clip mode; a pure function of the world point,
// so computing them once per vertex gives the reference's values).
__device__ __forceinline__ float edge_len2(const SplitParams& P, const float* A, const float* B, const ClipPoint& a,
                                           const ClipPoint& b) {
    if (P.mode == 0) {
        const float dx = __fsub_rn(B[0], A[0]), dy = __fsub_rn(B[1], A[1]), dz = __fsub_rn(B[2], A[2]);
        return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    }
    if (!a.inside || !b.inside) return 0.f;
    const float dx = __fmul_rn(__fsub_rn(a.n[0], b.n[0]), P.aspect), dy = __fsub_rn(a.n[1], b.n[1]);
    return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
}

// The split point of edge (A, B): the midpoint in world space, or the point
// whose projection is the NDC midpoint (remesh_clip.cpp:100-145).
__device__ __forceinline__ void split_point(const SplitParams& P, const float* A, const float* B, const ClipPoint& a,
                                            const ClipPoint& b, float* C) {
    if (P.mode == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) C[k] = __fmul_rn(0.5f, __fadd_rn(A[k], B[k]));
        return;
    }
    const float nx = __fmul_rn(0.5f, __fadd_rn(a.n[0], b.n[0]));
    const float ny = __fmul_rn(0.5f, __fadd_rn(a.n[1], b.n[1]));
    const float dx = __fsub_rn(b.c[0], a.c[0]), dy = __fsub_rn(b.c[1], a.c[1]), dw = __fsub_rn(b.c[3], a.c[3]);
    const float ax = __fsub_rn(a.c[0], __fmul_rn(nx, a.c[3])), ay = __fsub_rn(a.c[1], __fmul_rn(ny, a.c[3]));
    const float bx = __fsub_rn(dx, __fmul_rn(nx, dw)), by = __fsub_rn(dy, __fmul_rn(ny, dw));
    const float den = __fadd_rn(__fmul_rn(bx, bx), __fmul_rn(by, by));
    const float tB = den != 0.f ? __fdiv_rn(-__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), den) : 0.5f;
    const float tA = __fsub_rn(1.f, tB);
#pragma unroll
    for (int k = 0; k < 3; ++k) C[k] = __fadd_rn(__fmul_rn(tA, A[k]), __fmul_rn(tB, B[k]));
}

// The longest considered edge of a node: e = 0 (0,1), 1 (1,2), 2 (2,0),
// first of equals; -1 when no edge is considered.
__device__ __forceinline__ int longest_edge(const SplitParams& P, const SplitNode& cur, const ClipPoint* q,
                                            float& best) {
    int e = -1;
    best = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float l2 = edge_len2(P, cur.p + k * 3, cur.p + ((k + 1) % 3) * 3, q[k], q[(k + 1) % 3]);
        const bool considered = P.mode == 0 || l2 > 0.f;
        if (considered && (e < 0 || l2 > best)) { e = k; best = l2; }
    }
    return e;
}

__device__ __forceinline__ void node_clip_points(const SplitParams& P, const SplitNode& n, ClipPoint* q) {
    if (P.mode == 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) q[k] = clip_point(P, n.p + k * 3);
    }
}

// Splits node cur at edge e as split number k of its family: the first child
// (a, mA, cA) keeps the slot, the second (mB, b, c) takes slot fbase + k;
// mA = vbase + 3k, mB = mA + 1, cA = mA + 2.  EMIT writes the three new
// vertices and the new slot's face mapping (family t) and flag.
template <bool EMIT>
__device__ __forceinline__ void split_node(const SplitParams& P, const SplitNode& cur, const ClipPoint* q, int e,
                                           int64_t k, int64_t vbase, int64_t fbase, int t, SplitNode& first,
                                           SplitNode& second, float* __restrict__ out_verts, int* __restrict__ map,
                                           int* __restrict__ flag) {
    const int ia = e, ib = (e + 1) % 3, ic = (e + 2) % 3;  // edge (a, b), opposite c
    float C[3];
    split_point(P, cur.p + ia * 3, cur.p + ib * 3, q[ia], q[ib], C);
    const int mA = (int)(vbase + 3 * k), mB = mA + 1, cA = mA + 2;
    second.slot = (int)(fbase + k);
    second.id[0] = mB; second.id[1] = cur.id[ib]; second.id[2] = cur.id[ic];
    first.slot = cur.slot;
    first.id[0] = cur.id[ia]; first.id[1] = mA; first.id[2] = cA;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        second.p[j] = C[j];
        second.p[3 + j] = cur.p[ib * 3 + j];
        second.p[6 + j] = cur.p[ic * 3 + j];
        first.p[j] = cur.p[ia * 3 + j];
        first.p[3 + j] = C[j];
        first.p[6 + j] = cur.p[ic * 3 + j];
    }
    if (EMIT) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            out_verts[(size_t)mA * 3 + j] = C[j];
            out_verts[(size_t)mB * 3 + j] = C[j];
            out_verts[(size_t)cA * 3 + j] = cur.p[ic * 3 + j];
        }
        map[second.slot] = t;
        flag[second.slot] = 0;
    }
}

__device__ __forceinline__ SplitNode family_root(int t, const float* __restrict__ verts, const int* __restrict__ faces) {
    SplitNode n;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        n.id[k] = faces[(size_t)t * 3 + k];
#pragma unroll
        for (int j = 0; j < 3; ++j) n.p[k * 3 + j] = verts[(size_t)n.id[k] * 3 + j];
    }
    n.slot = t;
    return n;
}

// Walks the split tree below `root` depth first (first child before second
// child), numbering its splits k0, k0 + 1, ...  Counting pass (EMIT false):
// returns the number of splits.  Emitting pass: writes the faces of its
// leaves, its new vertices (from vbase) and new slots (from fbase).  Both
// passes take the same decisions; a walk that would exceed max_splits (or
// the stack) stops splitting and raises DS_STATUS_SPLIT_LIMIT, which the host
// turns into an error after the counting pass.  `quota` counts down the
// cut-off-length splits the walk may still take (a split budget's ties).
template <bool EMIT>
__device__ int64_t walk_subtree(const SplitParams& P, SplitPlan plan, int quota, SplitNode cur, bool splittable,
                                int64_t max_splits, int64_t k0, int64_t vbase, int64_t fbase, int t,
                                float* __restrict__ out_verts, int* __restrict__ out_faces, int* __restrict__ map,
                                int* __restrict__ flag, int* __restrict__ status,
                                unsigned long long* __restrict__ total) {
    SplitNode stack[kSplitStack];
    int top = 0;
    ClipPoint q[3];  // clip points of cur's corners (clip mode)
    node_clip_points(P, cur, q);
    int64_t splits = 0;
    bool stop = !splittable;
    while (true) {
        float best = 0.f;
        const int e = stop ? -1 : longest_edge(P, cur, q, best);
        const bool tie = quota > 0 && best == plan.tie2;
        const bool split = e >= 0 && best > 0.f && (best >= plan.tau2 || tie);
        if (split && (top == kSplitStack || splits >= max_splits)) {
            atomicOr(status, DS_STATUS_SPLIT_LIMIT);  // the family stops here; the host reports it
            stop = true;
            continue;
        }
        if (split) {
            // the call's total, charged every 256 splits of a walk
            if (!EMIT && splits > 0 && (splits & 255) == 0 &&
                atomicAdd(total, 256ull) > (unsigned long long)kMaxTotalSplits) {
                atomicOr(status, DS_STATUS_SPLIT_LIMIT);
                stop = true;
                continue;
            }
            if (tie && !(best >= plan.tau2)) --quota;
            SplitNode first, second;
            split_node<EMIT>(P, cur, q, e, k0 + splits, vbase, fbase, t, first, second, out_verts, map, flag);
            ++splits;
            const int ia = e, ic = (e + 2) % 3;
            stack[top++] = second;
            cur = first;
            if (P.mode == 1) {  // corners (a, C, c)
                const ClipPoint qa = q[ia], qc = q[ic];
                q[0] = qa;
                q[1] = clip_point(P, cur.p + 3);
                q[2] = qc;
            }
            continue;
        }
        if (EMIT) {
#pragma unroll
            for (int k = 0; k < 3; ++k) out_faces[(size_t)cur.slot * 3 + k] = cur.id[k];
        }
        if (top == 0) break;
        cur = stack[--top];
        node_clip_points(P, cur, q);
    }
    return splits;
}

// A family's split tree is walked in two parts, so that one large family
// does not serialise the launch: its top kTopLevels levels breadth first (by
// one thread per family, split_top_kernel), then each of the up to
// 2^kTopLevels subtrees hanging below them depth first (one thread per
// subtree, split_task_kernel).  A family's splits are numbered in that order:
// the top splits level by level, left to right (first child before second),
// then the subtrees left to right, each in depth-first order.  The top
// kernel records the split number of every top node in a heap-indexed table
// (node v has children 2v, 2v + 1; -1: no split there), from which a subtree
// task rebuilds its root by re-walking the D splits above it.  Families with
// a tie quota (a split budget's cut-off) are walked depth first by the top
// kernel alone, since their quota is consumed in walk order.
constexpr int kTopLevels = 5;
constexpr int kTopNodes = 1 << kTopLevels;  // subtrees per family; also the size of the heap table
constexpr short kSerialFamily = -2;        // table[0] of a family walked whole by the top kernel

template <bool EMIT>
__global__ void __launch_bounds__(kSplitThreads) split_top_kernel(
    SplitParams P, const SplitPlan* __restrict__ plan_dev, SplitPlan plan_arg, int N, int M,
    const float* __restrict__ verts, const int* __restrict__ faces, const int* __restrict__ valid,
    const int* __restrict__ quota, short* __restrict__ table, int* __restrict__ top_count,
    const int64_t* __restrict__ offsets, float* __restrict__ out_verts, int* __restrict__ out_faces,
    int* __restrict__ map, int* __restrict__ flag, int* __restrict__ status, unsigned long long* __restrict__ total) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const SplitPlan plan = EMIT ? *plan_dev : plan_arg;
    const bool splittable = P.mode == 0 || valid == nullptr || valid[t] > 0;
    short* tab = table + (size_t)t * kTopNodes;
    const int64_t o = EMIT ? offsets[t] : 0, n = EMIT ? offsets[t + 1] - o : 0;
    const int64_t vbase = N + 3 * o, fbase = M + o;
    if (EMIT) {
        map[t] = t;
        flag[t] = n == 0 ? 1 : 0;
    }
    const int qt = quota ? quota[t] : 0;
    if (qt > 0) {  // a tie quota: the whole family depth first, here
        const int64_t c = walk_subtree<EMIT>(P, plan, qt, family_root(t, verts, faces), EMIT ? n > 0 : splittable,
                                             EMIT ? n : kMaxFamilySplits, 0, vbase, fbase, t, out_verts, out_faces,
                                             map, flag, status, total);
        if (!EMIT) {
            top_count[t] = (int)c;
            tab[0] = kSerialFamily;
        }
        return;
    }
    SplitNode front[kTopNodes / 2], next[kTopNodes];
    int fv[kTopNodes / 2], nv[kTopNodes];  // heap indices of the frontier nodes
    int nf = 1;
    front[0] = family_root(t, verts, faces);
    fv[0] = 1;
    if (!EMIT) {
        for (int i = 0; i < kTopNodes; ++i) tab[i] = -1;
    }
    int k = 0;
    const bool can = EMIT ? n > 0 : splittable;
    for (int level = 0; level < kTopLevels && nf > 0; ++level) {
        int nn = 0;
        for (int i = 0; i < nf; ++i) {
            const SplitNode cur = front[i];
            ClipPoint q[3];
            node_clip_points(P, cur, q);
            float best = 0.f;
            const int e = can ? longest_edge(P, cur, q, best) : -1;
            if (e >= 0 && best > 0.f && best >= plan.tau2 && (!EMIT || k < n)) {
                if (!EMIT) tab[fv[i]] = (short)k;
                split_node<EMIT>(P, cur, q, e, k, vbase, fbase, t, next[nn], next[nn + 1], out_verts, map, flag);
                nv[nn] = 2 * fv[i];
                nv[nn + 1] = 2 * fv[i] + 1;
                nn += 2;
                ++k;
            } else if (EMIT) {
#pragma unroll
                for (int j = 0; j < 3; ++j) out_faces[(size_t)cur.slot * 3 + j] = cur.id[j];
            }
        }
        if (level + 1 == kTopLevels) break;  // next[] holds the subtree roots: the tasks' work
        for (int i = 0; i < nn; ++i) {
            front[i] = next[i];
            fv[i] = nv[i];
        }
        nf = nn;
    }
    if (!EMIT) top_count[t] = k;
}

// Subtree task j of family t: rebuilds its root from the top table (the path
// of first / second children given by the bits of j, top level first) and
// walks it depth first.  Counting pass: task_counts[t * kTopNodes + j].
// Emitting pass: its splits are numbered after the family's top splits and
// the subtrees to its left (task_scan: inclusive scan of the task counts).
template <bool EMIT>
__global__ void __launch_bounds__(kSplitThreads) split_task_kernel(
    SplitParams P, const SplitPlan* __restrict__ plan_dev, SplitPlan plan_arg, int N, int M,
    const float* __restrict__ verts, const int* __restrict__ faces, const short* __restrict__ table,
    const int* __restrict__ top_count, int* __restrict__ task_counts, const int* __restrict__ task_scan,
    const int64_t* __restrict__ offsets, float* __restrict__ out_verts, int* __restrict__ out_faces,
    int* __restrict__ map, int* __restrict__ flag, int* __restrict__ status, unsigned long long* __restrict__ total) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (int64_t)M * kTopNodes) return;
    const int t = (int)(gid / kTopNodes), j = (int)(gid % kTopNodes);
    const SplitPlan plan = EMIT ? *plan_dev : plan_arg;
    const short* tab = table + (size_t)t * kTopNodes;
    if (!EMIT) task_counts[gid] = 0;
    if (tab[0] == kSerialFamily) return;
    const int64_t o = EMIT ? offsets[t] : 0, n = EMIT ? offsets[t + 1] - o : 0;
    if (EMIT && n == 0) return;  // nothing of this family splits (the count was reset)
    const int64_t vbase = N + 3 * o, fbase = M + o;
    SplitNode cur = family_root(t, verts, faces);
    int v = 1;
    for (int level = 0; level < kTopLevels; ++level) {
        const int k = tab[v];
        if (k < 0) return;  // the path ends above this subtree: no task
        ClipPoint q[3];
        node_clip_points(P, cur, q);
        float best = 0.f;
        const int e = longest_edge(P, cur, q, best);  // the split the top kernel made
        SplitNode first, second;
        split_node<false>(P, cur, q, e, k, vbase, fbase, t, first, second, nullptr, nullptr, nullptr);
        const int bit = (j >> (kTopLevels - 1 - level)) & 1;
        cur = bit ? second : first;
        v = 2 * v + bit;
    }
    if (!EMIT) {
        task_counts[gid] = (int)walk_subtree<false>(P, plan, 0, cur, true, kMaxFamilySplits, 0, 0, 0, t, nullptr,
                                                    nullptr, nullptr, nullptr, status, total);
        return;
    }
    const int64_t fam0 = t > 0 ? task_scan[(int64_t)t * kTopNodes - 1] : 0;  // tasks of earlier families
    const int mine = task_scan[gid] - (gid > 0 ? task_scan[gid - 1] : 0);
    const int64_t k0 = top_count[t] + (task_scan[gid] - mine - fam0);
    if (k0 + mine > n) {  // inconsistent with the offsets given: write nothing out of range
        atomicOr(status, DS_STATUS_SPLIT_LIMIT);
        return;
    }
    walk_subtree<true>(P, plan, 0, cur, mine > 0, mine, k0, vbase, fbase, t, out_verts, out_faces, map, flag, status,
                       nullptr);
}

// counts[t] = the family's top splits + its subtree tasks' splits.
__global__ void split_family_kernel(int M, const int* __restrict__ top_count, const int* __restrict__ task_scan,
                                    int* __restrict__ counts, int* __restrict__ status) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const int64_t hi = task_scan[(int64_t)t * kTopNodes + kTopNodes - 1];
    const int64_t lo = t > 0 ? task_scan[(int64_t)t * kTopNodes - 1] : 0;
    const int64_t c = top_count[t] + (hi - lo);
    if (c > kMaxFamilySplits) atomicOr(status, DS_STATUS_SPLIT_LIMIT);
    counts[t] = (int)(c < kMaxFamilySplits ? c : kMaxFamilySplits);
}

// Largest considered squared edge length over the faces that may split (as
// the bits of a non-negative float, which order like the values).
__global__ void __launch_bounds__(kSplitThreads) split_max_edge_kernel(SplitParams P, int M,
                                                                       const float* __restrict__ verts,
                                                                       const int* __restrict__ faces,
                                                                       const int* __restrict__ valid,
                                                                       unsigned* __restrict__ max_bits) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M || !(P.mode == 0 || valid == nullptr || valid[t] > 0)) return;
    float p[9];
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) p[k * 3 + j] = verts[(size_t)faces[(size_t)t * 3 + k] * 3 + j];
    ClipPoint q[3];
    for (int k = 0; k < 3; ++k) q[k] = P.mode == 1 ? clip_point(P, p + k * 3) : ClipPoint{};
    float best = 0.f;
    for (int k = 0; k < 3; ++k) best = fmaxf(best, edge_len2(P, p + k * 3, p + ((k + 1) % 3) * 3, q[k], q[(k + 1) % 3]));
    atomicMax(max_bits, __float_as_uint(best));
}

// quota[t] = the share of face t in the first `extra` cut-off splits, faces in
// index order: clamp(extra - before[t], 0, ties[t]).
__global__ void split_quota_kernel(int M, const int* __restrict__ ties, const int64_t* __restrict__ before,
                                   int64_t extra, int* __restrict__ quota) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const int64_t q = extra - before[t];
    quota[t] = q <= 0 ? 0 : (q < ties[t] ? (int)q : ties[t]);
}

__global__ void split_diff_kernel(int M, const int* __restrict__ a, int* __restrict__ b) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < M) b[t] -= a[t];
}

__global__ void copy_floats_kernel(int64_t n, const float* __restrict__ src, float* __restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

static int make_params(int mode, const float* mvp_host, float aspect_wh, SplitParams& P) {
    DS_CHECK_ARG(mode == 0 || mode == 1, "split_soup: mode %d is neither 0 (world) nor 1 (clip)", mode);
    DS_CHECK_ARG(mode == 0 || mvp_host != nullptr, "split_soup: clip mode needs the MVP");
    P.mode = mode;
    for (int i = 0; i < 16; ++i) P.m[i] = mode == 1 ? mvp_host[i] : 0.f;
    P.aspect = aspect_wh;
    return DS_OK;
}

static size_t al256(size_t n) { return (n + 255) & ~(size_t)255; }

// The count call's workspace: per-face counts and quotas, the scan's
// partials, and a small block of scalars that the emit call reads back.
struct SplitWs {
    int* counts;
    int* quota;
    short* table;      // per family: split numbers of its top nodes (heap order)
    int* top_count;    // per family: splits of its top levels (or of the whole family, walked serially)
    int* task_counts;  // per (family, subtree): splits of the subtree
    int* task_scan;    // inclusive scan of task_counts
    void* scan;
    void* scan_tasks;
    unsigned long long* total;  // limit accounting of a counting pass
    int* probe_status;          // status of the current counting pass
    unsigned* max_bits;         // largest edge (split budget)
    SplitPlan* plan;            // the plan the emit call follows
};

static SplitWs carve_split(void* ws, int M, size_t* bytes) {
    const size_t m = (size_t)(M > 0 ? M : 1);
    char* p = reinterpret_cast<char*>(ws);
    size_t o = 0;
    SplitWs w;
    w.counts = reinterpret_cast<int*>(p + o); o += al256(m * sizeof(int));
    w.quota = reinterpret_cast<int*>(p + o); o += al256(m * sizeof(int));
    w.table = reinterpret_cast<short*>(p + o); o += al256(m * kTopNodes * sizeof(short));
    w.top_count = reinterpret_cast<int*>(p + o); o += al256(m * sizeof(int));
    w.task_counts = reinterpret_cast<int*>(p + o); o += al256(m * kTopNodes * sizeof(int));
    w.task_scan = reinterpret_cast<int*>(p + o); o += al256(m * kTopNodes * sizeof(int));
    w.scan = p + o; o += al256(scan_workspace_bytes((int64_t)m));
    w.scan_tasks = p + o; o += al256(scan_workspace_bytes((int64_t)m * kTopNodes));
    w.total = reinterpret_cast<unsigned long long*>(p + o);
    w.probe_status = reinterpret_cast<int*>(p + o + 8);
    w.max_bits = reinterpret_cast<unsigned*>(p + o + 12);
    w.plan = reinterpret_cast<SplitPlan*>(p + o + 16);
    o += 256;
    if (bytes) *bytes = o;
    return w;
}

// One counting pass under `plan` (quotas when given): per-face counts into
// w.counts, their exclusive scan into offsets [M+1]; returns the total, or -1
// when a family or the call exceeded the limits.
static int64_t count_pass(const SplitParams& P, SplitPlan plan, const int* quota, int M, const float* verts,
                          const int* faces, const int* valid, int64_t* offsets, const SplitWs& w, cudaStream_t st,
                          int* rc) {
    *rc = DS_OK;
    if (cudaMemsetAsync(w.total, 0, 16, st) != cudaSuccess) { *rc = check_launch("split_soup_count"); return -1; }
    if (M > 0) {
        split_top_kernel<false><<<blocks_for(M, kSplitThreads), kSplitThreads, 0, st>>>(
            P, nullptr, plan, 0, M, verts, faces, valid, quota, w.table, w.top_count, nullptr, nullptr, nullptr,
            nullptr, nullptr, w.probe_status, w.total);
        split_task_kernel<false><<<blocks_for((int64_t)M * kTopNodes, kSplitThreads), kSplitThreads, 0, st>>>(
            P, nullptr, plan, 0, M, verts, faces, w.table, w.top_count, w.task_counts, nullptr, nullptr, nullptr,
            nullptr, nullptr, nullptr, w.probe_status, w.total);
        if ((*rc = device_scan<int, int>(w.task_counts, (int64_t)M * kTopNodes, w.task_scan, true, w.scan_tasks, st)))
            return -1;
        split_family_kernel<<<blocks_for(M, kSplitThreads), kSplitThreads, 0, st>>>(M, w.top_count, w.task_scan,
                                                                                     w.counts, w.probe_status);
    }
    int64_t* total_dev = nullptr;
    if ((*rc = device_scan<int, int64_t>(w.counts, M, offsets, false, w.scan, st, &total_dev))) return -1;
    int64_t total = 0;
    int pst = 0;
    if (cudaMemcpyAsync(offsets + M, total_dev, sizeof(int64_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(&total, total_dev, sizeof(int64_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&pst, w.probe_status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        *rc = check_launch("split_soup_count");
        return -1;
    }
    if ((*rc = check_launch("split_soup_count"))) return -1;
    return (pst & DS_STATUS_SPLIT_LIMIT) ? -1 : total;
}

static float bits_float(unsigned b) { float f; std::memcpy(&f, &b, 4); return f; }
static unsigned float_bits(float f) { unsigned b; std::memcpy(&b, &f, 4); return b; }

}  // namespace dsb

using namespace dsb;

extern "C" {

size_t ds_split_soup_workspace_size(int M) {
    size_t b = 0;
    carve_split(nullptr, M, &b);
    return b;
}

int ds_split_soup_count(int mode, const float* mvp_host, float aspect_wh, float tau, int num_splits, int N,
                        const float* verts, int M, const int* faces, const int* valid, int64_t* split_offsets,
                        int64_t* total_splits_host, void* workspace, size_t workspace_bytes, int* status,
                        ds_stream_t stream) {
    SplitParams P;
    int rc = make_params(mode, mvp_host, aspect_wh, P);
    if (rc) return rc;
    DS_CHECK_ARG(N >= 0 && M >= 0 && total_splits_host && split_offsets && status, "split_soup: bad arguments");
    DS_CHECK_ARG(M == 0 || (verts && faces), "split_soup: null pointer");
    DS_CHECK_ARG(workspace && workspace_bytes >= ds_split_soup_workspace_size(M), "split_soup: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const SplitWs w = carve_split(workspace, M, nullptr);
    const int* vmask = mode == 1 ? valid : nullptr;
    // world: tau; clip: tau = 2 * tau_ratio (NDC spans 2 per image height)
    const float tt = mode == 0 ? tau : 2.0f * tau;
    const float tau2 = tt * tt;
    SplitPlan plan{INFINITY, 0.f};  // splits nothing
    if (M > 0) DS_CUDA(cudaMemsetAsync(w.quota, 0, (size_t)M * sizeof(int), st));
    DS_CUDA(cudaMemsetAsync(w.probe_status, 0, sizeof(int), st));
    int64_t total = 0;
    if (num_splits < 0 && tau > 0.f) {
        // threshold mode (the *_until functions): every edge of at least tau
        plan = SplitPlan{tau2, 0.f};
        total = count_pass(P, plan, nullptr, M, verts, faces, vmask, split_offsets, w, st, &rc);
        if (rc) return rc;
        if (total < 0) DS_CUDA(cudaMemcpyAsync(status, w.probe_status, sizeof(int), cudaMemcpyDeviceToDevice, st));
    } else if (num_splits > 0 && M > 0) {
        // split budget K: the reference pops edges longest first until K splits, so it performs the K longest
        // splits of all the faces' split trees (a child's edges are shorter than the edge its parent split).
        // Search the squared length lam with count(lam) <= K < count(prev(lam)); the R = K - count(lam) missing
        // splits are edges of exactly prev(lam), taken in face order (the reference's heap takes such ties in
        // an unspecified order).
        const int64_t K = num_splits;
        if (tau > 0.f) {
            total = count_pass(P, SplitPlan{tau2, 0.f}, nullptr, M, verts, faces, vmask, split_offsets, w, st, &rc);
            if (rc) return rc;
            if (total >= 0 && total <= K) plan = SplitPlan{tau2, 0.f};
        }
        if (!(plan.tau2 < INFINITY)) {
            DS_CUDA(cudaMemsetAsync(w.max_bits, 0, sizeof(unsigned), st));
            split_max_edge_kernel<<<blocks_for(M, kSplitThreads), kSplitThreads, 0, st>>>(P, M, verts, faces, vmask,
                                                                                        w.max_bits);
            unsigned hi_bits = 0;
            DS_CUDA(cudaMemcpyAsync(&hi_bits, w.max_bits, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
            DS_CUDA(cudaStreamSynchronize(st));
            const unsigned floor_bits = tau > 0.f ? float_bits(tau2) : 1u;  // lam stays >= tau^2 (> 0)
            if (hi_bits == 0 || hi_bits < floor_bits) {
                total = 0;  // nothing reaches the threshold
            } else {
                // count(hi) <= K is not certain (equal longest edges): walk down until count > K or the floor
                unsigned ok = hi_bits + 1, bad = 0;  // count(ok) <= K, count(bad) > K
                bool have_bad = false;
                unsigned probe = hi_bits;
                for (int it = 0; it < 64 && !have_bad; ++it) {
                    const int64_t c = count_pass(P, SplitPlan{bits_float(probe), 0.f}, nullptr, M, verts, faces,
                                                 vmask, split_offsets, w, st, &rc);
                    if (rc) return rc;
                    if (c < 0 || c > K) { bad = probe; have_bad = true; break; }
                    ok = probe;
                    if (probe == floor_bits) break;
                    // halve the squared length (one exponent step), not below the floor
                    probe = probe > floor_bits + (1u << 23) ? probe - (1u << 23) : floor_bits;
                }
                if (have_bad) {
                    while (ok - bad > 1) {
                        const unsigned mid = bad + (ok - bad) / 2;
                        const int64_t c = count_pass(P, SplitPlan{bits_float(mid), 0.f}, nullptr, M, verts, faces,
                                                     vmask, split_offsets, w, st, &rc);
                        if (rc) return rc;
                        if (c < 0 || c > K) bad = mid; else ok = mid;
                    }
                }
                // lam = the smallest length whose count fits; when even the longest edges exceed the budget,
                // lam lies above them and only the cut-off ties are split
                plan = SplitPlan{bits_float(ok), have_bad ? bits_float(ok - 1) : 0.f};
                total = count_pass(P, SplitPlan{plan.tau2, 0.f}, nullptr, M, verts, faces, vmask, split_offsets, w,
                                   st, &rc);
                if (rc) return rc;
                const int64_t extra = K - total;
                if (have_bad && total >= 0 && extra > 0) {
                    // ties[t] = count_t(prev(lam)) - count_t(lam); quota = their first `extra` in face order
                    DS_CUDA(cudaMemcpyAsync(w.quota, w.counts, (size_t)M * sizeof(int), cudaMemcpyDeviceToDevice,
                                            st));
                    const int64_t c2 = count_pass(P, SplitPlan{plan.tie2, 0.f}, nullptr, M, verts, faces, vmask,
                                                  split_offsets, w, st, &rc);
                    if (rc) return rc;
                    if (c2 < 0) {
                        total = -1;
                    } else {
                        split_diff_kernel<<<blocks_for(M, kSplitThreads), kSplitThreads, 0, st>>>(M, w.quota,
                                                                                                   w.counts);
                        if ((rc = device_scan<int, int64_t>(w.counts, M, split_offsets, false, w.scan, st))) return rc;
                        split_quota_kernel<<<blocks_for(M, kSplitThreads), kSplitThreads, 0, st>>>(
                            M, w.counts, split_offsets, extra, w.quota);
                        total = count_pass(P, plan, w.quota, M, verts, faces, vmask, split_offsets, w, st, &rc);
                        if (rc) return rc;
                    }
                } else {
                    plan.tie2 = 0.f;
                }
            }
        }
        if (total < 0) DS_CUDA(cudaMemcpyAsync(status, w.probe_status, sizeof(int), cudaMemcpyDeviceToDevice, st));
    }
    if (total == 0) {
        // nothing to split: zero offsets
        plan = SplitPlan{INFINITY, 0.f};
        if (M > 0) {
            DS_CUDA(cudaMemsetAsync(w.counts, 0, (size_t)M * sizeof(int), st));
            DS_CUDA(cudaMemsetAsync(w.table, 0xff, (size_t)M * kTopNodes * sizeof(short), st));  // every entry -1
            DS_CUDA(cudaMemsetAsync(w.top_count, 0, (size_t)M * sizeof(int), st));
            DS_CUDA(cudaMemsetAsync(w.task_scan, 0, (size_t)M * kTopNodes * sizeof(int), st));
        }
        if ((rc = device_scan<int, int64_t>(w.counts, M, split_offsets, false, w.scan, st))) return rc;
        DS_CUDA(cudaMemsetAsync(split_offsets + M, 0, sizeof(int64_t), st));
        total = 0;
    }
    if (total < 0) {
        int one = DS_STATUS_SPLIT_LIMIT;
        DS_CUDA(cudaMemcpyAsync(status, &one, sizeof(int), cudaMemcpyHostToDevice, st));
        total = 0;
    }
    DS_CUDA(cudaMemcpyAsync(w.plan, &plan, sizeof(SplitPlan), cudaMemcpyHostToDevice, st));
    DS_CUDA(cudaStreamSynchronize(st));
    *total_splits_host = total;
    return check_launch("split_soup_count");
}

int ds_split_soup_emit(int mode, const float* mvp_host, float aspect_wh, int N, const float* verts, int M,
                       const int* faces, const int64_t* split_offsets, int64_t total_splits, const void* workspace,
                       float* out_verts, int* out_faces, int* out_map, int* out_flag, int* status,
                       ds_stream_t stream) {
    SplitParams P;
    int rc = make_params(mode, mvp_host, aspect_wh, P);
    if (rc) return rc;
    DS_CHECK_ARG(N >= 0 && M >= 0 && total_splits >= 0 && split_offsets && status && workspace,
                 "split_soup: bad arguments");
    DS_CHECK_ARG((int64_t)N + 3 * total_splits <= 0x7fffffff && (int64_t)M + total_splits <= 0x7fffffff,
                 "split_soup: %lld splits exceed the int32 vertex and face indices", (long long)total_splits);
    DS_CHECK_ARG(M == 0 || (verts && faces && out_verts && out_faces && out_map && out_flag),
                 "split_soup: null pointer");
    const SplitWs w = carve_split(const_cast<void*>(workspace), M, nullptr);
    cudaStream_t st = (cudaStream_t)stream;
    if (N > 0) {
        const unsigned b = blocks_for((int64_t)N * 3), cap = (unsigned)sm_count() * 8;
        copy_floats_kernel<<<b < cap ? b : cap, kThreads, 0, st>>>((int64_t)N * 3,
                                                                                                   verts, out_verts);
    }
    if (M > 0) {
        split_top_kernel<true><<<blocks_for(M, kSplitThreads), kSplitThreads, 0, st>>>(
            P, w.plan, SplitPlan{}, N, M, verts, faces, nullptr, w.quota, w.table, w.top_count, split_offsets,
            out_verts, out_faces, out_map, out_flag, status, nullptr);
        split_task_kernel<true><<<blocks_for((int64_t)M * kTopNodes, kSplitThreads), kSplitThreads, 0, st>>>(
            P, w.plan, SplitPlan{}, N, M, verts, faces, w.table, w.top_count, nullptr, w.task_scan, split_offsets,
            out_verts, out_faces, out_map, out_flag, status, nullptr);
    }
    return check_launch("split_soup_emit");
}

}  // extern "C"
