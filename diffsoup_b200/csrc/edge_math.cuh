// diffsoup_b200/csrc/edge_math.cuh -- per-pixel edge-gradient estimator and
// per-fragment opacity auxiliary gradient (kenji-tojo/diffsoup
// src/cuda/rasterize.cu:489-971), shared by the operator kernels and the
// fused training step.
#pragma once

#include "geometry.cuh"
#include "tiled.cuh"

namespace dsb {

// Segment (x0,y0)-(x1,y1) against (x2,y2)-(x3,y3) (rasterize.cu:493-544).
__device__ __forceinline__ bool segment_intersect2d(float x0, float y0, float x1, float y1, float x2, float y2,
                                                    float x3, float y3, float& ix, float& iy) {
    const float eps = 1e-7f;
    const float rx = x1 - x0, ry = y1 - y0, sx = x3 - x2, sy = y3 - y2;
    const float denom = rx * sy - ry * sx;
    const float qpx = x2 - x0, qpy = y2 - y0;
    if (fabsf(denom) <= eps) {
        const float cr = qpx * ry - qpy * rx;
        if (fabsf(cr) > eps) return false;
        const float rr = rx * rx + ry * ry;
        if (rr < eps) return false;
        const float t0 = ((x2 - x0) * rx + (y2 - y0) * ry) / rr;
        const float t1 = ((x3 - x0) * rx + (y3 - y0) * ry) / rr;
        const float tmin = fminf(t0, t1), tmax = fmaxf(t0, t1);
        if (tmax < -eps || tmin > 1.f + eps) return false;
        const float t = fmaxf(0.f, fminf(1.f, 0.5f * (fmaxf(0.f, tmin) + fminf(1.f, tmax))));
        ix = x0 + t * rx; iy = y0 + t * ry;
        return true;
    }
    const float t = (qpx * sy - qpy * sx) / denom;
    const float u = (qpx * ry - qpy * rx) / denom;
    if (t < -eps || t > 1.f + eps || u < -eps || u > 1.f + eps) return false;
    ix = x0 + t * rx; iy = y0 + t * ry;
    return true;
}

// Which triangle edge the pixel-pair segment crosses, and the perspective-
// correct edge weights at the crossing (rasterize.cu:546-604).
// As find_edge_intersection, given the vertices' NDC rx, ry (x / w, y / w).
__device__ __forceinline__ bool find_edge_intersection_ndc(const float4 P[3], const float rx[3], const float ry[3],
                                                           float x0, float y0, float x1, float y1, int& i0, int& i1,
                                                           float& s0, float& s1) {
    float ix = 0.f, iy = 0.f;
    if (segment_intersect2d(x0, y0, x1, y1, rx[0], ry[0], rx[1], ry[1], ix, iy)) { i0 = 0; i1 = 1; }
    else if (segment_intersect2d(x0, y0, x1, y1, rx[1], ry[1], rx[2], ry[2], ix, iy)) { i0 = 1; i1 = 2; }
    else if (segment_intersect2d(x0, y0, x1, y1, rx[2], ry[2], rx[0], ry[0], ix, iy)) { i0 = 2; i1 = 0; }
    else return false;
    const float4 A = i0 == 0 ? P[0] : (i0 == 1 ? P[1] : P[2]);
    const float4 Bv = i1 == 0 ? P[0] : (i1 == 1 ? P[1] : P[2]);
    const float dx = Bv.x - A.x, dy = Bv.y - A.y, dw = Bv.w - A.w;
    const float ax = A.x - ix * A.w, ay = A.y - iy * A.w;
    const float bx = dx - ix * dw, by = dy - iy * dw;
    const float den = bx * bx + by * by;
    const float t = den != 0.f ? -(ax * bx + ay * by) / den : 0.5f;
    s0 = 1.f - t; s1 = t;
    return true;
}

__device__ __forceinline__ bool find_edge_intersection(const float4 P[3], float x0, float y0, float x1, float y1,
                                                       int& i0, int& i1, float& s0, float& s1) {
    float rx[3], ry[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { rx[k] = P[k].x / P[k].w; ry[k] = P[k].y / P[k].w; }
    return find_edge_intersection_ndc(P, rx, ry, x0, y0, x1, y1, i0, i1, s0, s1);
}

// Unit normal of the triangle in NDC (rasterize.cu:608-633).
__device__ __forceinline__ bool tri_normal_ndc(const float4 P[3], float n[3]) {
    if (fabsf(P[0].w) < 1e-30f || fabsf(P[1].w) < 1e-30f || fabsf(P[2].w) < 1e-30f) return false;
    const float X0 = P[0].x / P[0].w, Y0 = P[0].y / P[0].w, Z0 = P[0].z / P[0].w;
    const float X1 = P[1].x / P[1].w, Y1 = P[1].y / P[1].w, Z1 = P[1].z / P[1].w;
    const float X2 = P[2].x / P[2].w, Y2 = P[2].y / P[2].w, Z2 = P[2].z / P[2].w;
    const float e1x = X1 - X0, e1y = Y1 - Y0, e1z = Z1 - Z0;
    const float e2x = X2 - X0, e2y = Y2 - Y0, e2z = Z2 - Z0;
    const float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const float l2 = nx * nx + ny * ny + nz * nz;
    if (!(l2 > 0.f)) return false;
    const float il = rsqrtf(l2);
    n[0] = nx * il; n[1] = ny * il; n[2] = nz * il;
    return true;
}

// 2D boundary displacement of an intersection line (rasterize.cu:636-651).
__device__ __forceinline__ void db_dp_2d(float nvx, float nvy, float nfx, float nfy, float& dbx, float& dby) {
    float il = rsqrtf(fmaxf(1e-30f, nvx * nvx + nvy * nvy)); nvx *= il; nvy *= il;
    il = rsqrtf(fmaxf(1e-30f, nfx * nfx + nfy * nfy)); nfx *= il; nfy *= il;
    const float bx = -nfy, by = nfx;
    const float den = bx * nvx + by * nvy;
    const float s = fabsf(den) > 1e-12f ? bx / den : 0.f;
    dbx = s * nvx; dby = s * nvy;
}

struct EdgeAccum {
    float g[12];
    bool any;
};

// Interior / implicit-edge contribution at the pixel-pair midpoint
// (rasterize.cu:727-746, :811-835, :843-863).
__device__ __forceinline__ void add_mid_contrib(float mx, float my, const float4 P[3], float gx, float gy, float gz,
                                                bool use_z, EdgeAccum& a) {
    float b0, b1, cz, cw;
    if (!intersect_triangle(my, mx, P[0], P[1], P[2], b0, b1, cz, cw)) return;
    const float b2 = 1.f - b0 - b1;
    const float cx = mx * cw, cy = my * cw;
    const float iw = 1.f / cw, iw2 = iw * iw;
    const float gsum = use_z ? gx * cx + gy * cy + gz * cz : gx * cx + gy * cy;
    const float bb[3] = {b0, b1, b2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a.g[k * 4 + 0] += bb[k] * gx * iw;
        a.g[k * 4 + 1] += bb[k] * gy * iw;
        if (use_z) a.g[k * 4 + 2] += bb[k] * gz * iw;
        a.g[k * 4 + 3] += -bb[k] * gsum * iw2;
    }
    a.any = true;
}

// Edge-gradient estimator of one pixel (rasterize.cu:663-892).  Pixel
// buffers are addressed as base + y*W + x with `base` the view's first pixel;
// posb holds the view's clip positions.  Returns the pixel's triangle (or -1)
// and its clip-space vertex gradients in acc.g[vertex*4 + xyzw].
//
// `pair_once`: an interior pair (both pixels on the same triangle) gives the
// same contribution from either pixel (the adjoint and the pixel offset both
// change sign), so with pair_once the pair is evaluated only from the pixel on
// its left/bottom and counted twice; the caller then runs every pixel.
__device__ __forceinline__ int edge_grad_pixel(int b, int y0, int x0, int H, int W, int C,
                                               const float* __restrict__ color, const float* __restrict__ grad_color,
                                               const float* __restrict__ rast, const float* __restrict__ posb,
                                               const int* __restrict__ tri, int64_t base, EdgeAccum& acc,
                                               bool pair_once = false) {
    (void)b;
#pragma unroll
    for (int k = 0; k < 12; ++k) acc.g[k] = 0.f;
    acc.any = false;
    const int64_t pix0 = base + (int64_t)y0 * W + x0;
    const float4 r0 = reinterpret_cast<const float4*>(rast)[pix0];
    const int it0 = (int)r0.w - 1;
    if (it0 < 0) return -1;
    const float depth0 = r0.z;
    const float nx0 = -1.f + 2.f * ((float)x0 + 0.5f) / (float)W;
    const float ny0 = -1.f + 2.f * ((float)y0 + 0.5f) / (float)H;
    float4 P0[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) P0[k] = load_vertex(posb, __ldg(tri + it0 * 3 + k));
    const float* c0 = color + pix0 * C;
    const float* g0 = grad_color + pix0 * C;
#pragma unroll 1
    for (int e = 0; e < 4; ++e) {
        // neighbour offsets (+x, -x, -y, +y) as in rasterize.cu:691-692
        const int DX = (e == 0) - (e == 1);
        const int DY = (e == 3) - (e == 2);
        const int y1 = y0 + DY, x1 = x0 + DX;
        if (y1 < 0 || y1 >= H || x1 < 0 || x1 >= W) continue;
        const int64_t pix1 = base + (int64_t)y1 * W + x1;
        const float4 r1 = reinterpret_cast<const float4*>(rast)[pix1];
        const float depth1 = r1.z;
        const int it1 = (int)r1.w - 1;
        const bool interior = it1 == it0;
        if (pair_once && interior && (DX < 0 || DY < 0)) continue;  // counted by the neighbour
        const float* c1 = color + pix1 * C;
        const float* g1 = grad_color + pix1 * C;
        float adj = 0.f;
        for (int i = 0; i < C; ++i) adj += 0.5f * (g0[i] + g1[i]) * (c0[i] - c1[i]);
        if (adj == 0.f) continue;
        const float gx = adj * (float)DX * (float)W / 2.f;
        const float gy = adj * (float)DY * (float)H / 2.f;
        const float nx1 = -1.f + 2.f * ((float)x1 + 0.5f) / (float)W;
        const float ny1 = -1.f + 2.f * ((float)y1 + 0.5f) / (float)H;
        const float mx = 0.5f * (nx0 + nx1), my = 0.5f * (ny0 + ny1);
        if (interior) {  // not an edge
            const float m = pair_once ? 2.f : 1.f;
            add_mid_contrib(mx, my, P0, m * gx, m * gy, 0.f, false, acc);
            continue;
        }
        float tb0, tb1, cz1, cw1;
        if (intersect_triangle(ny1, nx1, P0[0], P0[1], P0[2], tb0, tb1, cz1, cw1)) {
            // implicit edge: triangle intersection or opacity edge
            const float d1_it0 = cz1 / cw1;
            if (it1 >= 0 && depth1 < d1_it0) {
                float4 P1[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) P1[k] = load_vertex(posb, __ldg(tri + it1 * 3 + k));
                float cz0, cw0;
                if (intersect_triangle(ny0, nx0, P1[0], P1[1], P1[2], tb0, tb1, cz0, cw0)) {
                    const float d0_it1 = cz0 / cw0;
                    if (depth0 < d0_it1) {  // triangle intersection
                        float nv[3], nf[3];
                        if (tri_normal_ndc(P0, nv) && tri_normal_ndc(P1, nf)) {
                            float gxn = 0.f, gyn = 0.f, gzn = 0.f;
                            if (DX != 0) {
                                float dbx, dbz;
                                db_dp_2d(nv[0], nv[2], nf[0], nf[2], dbx, dbz);
                                gxn = gx * dbx; gzn = gx * dbz;
                            } else {
                                float dby, dbz;
                                db_dp_2d(nv[1], nv[2], nf[1], nf[2], dby, dbz);
                                gyn = gy * dby; gzn = gy * dbz;
                            }
                            add_mid_contrib(mx, my, P0, gxn, gyn, gzn, true, acc);
                        }
                    }
                }
            } else if (it1 < 0 || depth0 < depth1) {  // active opacity edge
                add_mid_contrib(mx, my, P0, gx, gy, 0.f, false, acc);
            }
        } else if (it1 < 0 || depth0 < depth1) {  // active geometric edge
            int i0, i1;
            float s0, s1;
            if (find_edge_intersection(P0, nx0, ny0, nx1, ny1, i0, i1, s0, s1)) {
                const float4 A = i0 == 0 ? P0[0] : (i0 == 1 ? P0[1] : P0[2]);
                const float4 Bv = i1 == 0 ? P0[0] : (i1 == 1 ? P0[1] : P0[2]);
                const float cx = s0 * A.x + s1 * Bv.x;
                const float cy = s0 * A.y + s1 * Bv.y;
                const float cw = s0 * A.w + s1 * Bv.w;
                const float iw = 1.f / cw, iw2 = iw * iw;
                const float gsum = gx * cx + gy * cy;
#pragma unroll
                for (int k = 0; k < 3; ++k) {  // static indices: no local-memory array
                    const float s = k == i0 ? s0 : (k == i1 ? s1 : 0.f);
                    if (k == i0 || k == i1) {
                        acc.g[k * 4 + 0] += s * gx * iw;
                        acc.g[k * 4 + 1] += s * gy * iw;
                        acc.g[k * 4 + 3] += -s * gsum * iw2;
                    }
                }
                acc.any = true;
            }
        }
    }
    return it0;
}

// The estimator of edge_grad_pixel for a colour of 3 channels, reorganised
// for SIMT execution.
//
// * Each interior pair (both pixels on the same triangle) is evaluated once,
//   from its left/bottom pixel, and counted twice (the adjoint and the pixel
//   offset both change sign, so the two evaluations the reference makes are
//   equal).
// * The triangle's edge functions A_k are affine in the NDC point (the
//   w-products of the homogeneous cross product cancel), so they are
//   evaluated once at the pixel centre with the reference's arithmetic and
//   stepped to the neighbour centre and the pair midpoint.  The
//   barycentrics are b_k = A_k / sum A, so coverage is a sign test, and with
//   cw = sum b_k w_k a midpoint's weights b_k / cw are A_k / sum(A_k w_k):
//   one reciprocal per point.
// * A silhouette pair leaves the triangle through the edge whose function
//   changes sign first along the segment between the two centres: the
//   crossing parameter is A_k(p0) / (A_k(p0) - A_k(p1)), which replaces the
//   reference's three segment-segment tests (rasterize.cu:546-604) and gives
//   the same edge except within rounding of a vertex (ties go to the edge
//   the reference tests first).  The perspective-correct position along
//   that edge follows rasterize.cu:585-603.
// * Every pair type ends in one accumulation: weights on the triangle's
//   three vertices at the evaluation point and its clip coordinates
//   (rasterize.cu:727-746 for midpoints, :868-891 for edge crossings).
// Magnitudes use approximate reciprocals; comparisons that decide a pair's
// case use correctly rounded divisions, as the reference does.

// The triangle-intersection case (rasterize.cu:760-809): the neighbour's
// triangle it1 hides it0 there and lies behind it0 at this pixel.  Returns
// false when the pair contributes nothing; else the gradient direction.
__device__ __forceinline__ bool intersection_pair(const float4 P0[3], const TriVerts* __restrict__ tverts, int it1,
                                               float depth0, float nx0, float ny0, int DX, float gx, float gy,
                                               float& gxn, float& gyn, float& gzn) {
    const TriVerts v = tverts[it1];
    float tb0, tb1, cz0, cw0;
    if (!intersect_triangle(ny0, nx0, v.p0, v.p1, v.p2, tb0, tb1, cz0, cw0)) return false;
    if (!(depth0 < cz0 / cw0)) return false;
    const float4 P1[3] = {v.p0, v.p1, v.p2};
    float nv[3], nf[3];
    if (!(tri_normal_ndc(P0, nv) && tri_normal_ndc(P1, nf))) return false;
    gxn = gyn = gzn = 0.f;
    if (DX != 0) {
        float dbx, dbz;
        db_dp_2d(nv[0], nv[2], nf[0], nf[2], dbx, dbz);
        gxn = gx * dbx; gzn = gx * dbz;
    } else {
        float dby, dbz;
        db_dp_2d(nv[1], nv[2], nf[1], nf[2], dby, dbz);
        gyn = gy * dby; gzn = gy * dbz;
    }
    return true;
}

// A 16x16 screen tile of the pixel buffers with a one-pixel border, staged
// in shared memory by the edge-gradient kernel: per pixel its triangle
// (-1 background, kOutside beyond the view), depth, colour, dL/dcolour and
// the far depth bound of its triangle.
constexpr int kHaloW = DS_TILE + 2;
constexpr int kHaloN = kHaloW * kHaloW;
constexpr int kOutside = -2;

struct EdgeHalo {
    int it[kHaloN];
    float dep[kHaloN];
    float zhi[kHaloN];
    float c[3][kHaloN];
    float g[3][kHaloN];
};

// One pixel pair of the staged estimator: the pixel's frame (its triangle's
// clip vertices, the edge functions at its centre and their NDC
// derivatives) and the pair's neighbour offset.
struct EdgeFrame {
    float4 P[3];
    float A[3], ax[3], ay[3];
    float nx, ny, depth, sgn;
};

// Adds u_k (ge_x, ge_y, ge_z, -q) to vertex k's clip-space gradient.
__device__ __forceinline__ void edge_accumulate(EdgeAccum& acc, float u0, float u1, float u2, float ge_x, float ge_y,
                                                float ge_z, float q) {
    const float uv[3] = {u0, u1, u2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        acc.g[k * 4 + 0] += uv[k] * ge_x;
        acc.g[k * 4 + 1] += uv[k] * ge_y;
        acc.g[k * 4 + 2] += uv[k] * ge_z;
        acc.g[k * 4 + 3] -= uv[k] * q;
    }
    acc.any = true;
}

// Contribution at the pair midpoint (centre + (hx, hy)): b_k / cw =
// A_k / sum(A_k w_k) and cz / cw = sum(A_k z_k) / sum(A_k w_k).  Nothing
// when the midpoint lies outside the triangle.
__device__ __forceinline__ void edge_midpoint(const EdgeFrame& f, float hx, float hy, float ge_x, float ge_y,
                                              float ge_z, EdgeAccum& acc) {
    float Am[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) Am[k] = fmaf(f.ay[k], hy, fmaf(f.ax[k], hx, f.A[k]));
    const float Sm = Am[0] + Am[1] + Am[2];
    if (!(Sm != 0.f && Am[0] * Sm >= 0.f && Am[1] * Sm >= 0.f && Am[2] * Sm >= 0.f)) return;
    const float Ws = Am[0] * f.P[0].w + Am[1] * f.P[1].w + Am[2] * f.P[2].w;
    const float Zs = Am[0] * f.P[0].z + Am[1] * f.P[1].z + Am[2] * f.P[2].z;
    const float iW = __fdividef(1.f, Ws);
    const float q = ge_x * (f.nx + hx) + ge_y * (f.ny + hy) + ge_z * (Zs * iW);
    edge_accumulate(acc, Am[0] * iW, Am[1] * iW, Am[2] * iW, ge_x, ge_y, ge_z, q);
}

// The pair's neighbour offset, adjoint direction and edge functions at the
// neighbour centre (recomputed from the staged tile).
struct EdgePair {
    int DX, DY, n;
    float gx, gy, hx, hy;
    float A1[3];
};

// Adjoint of the colour step between staged pixels a and b.
__device__ __forceinline__ float pair_adjoint(const EdgeHalo& h, int a, int b) {
    float adj = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) adj += 0.5f * (h.g[i][a] + h.g[i][b]) * (h.c[i][a] - h.c[i][b]);
    return adj;
}

// The pair towards neighbour e given its adjoint.
__device__ __forceinline__ EdgePair edge_pair(const EdgeFrame& f, int hidx, int e, float adj, int H, int W, float sx,
                                              float sy) {
    EdgePair p;
    p.DX = (e == 0) - (e == 1);
    p.DY = (e == 3) - (e == 2);
    p.n = hidx + p.DX + p.DY * kHaloW;
    p.gx = adj * (float)p.DX * (float)W / 2.f;
    p.gy = adj * (float)p.DY * (float)H / 2.f;
    p.hx = 0.5f * (float)p.DX * sx;
    p.hy = 0.5f * (float)p.DY * sy;
#pragma unroll
    for (int k = 0; k < 3; ++k) p.A1[k] = fmaf(f.ay[k], 2.f * p.hy, fmaf(f.ax[k], 2.f * p.hx, f.A[k]));
    return p;
}

// Edge-gradient estimator of one pixel from the staged tile: the pixel's
// triangle (or -1) is returned and its clip-space vertex gradients are in
// acc.g[vertex*4 + xyzw].  A first pass over the four neighbours only
// classifies the pairs (keeping each marked pair's adjoint in
// adj[e * kEdgeLanes]); interior and opacity-edge pairs (midpoint
// contributions), geometric-edge pairs and pairs that may be triangle
// intersections are then evaluated in three passes, where round k of a pass
// takes each lane's k-th pair of that kind, so that the lanes of a warp run
// the same case together.
// `active` false: the lane has no pixel (it takes part in the warp-wide steps only).
constexpr int kEdgeLanes = DS_TILE * DS_TILE;  // threads of the edge kernel: the stride of adj

__device__ __forceinline__ int edge_grad_pixel_staged(const EdgeHalo& h, int hidx, int y0, int x0, int H, int W,
                                                      const TriVerts* __restrict__ tverts, EdgeAccum& acc,
                                                      float* adj, bool active = true) {
#pragma unroll
    for (int k = 0; k < 12; ++k) acc.g[k] = 0.f;
    acc.any = false;
    const int it0 = active ? h.it[hidx] : -1;
    unsigned mid = 0u, geo = 0u, isect = 0u;  // pairs (bit e) of the midpoint, edge-crossing and intersection passes
    EdgeFrame f;
    // pixel-centre NDC with one reciprocal per axis (this path is compared to
    // the oracle with a tolerance; the 1-ulp difference is far below it)
    const float sx = 2.f / (float)W, sy = 2.f / (float)H;
    if (it0 >= 0) {
        f.depth = h.dep[hidx];
        f.nx = -1.f + ((float)x0 + 0.5f) * sx;
        f.ny = -1.f + ((float)y0 + 0.5f) * sy;
        {
            const TriVerts v = tverts[it0];
            f.P[0] = v.p0; f.P[1] = v.p1; f.P[2] = v.p2;
        }
        float As;
        edge_terms(f.ny, f.nx, f.P[0], f.P[1], f.P[2], f.A[0], f.A[1], f.A[2], As);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float4 u = f.P[(k + 1) % 3], v = f.P[(k + 2) % 3];
            f.ax[k] = u.y * v.w - u.w * v.y;
            f.ay[k] = u.w * v.x - u.x * v.w;
        }
        f.sgn = As > 0.f ? 1.f : -1.f;  // orientation of the inside near the pixel
        // neighbours (+x, -x, -y, +y) as in rasterize.cu:691-692
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (As == 0.f) break;
            const int DX = (e == 0) - (e == 1);
            const int DY = (e == 3) - (e == 2);
            const int n = hidx + DX + DY * kHaloW;
            const int it1 = h.it[n];
            if (it1 == kOutside) continue;  // no neighbour in the view
            const bool interior = it1 == it0;
            if (interior && (DX < 0 || DY < 0)) continue;  // interior pair counted by the neighbour
            const float a = pair_adjoint(h, hidx, n);
            const EdgePair p = edge_pair(f, hidx, e, a, H, W, sx, sy);
            if (p.gx == 0.f && p.gy == 0.f) continue;  // zero adjoint
            adj[e * kEdgeLanes] = a;
            if (interior) {
                mid |= 1u << e;
                continue;
            }
            const float depth1 = h.dep[n];
            const float S1 = p.A1[0] + p.A1[1] + p.A1[2];
            if (S1 != 0.f && p.A1[0] * S1 >= 0.f && p.A1[1] * S1 >= 0.f && p.A1[2] * S1 >= 0.f) {
                // the neighbour centre lies inside it0: implicit edge
                const float z1 = p.A1[0] * f.P[0].z + p.A1[1] * f.P[1].z + p.A1[2] * f.P[2].z;
                const float w1 = p.A1[0] * f.P[0].w + p.A1[1] * f.P[1].w + p.A1[2] * f.P[2].w;
                if (it1 >= 0 && depth1 < z1 / w1) {
                    // it1 hides it0 at the neighbour: a triangle intersection, which needs it1
                    // behind depth0 at this pixel (never when its far depth bound is in front)
                    if (!(h.zhi[n] < f.depth)) isect |= 1u << e;
                } else if (it1 < 0 || f.depth < depth1) {  // active opacity edge
                    mid |= 1u << e;
                }
            } else if (it1 < 0 || f.depth < depth1) {  // active geometric edge
                geo |= 1u << e;
            }
        }
    }
    // midpoint contributions (interior pairs, counted twice, and opacity edges), in neighbour order;
    // pass k takes each lane's k-th marked pair, so that the lanes evaluate them together
    const int nmid = __reduce_max_sync(0xffffffffu, (unsigned)__popc(mid));
    for (int r = 0; r < nmid; ++r) {
        if (mid == 0u) continue;
        const int e = __ffs(mid) - 1;
        mid &= mid - 1u;
        const EdgePair p = edge_pair(f, hidx, e, adj[e * kEdgeLanes], H, W, sx, sy);
        const float m = h.it[p.n] == it0 ? 2.f : 1.f;
        edge_midpoint(f, p.hx, p.hy, m * p.gx, m * p.gy, 0.f, acc);
    }
    // geometric edges: the exit edge is the first edge function to change sign along p0 -> p1,
    // in the reference's test order (0,1) = k 2, (1,2) = k 0, (2,0) = k 1
    const int ngeo = __reduce_max_sync(0xffffffffu, (unsigned)__popc(geo));
    for (int r = 0; r < ngeo; ++r) {
        if (geo == 0u) continue;
        const int e = __ffs(geo) - 1;
        geo &= geo - 1u;
        const EdgePair p = edge_pair(f, hidx, e, adj[e * kEdgeLanes], H, W, sx, sy);
        float tb = 2.f;
        int kb = -1;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int k = (j + 2) % 3;
            const float s0 = fmaxf(f.sgn * f.A[k], 0.f), s1 = f.sgn * p.A1[k];
            if (s1 <= 0.f && s1 < s0) {
                const float t = __fdividef(s0, s0 - s1);
                if (t < tb) { tb = t; kb = k; }
            }
        }
        if (kb < 0) continue;
        const float ix = f.nx + tb * (2.f * p.hx), iy = f.ny + tb * (2.f * p.hy);
        const float4 Av = kb == 0 ? f.P[1] : (kb == 1 ? f.P[2] : f.P[0]);
        const float4 Bv = kb == 0 ? f.P[2] : (kb == 1 ? f.P[0] : f.P[1]);
        const float dx = Bv.x - Av.x, dy = Bv.y - Av.y, dw = Bv.w - Av.w;
        const float qx = Av.x - ix * Av.w, qy = Av.y - iy * Av.w;
        const float bx = dx - ix * dw, by = dy - iy * dw;
        const float den = bx * bx + by * by;
        const float t = den != 0.f ? -__fdividef(qx * bx + qy * by, den) : 0.5f;
        const float s0 = 1.f - t, s1 = t;
        const float cw = s0 * Av.w + s1 * Bv.w;
        const float iw = __fdividef(1.f, cw);
        const float cx = s0 * Av.x + s1 * Bv.x, cy = s0 * Av.y + s1 * Bv.y;
        // vertices (i0, i1) = (kb + 1, kb + 2) mod 3 carry (s0, s1)
        const float v0 = s0 * iw, v1 = s1 * iw;
        edge_accumulate(acc, kb == 0 ? 0.f : (kb == 1 ? v1 : v0), kb == 1 ? 0.f : (kb == 2 ? v1 : v0),
                        kb == 2 ? 0.f : (kb == 0 ? v1 : v0), p.gx, p.gy, 0.f, (p.gx * cx + p.gy * cy) * iw);
    }
    // possible triangle intersections (rasterize.cu:760-809)
    const int nisect = __reduce_max_sync(0xffffffffu, (unsigned)__popc(isect));
    for (int r = 0; r < nisect; ++r) {
        if (isect == 0u) continue;
        const int e = __ffs(isect) - 1;
        isect &= isect - 1u;
        const EdgePair p = edge_pair(f, hidx, e, adj[e * kEdgeLanes], H, W, sx, sy);
        float ge_x, ge_y, ge_z;
        if (intersection_pair(f.P, tverts, h.it[p.n], f.depth, f.nx, f.ny, p.DX, p.gx, p.gy, ge_x, ge_y, ge_z))
            edge_midpoint(f, p.hx, p.hy, ge_x, ge_y, ge_z, acc);
    }
    return it0;
}

// Per-fragment gradient of the opacity auxiliary objective
// (rasterize.cu:955-970): +L/alpha for the visible fragment, -L/(1-alpha)
// for the others in front of the surface or on empty pixels.
__device__ __forceinline__ float aux_alpha_grad(float loss, float alpha, bool visible) {
    const float eps = 1e-5f;
    return visible ? loss / fmaxf(alpha, eps) : -(loss / fmaxf(1.f - alpha, eps));
}

}  // namespace dsb
