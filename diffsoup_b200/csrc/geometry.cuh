// diffsoup_b200/csrc/geometry.cuh -- per-triangle and per-pixel device math
// shared by the fragment, tiled and shading kernels.  Each function follows
// the reference's arithmetic (kenji-tojo/diffsoup, cited file:line) so that
// triangle IDs, barycentrics and depths match it bit for bit.
#pragma once

#include "common.cuh"

namespace dsb {

// Outcode against the six clip planes (rasterize.cu:10-16).
__device__ __forceinline__ int outcode4(float x, float y, float z, float w) {
    int c = 0;
    c |= (x < -w) ? 1 : 0;  c |= (x > w) ? 2 : 0;
    c |= (y < -w) ? 4 : 0;  c |= (y > w) ? 8 : 0;
    c |= (z < -w) ? 16 : 0; c |= (z > w) ? 32 : 0;
    return c;
}

// NDC bounds with non-finite guards and clamping (rasterize.cu:18-41).
__device__ __forceinline__ void accum_ndc4(float x, float y, float z, float w, float& xmin, float& ymin,
                                           float& zmin, float& xmax, float& ymax, float& zmax) {
    const float invw = __fdiv_rn(1.f, w);
    float nx = __fmul_rn(x, invw), ny = __fmul_rn(y, invw), nz = __fmul_rn(z, invw);
    if (!isfinite(nx)) nx = nx > 0.f ? 1.f : -1.f;
    if (!isfinite(ny)) ny = ny > 0.f ? 1.f : -1.f;
    if (!isfinite(nz)) nz = nz > 0.f ? 1.f : -1.f;
    nx = fminf(1.f, fmaxf(-1.f, nx));
    ny = fminf(1.f, fmaxf(-1.f, ny));
    nz = fminf(1.f, fmaxf(-1.f, nz));
    xmin = fminf(xmin, nx); xmax = fmaxf(xmax, nx);
    ymin = fminf(ymin, ny); ymax = fmaxf(ymax, ny);
    zmin = fminf(zmin, nz); zmax = fmaxf(zmax, nz);
}

// Screen rectangle of a clip-space triangle (rasterize.cu:76-136):
// returns false when culled; otherwise rows [h0, h0+hlen) and columns
// [w0, w0+wlen) bound every pixel the triangle can cover.
__device__ __forceinline__ bool triangle_rect(int H, int W, float4 p0, float4 p1, float4 p2, int& h0, int& hlen,
                                              int& w0, int& wlen) {
    h0 = hlen = w0 = wlen = 0;
    if (!(p0.w > 0.f && p1.w > 0.f && p2.w > 0.f)) return false;
    const int c0 = outcode4(p0.x, p0.y, p0.z, p0.w);
    const int c1 = outcode4(p1.x, p1.y, p1.z, p1.w);
    const int c2 = outcode4(p2.x, p2.y, p2.z, p2.w);
    if ((c0 & c1 & c2) != 0) return false;
    float xmin = 1.f, ymin = 1.f, zmin = 1.f, xmax = -1.f, ymax = -1.f, zmax = -1.f;
    accum_ndc4(p0.x, p0.y, p0.z, p0.w, xmin, ymin, zmin, xmax, ymax, zmax);
    accum_ndc4(p1.x, p1.y, p1.z, p1.w, xmin, ymin, zmin, xmax, ymax, zmax);
    accum_ndc4(p2.x, p2.y, p2.z, p2.w, xmin, ymin, zmin, xmax, ymax, zmax);
    if (zmax < -1.f || zmin > 1.f) return false;
    const float fH = (float)H, fW = (float)W;
    float x0f = __fmul_rn(__fmul_rn(0.5f, __fadd_rn(xmin, 1.f)), fW);
    float x1f = __fmul_rn(__fmul_rn(0.5f, __fadd_rn(xmax, 1.f)), fW);
    float y0f = __fmul_rn(__fmul_rn(0.5f, __fadd_rn(ymin, 1.f)), fH);
    float y1f = __fmul_rn(__fmul_rn(0.5f, __fadd_rn(ymax, 1.f)), fH);
    if (x0f > x1f) { const float t = x0f; x0f = x1f; x1f = t; }
    if (y0f > y1f) { const float t = y0f; y0f = y1f; y1f = t; }
    const int a0 = max((int)floorf(x0f), 0);
    const int a1 = min((int)floorf(x1f), W - 1) + 1;
    const int b0 = max((int)floorf(y0f), 0);
    const int b1 = min((int)floorf(y1f), H - 1) + 1;
    const int wl = max(a1 - a0, 0), hl = max(b1 - b0, 0);
    if (wl == 0 || hl == 0) return false;
    h0 = b0; hlen = hl; w0 = a0; wlen = wl;
    return true;
}

// Homogeneous 2D edge-function coverage test (rasterize.cu:170-206), in two
// stages so that a warp can skip the divisions when none of its lanes needs
// them: edge_terms() gives the three edge functions and their sum,
// surely_outside() rejects what the full test is certain to reject, and
// finish_coverage() completes the reference's test bit for bit.
__device__ __forceinline__ void edge_terms(float ndc_y, float ndc_x, float4 p0, float4 p1, float4 p2, float& A0,
                                           float& A1, float& A2, float& A) {
    const float q0x = sub_mul(p0.x, ndc_x, p0.w), q0y = sub_mul(p0.y, ndc_y, p0.w);
    const float q1x = sub_mul(p1.x, ndc_x, p1.w), q1y = sub_mul(p1.y, ndc_y, p1.w);
    const float q2x = sub_mul(p2.x, ndc_x, p2.w), q2y = sub_mul(p2.y, ndc_y, p2.w);
    A0 = cross2(q1x, q2y, q1y, q2x);
    A1 = cross2(q2x, q0y, q2y, q0x);
    A2 = cross2(q0x, q1y, q0y, q1x);
    A = __fadd_rn(__fadd_rn(A0, A1), A2);
}

// True only where the reference's test fails.  A == 0 is its own rejection.
// Otherwise, with 2^-60 <= |A| <= 2^60 (so 1/A rounds to a normal float):
//  * b0 = A0 * (1/A) is negative (and nonzero) when A0 has the sign opposite
//    to A and |A0| > 2^-100 |A|; likewise b1;
//  * b0 + b1 rounds above 1 when A2 has the sign opposite to A and
//    |A2| > 2^-20 (|A| + |A0| + |A1|): from A = rn(rn(A0 + A1) + A2),
//    (b0 + b1) >= (1 - 2u)(1 + k - 2u - uk - um) with u = 2^-24,
//    k = -A2/A and m = (|A0| + |A1|)/|A|, which exceeds 1 once k > 16u(1 + m).
// Written without branches: with s_k = A_k oriented by the sign of A, "A_k
// nonzero, of the opposite sign and |A_k| > m" is s_k < -m (m >= 0; NaN
// compares false either way).
__device__ __forceinline__ bool surely_outside(float A0, float A1, float A2, float A) {
    const float aA = fabsf(A);
    const bool negA = A < 0.f;
    const float s0 = negA ? -A0 : A0, s1 = negA ? -A1 : A1, s2 = negA ? -A2 : A2;
    const float m01 = aA * 0x1p-100f;
    const float m2 = 0x1p-20f * (aA + fabsf(A0) + fabsf(A1));
    const bool in_range = aA >= 0x1p-60f && aA <= 0x1p60f;
    return A == 0.f || (in_range && (s0 < -m01 || s1 < -m01 || s2 < -m2));
}

// True only when no pixel centre of a block, whose pixel-centre NDC
// coordinates span [xa, xb] x [ya, yb], can pass the reference's coverage
// test.  The edge terms are affine in the NDC point, so over the block their
// extremes (and those of |A| + |A0| + |A1|, a convex function) lie at its
// corners.  The reference's A_k at any pixel, and the value computed here at
// a corner, differ from the exact affine value by at most
// 4u (|q1x q2y| + |q1y q2x|) (u = 2^-24); the margins t_k = 2^-18 S_k, with
// S_k a bound of those products over the block, cover both.  The block is
// rejected when A keeps one sign with 2^-60 <= |A| <= 2^60 everywhere and
// b0 or b1 is negative everywhere, or the b2 condition of surely_outside
// holds everywhere.  NaN anywhere rejects nothing.
__device__ __forceinline__ bool block_surely_outside(float4 p0, float4 p1, float4 p2, float xa, float xb, float ya,
                                                     float yb) {
    // bounds of |q| = |p.xy - ndc p.w| over the block, and the margins
    float t0, t1, t2;
    {
        const float qx0 = fmaxf(fabsf(p0.x - xa * p0.w), fabsf(p0.x - xb * p0.w));
        const float qx1 = fmaxf(fabsf(p1.x - xa * p1.w), fabsf(p1.x - xb * p1.w));
        const float qx2 = fmaxf(fabsf(p2.x - xa * p2.w), fabsf(p2.x - xb * p2.w));
        const float qy0 = fmaxf(fabsf(p0.y - ya * p0.w), fabsf(p0.y - yb * p0.w));
        const float qy1 = fmaxf(fabsf(p1.y - ya * p1.w), fabsf(p1.y - yb * p1.w));
        const float qy2 = fmaxf(fabsf(p2.y - ya * p2.w), fabsf(p2.y - yb * p2.w));
        t0 = 0x1p-18f * (qx1 * qy2 + qy1 * qx2);
        t1 = 0x1p-18f * (qx2 * qy0 + qy2 * qx0);
        t2 = 0x1p-18f * (qx0 * qy1 + qy0 * qx1);
    }
    const float tA = t0 + t1 + t2;
    bool pos = false, r0 = true, r1 = true;
    float m = 0.f, a2 = -INFINITY;  // max of |A| + |A0| + |A1| and of the signed A2 over the corners
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float A0, A1, A2, A;
        edge_terms((c & 2) ? yb : ya, (c & 1) ? xb : xa, p0, p1, p2, A0, A1, A2, A);
        const float aA = fabsf(A);
        if (c == 0) pos = A > 0.f;
        if (!(aA - tA >= 0x1p-60f && aA + tA <= 0x1p60f) || (A > 0.f) != pos) return false;
        r0 = r0 && (pos ? A0 : -A0) < -t0;
        r1 = r1 && (pos ? A1 : -A1) < -t1;
        m = fmaxf(m, aA + fabsf(A0) + fabsf(A1));
        a2 = fmaxf(a2, pos ? A2 : -A2);
    }
    if (r0 || r1) return true;
    return a2 < -(t2 + 0x1p-19f * (m + tA));
}

// Per-triangle data of the block test of the rasterizer's staging pass:
// e[k] = (ox, oy, oc, m) such that, for any block of pixel centres inside
// the rect the record was built for, no centre can pass the reference's
// coverage test when  max over the block of ox x + oy y + oc  <  -m  for
// some k.  (ox, oy, oc) is the exact affine edge function E_k of
// edge_terms (the w-products cancel), oriented so that the inside is
// positive, and m bounds the difference between E_k and the reference's
// FP32 value A_k, the evaluation of the rounded coefficients, and the
// conditions under which surely_outside() rejects.  A record that
// rejects nothing has oc = 1, m = 0.
struct __align__(16) TriEdges {
    float4 e[3];
};

// Builds the TriEdges of a triangle over the pixel-centre NDC rect
// [xa, xb] x [ya, yb] (every |coordinate| <= 1).  The arithmetic is FP64:
// products of two floats are exact, so the coefficients carry one rounding.
//  * Bounds: |q| = |p.xy - ndc p.w| over the rect is largest at its ends;
//    with S_k = Qx_u Qy_v + Qy_u Qx_v, the reference's A_k differs from E_k
//    by at most t_k = 2^-18 S_k (as in block_surely_outside), and its
//    A = rn(rn(A0 + A1) + A2) from S = sum E_k by at most
//    tA = t0 + t1 + t2 + 2^-22 (|E0| + |E1| + |E2|).
//  * S is affine, so its extremes over the rect lie at corners; the test
//    needs one sign with 2^-60 <= |A| <= 2^60 over the rect.
//  * k = 0, 1: A_k of the opposite sign to A with |A_k| > 2^-100 |A|
//    rejects (surely_outside); margin t_k + 2^-99 max|A|.
//  * k = 2: A2 of the opposite sign with |A2| > 2^-20 (|A| + |A0| + |A1|)
//    rejects; margin t_2 + 2^-19 (max|A| + max|A0| + max|A1|).
//  * The block maximum is computed in FP32 from the rounded coefficients,
//    within 2^-22 (|ox| + |oy| + |oc|) for |x|, |y| <= 1; margin 2^-21 of it.
__device__ inline TriEdges tri_edges_over_rect(float4 p0, float4 p1, float4 p2, float xa, float xb, float ya,
                                               float yb) {
    TriEdges out;
    const double4 P[3] = {make_double4(p0.x, p0.y, p0.z, p0.w), make_double4(p1.x, p1.y, p1.z, p1.w),
                          make_double4(p2.x, p2.y, p2.z, p2.w)};
    double Qx[3], Qy[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        Qx[i] = fmax(fabs(P[i].x - (double)xa * P[i].w), fabs(P[i].x - (double)xb * P[i].w)) * (1.0 + 0x1p-20);
        Qy[i] = fmax(fabs(P[i].y - (double)ya * P[i].w), fabs(P[i].y - (double)yb * P[i].w)) * (1.0 + 0x1p-20);
    }
    double ax[3], ay[3], c[3], t[3], emax[3];
    const double cx[2] = {(double)xa, (double)xb}, cy[2] = {(double)ya, (double)yb};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double4 u = P[(k + 1) % 3], v = P[(k + 2) % 3];
        ax[k] = u.y * v.w - u.w * v.y;
        ay[k] = u.w * v.x - u.x * v.w;
        c[k] = u.x * v.y - u.y * v.x;
        t[k] = 0x1p-18 * (Qx[(k + 1) % 3] * Qy[(k + 2) % 3] + Qy[(k + 1) % 3] * Qx[(k + 2) % 3]);
        double m = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) m = fmax(m, fabs(c[k] + ax[k] * cx[j & 1] + ay[k] * cy[j >> 1]));
        emax[k] = m + t[k];
    }
    const double tA = t[0] + t[1] + t[2] + 0x1p-22 * (emax[0] + emax[1] + emax[2]);
    const double sx = ax[0] + ax[1] + ax[2], sy = ay[0] + ay[1] + ay[2], sc = c[0] + c[1] + c[2];
    double slo = INFINITY, shi = -INFINITY;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double s = sc + sx * cx[j & 1] + sy * cy[j >> 1];
        slo = fmin(slo, s);
        shi = fmax(shi, s);
    }
    double sgn = 0.0;
    if (slo - tA >= 0x1p-60 && shi + tA <= 0x1p60) sgn = 1.0;
    else if (-shi - tA >= 0x1p-60 && -slo + tA <= 0x1p60) sgn = -1.0;
    const double amax = fmax(fabs(slo), fabs(shi)) + tA;
    const double m01 = 0x1p-99 * amax, m2 = 0x1p-19 * (amax + emax[0] + emax[1]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double m = t[k] + (k == 2 ? m2 : m01) + 0x1p-21 * (fabs(ax[k]) + fabs(ay[k]) + fabs(c[k]));
        const float mf = (float)(m * (1.0 + 0x1p-20));
        const bool ok = sgn != 0.0 && isfinite(m) && isfinite(mf);
        out.e[k] = ok ? make_float4((float)(sgn * ax[k]), (float)(sgn * ay[k]), (float)(sgn * c[k]), mf)
                      : make_float4(0.f, 0.f, 1.f, 0.f);
    }
    return out;
}

// True when the TriEdges record proves that no pixel centre of the block
// [xa, xb] x [ya, yb] (inside the record's rect) is covered.
__device__ __forceinline__ bool edges_reject_block(const TriEdges& r, float xa, float xb, float ya, float yb) {
    bool out = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float4 e = r.e[k];
        const float v = fmaf(e.x, e.x > 0.f ? xb : xa, fmaf(e.y, e.y > 0.f ? yb : ya, e.z));
        out = out || v < -e.w;
    }
    return out;
}

// Remainder of intersect_triangle given its edge terms (A != 0).
__device__ __forceinline__ bool finish_coverage(float A0, float A1, float A, float4 p0, float4 p1, float4 p2,
                                                float& b0, float& b1, float& z, float& w) {
    const float invA = __frcp_rn(A);  // == 1.f / A, correctly rounded
    b0 = __fmul_rn(A0, invA);
    b1 = __fmul_rn(A1, invA);
    const float b2 = __fsub_rn(__fsub_rn(1.f, b0), b1);
    z = dot3_z(b0, p0.z, b1, p1.z, b2, p2.z);
    w = dot3_w(b0, p0.w, b1, p1.w, b2, p2.w);
    return b0 >= 0.f && b1 >= 0.f && __fadd_rn(b0, b1) <= 1.f;
}

__device__ __forceinline__ bool intersect_triangle(float ndc_y, float ndc_x, float4 p0, float4 p1, float4 p2,
                                                   float& b0, float& b1, float& z, float& w) {
    float A0, A1, A2, A;
    edge_terms(ndc_y, ndc_x, p0, p1, p2, A0, A1, A2, A);
    if (surely_outside(A0, A1, A2, A)) return false;
    return finish_coverage(A0, A1, A, p0, p1, p2, b0, b1, z, w);
}

// Fragment test of compute_fragments (rasterize.cu:257-268): covered and
// depth = z / w within [-1, 1].
__device__ __forceinline__ bool fragment_at(float ndc_y, float ndc_x, float4 p0, float4 p1, float4 p2, float& b0,
                                            float& b1, float& depth) {
    float z, w;
    if (!intersect_triangle(ndc_y, ndc_x, p0, p1, p2, b0, b1, z, w)) return false;
    depth = __fdiv_rn(z, w);
    return depth >= -1.f && depth <= 1.f;
}

__device__ __forceinline__ float4 load_vertex(const float* pos, int v) {
    return __ldg(reinterpret_cast<const float4*>(pos) + v);
}

// ---------------------------------------------------------------------------
// Multi-resolution barycentric lattice (multires.cu:10-68, multires.cuh:8-20)
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t feats_at_level(uint32_t level) {
    return level == 0u ? 3u : (((1u << (level - 1u)) + 1u) * ((1u << level) + 1u));
}

__host__ __device__ __forceinline__ uint32_t total_feats(uint32_t lo, uint32_t hi) {
    uint32_t s = 0;
    for (uint32_t l = lo; l <= hi; ++l) s += feats_at_level(l);
    return s;
}

// Sample indices and weights of the lattice cell containing (b0, b1).
__device__ __forceinline__ void lattice_cell(float b0, float b1, uint32_t level, uint32_t idx[3], float w[3]) {
    const uint32_t res = 1u << level;
    const float res_f = (float)res;
    float b0l = __fmul_rn(b0, res_f), b1l = __fmul_rn(b1, res_f);
    const uint32_t x = min((uint32_t)floorf(b0l), res - 1);
    const uint32_t y = min((uint32_t)floorf(b1l), res - 1 - x);
    b0l = __fsub_rn(b0l, (float)x);
    b1l = __fsub_rn(b1l, (float)y);
    const bool flip = __fadd_rn(b0l, b1l) > 1.f;
    const uint32_t fu = (uint32_t)flip;
    const uint32_t x0 = x + 1, y0 = y, x1 = x, y1 = y + 1;
    const uint32_t x2 = x + fu;
    const uint32_t y2 = min(y + fu, res - x2);
    idx[0] = (x0 + y0) * (x0 + y0 + 1) / 2 + y0;
    idx[1] = (x1 + y1) * (x1 + y1 + 1) / 2 + y1;
    idx[2] = (x2 + y2) * (x2 + y2 + 1) / 2 + y2;
    // Weights of multires.cu:50-53; flip is 0 or 1, so these are exact selects.
    w[0] = flip ? __fsub_rn(1.f, b1l) : b0l;
    w[1] = flip ? __fsub_rn(1.f, b0l) : b1l;
    w[2] = __fsub_rn(__fsub_rn(1.f, w[0]), w[1]);
}

// Scalar lattice interpolation over levels [lo, hi] of one triangle's samples.
__device__ __forceinline__ float interp_scalar(float b0, float b1, uint32_t lo, uint32_t hi, const float* src) {
    float acc = 0.f;
    uint32_t off = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; float w[3];
        lattice_cell(b0, b1, l, idx, w);
        acc = madd(acc, w[0], __ldg(src + off + idx[0]));
        acc = madd(acc, w[1], __ldg(src + off + idx[1]));
        acc = madd(acc, w[2], __ldg(src + off + idx[2]));
        off += feats_at_level(l);
    }
    return acc;
}

// interp_scalar over one level (lo == hi): the same operations without the
// level loop.
__device__ __forceinline__ float interp_level(float b0, float b1, uint32_t level, const float* src) {
    uint32_t idx[3]; float w[3];
    lattice_cell(b0, b1, level, idx, w);
    float acc = 0.f;
    acc = madd(acc, w[0], __ldg(src + idx[0]));
    acc = madd(acc, w[1], __ldg(src + idx[1]));
    acc = madd(acc, w[2], __ldg(src + idx[2]));
    return acc;
}

// Triangular-number inverse of multires.cu:314-325.
__device__ __forceinline__ void index_to_xy(uint32_t idx, uint32_t& x, uint32_t& y) {
    const float fi = (float)idx;
    const uint32_t n = (uint32_t)floorf(__fmul_rn(__fsub_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(8.f, fi), 1.f)), 1.f), 0.5f));
    const uint32_t Tn = (n * (n + 1u)) >> 1;
    y = idx - Tn;
    x = n - y;
}

// ---------------------------------------------------------------------------
// View direction from the inverse MVP (encoding.cu:9-53), unit vector from the
// far plane towards the camera.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void view_direction(float ndc_x, float ndc_y, const float* M, float d[3]) {
    float wn[3], wf[3];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const float nz = s == 0 ? -1.f : 1.f;
        float c[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) c[r] = M[r * 4 + 0] * ndc_x + M[r * 4 + 1] * ndc_y + M[r * 4 + 2] * nz + M[r * 4 + 3];
        const float iw = 1.f / c[3];
        float* o = s == 0 ? wn : wf;
        o[0] = c[0] * iw; o[1] = c[1] * iw; o[2] = c[2] * iw;
    }
    const float dx = wn[0] - wf[0], dy = wn[1] - wf[1], dz = wn[2] - wf[2];
    const float il = rsqrtf(dx * dx + dy * dy + dz * dz);
    d[0] = dx * il; d[1] = dy * il; d[2] = dz * il;
}

// Real spherical-harmonic basis up to degree 2 (encoding.cu:55-85).
__device__ __forceinline__ void sh2_basis(float x, float y, float z, float* sh) {
    const float C0 = 0.28209479177387814f, C1 = 0.4886025119029199f;
    const float C2a = 1.0925484305920792f, C2b = 0.31539156525252005f, C2c = 0.5462742152960396f;
    sh[0] = C0;
    sh[1] = -C1 * y; sh[2] = C1 * z; sh[3] = -C1 * x;
    const float xx = x * x, yy = y * y, zz = z * z;
    sh[4] = C2a * (x * y); sh[5] = -C2a * (y * z); sh[6] = C2b * (2.f * zz - xx - yy);
    sh[7] = -C2a * (x * z); sh[8] = C2c * (xx - yy);
}

}  // namespace dsb
