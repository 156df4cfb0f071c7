// oracle/oracle.cpp -- CPU restatement of DiffSoup's rasterize-and-shade kernels.
//
// TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
// in diffsoup_b200/csrc: only tests/, __graft_entry__.smoke() and the CPU
// baseline leg of bench.py load it.  The product path never calls into it.
//
// Every function restates one kernel of the reference (kenji-tojo/diffsoup),
// cited as file:line inside that project.  Arithmetic follows the reference's
// FP32 operation order exactly.  Because nvcc contracts a*b+c into FMA by
// default, the FP32 entry points take a `variant` bit mask that selects where
// a fused multiply-add is applied (see the V_* flags below); variant 0 is
// plain IEEE single precision with every operation rounded (what the
// reference produces when built with -fmad=false).  The same code is also
// instantiated in double precision for the FP64 error reports.
//
// Build: g++ -O2 -fopenmp -ffp-contract=off -shared -fPIC (see oracle/Makefile).
// -ffp-contract=off is required: contraction is chosen explicitly below.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <climits>
#include <vector>
#include <algorithm>
#include <type_traits>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// FMA-contraction variants (FP32 only)
// ---------------------------------------------------------------------------
enum : int {
    V_Q = 1,          // q = p.xy - ndc * p.w  ->  fma(-ndc, p.w, p.xy)
    V_CROSS = 2,      // A_i = a*b - c*d fused
    V_CROSS_ALT = 4,  //   0: fma(a, b, -(c*d))   1: fma(-c, d, a*b)
    V_DOT = 8,        // z, w = b0*p0 + b1*p1 + b2*p2 fused
    V_DOT_SHIFT = 4,  //   pattern of z in bits 4..5 (see dot3)
    V_INTERP = 64,    // multires accumulation out += w*f fused
    V_DOTW_SHIFT = 7, //   pattern of w in bits 7..8 (see dot3)
};

template <typename T> constexpr bool is_f32() { return std::is_same<T, float>::value; }

template <typename T>
inline T sub_mul(T a, T b, T c, int v) {  // a - b*c
    if (is_f32<T>() && (v & V_Q)) return std::fma(-b, c, a);
    return a - b * c;
}

template <typename T>
inline T cross2(T a, T b, T c, T d, int v) {  // a*b - c*d
    if (is_f32<T>() && (v & V_CROSS)) {
        if (v & V_CROSS_ALT) return std::fma(-c, d, a * b);
        return std::fma(a, b, -(c * d));
    }
    return a * b - c * d;
}

template <typename T>
inline T dot3(T b0, T x0, T b1, T x1, T b2, T x2, int v, int shift) {  // b0*x0 + b1*x1 + b2*x2
    if (is_f32<T>() && (v & V_DOT)) {
        switch ((v >> shift) & 3) {
            case 0: return std::fma(b2, x2, std::fma(b1, x1, b0 * x0));
            case 1: return std::fma(b2, x2, std::fma(b0, x0, b1 * x1));
            case 2: return std::fma(b1, x1, std::fma(b0, x0, b2 * x2));
            default: return std::fma(b0, x0, std::fma(b1, x1, b2 * x2));
        }
    }
    return b0 * x0 + b1 * x1 + b2 * x2;
}

template <typename T>
inline T madd(T acc, T w, T f, int v) {  // acc + w*f
    if (is_f32<T>() && (v & V_INTERP)) return std::fma(w, f, acc);
    return acc + w * f;
}

inline void atomic_add_d(double* p, double x) {
#pragma omp atomic
    *p += x;
}

inline uint32_t float_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

// ---------------------------------------------------------------------------
// Triangle rectangles: rasterize.cu:10-137
// ---------------------------------------------------------------------------
inline int outcode4(float x, float y, float z, float w) {  // rasterize.cu:10-16
    int c = 0;
    c |= (x < -w) ? 1 : 0;  c |= (x > w) ? 2 : 0;
    c |= (y < -w) ? 4 : 0;  c |= (y > w) ? 8 : 0;
    c |= (z < -w) ? 16 : 0; c |= (z > w) ? 32 : 0;
    return c;
}

inline void accum_ndc4(float x, float y, float z, float w,  // rasterize.cu:18-41
                       float& xmin, float& ymin, float& zmin,
                       float& xmax, float& ymax, float& zmax) {
    const float invw = 1.f / w;
    float nx = x * invw, ny = y * invw, nz = z * invw;
    if (!std::isfinite(nx)) nx = (nx > 0.f ? 1.f : -1.f);
    if (!std::isfinite(ny)) ny = (ny > 0.f ? 1.f : -1.f);
    if (!std::isfinite(nz)) nz = (nz > 0.f ? 1.f : -1.f);
    nx = std::fmin(1.f, std::fmax(-1.f, nx));
    ny = std::fmin(1.f, std::fmax(-1.f, ny));
    nz = std::fmin(1.f, std::fmax(-1.f, nz));
    xmin = std::fmin(xmin, nx); xmax = std::fmax(xmax, nx);
    ymin = std::fmin(ymin, ny); ymax = std::fmax(ymax, ny);
    zmin = std::fmin(zmin, nz); zmax = std::fmax(zmax, nz);
}

// rect = (h0, h_len, w0, w_len); all zero when culled.  rasterize.cu:43-137
inline void triangle_rect(int H, int W, const float* p0, const float* p1, const float* p2, int rect[4]) {
    rect[0] = rect[1] = rect[2] = rect[3] = 0;
    if (!(p0[3] > 0.f && p1[3] > 0.f && p2[3] > 0.f)) return;
    const int c0 = outcode4(p0[0], p0[1], p0[2], p0[3]);
    const int c1 = outcode4(p1[0], p1[1], p1[2], p1[3]);
    const int c2 = outcode4(p2[0], p2[1], p2[2], p2[3]);
    if ((c0 & c1 & c2) != 0) return;
    float xmin = 1.f, ymin = 1.f, zmin = 1.f, xmax = -1.f, ymax = -1.f, zmax = -1.f;
    accum_ndc4(p0[0], p0[1], p0[2], p0[3], xmin, ymin, zmin, xmax, ymax, zmax);
    accum_ndc4(p1[0], p1[1], p1[2], p1[3], xmin, ymin, zmin, xmax, ymax, zmax);
    accum_ndc4(p2[0], p2[1], p2[2], p2[3], xmin, ymin, zmin, xmax, ymax, zmax);
    if (zmax < -1.f || zmin > 1.f) return;
    const float fH = (float)H, fW = (float)W;
    float x0f = 0.5f * (xmin + 1.f) * fW;
    float x1f = 0.5f * (xmax + 1.f) * fW;
    float y0f = 0.5f * (ymin + 1.f) * fH;
    float y1f = 0.5f * (ymax + 1.f) * fH;
    if (x0f > x1f) std::swap(x0f, x1f);
    if (y0f > y1f) std::swap(y0f, y1f);
    const int w0 = std::max((int)std::floor(x0f), 0);
    const int w1 = std::min((int)std::floor(x1f), W - 1) + 1;
    const int h0 = std::max((int)std::floor(y0f), 0);
    const int h1 = std::min((int)std::floor(y1f), H - 1) + 1;
    const int w_len = std::max(w1 - w0, 0);
    const int h_len = std::max(h1 - h0, 0);
    if (w_len == 0 || h_len == 0) return;
    rect[0] = h0; rect[1] = h_len; rect[2] = w0; rect[3] = w_len;
}

// Pixel-centre NDC: rasterize.cu:250-251 (row 0 is the bottom, ndc y = -1).
template <typename T>
inline T pix_ndc(int i, int n) { return T(-1) + T(2) * (T(i) + T(0.5)) / T(n); }

// Homogeneous edge-function coverage test: rasterize.cu:170-206.
template <typename T>
inline bool intersect_triangle(T ndc_y, T ndc_x, const T* P0, const T* P1, const T* P2,
                               T& b0, T& b1, T& out_z, T& out_w, int v) {
    const T q0x = sub_mul(P0[0], ndc_x, P0[3], v), q0y = sub_mul(P0[1], ndc_y, P0[3], v);
    const T q1x = sub_mul(P1[0], ndc_x, P1[3], v), q1y = sub_mul(P1[1], ndc_y, P1[3], v);
    const T q2x = sub_mul(P2[0], ndc_x, P2[3], v), q2y = sub_mul(P2[1], ndc_y, P2[3], v);
    const T A0 = cross2(q1x, q2y, q1y, q2x, v);
    const T A1 = cross2(q2x, q0y, q2y, q0x, v);
    const T A2 = cross2(q0x, q1y, q0y, q1x, v);
    const T A = A0 + A1 + A2;
    if (A == T(0)) return false;
    const T invA = T(1) / A;
    b0 = A0 * invA;
    b1 = A1 * invA;
    const T b2 = T(1) - b0 - b1;
    out_z = dot3(b0, P0[2], b1, P1[2], b2, P2[2], v, V_DOT_SHIFT);
    out_w = dot3(b0, P0[3], b1, P1[3], b2, P2[3], v, V_DOTW_SHIFT);
    return b0 >= T(0) && b1 >= T(0) && b0 + b1 <= T(1);
}

// ---------------------------------------------------------------------------
// Multi-resolution barycentric lattice: multires.cu:10-128, multires.cuh:8-20
// ---------------------------------------------------------------------------
inline uint32_t feats_at_level(uint32_t level) {
    return level == 0u ? 3u : (((1u << (level - 1u)) + 1u) * ((1u << level) + 1u));
}
inline uint32_t total_feats(uint32_t lo, uint32_t hi) {
    uint32_t s = 0;
    for (uint32_t l = lo; l <= hi; ++l) s += feats_at_level(l);
    return s;
}

// Lattice cell of (b0,b1) at `level`: three sample indices and weights.
// The cell arithmetic is done in FP32 as in the reference (multires.cu:22-53);
// the weights are then promoted to T.
template <typename T>
inline void lattice_cell(float b0, float b1, uint32_t level, uint32_t idx[3], T w[3]) {
    const uint32_t res = 1u << level;
    const float res_f = (float)res;
    float b0l = b0 * res_f, b1l = b1 * res_f;
    const float fl0 = std::floor(b0l), fl1 = std::floor(b1l);
    // static_cast<uint32_t>(floorf(x)) of a negative value is undefined in C++;
    // on the GPU (cvt.rzi.u32) it saturates to 0.  Barycentrics of covered
    // fragments are >= 0, so this only matters for out-of-range inputs.
    const uint32_t fx = fl0 <= 0.f ? 0u : (uint32_t)fl0;
    const uint32_t fy = fl1 <= 0.f ? 0u : (uint32_t)fl1;
    const uint32_t x = std::min(fx, res - 1);
    const uint32_t y = std::min(fy, res - 1 - x);
    b0l = b0l - (float)x;
    b1l = b1l - (float)y;
    const bool flip = b0l + b1l > 1.f;
    const uint32_t fu = (uint32_t)flip;
    const float ff = (float)flip;
    const uint32_t x0 = x + 1, y0 = y, x1 = x, y1 = y + 1;
    const uint32_t x2 = x + fu;
    const uint32_t y2 = std::min(y + fu, res - x2);
    idx[0] = (x0 + y0) * (x0 + y0 + 1) / 2 + y0;
    idx[1] = (x1 + y1) * (x1 + y1 + 1) / 2 + y1;
    idx[2] = (x2 + y2) * (x2 + y2 + 1) / 2 + y2;
    // The products by flip in {0,1} are exact, so contraction cannot change them.
    const float w0 = (1.f - ff) * b0l + ff * (1.f - b1l);
    const float w1 = (1.f - ff) * b1l + ff * (1.f - b0l);
    const float w2 = 1.f - w0 - w1;
    w[0] = (T)w0; w[1] = (T)w1; w[2] = (T)w2;
}

// multires.cu:10-68 (out accumulates; caller zeroes it)
template <typename T, typename F>
inline void interp(float b0, float b1, uint32_t lo, uint32_t hi, uint32_t C,
                   const F* feats, T* out, int v) {
    uint32_t offset = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; T w[3];
        lattice_cell<T>(b0, b1, l, idx, w);
        const F* lf = feats + (size_t)offset * C;
        for (int i = 0; i < 3; ++i)
            for (uint32_t j = 0; j < C; ++j)
                out[j] = madd<T>(out[j], w[i], (T)lf[(size_t)idx[i] * C + j], v);
        offset += feats_at_level(l);
    }
}

// multires.cu:70-128 (scatter into double accumulators)
template <typename T>
inline void interp_backward(float b0, float b1, uint32_t lo, uint32_t hi, uint32_t C,
                            double* grad_feats, const T* grad_out) {
    uint32_t offset = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; T w[3];
        lattice_cell<T>(b0, b1, l, idx, w);
        double* lg = grad_feats + (size_t)offset * C;
        for (int i = 0; i < 3; ++i)
            for (uint32_t j = 0; j < C; ++j)
                atomic_add_d(&lg[(size_t)idx[i] * C + j], (double)(grad_out[j] * w[i]));
        offset += feats_at_level(l);
    }
}

// multires.cu:314-325
inline void index_to_xy(uint32_t idx, uint32_t& x, uint32_t& y) {
    const float fi = (float)idx;
    const uint32_t n = (uint32_t)std::floor((std::sqrt(8.f * fi + 1.f) - 1.f) * 0.5f);
    const uint32_t Tn = (n * (n + 1u)) >> 1;
    y = idx - Tn;
    x = n - y;
}

// ---------------------------------------------------------------------------
// Counter-based RNG for the stochastic opacity threshold: Philox-4x32-10
// (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011).  Counter = (pixel, tri, view, iter), key = seed.
// ---------------------------------------------------------------------------
inline void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)M0 * ctr[0];
        const uint64_t p1 = (uint64_t)M1 * ctr[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        const uint32_t n1 = lo1;
        const uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        const uint32_t n3 = lo0;
        ctr[0] = n0; ctr[1] = n1; ctr[2] = n2; ctr[3] = n3;
        k0 += W0; k1 += W1;
    }
}

inline float opacity_threshold(uint64_t seed, uint32_t iter, uint32_t view, uint32_t pixel, uint32_t tri) {
    uint32_t c[4] = {pixel, tri, view, iter};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    return (float)(c[0] >> 8) * (1.0f / 16777216.0f);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int orc_omp_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

uint32_t orc_feats_at_level(uint32_t level) { return feats_at_level(level); }

float orc_opacity_threshold(uint64_t seed, uint32_t iter, uint32_t view, uint32_t pixel, uint32_t tri) {
    return opacity_threshold(seed, iter, view, pixel, tri);
}

// rasterize.cu:139-168.  rects [B*T,4], prefix [B*T] inclusive (int64 here so
// the oracle never overflows); returns the total bbox-pixel count.
int64_t orc_triangle_rects(int H, int W, int B, int V, const float* pos, int T, const int* tri,
                           int* rects, int64_t* prefix) {
    const int64_t n = (int64_t)B * T;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int64_t b = i / T, t = i % T;
        const float* P = pos + (size_t)b * V * 4;
        triangle_rect(H, W, P + (size_t)tri[t * 3 + 0] * 4, P + (size_t)tri[t * 3 + 1] * 4,
                      P + (size_t)tri[t * 3 + 2] * 4, rects + i * 4);
    }
    int64_t acc = 0;
    for (int64_t i = 0; i < n; ++i) { acc += (int64_t)rects[i * 4 + 1] * rects[i * 4 + 3]; prefix[i] = acc; }
    return acc;
}

// rasterize.cu:208-277.  frag_pix must be pre-filled with -1 by the caller
// (rasterize.py:69); rejected bbox pixels keep -1.
void orc_fragments(int variant, int H, int W, int B, int V, const float* pos, int T, const int* tri,
                   const int* rects, const int64_t* prefix, int* frag_pix, float* frag_attrs) {
    const int64_t n = (int64_t)B * T;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        const int* r = rects + i * 4;
        if (r[1] <= 0 || r[3] <= 0) continue;
        const int b = (int)(i / T), t = (int)(i % T);
        const float* P = pos + (size_t)b * V * 4;
        const float* P0 = P + (size_t)tri[t * 3 + 0] * 4;
        const float* P1 = P + (size_t)tri[t * 3 + 1] * 4;
        const float* P2 = P + (size_t)tri[t * 3 + 2] * 4;
        const int64_t base = i == 0 ? 0 : prefix[i - 1];
        const int64_t cnt = (int64_t)r[1] * r[3];
        for (int64_t l = 0; l < cnt; ++l) {
            const int y = r[0] + (int)(l / r[3]);
            const int x = r[2] + (int)(l % r[3]);
            if (x < 0 || x >= W || y < 0 || y >= H) continue;
            const float ndc_y = pix_ndc<float>(y, H), ndc_x = pix_ndc<float>(x, W);
            float b0, b1, z, w;
            if (!intersect_triangle<float>(ndc_y, ndc_x, P0, P1, P2, b0, b1, z, w, variant)) continue;
            const float depth = z / w;
            if (!(depth >= -1.f && depth <= 1.f)) continue;
            const int64_t k = base + l;
            frag_pix[k * 3 + 0] = b; frag_pix[k * 3 + 1] = y; frag_pix[k * 3 + 2] = x;
            frag_attrs[k * 4 + 0] = b0; frag_attrs[k * 4 + 1] = b1;
            frag_attrs[k * 4 + 2] = depth; frag_attrs[k * 4 + 3] = (float)(t + 1);
        }
    }
}

// rasterize.cu:402-487, order preserving (the reference's block order is
// nondeterministic; within-view fragment order here is triangle order).
int64_t orc_filter_valid(int64_t n, const int* frag_pix, const float* frag_attrs,
                         int* pix_out, float* attrs_out) {
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (frag_pix[i * 3] < 0) continue;
        std::memcpy(pix_out + k * 3, frag_pix + i * 3, 12);
        std::memcpy(attrs_out + k * 4, frag_attrs + i * 4, 16);
        ++k;
    }
    return k;
}

// multires.cu:130-156 (FP32 with variant).
void orc_multires_alpha(int variant, int64_t nf, const float* frag_attrs, int lo, int hi,
                        const float* alpha_src, float* frag_alpha) {
    const uint32_t S = total_feats(lo, hi);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nf; ++i) {
        const int t = (int)frag_attrs[i * 4 + 3] - 1;
        if (t < 0) continue;
        float a = 0.f;
        interp<float, float>(frag_attrs[i * 4], frag_attrs[i * 4 + 1], lo, hi, 1,
                             alpha_src + (size_t)t * S, &a, variant);
        frag_alpha[i] = a;
    }
}

// multires.cu:178-202, accumulated in double then rounded.
void orc_multires_alpha_backward(int64_t nf, const float* frag_attrs, int lo, int hi, int T,
                                 double* grad_alpha_src, const double* grad_frag_alpha) {
    const uint32_t S = total_feats(lo, hi);
    (void)T;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nf; ++i) {
        const int t = (int)frag_attrs[i * 4 + 3] - 1;
        if (t < 0) continue;
        const double g = grad_frag_alpha[i];
        interp_backward<double>(frag_attrs[i * 4], frag_attrs[i * 4 + 1], lo, hi, 1,
                                grad_alpha_src + (size_t)t * S, &g);
    }
}

// Per-fragment thresholds: 0.5 when seed == 0 and iter == UINT32_MAX
// (stochastic=False, multires.py:99-100), else Philox keyed by
// (view, y*W+x, tri).
void orc_fragment_thresholds(int64_t nf, const int* frag_pix, const float* frag_attrs, int W,
                             int stochastic, uint64_t seed, uint32_t iter, float* thresh) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nf; ++i) {
        if (!stochastic) { thresh[i] = 0.5f; continue; }
        const int b = frag_pix[i * 3], y = frag_pix[i * 3 + 1], x = frag_pix[i * 3 + 2];
        const int t = (int)frag_attrs[i * 4 + 3] - 1;
        thresh[i] = opacity_threshold(seed, iter, (uint32_t)b, (uint32_t)(y * W + x), (uint32_t)t);
    }
}

// rasterize.cu:307-400.  Packed key (bits(z+2) << 32 | fragment index), min
// wins; the winner's attrs are gathered into rast (zeros elsewhere).
void orc_depth_test(int B, int H, int W, int64_t nf, const int* frag_pix, const float* frag_attrs,
                    const float* frag_alpha, const float* alpha_thresh, float* rast) {
    const int64_t npix = (int64_t)B * H * W;
    std::vector<uint64_t> best((size_t)npix, (uint64_t)LLONG_MAX);
    std::vector<int64_t> who((size_t)npix, -1);
    for (int64_t i = 0; i < nf; ++i) {
        const int b = frag_pix[i * 3];
        if (b < 0) continue;
        const int64_t p = (int64_t)b * H * W + (int64_t)frag_pix[i * 3 + 1] * W + frag_pix[i * 3 + 2];
        if (frag_alpha[i] < alpha_thresh[i]) continue;
        const float zw = frag_attrs[i * 4 + 2];
        if (zw <= -1.f || !std::isfinite(zw)) continue;
        const uint64_t key = ((uint64_t)float_bits(zw + 2.f) << 32) | (uint64_t)(uint32_t)i;
        if (key < best[p]) { best[p] = key; who[p] = i; }
    }
    std::memset(rast, 0, sizeof(float) * (size_t)npix * 4);
    for (int64_t p = 0; p < npix; ++p)
        if (who[p] >= 0) std::memcpy(rast + p * 4, frag_attrs + who[p] * 4, 16);
}

// Composite of rasterize_multires_triangle_alpha (multires.py:52-102) for one
// call: rects -> fragments -> compaction -> alpha -> threshold -> depth test.
// Processed view by view (the reference's int32 counts overflow otherwise).
// Returns the number of covered fragments (before the depth test).
int64_t orc_rasterize_alpha(int variant, int H, int W, int B, int V, const float* pos, int T,
                            const int* tri, int level, const float* alpha_src, int stochastic,
                            uint64_t seed, uint32_t iter, int view0, float* rast) {
    int64_t total_frags = 0;
    const int64_t npix = (int64_t)H * W;
    for (int b = 0; b < B; ++b) {
        const float* P = pos + (size_t)b * V * 4;
        std::vector<int> rects((size_t)T * 4);
        std::vector<int64_t> prefix((size_t)T);
        const int64_t nbb = orc_triangle_rects(H, W, 1, V, P, T, tri, rects.data(), prefix.data());
        std::vector<int> fpix((size_t)nbb * 3, -1);
        std::vector<float> fattr((size_t)nbb * 4, 0.f);
        orc_fragments(variant, H, W, 1, V, P, T, tri, rects.data(), prefix.data(), fpix.data(), fattr.data());
        std::vector<int> cpix((size_t)nbb * 3);
        std::vector<float> cattr((size_t)nbb * 4);
        const int64_t nf = orc_filter_valid(nbb, fpix.data(), fattr.data(), cpix.data(), cattr.data());
        for (int64_t i = 0; i < nf; ++i) cpix[i * 3] = view0 + b;
        std::vector<float> alpha((size_t)nf, 0.f), thr((size_t)nf);
        orc_multires_alpha(variant, nf, cattr.data(), level, level, alpha_src, alpha.data());
        orc_fragment_thresholds(nf, cpix.data(), cattr.data(), W, stochastic, seed, iter, thr.data());
        for (int64_t i = 0; i < nf; ++i) cpix[i * 3] = 0;
        orc_depth_test(1, H, W, nf, cpix.data(), cattr.data(), alpha.data(), thr.data(), rast + b * npix * 4);
        total_frags += nf;
    }
    return total_frags;
}

// ---------------------------------------------------------------------------
// Per-pixel feature interpolation: multires.cu:224-311
// ---------------------------------------------------------------------------
void orc_multires_color_f32(int variant, int B, int H, int W, const float* rast, int lo, int hi, int C,
                            const float* feat, float* out) {
    const uint32_t S = total_feats(lo, hi);
    const int64_t n = (int64_t)B * H * W;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int t = (int)rast[i * 4 + 3] - 1;
        if (t < 0) continue;
        interp<float, float>(rast[i * 4], rast[i * 4 + 1], lo, hi, C, feat + (size_t)t * S * C, out + i * C, variant);
    }
}

void orc_multires_color_f64(int B, int H, int W, const float* rast, int lo, int hi, int C,
                            const double* feat, double* out) {
    const uint32_t S = total_feats(lo, hi);
    const int64_t n = (int64_t)B * H * W;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int t = (int)rast[i * 4 + 3] - 1;
        if (t < 0) continue;
        interp<double, double>(rast[i * 4], rast[i * 4 + 1], lo, hi, C, feat + (size_t)t * S * C, out + i * C, 0);
    }
}

// grad_feat (double, zeroed by caller) += scatter of grad_out.
void orc_multires_color_backward(int B, int H, int W, const float* rast, int lo, int hi, int C,
                                 double* grad_feat, const double* grad_out) {
    const uint32_t S = total_feats(lo, hi);
    const int64_t n = (int64_t)B * H * W;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int t = (int)rast[i * 4 + 3] - 1;
        if (t < 0) continue;
        interp_backward<double>(rast[i * 4], rast[i * 4 + 1], lo, hi, C, grad_feat + (size_t)t * S * C, grad_out + i * C);
    }
}

// ---------------------------------------------------------------------------
// Cross-level accumulation: multires.cu:329-430
// ---------------------------------------------------------------------------
void orc_accumulate_forward_f64(int T, int lo, int hi, int target, int C, const double* feat, double* out) {
    const uint32_t S = total_feats(lo, hi), ST = feats_at_level(target);
    const float Rf = (float)(1u << target);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)T * ST; ++i) {
        const uint32_t t = (uint32_t)(i / ST), k = (uint32_t)(i % ST);
        uint32_t x, y; index_to_xy(k, x, y);
        const float b0 = (float)x / Rf, b1 = (float)y / Rf;
        double* o = out + (size_t)i * C;
        for (int c = 0; c < C; ++c) o[c] = 0.0;
        interp<double, double>(b0, b1, lo, hi, C, feat + (size_t)t * S * C, o, 0);
    }
}

void orc_accumulate_forward_f32(int variant, int T, int lo, int hi, int target, int C, const float* feat, float* out) {
    const uint32_t S = total_feats(lo, hi), ST = feats_at_level(target);
    const float Rf = (float)(1u << target);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)T * ST; ++i) {
        const uint32_t t = (uint32_t)(i / ST), k = (uint32_t)(i % ST);
        uint32_t x, y; index_to_xy(k, x, y);
        const float b0 = (float)x / Rf, b1 = (float)y / Rf;
        float* o = out + (size_t)i * C;
        for (int c = 0; c < C; ++c) o[c] = 0.f;
        interp<float, float>(b0, b1, lo, hi, C, feat + (size_t)t * S * C, o, variant);
    }
}

void orc_accumulate_backward(int T, int lo, int hi, int target, int C, double* grad_feat, const double* grad_out) {
    const uint32_t S = total_feats(lo, hi), ST = feats_at_level(target);
    const float Rf = (float)(1u << target);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)T * ST; ++i) {
        const uint32_t t = (uint32_t)(i / ST), k = (uint32_t)(i % ST);
        uint32_t x, y; index_to_xy(k, x, y);
        const float b0 = (float)x / Rf, b1 = (float)y / Rf;
        interp_backward<double>(b0, b1, lo, hi, C, grad_feat + (size_t)t * S * C, grad_out + (size_t)i * C);
    }
}

// ---------------------------------------------------------------------------
// View-direction encodings: encoding.cu:9-118
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {
template <typename T>
inline void view_direction(T ndc_x, T ndc_y, const T* M, T d[3]) {  // encoding.cu:9-53
    T wn[3] = {0, 0, 0}, wf[3] = {0, 0, 0};
    for (int s = 0; s < 2; ++s) {
        const T nz = s == 0 ? T(-1) : T(1);
        T c[4];
        for (int r = 0; r < 4; ++r) c[r] = M[r * 4 + 0] * ndc_x + M[r * 4 + 1] * ndc_y + M[r * 4 + 2] * nz + M[r * 4 + 3];
        const T iw = T(1) / c[3];
        T* o = s == 0 ? wn : wf;
        o[0] = c[0] * iw; o[1] = c[1] * iw; o[2] = c[2] * iw;
    }
    const T dx = wn[0] - wf[0], dy = wn[1] - wf[1], dz = wn[2] - wf[2];
    const T il = T(1) / std::sqrt(dx * dx + dy * dy + dz * dz);
    d[0] = dx * il; d[1] = dy * il; d[2] = dz * il;
}

template <typename T>
inline void sh2(T x, T y, T z, T* sh) {  // encoding.cu:56-85
    const T C0 = T(0.28209479177387814), C1 = T(0.4886025119029199);
    const T C20 = T(1.0925484305920792), C21 = T(-1.0925484305920792), C22 = T(0.31539156525252005),
            C23 = T(-1.0925484305920792), C24 = T(0.5462742152960396);
    sh[0] = C0;
    sh[1] = -C1 * y; sh[2] = C1 * z; sh[3] = -C1 * x;
    const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
    sh[4] = C20 * xy; sh[5] = C21 * yz; sh[6] = C22 * (T(2) * zz - xx - yy); sh[7] = C23 * xz; sh[8] = C24 * (xx - yy);
}

template <typename T>
void encode_view(int B, int H, int W, const float* rast, const T* inv_mvp, T* enc, int sh) {
    const int64_t n = (int64_t)B * H * W;
    const int K = sh ? 9 : 3;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int b = (int)(i / ((int64_t)H * W));
        const int y = (int)((i % ((int64_t)H * W)) / W), x = (int)((i % ((int64_t)H * W)) % W);
        if ((int)rast[i * 4 + 3] - 1 < 0) continue;
        T d[3];
        view_direction<T>(pix_ndc<T>(x, W), pix_ndc<T>(y, H), inv_mvp + (size_t)b * 16, d);
        if (sh) sh2<T>(d[0], d[1], d[2], enc + i * K);
        else { enc[i * 3] = d[0]; enc[i * 3 + 1] = d[1]; enc[i * 3 + 2] = d[2]; }
    }
}

// ---------------------------------------------------------------------------
// Edge gradients: rasterize.cu:489-903
// ---------------------------------------------------------------------------
template <typename T>
bool segment_intersect2d(T x0, T y0, T x1, T y1, T x2, T y2, T x3, T y3, T& ix, T& iy) {  // :493-544
    const T eps = T(1e-7f);
    const T rx = x1 - x0, ry = y1 - y0, sx = x3 - x2, sy = y3 - y2;
    const T denom = rx * sy - ry * sx;
    const T qpx = x2 - x0, qpy = y2 - y0;
    if (std::fabs(denom) <= eps) {
        const T cr = qpx * ry - qpy * rx;
        if (std::fabs(cr) > eps) return false;
        const T rr = rx * rx + ry * ry;
        if (rr < eps) return false;
        const T t0 = ((x2 - x0) * rx + (y2 - y0) * ry) / rr;
        const T t1 = ((x3 - x0) * rx + (y3 - y0) * ry) / rr;
        const T tmin = std::min(t0, t1), tmax = std::max(t0, t1);
        if (tmax < -eps || tmin > T(1) + eps) return false;
        const T t = std::max(T(0), std::min(T(1), T(0.5) * (std::max(T(0), tmin) + std::min(T(1), tmax))));
        ix = x0 + t * rx; iy = y0 + t * ry;
        return true;
    }
    const T t = (qpx * sy - qpy * sx) / denom;
    const T u = (qpx * ry - qpy * rx) / denom;
    if (t < -eps || t > T(1) + eps || u < -eps || u > T(1) + eps) return false;
    ix = x0 + t * rx; iy = y0 + t * ry;
    return true;
}

template <typename T>
bool find_edge_intersection(const T* P[3], T x0, T y0, T x1, T y1, int& i0, int& i1, T& s0, T& s1) {  // :546-604
    T r[3][2];
    for (int k = 0; k < 3; ++k) { r[k][0] = P[k][0] / P[k][3]; r[k][1] = P[k][1] / P[k][3]; }
    T ix = 0, iy = 0;
    if (segment_intersect2d(x0, y0, x1, y1, r[0][0], r[0][1], r[1][0], r[1][1], ix, iy)) { i0 = 0; i1 = 1; }
    else if (segment_intersect2d(x0, y0, x1, y1, r[1][0], r[1][1], r[2][0], r[2][1], ix, iy)) { i0 = 1; i1 = 2; }
    else if (segment_intersect2d(x0, y0, x1, y1, r[2][0], r[2][1], r[0][0], r[0][1], ix, iy)) { i0 = 2; i1 = 0; }
    else return false;
    const T* A = P[i0]; const T* Bv = P[i1];
    const T dx = Bv[0] - A[0], dy = Bv[1] - A[1], dw = Bv[3] - A[3];
    const T ax = A[0] - ix * A[3], ay = A[1] - iy * A[3];
    const T bx = dx - ix * dw, by = dy - iy * dw;
    const T den = bx * bx + by * by;
    const T t = den != T(0) ? -(ax * bx + ay * by) / den : T(0.5);
    s0 = T(1) - t; s1 = t;
    return true;
}

template <typename T>
bool tri_normal_ndc(const T* P[3], T n[3]) {  // :608-633
    for (int k = 0; k < 3; ++k) if (std::fabs(P[k][3]) < T(1e-30f)) return false;
    T X[3], Y[3], Z[3];
    for (int k = 0; k < 3; ++k) { X[k] = P[k][0] / P[k][3]; Y[k] = P[k][1] / P[k][3]; Z[k] = P[k][2] / P[k][3]; }
    const T e1x = X[1] - X[0], e1y = Y[1] - Y[0], e1z = Z[1] - Z[0];
    const T e2x = X[2] - X[0], e2y = Y[2] - Y[0], e2z = Z[2] - Z[0];
    const T nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const T l2 = nx * nx + ny * ny + nz * nz;
    if (!(l2 > T(0))) return false;
    const T il = T(1) / std::sqrt(l2);
    n[0] = nx * il; n[1] = ny * il; n[2] = nz * il;
    return true;
}

template <typename T>
void db_dp_2d(T nvx, T nvy, T nfx, T nfy, T& dbx, T& dby) {  // :636-651
    T il = T(1) / std::sqrt(std::max(T(1e-30f), nvx * nvx + nvy * nvy)); nvx *= il; nvy *= il;
    il = T(1) / std::sqrt(std::max(T(1e-30f), nfx * nfx + nfy * nfy)); nfx *= il; nfy *= il;
    const T bx = -nfy, by = nfx;
    const T den = bx * nvx + by * nvy;
    const T s = std::fabs(den) > T(1e-12f) ? bx / den : T(0);
    dbx = s * nvx; dby = s * nvy;
}

// Adds the interior/implicit-edge contribution at the pixel-pair midpoint
// (rasterize.cu:727-746, :811-835, :843-863).
template <typename T>
void add_mid_contrib(T ndc_mid_x, T ndc_mid_y, const T* P[3], T gx, T gy, T gz, bool use_z, T g[12], int v) {
    T b0, b1, cz, cw;
    if (!intersect_triangle<T>(ndc_mid_y, ndc_mid_x, P[0], P[1], P[2], b0, b1, cz, cw, v)) return;
    const T b2 = T(1) - b0 - b1;
    const T cx = ndc_mid_x * cw, cy = ndc_mid_y * cw;
    const T iw = T(1) / cw, iw2 = iw * iw;
    const T gsum = use_z ? gx * cx + gy * cy + gz * cz : gx * cx + gy * cy;
    const T bb[3] = {b0, b1, b2};
    for (int k = 0; k < 3; ++k) {
        g[k * 4 + 0] += bb[k] * gx * iw;
        g[k * 4 + 1] += bb[k] * gy * iw;
        if (use_z) g[k * 4 + 2] += bb[k] * gz * iw;
        g[k * 4 + 3] += -bb[k] * gsum * iw2;
    }
}

template <typename T>
void edge_grad(int B, int H, int W, int C, const T* color, const T* grad_color, const float* rast,
               int V, const T* pos, const int* tri, double* grad_pos, int v) {  // :653-903
    const int64_t n = (int64_t)B * H * W;
    const int DY[4] = {0, 0, -1, 1}, DX[4] = {1, -1, 0, 0};
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t idx = 0; idx < n; ++idx) {
        const int b = (int)(idx / ((int64_t)H * W));
        const int y0 = (int)((idx % ((int64_t)H * W)) / W), x0 = (int)((idx % ((int64_t)H * W)) % W);
        const T nx0 = pix_ndc<T>(x0, W), ny0 = pix_ndc<T>(y0, H);
        const int64_t pix0 = idx;
        const T depth0 = (T)rast[pix0 * 4 + 2];
        const int it0 = (int)rast[pix0 * 4 + 3] - 1;
        if (it0 < 0) continue;
        const int* v0 = tri + it0 * 3;
        const T* bp = pos + (size_t)b * V * 4;
        const T* P0[3] = {bp + (size_t)v0[0] * 4, bp + (size_t)v0[1] * 4, bp + (size_t)v0[2] * 4};
        const T* c0 = color + pix0 * C; const T* g0 = grad_color + pix0 * C;
        T g[12] = {0};
        for (int e = 0; e < 4; ++e) {
            const int y1 = y0 + DY[e], x1 = x0 + DX[e];
            if (y1 < 0 || y1 >= H || x1 < 0 || x1 >= W) continue;
            const int64_t pix1 = (int64_t)b * H * W + (int64_t)y1 * W + x1;
            const T depth1 = (T)rast[pix1 * 4 + 2];
            const int it1 = (int)rast[pix1 * 4 + 3] - 1;
            const T* c1 = color + pix1 * C; const T* g1 = grad_color + pix1 * C;
            T adj = 0;
            for (int i = 0; i < C; ++i) adj += T(0.5) * (g0[i] + g1[i]) * (c0[i] - c1[i]);
            if (adj == T(0)) continue;
            const T gx = adj * T(DX[e]) * T(W) / T(2);
            const T gy = adj * T(DY[e]) * T(H) / T(2);
            const T nx1 = pix_ndc<T>(x1, W), ny1 = pix_ndc<T>(y1, H);
            const T mx = T(0.5) * (nx0 + nx1), my = T(0.5) * (ny0 + ny1);
            if (it1 == it0) { add_mid_contrib<T>(mx, my, P0, gx, gy, T(0), false, g, v); continue; }
            T cz1, cw1, tb0, tb1;
            const bool hit1 = intersect_triangle<T>(ny1, nx1, P0[0], P0[1], P0[2], tb0, tb1, cz1, cw1, v);
            if (hit1) {
                const T d1_it0 = cz1 / cw1;
                if (it1 >= 0 && depth1 < d1_it0) {
                    const int* v1 = tri + it1 * 3;
                    const T* P1[3] = {bp + (size_t)v1[0] * 4, bp + (size_t)v1[1] * 4, bp + (size_t)v1[2] * 4};
                    T cz0, cw0;
                    if (intersect_triangle<T>(ny0, nx0, P1[0], P1[1], P1[2], tb0, tb1, cz0, cw0, v)) {
                        const T d0_it1 = cz0 / cw0;
                        if (depth0 < d0_it1) {
                            T nv[3], nf[3];
                            if (tri_normal_ndc<T>(P0, nv) && tri_normal_ndc<T>(P1, nf)) {
                                T gxn = 0, gyn = 0, gzn = 0;
                                if (DX[e] != 0) { T dbx, dbz; db_dp_2d<T>(nv[0], nv[2], nf[0], nf[2], dbx, dbz); gxn = gx * dbx; gzn = gx * dbz; }
                                else { T dby, dbz; db_dp_2d<T>(nv[1], nv[2], nf[1], nf[2], dby, dbz); gyn = gy * dby; gzn = gy * dbz; }
                                add_mid_contrib<T>(mx, my, P0, gxn, gyn, gzn, true, g, v);
                            }
                        }
                    }
                } else if (it1 < 0 || depth0 < depth1) {
                    add_mid_contrib<T>(mx, my, P0, gx, gy, T(0), false, g, v);
                }
            } else if (it1 < 0 || depth0 < depth1) {
                int i0, i1; T s0, s1;
                if (find_edge_intersection<T>(P0, nx0, ny0, nx1, ny1, i0, i1, s0, s1)) {
                    const T cx = s0 * P0[i0][0] + s1 * P0[i1][0];
                    const T cy = s0 * P0[i0][1] + s1 * P0[i1][1];
                    const T cw = s0 * P0[i0][3] + s1 * P0[i1][3];
                    const T iw = T(1) / cw, iw2 = iw * iw;
                    const T gsum = gx * cx + gy * cy;
                    g[i0 * 4 + 0] += s0 * gx * iw; g[i1 * 4 + 0] += s1 * gx * iw;
                    g[i0 * 4 + 1] += s0 * gy * iw; g[i1 * 4 + 1] += s1 * gy * iw;
                    g[i0 * 4 + 3] += -s0 * gsum * iw2; g[i1 * 4 + 3] += -s1 * gsum * iw2;
                }
            }
        }
        double* gp = grad_pos + (size_t)b * V * 4;
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 4; ++j) atomic_add_d(&gp[(size_t)v0[k] * 4 + j], (double)g[k * 4 + j]);
    }
}

// Opacity auxiliary gradient per fragment: rasterize.cu:923-971.
template <typename T>
void aux_fragment_grad(int H, int W, int C, const T* color, const T* target, const float* rast,
                       int64_t nf, const int* frag_pix, const float* frag_attrs, const T* frag_alpha,
                       T* grad_frag_alpha) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nf; ++i) {
        const int b = frag_pix[i * 3];
        if (b < 0) continue;
        const int64_t p = (int64_t)b * H * W + (int64_t)frag_pix[i * 3 + 1] * W + frag_pix[i * 3 + 2];
        const float zf = frag_attrs[i * 4 + 2];
        const int tf = (int)frag_attrs[i * 4 + 3] - 1;
        const float zp = rast[p * 4 + 2];
        const int tp = (int)rast[p * 4 + 3] - 1;
        if (tp >= 0 && zf > zp) continue;
        T loss = 0;
        for (int c = 0; c < C; ++c) loss += std::fabs(color[p * C + c] - target[p * C + c]);
        const T eps = T(1e-5f);
        const T a = frag_alpha[i];
        if (tp >= 0 && tf == tp) grad_frag_alpha[i] += loss / std::max(a, eps);
        else grad_frag_alpha[i] -= loss / std::max(T(1) - a, eps);
    }
}
}  // namespace

extern "C" {

void orc_encode_view_f32(int B, int H, int W, const float* rast, const float* inv_mvp, float* enc, int sh) {
    encode_view<float>(B, H, W, rast, inv_mvp, enc, sh);
}
void orc_encode_view_f64(int B, int H, int W, const float* rast, const double* inv_mvp, double* enc, int sh) {
    encode_view<double>(B, H, W, rast, inv_mvp, enc, sh);
}

// grad_pos: double [B,V,4], zeroed by the caller.
void orc_edge_grad_f32(int variant, int B, int H, int W, int C, const float* color, const float* grad_color,
                       const float* rast, int V, const float* pos, const int* tri, double* grad_pos) {
    edge_grad<float>(B, H, W, C, color, grad_color, rast, V, pos, tri, grad_pos, variant);
}
void orc_edge_grad_f64(int B, int H, int W, int C, const double* color, const double* grad_color, const float* rast,
                       int V, const double* pos, const int* tri, double* grad_pos) {
    edge_grad<double>(B, H, W, C, color, grad_color, rast, V, pos, tri, grad_pos, 0);
}

void orc_aux_fragment_grad_f32(int H, int W, int C, const float* color, const float* target, const float* rast,
                               int64_t nf, const int* frag_pix, const float* frag_attrs, const float* frag_alpha,
                               float* grad_frag_alpha) {
    aux_fragment_grad<float>(H, W, C, color, target, rast, nf, frag_pix, frag_attrs, frag_alpha, grad_frag_alpha);
}

// Composite of _OpacityAuxLossFn.forward (rasterize.py:147-190): recompute the
// fragments, alpha, per-fragment aux gradient and its lattice adjoint.
// grad_alpha_src: double [T,S] zeroed by caller (unscaled, as in the reference
// before the 1/numel weight of rasterize.py:183-195).  Alpha and the per-
// fragment gradient are evaluated in T = double when f64 != 0.
void orc_opacity_aux(int variant, int f64, int B, int H, int W, int C, const void* color, const void* target,
                     const float* rast, int V, const float* pos, int T, const int* tri, int level,
                     const void* alpha_src, double* grad_alpha_src) {
    const uint32_t S = feats_at_level((uint32_t)level);
    for (int b = 0; b < B; ++b) {
        const float* P = pos + (size_t)b * V * 4;
        std::vector<int> rects((size_t)T * 4);
        std::vector<int64_t> prefix((size_t)T);
        const int64_t nbb = orc_triangle_rects(H, W, 1, V, P, T, tri, rects.data(), prefix.data());
        std::vector<int> fpix((size_t)nbb * 3, -1);
        std::vector<float> fattr((size_t)nbb * 4, 0.f);
        orc_fragments(variant, H, W, 1, V, P, T, tri, rects.data(), prefix.data(), fpix.data(), fattr.data());
        std::vector<int> cpix((size_t)nbb * 3);
        std::vector<float> cattr((size_t)nbb * 4);
        const int64_t nf = orc_filter_valid(nbb, fpix.data(), fattr.data(), cpix.data(), cattr.data());
        for (int64_t i = 0; i < nf; ++i) cpix[i * 3] = b;
        std::vector<double> gfa((size_t)nf, 0.0);
        if (f64) {
            const double* as = (const double*)alpha_src;
            std::vector<double> alpha((size_t)nf, 0.0), g((size_t)nf, 0.0);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < nf; ++i) {
                const int t = (int)cattr[i * 4 + 3] - 1;
                double a = 0.0;
                interp<double, double>(cattr[i * 4], cattr[i * 4 + 1], level, level, 1, as + (size_t)t * S, &a, 0);
                alpha[i] = a;
            }
            aux_fragment_grad<double>(H, W, C, (const double*)color, (const double*)target, rast, nf, cpix.data(),
                                      cattr.data(), alpha.data(), g.data());
            gfa = g;
        } else {
            std::vector<float> alpha((size_t)nf, 0.f), g((size_t)nf, 0.f);
            orc_multires_alpha(variant, nf, cattr.data(), level, level, (const float*)alpha_src, alpha.data());
            aux_fragment_grad<float>(H, W, C, (const float*)color, (const float*)target, rast, nf, cpix.data(),
                                     cattr.data(), alpha.data(), g.data());
            for (int64_t i = 0; i < nf; ++i) gfa[i] = g[i];
        }
        orc_multires_alpha_backward(nf, cattr.data(), level, level, T, grad_alpha_src, gfa.data());
    }
}

// Projection of the batched training step (examples/utils.py:412-426) with the
// fixed fused order of the product kernel: ((M[r][3] + M[r][0] x) + M[r][1] y)
// + M[r][2] z, each step one fma.
void orc_project_f32(int B, int V, const float* verts, const float* mvp, float* pos) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)B * V; ++i) {
        const int b = (int)(i / V), v = (int)(i % V);
        const float* M = mvp + (size_t)b * 16;
        const float x = verts[(size_t)v * 3], y = verts[(size_t)v * 3 + 1], z = verts[(size_t)v * 3 + 2];
        for (int r = 0; r < 4; ++r)
            pos[i * 4 + r] = std::fma(M[r * 4 + 2], z, std::fma(M[r * 4 + 1], y, std::fma(M[r * 4 + 0], x, M[r * 4 + 3])));
    }
}

// Level accumulation + sigmoid as the product's step computes it in FP32
// (accumulate_to_level then torch.sigmoid, examples/02_synthetic.py:355-356).
void orc_accumulate_sigmoid_f32(int T, int lo, int hi, int target, int C, const float* feat, float* out) {
    orc_accumulate_forward_f32(64 | 0, T, lo, hi, target, C, feat, out);
    const int64_t n = (int64_t)T * feats_at_level((uint32_t)target) * C;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = 1.f / (1.f + std::exp(-out[i]));
}

// Exposes the coverage test for contraction-variant pinning.
int orc_intersect(int variant, float ndc_y, float ndc_x, const float* p0, const float* p1, const float* p2,
                  float* out4) {
    float b0 = 0, b1 = 0, z = 0, w = 0;
    const bool hit = intersect_triangle<float>(ndc_y, ndc_x, p0, p1, p2, b0, b1, z, w, variant);
    out4[0] = b0; out4[1] = b1; out4[2] = z; out4[3] = w;
    return hit ? 1 : 0;
}

}  // extern "C"
