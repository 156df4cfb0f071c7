// diffsoup_b200/csrc/common.cuh -- shared definitions of the sm_100a kernels.
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

#include "diffsoup_b200.h"

namespace dsb {

constexpr int kThreads = 256;

// Streaming multiprocessors of the current device (cudaDevAttrMultiProcessorCount,
// queried once per device and cached; 148 on a B200).  Grids of persistent and
// grid-stride kernels are sized from it.
int sm_count();

// Upper bound on the resident warps of a grid of 256-thread CTAs on the
// current device: 2048 threads per SM.
inline int64_t max_resident_warps() { return (int64_t)sm_count() * 64; }

inline unsigned blocks_for(int64_t n, int threads = kThreads) {
    return (unsigned)((n + threads - 1) / threads);
}

// Records a message for ds_last_error() and returns `code`.
int set_error(int code, const char* fmt, ...);

// Checks the launch and converts a CUDA error into a DS status.
int check_launch(const char* what);

#define DS_CHECK_ARG(cond, ...)                                          \
    do {                                                                 \
        if (!(cond)) return ::dsb::set_error(DS_ERR_ARG, __VA_ARGS__);   \
    } while (0)

#define DS_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ::dsb::set_error(DS_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// View of a packed pixel index: the last view whose pix_offset <= p.
__device__ __forceinline__ int view_of_pixel(const ds_view_desc* __restrict__ views, int B, int64_t p) {
    int lo = 0, hi = B - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&views[mid].pix_offset) <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// FP32 arithmetic with the rounding of the reference's default nvcc build.
//
// nvcc contracts a*b+c into one FMA by default, and which products it fuses
// decides the last bit of every barycentric and depth value.  The pattern
// below reproduces the reference (pinned bit for bit against its own build on
// the golden fixtures); the explicit intrinsics stop nvcc from re-contracting
// this code differently.  DSB_FMA_REF=0 selects plain IEEE rounding of every
// operation instead (the reference built with -fmad=false).
// ---------------------------------------------------------------------------
#ifndef DSB_FMA_REF
#define DSB_FMA_REF 1
#endif

// a - b*c
__device__ __forceinline__ float sub_mul(float a, float b, float c) {
#if DSB_FMA_REF
    return __fmaf_rn(-b, c, a);
#else
    return __fsub_rn(a, __fmul_rn(b, c));
#endif
}

// a*b - c*d
__device__ __forceinline__ float cross2(float a, float b, float c, float d) {
#if DSB_FMA_REF
    return __fmaf_rn(a, b, -__fmul_rn(c, d));
#else
    return __fsub_rn(__fmul_rn(a, b), __fmul_rn(c, d));
#endif
}

// b0*z0 + b1*z1 + b2*z2 for the interpolated clip z
__device__ __forceinline__ float dot3_z(float b0, float x0, float b1, float x1, float b2, float x2) {
#if DSB_FMA_REF
    return __fmaf_rn(b2, x2, __fmaf_rn(b1, x1, __fmul_rn(b0, x0)));
#else
    return __fadd_rn(__fadd_rn(__fmul_rn(b0, x0), __fmul_rn(b1, x1)), __fmul_rn(b2, x2));
#endif
}

// b0*w0 + b1*w1 + b2*w2 for the interpolated clip w (nvcc fuses this sum in a
// different order than the z sum)
__device__ __forceinline__ float dot3_w(float b0, float x0, float b1, float x1, float b2, float x2) {
#if DSB_FMA_REF
    return __fmaf_rn(b2, x2, __fmaf_rn(b0, x0, __fmul_rn(b1, x1)));
#else
    return __fadd_rn(__fadd_rn(__fmul_rn(b0, x0), __fmul_rn(b1, x1)), __fmul_rn(b2, x2));
#endif
}

// acc + w*f
__device__ __forceinline__ float madd(float acc, float w, float f) {
#if DSB_FMA_REF
    return __fmaf_rn(w, f, acc);
#else
    return __fadd_rn(acc, __fmul_rn(w, f));
#endif
}

// Pixel-centre NDC coordinate, -1 + 2 (i + 0.5) / n (rasterize.cu:250-251).
__device__ __forceinline__ float pix_ndc(int i, int n) {
    return __fadd_rn(-1.f, __fdiv_rn(__fmul_rn(2.f, __fadd_rn((float)i, 0.5f)), (float)n));
}

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon et al., SC 2011), used as the counter-based RNG of
// the stochastic opacity threshold: counter = (pixel, tri, view, iteration),
// key = 64-bit seed.  uniform = (word0 >> 8) * 2^-24 in [0, 1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float philox_uniform(uint64_t seed, uint32_t iter, uint32_t view, uint32_t pixel,
                                                uint32_t tri) {
    uint32_t c0 = pixel, c1 = tri, c2 = view, c3 = iter;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return (float)(c0 >> 8) * (1.0f / 16777216.0f);
}

// The same draw split in two: with counter (pixel, tri, view, iter), the
// first two rounds touch the triangle only through one word of round 0, so
// the rest of them is done once per (view, pixel) by philox_pixel and the
// per-triangle remainder is one wide multiply and two XORs before rounds
// 2..9 (philox_uniform_tri(philox_pixel(...), ...) == philox_uniform(...)).
struct PhiloxPixel {
    uint32_t c0, c1, x2, u;  // round-2 words 0 and 1, the pixel's part of word 2, the view's part of round 0
};

__device__ __forceinline__ PhiloxPixel philox_pixel(uint64_t seed, uint32_t iter, uint32_t view, uint32_t pixel) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    PhiloxPixel pp;
    pp.u = __umulhi(0xCD9E8D57u, view) ^ k0;
    const uint32_t c2 = __umulhi(0xD2511F53u, pixel) ^ iter ^ k1;
    pp.c0 = __umulhi(0xCD9E8D57u, c2) ^ (0xCD9E8D57u * view) ^ (k0 + 0x9E3779B9u);
    pp.c1 = 0xCD9E8D57u * c2;
    pp.x2 = (0xD2511F53u * pixel) ^ (k1 + 0xBB67AE85u);
    return pp;
}

__device__ __forceinline__ float philox_uniform_tri(const PhiloxPixel& pp, uint64_t seed, uint32_t tri) {
    const uint32_t w = pp.u ^ tri;
    uint32_t c0 = pp.c0, c1 = pp.c1, c2 = __umulhi(0xD2511F53u, w) ^ pp.x2, c3 = 0xD2511F53u * w;
    uint32_t k0 = (uint32_t)seed + 2u * 0x9E3779B9u, k1 = (uint32_t)(seed >> 32) + 2u * 0xBB67AE85u;
#pragma unroll
    for (int r = 2; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return (float)(c0 >> 8) * (1.0f / 16777216.0f);
}

// Packed depth key of rasterize.cu:308-312: float bits of (z + 2) above a
// 32-bit tie-break (fragment order, i.e. triangle index within a view).
__device__ __forceinline__ unsigned long long depth_key(float z, uint32_t tie) {
    return ((unsigned long long)__float_as_uint(__fadd_rn(z, 2.f)) << 32) | tie;
}

}  // namespace dsb
