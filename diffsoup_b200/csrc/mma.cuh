// diffsoup_b200/csrc/mma.cuh -- warp-level BF16 tensor-core helpers for the
// per-pixel shading MLP (m16n8k16, FP32 accumulation).
//
// All operands are staged in shared memory as row-major bf16 tiles; ldmatrix
// (optionally .trans) turns them into fragments, so the same smem copy of a
// weight matrix serves both W (forward) and W^T (backward), and activation
// rows serve as K-major operands of the weight-gradient products.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace dsb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// D = A(16x16, row) * B(16x8, col) + D
__device__ __forceinline__ void mma_16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void ldsm_x4(uint32_t r[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t r[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x2(uint32_t r[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x2_t(uint32_t r[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p)));
}

// Fragment loaders.  `ld` is the row stride in bf16 elements.
// A (16 x 16) from a row-major [m][k] tile at (m0, k0).
__device__ __forceinline__ void load_a(uint32_t a[4], const __nv_bfloat16* s, int ld, int m0, int k0) {
    const int l = threadIdx.x & 31;
    ldsm_x4(a, s + (m0 + (l & 15)) * ld + k0 + (l >> 4) * 8);
}

// A (16 x 16) from a row-major [k][m] tile (A = tile^T) at (k0, m0).
__device__ __forceinline__ void load_a_t(uint32_t a[4], const __nv_bfloat16* s, int ld, int k0, int m0) {
    const int l = threadIdx.x & 31;
    const int mi = l >> 3, r = l & 7;
    ldsm_x4_t(a, s + (k0 + r + (mi >> 1) * 8) * ld + m0 + (mi & 1) * 8);
}

// B (16 x 8) from a row-major [n][k] tile (B[k][n] = tile[n][k]) at (n0, k0).
__device__ __forceinline__ void load_b(uint32_t b[2], const __nv_bfloat16* s, int ld, int n0, int k0) {
    const int l = threadIdx.x & 15;
    ldsm_x2(b, s + (n0 + (l & 7)) * ld + k0 + (l >> 3) * 8);
}

// B (16 x 8) from a row-major [k][n] tile at (k0, n0).
__device__ __forceinline__ void load_b_t(uint32_t b[2], const __nv_bfloat16* s, int ld, int k0, int n0) {
    const int l = threadIdx.x & 15;
    ldsm_x2_t(b, s + (k0 + (l & 7) + (l >> 3) * 8) * ld + n0);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

}  // namespace dsb
