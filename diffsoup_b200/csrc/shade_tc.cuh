// diffsoup_b200/csrc/shade_tc.cuh -- the fused shading step for the wide
// shading MLP (16 features + 3-D view direction -> 64 -> 64 -> 3, BF16
// operands) on the 5th-generation tensor cores: tcgen05.mma with operands in
// shared memory and accumulators in tensor memory (TMEM).
//
// Same pixel arithmetic as shade_step_kernel<ShadeCfg<16,32,64,2>> (shade.cuh):
// feature gather (multires.cu:224-247), view direction (encoding.cu:28-53),
// ColorMLP (multires.py:171-207) with the residual blend, MSE loss, MLP
// backward and the feature scatter (multires.cu:268-292).  Organisation:
//
//   * a CTA of 128 threads shades tiles of 128 consecutive pixels; thread i
//     owns pixel row i of the tile, which is also TMEM lane i, so every
//     epilogue (bias, ReLU, blend, gate) reads its own accumulator row with
//     tcgen05.ld and writes its own operand row to shared memory;
//   * one thread issues the MMAs of a stage and commits them to an mbarrier;
//     the CTA waits (bounded), runs the epilogue, fences the shared-memory
//     writes to the async proxy and syncs before the next stage;
//   * operand tiles are stored pixel-major in 8x8 core matrices with no
//     swizzle: (column / 8) * 2048 + (pixel / 8) * 128 + (pixel % 8) * 16 +
//     (column % 8) * 2 bytes.  Read as a K-major operand (pixels as M, columns
//     as K) the core matrices are 2048 bytes apart along K and 128 along M;
//     read as an MN-major operand (columns as M or N, pixels as K) the same
//     bytes serve the transposed matrix, 128 apart along K and 2048 along
//     M/N -- so each tile feeds both its forward product and the
//     weight-gradient product that needs its transpose;
//   * the weight gradients accumulate in TMEM across all tiles of the CTA
//     (enable_input_d), with the pixel count as K: gW0 = dZ1^T [X | 1],
//     gW1^T = [H1 | 1]^T dZ2 and gWo^T = [H2 | 1]^T dZo, where the column of
//     ones (input 19, hidden column 64) gives the bias gradients in the same
//     products.  M is 128 in every product; rows past the real ones (hidden
//     64..127, augmented columns 80..127) read shared memory that stays zero.
//     They are read back once, at the end of the kernel.
//
// TMEM (256 columns per CTA, two CTAs per SM): R1 = columns 0-63 (Z1, then
// the logits, then dH1), R2 = 64-127 (Z2, then dH2, then dX), G0 = 128-159,
// G1 = 160-223, Go = 224-239.
#pragma once

#include "shade.cuh"

namespace dsb {
namespace tc {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle: start address, the byte
// distance between core matrices adjacent along K (leading) and along M/N
// (stride); bits 46-47 hold the descriptor version (1).
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t k_stride, uint32_t mn_stride) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((k_stride >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((mn_stride >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D fp32, A and B bf16, M = 128, N,
// A / B MN-major (transposed) when a_mn / b_mn.
__host__ __device__ constexpr uint32_t idesc(int n, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// Bounded wait for the mbarrier phase; false when it gave up.
__device__ __forceinline__ bool wait(uint32_t mbar, uint32_t phase) {
    uint32_t done = 0;
    for (int it = 0; it < (1 << 20) && !done; ++it) {
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
    }
    return done != 0;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive fp32 columns of the calling thread's lane.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of (row, col) in a pixel-major operand tile of 128 rows.
__host__ __device__ constexpr uint32_t tile_off(int row, int col) {
    return (uint32_t)((col >> 3) * 2048 + (row >> 3) * 128 + (row & 7) * 16 + (col & 7) * 2);
}

// Byte offset of (n, k) in a K-major weight tile of N rows.
__host__ __device__ constexpr uint32_t wtile_off(int N, int n, int k) {
    return (uint32_t)((k >> 3) * (N * 16) + (n >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
}

}  // namespace tc

constexpr int kTcThreads = 128;
constexpr int kTcCols = 256;  // TMEM columns per CTA

// Shared memory of shade_tc_kernel (dynamic; 1024-byte aligned base).
struct __align__(1024) TcSmem {
    unsigned char X[8192];      // [X | 1]: 128 x 32 (input 19 = 1 on covered pixels)
    unsigned char RA[32768];    // [H1 | 1] (128 x 80, columns up to 127 zero), then dZ1 (128 x 64, rest zero)
    unsigned char RB[32768];    // [H2 | 1], then dZ2
    unsigned char DZO[4096];    // dL/dlogits, 128 x 16 (outputs 3..15 zero)
    unsigned char W0[4096];     // B of Z1 = X W0^T: [64 x 32]
    unsigned char W1[8192];     // B of Z2 = H1 W1^T: [64 x 64]
    unsigned char WO[2048];     // B of logits = H2 Wo^T: [16 x 64]
    unsigned char WOT[2048];    // B of dH2 = dZo Wo: [64 x 16]
    unsigned char W1T[8192];    // B of dH1 = dZ2 W1: [64 x 64]
    unsigned char W0T[4096];    // B of dX = dZ1 W0: [32 x 64]
    float b0[64], b1[64], bo[4];
    float loss[kTcThreads / 32];
    unsigned long long mbar;
    uint32_t tmem;
};

__global__ void __launch_bounds__(kTcThreads, 2) shade_tc_kernel(ShadeArgs a) {
    using K = ShadeCfg<16, 32, 64, 2>;
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const float* P = a.params;

    // ---- set-up: zero the operand tiles, weights as bf16 tiles, TMEM, mbarrier --
    for (int i = tid; i < (int)(offsetof(TcSmem, W0) / 16); i += kTcThreads)
        reinterpret_cast<uint4*>(&sm)[i] = make_uint4(0u, 0u, 0u, 0u);
    auto put_w = [&](unsigned char* base, int N, int n, int k, float v) {
        *reinterpret_cast<__nv_bfloat16*>(base + tc::wtile_off(N, n, k)) = __float2bfloat16_rn(v);
    };
    for (int i = tid; i < 64 * 32; i += kTcThreads) {  // W0 [h][in], W0T [in][h]
        const int h = i / 32, in = i % 32;
        const float v = in < K::IN_REAL ? P[K::P_W0 + h * K::IN_REAL + in] : 0.f;
        put_w(sm.W0, 64, h, in, v);
        put_w(sm.W0T, 32, in, h, v);
    }
    for (int i = tid; i < 64 * 64; i += kTcThreads) {  // W1 [o][i], W1T [i][o]
        const int o = i / 64, in = i % 64;
        const float v = P[K::P_WH + o * 64 + in];
        put_w(sm.W1, 64, o, in, v);
        put_w(sm.W1T, 64, in, o, v);
    }
    for (int i = tid; i < 16 * 64; i += kTcThreads) {  // WO [o][h], WOT [h][o]
        const int o = i / 64, h = i % 64;
        const float v = o < 3 ? P[K::P_WO + o * 64 + h] : 0.f;
        put_w(sm.WO, 16, o, h, v);
        put_w(sm.WOT, 64, h, o, v);
    }
    for (int i = tid; i < 64; i += kTcThreads) {
        sm.b0[i] = P[K::P_B0 + i];
        sm.b1[i] = P[K::P_WH + 64 * 64 + i];
    }
    if (tid < 4) sm.bo[tid] = tid < 3 ? P[K::P_BO + tid] : 0.f;
    if (warp == 0) {
        static_assert(kTcCols == 256, "the allocation below names 256 columns");
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(tc::saddr(&sm.tmem))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::saddr(&sm.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::proxy_fence();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = sm.tmem;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's lanes
    const uint32_t R1 = tmem, R2 = tmem + 64, G0 = tmem + 128, G1 = tmem + 160, GO = tmem + 224;  // lane 0
    const uint32_t mbar = tc::saddr(&sm.mbar);
    const uint32_t sX = tc::saddr(sm.X), sA = tc::saddr(sm.RA), sB = tc::saddr(sm.RB), sZ = tc::saddr(sm.DZO);
    const uint32_t sW0 = tc::saddr(sm.W0), sW1 = tc::saddr(sm.W1), sWO = tc::saddr(sm.WO);
    const uint32_t sWOT = tc::saddr(sm.WOT), sW1T = tc::saddr(sm.W1T), sW0T = tc::saddr(sm.W0T);
    uint32_t phase = 0;
    bool g_started = false, failed = false;
    float loss_acc = 0.f;

    // one stage: the CTA syncs (operand rows visible to the async proxy),
    // thread 0 issues `issue`, commits, and every thread waits for it
    auto stage = [&](auto issue) -> bool {
        tc::proxy_fence();
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        if (tid == 0) {
            issue();
            tc::commit(mbar);
        }
        const bool ok = tc::wait(mbar, phase);
        phase ^= 1u;
        tc::fence_after();
        return __syncthreads_and(ok) != 0;
    };
    auto st_row16 = [&](unsigned char* base, int chunk, const uint32_t (&u)[4]) {
        *reinterpret_cast<uint4*>(base + tc::tile_off(tid, chunk * 8)) = make_uint4(u[0], u[1], u[2], u[3]);
    };

    const int64_t ntiles = (a.num_pixels + kTcThreads - 1) / kTcThreads;
    // ---- the pixel front, one tile ahead: the next tile's rast entry is requested before this tile's
    // first product, its feature samples and target after that product (their latency hides behind
    // the remaining products), and they are interpolated when this tile is done ---------------------
    auto issue_rast = [&](int64_t tl, float4& r) {
        const int64_t q = tl * kTcThreads + tid;
        r = make_float4(0.f, 0.f, 0.f, 0.f);
        if (tl < ntiles && q < a.num_pixels) r = reinterpret_cast<const float4*>(a.rast)[q];
    };
    auto issue_feat = [&](int64_t tl, const float4& r, uint4 (&u)[3][2], uint32_t (&ix)[3], float (&wg)[3],
                          float (&tg)[3]) {
        const int64_t q = tl * kTcThreads + tid;
        const bool ok = tl < ntiles && q < a.num_pixels;
        const int tt = (int)r.w - 1;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ix[k] = 0u; wg[k] = 0.f; tg[k] = 0.f;
            u[k][0] = u[k][1] = make_uint4(0u, 0u, 0u, 0u);
        }
        if (ok && tt >= 0) {
            lattice_cell(r.x, r.y, (uint32_t)a.level, ix, wg);
            const __nv_bfloat16* tf = a.feat + (size_t)tt * a.S * 16;
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    u[k][h] = __ldg(reinterpret_cast<const uint4*>(tf + (size_t)ix[k] * 16 + 8 * h));
        }
        if (ok) {
#pragma unroll
            for (int c = 0; c < 3; ++c) tg[c] = target_at(a, q, c);
        }
    };
    float4 r_cur;
    uint4 u_cur[3][2];
    uint32_t ix_cur[3];
    float wg_cur[3], tg_cur[3];
    issue_rast(blockIdx.x, r_cur);
    issue_feat(blockIdx.x, r_cur, u_cur, ix_cur, wg_cur, tg_cur);
    for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
        // ---------------- pixel front: interpolated features, view direction ----------
        const int64_t p = tile * kTcThreads + tid;
        const bool valid = p < a.num_pixels;
        const float4 r = r_cur;
        const int t = (int)r.w - 1;
        const bool mask = valid && t >= 0;
        float x[K::IN_REAL];
#pragma unroll
        for (int c = 0; c < K::IN_REAL; ++c) x[c] = 0.f;
        uint32_t idx[3];
        float wgt[3], tgt[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) { idx[k] = ix_cur[k]; wgt[k] = wg_cur[k]; tgt[k] = tg_cur[k]; }
        if (mask) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint4 u = u_cur[k][h];
                    const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 f = __bfloat1622float2(h2[j]);
                        x[8 * h + 2 * j] = __fmaf_rn(wgt[k], f.x, x[8 * h + 2 * j]);
                        x[8 * h + 2 * j + 1] = __fmaf_rn(wgt[k], f.y, x[8 * h + 2 * j + 1]);
                    }
                }
            }
            const int b = view_of_pixel(a.views, a.B, p);
            const ds_view_desc vd = a.views[b];
            const int local = (int)(p - vd.pix_offset);
            const int py = local / vd.W, px = local - py * vd.W;
            float M[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) M[k] = __ldg(a.inv_mvp + (size_t)b * 16 + k);
            float d[3];
            view_direction(pix_ndc(px, vd.W), pix_ndc(py, vd.H), M, d);
            x[16] = d[0]; x[17] = d[1]; x[18] = d[2];
        }
        const int64_t next = tile + gridDim.x;
        float4 r_next;
        issue_rast(next, r_next);
        if (!__syncthreads_or(mask)) {  // no covered pixel in the tile: background colour 1, no MLP and no gradients
            if (valid) {
                float l1 = 0.f;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float diff = 1.f - tgt[c];
                    loss_acc += diff * diff;
                    a.color[p * 3 + c] = 1.f;
                    a.grad_color[p * 3 + c] = 2.f * diff * a.inv_n;
                    l1 += fabsf(diff);
                }
                a.l1[p] = l1;
            }
            r_cur = r_next;
            issue_feat(next, r_cur, u_cur, ix_cur, wg_cur, tg_cur);
            continue;
        }
        {  // [X | 1] row
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) {
                uint32_t u[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c0 = ch * 8 + 2 * j;
                    const float v0 = c0 < 19 ? x[c0 < 19 ? c0 : 0] : (c0 == 19 && mask ? 1.f : 0.f);
                    const float v1 = c0 + 1 < 19 ? x[c0 + 1 < 19 ? c0 + 1 : 0] : (c0 + 1 == 19 && mask ? 1.f : 0.f);
                    u[j] = pack_bf16(v0, v1);
                }
                st_row16(sm.X, ch, u);
            }
        }
        // ---------------- forward ---------------------------------------------------
        // Z1 = X W0^T -> R1
        if (!stage([&] {
                for (int ks = 0; ks < 2; ++ks)
                    tc::mma(R1, tc::desc(sX + ks * 4096, 2048, 128), tc::desc(sW0 + ks * 2048, 1024, 128),
                            tc::idesc(64, 0, 0), ks > 0);
            })) { failed = true; break; }
        // [H1 | 1] = [relu(Z1 + b0) | 1]
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            float v[16];
            tc::ld16(lane_base + q4 * 16, v);
            tc::wait_ld();
            uint32_t u0[4], u1[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                u0[j] = pack_bf16(fmaxf(v[2 * j] + sm.b0[q4 * 16 + 2 * j], 0.f),
                                  fmaxf(v[2 * j + 1] + sm.b0[q4 * 16 + 2 * j + 1], 0.f));
                u1[j] = pack_bf16(fmaxf(v[8 + 2 * j] + sm.b0[q4 * 16 + 8 + 2 * j], 0.f),
                                  fmaxf(v[8 + 2 * j + 1] + sm.b0[q4 * 16 + 8 + 2 * j + 1], 0.f));
            }
            st_row16(sm.RA, 2 * q4, u0);
            st_row16(sm.RA, 2 * q4 + 1, u1);
        }
        {
            const uint32_t one[4] = {pack_bf16(mask ? 1.f : 0.f, 0.f), 0u, 0u, 0u}, zero[4] = {0u, 0u, 0u, 0u};
            st_row16(sm.RA, 8, one);
            st_row16(sm.RA, 9, zero);
        }
        r_cur = r_next;
        issue_feat(next, r_cur, u_cur, ix_cur, wg_cur, tg_cur);  // the next tile's samples, in flight from here
        // Z2 = H1 W1^T -> R2
        if (!stage([&] {
                for (int ks = 0; ks < 4; ++ks)
                    tc::mma(R2, tc::desc(sA + ks * 4096, 2048, 128), tc::desc(sW1 + ks * 2048, 1024, 128),
                            tc::idesc(64, 0, 0), ks > 0);
            })) { failed = true; break; }
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            float v[16];
            tc::ld16(lane_base + 64 + q4 * 16, v);
            tc::wait_ld();
            uint32_t u0[4], u1[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                u0[j] = pack_bf16(fmaxf(v[2 * j] + sm.b1[q4 * 16 + 2 * j], 0.f),
                                  fmaxf(v[2 * j + 1] + sm.b1[q4 * 16 + 2 * j + 1], 0.f));
                u1[j] = pack_bf16(fmaxf(v[8 + 2 * j] + sm.b1[q4 * 16 + 8 + 2 * j], 0.f),
                                  fmaxf(v[8 + 2 * j + 1] + sm.b1[q4 * 16 + 8 + 2 * j + 1], 0.f));
            }
            st_row16(sm.RB, 2 * q4, u0);
            st_row16(sm.RB, 2 * q4 + 1, u1);
        }
        {
            const uint32_t one[4] = {pack_bf16(mask ? 1.f : 0.f, 0.f), 0u, 0u, 0u}, zero[4] = {0u, 0u, 0u, 0u};
            st_row16(sm.RB, 8, one);
            st_row16(sm.RB, 9, zero);
        }
        // logits = H2 Wo^T -> R1 columns 0..15
        if (!stage([&] {
                for (int ks = 0; ks < 4; ++ks)
                    tc::mma(R1, tc::desc(sB + ks * 4096, 2048, 128), tc::desc(sWO + ks * 512, 256, 128),
                            tc::idesc(16, 0, 0), ks > 0);
            })) { failed = true; break; }
        // ---------------- blend, loss, dL/dcolour --------------------------------------
        float dz[3] = {0.f, 0.f, 0.f}, dxd[4] = {0.f, 0.f, 0.f, 0.f};
        {
            float v[16];
            tc::ld16(lane_base, v);
            tc::wait_ld();
            if (valid) {
                const float res = x[3];
                float l1 = 0.f;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float s = mask ? 1.f / (1.f + expf(-(v[c] + sm.bo[c]))) : 0.f;
                    const float col = mask ? (1.f - res) * x[c] + res * s : 1.f;
                    const float diff = col - tgt[c];
                    loss_acc += diff * diff;
                    const float gc = 2.f * diff * a.inv_n;
                    a.color[p * 3 + c] = col;
                    a.grad_color[p * 3 + c] = gc;
                    l1 += fabsf(diff);
                    if (mask) {
                        dxd[c] = (1.f - res) * gc;
                        dxd[3] += (s - x[c]) * gc;
                        dz[c] = res * gc * s * (1.f - s);
                    }
                }
                a.l1[p] = l1;
            }
            const uint32_t u[4] = {pack_bf16(dz[0], dz[1]), pack_bf16(dz[2], 0.f), 0u, 0u};
            const uint32_t zero[4] = {0u, 0u, 0u, 0u};
            st_row16(sm.DZO, 0, u);
            st_row16(sm.DZO, 1, zero);
        }
        // ---------------- backward ---------------------------------------------------
        // dH2 = dZo Wo -> R2;  gWo^T += [H2 | 1]^T dZo -> Go
        const uint32_t gacc = g_started ? 1u : 0u;
        if (!stage([&] {
                tc::mma(R2, tc::desc(sZ, 2048, 128), tc::desc(sWOT, 1024, 128), tc::idesc(64, 0, 0), 0u);
                for (int ks = 0; ks < 8; ++ks)
                    tc::mma(GO, tc::desc(sB + ks * 256, 128, 2048), tc::desc(sZ + ks * 256, 128, 2048),
                            tc::idesc(16, 1, 1), ks > 0 ? 1u : gacc);
            })) { failed = true; break; }
        // dZ2 = dH2 * relu'(H2) -> RB (H2 has been read by the products above)
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            float v[16];
            tc::ld16(lane_base + 64 + q4 * 16, v);
            tc::wait_ld();
#pragma unroll
            for (int hf = 0; hf < 2; ++hf) {
                const int ch = 2 * q4 + hf;
                const uint4 hv = *reinterpret_cast<const uint4*>(sm.RB + tc::tile_off(tid, ch * 8));
                const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
                uint32_t u[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const __nv_bfloat162 h2 = *reinterpret_cast<const __nv_bfloat162*>(&hw[j]);
                    u[j] = pack_bf16(__low2float(h2) > 0.f ? v[8 * hf + 2 * j] : 0.f,
                                     __high2float(h2) > 0.f ? v[8 * hf + 2 * j + 1] : 0.f);
                }
                st_row16(sm.RB, ch, u);
            }
        }
        // dH1 = dZ2 W1 -> R1;  gW1^T += [H1 | 1]^T dZ2 -> G1
        if (!stage([&] {
                for (int ks = 0; ks < 4; ++ks)
                    tc::mma(R1, tc::desc(sB + ks * 4096, 2048, 128), tc::desc(sW1T + ks * 2048, 1024, 128),
                            tc::idesc(64, 0, 0), ks > 0);
                for (int ks = 0; ks < 8; ++ks)
                    tc::mma(G1, tc::desc(sA + ks * 256, 128, 2048), tc::desc(sB + ks * 256, 128, 2048),
                            tc::idesc(64, 1, 1), ks > 0 ? 1u : gacc);
            })) { failed = true; break; }
        // dZ1 = dH1 * relu'(H1) -> RA (columns 64..79 cleared: the transposed read wants zero rows there)
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            float v[16];
            tc::ld16(lane_base + q4 * 16, v);
            tc::wait_ld();
#pragma unroll
            for (int hf = 0; hf < 2; ++hf) {
                const int ch = 2 * q4 + hf;
                const uint4 hv = *reinterpret_cast<const uint4*>(sm.RA + tc::tile_off(tid, ch * 8));
                const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
                uint32_t u[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const __nv_bfloat162 h2 = *reinterpret_cast<const __nv_bfloat162*>(&hw[j]);
                    u[j] = pack_bf16(__low2float(h2) > 0.f ? v[8 * hf + 2 * j] : 0.f,
                                     __high2float(h2) > 0.f ? v[8 * hf + 2 * j + 1] : 0.f);
                }
                st_row16(sm.RA, ch, u);
            }
        }
        {
            const uint32_t zero[4] = {0u, 0u, 0u, 0u};
            st_row16(sm.RA, 8, zero);
            st_row16(sm.RA, 9, zero);
        }
        // dX = dZ1 W0 -> R2 columns 0..31;  gW0 += dZ1^T [X | 1] -> G0
        if (!stage([&] {
                for (int ks = 0; ks < 4; ++ks)
                    tc::mma(R2, tc::desc(sA + ks * 4096, 2048, 128), tc::desc(sW0T + ks * 1024, 512, 128),
                            tc::idesc(32, 0, 0), ks > 0);
                for (int ks = 0; ks < 8; ++ks)
                    tc::mma(G0, tc::desc(sA + ks * 256, 128, 2048), tc::desc(sX + ks * 256, 128, 2048),
                            tc::idesc(32, 1, 1), ks > 0 ? 1u : gacc);
            })) { failed = true; break; }
        g_started = true;
        // ---------------- feature-gradient scatter -------------------------------------
        {
            float v[16];
            tc::ld16(lane_base + 64, v);
            tc::wait_ld();
            if (mask) {
                float dx[16];
#pragma unroll
                for (int c = 0; c < 16; ++c) dx[c] = v[c] + (c < 4 ? dxd[c] : 0.f);
                float* tg = a.grad_feat + (size_t)t * a.S * 16;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    float* dst = tg + (size_t)idx[k] * 16;
#pragma unroll
                    for (int c = 0; c < 16; c += 4)
                        atomicAdd(reinterpret_cast<float4*>(dst + c), make_float4(wgt[k] * dx[c], wgt[k] * dx[c + 1],
                                                                                  wgt[k] * dx[c + 2],
                                                                                  wgt[k] * dx[c + 3]));
                }
            }
        }
    }

    // ---- the CTA's weight gradients from TMEM ---------------------------------------
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (failed) {
        if (tid == 0 && a.status) atomicOr(a.status, DS_STATUS_MMA_TIMEOUT);
    } else if (g_started) {
        float* gp = a.grad_params;
        // G0: row h (hidden), columns: inputs 0..18, 19 = bias
#pragma unroll
        for (int q2 = 0; q2 < 2; ++q2) {
            float v[16];
            tc::ld16(lane_base + 128 + q2 * 16, v);
            tc::wait_ld();
            if (tid < 64) {
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int in = q2 * 16 + c;
                    if (in < 19) atomicAdd(gp + K::P_W0 + tid * 19 + in, v[c]);
                    else if (in == 19) atomicAdd(gp + K::P_B0 + tid, v[c]);
                }
            }
        }
        // G1: row i (hidden-1 unit, 64 = bias), column o (hidden-2 unit): gW1[o][i]
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            float v[16];
            tc::ld16(lane_base + 160 + q4 * 16, v);
            tc::wait_ld();
            if (tid <= 64) {
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int o = q4 * 16 + c;
                    atomicAdd(gp + (tid < 64 ? K::P_WH + o * 64 + tid : K::P_WH + 64 * 64 + o), v[c]);
                }
            }
        }
        // Go: row h (hidden-2 unit, 64 = bias), columns o = 0..2: gWo[o][h]
        {
            float v[16];
            tc::ld16(lane_base + 224, v);
            tc::wait_ld();
            if (tid <= 64) {
#pragma unroll
                for (int o = 0; o < 3; ++o) atomicAdd(gp + (tid < 64 ? K::P_WO + o * 64 + tid : K::P_BO + o), v[o]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o);
    if ((tid & 31) == 0) sm.loss[warp] = loss_acc;
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < kTcThreads / 32; ++w) s += sm.loss[w];
        atomicAdd(a.loss_sum, s);
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem) : "memory");
}

}  // namespace dsb
