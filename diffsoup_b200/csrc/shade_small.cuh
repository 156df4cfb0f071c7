// diffsoup_b200/csrc/shade_small.cuh -- the fused shading step for the
// small MLP (8 features + 3 view-direction inputs -> 16 -> 3), with the MLP's
// activations kept in tensor-core fragments.
//
// Same arithmetic as shade_step_kernel (shade.cuh) for ShadeCfg<8,16,16,1>:
// bf16 operands, fp32 accumulation, fp32 biases.  What changes is where the
// intermediate tiles live.  The m16n8k16 accumulator of two adjacent n-tiles
// has exactly the register layout of the A operand of the next product
// (rows g, g+8; columns 2q, 2q+1 and 2q+8, 2q+9), so the hidden activations
// H and their gradient dZ1 go from one mma to the next in registers, and
// movmatrix (an 8x8 transpose within the warp) turns them, and the input
// tile X, into the transposed operands of the weight-gradient products.
// Shared memory keeps only the per-pixel rows: X on its way in (one 16-byte
// store per half row, then ldmatrix), the output logits, and dX on its way
// to the feature scatter.  Weights, biases and the weight gradients of the
// whole kernel stay in registers.
#pragma once

#include "shade.cuh"

namespace dsb {

// 8x8 b16 transpose across the warp (fragment layout in, fragment layout out).
__device__ __forceinline__ uint32_t movmatrix_t(uint32_t x) {
    uint32_t y;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;\n" : "=r"(y) : "r"(x));
    return y;
}

struct ShadeSmallWarp {
    __align__(16) __nv_bfloat16 X[32 * 24];  // per-pixel input rows, 16 used (48-byte stride)
    float scr[32 * 17];                      // per-pixel fp32 rows: logits, then dX
};

#ifndef DSB_SHADE_SMALL_WARPS
#define DSB_SHADE_SMALL_WARPS 8
#endif
constexpr int kShadeSmallWarps = DSB_SHADE_SMALL_WARPS;

struct ShadeSmallSmem {
    float g[ShadeCfg<8, 16, 16, 1>::NPARAM];  // CTA gradient accumulators (packed like the parameters)
    float loss[kShadeSmallWarps];
    ShadeSmallWarp w[kShadeSmallWarps];
};

#ifndef DSB_SHADE_SMALL_MIN_CTAS
#define DSB_SHADE_SMALL_MIN_CTAS 2  // resident 8-warp CTAs per SM the register budget is sized for
#endif

__global__ void __launch_bounds__(kShadeSmallWarps * 32, DSB_SHADE_SMALL_MIN_CTAS) shade_small_kernel(ShadeArgs a) {
    using K = ShadeCfg<8, 16, 16, 1>;
    constexpr int IN = K::IN_REAL;  // 11
    __shared__ ShadeSmallSmem sm;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const float* P = a.params;
    auto w0 = [&](int h, int i) { return i < IN ? P[K::P_W0 + h * IN + i] : 0.f; };
    auto wo = [&](int o, int h) { return o < 3 ? P[K::P_WO + o * 16 + h] : 0.f; };

    // ---- weights as fragments --------------------------------------------
    // Z1 = X W0^T: B[k = in][n = hidden] per hidden n-tile nt
    uint32_t bW0[2][2], bW0T[2][2], bWo[2], bWoT[2];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        const int h = nt * 8 + g;
        bW0[nt][0] = pack_bf16(w0(h, 2 * q), w0(h, 2 * q + 1));
        bW0[nt][1] = pack_bf16(w0(h, 2 * q + 8), w0(h, 2 * q + 9));
        // dX = dZ1 W0: B[k = hidden][n = in] per input n-tile nt
        const int i = nt * 8 + g;
        bW0T[nt][0] = pack_bf16(w0(2 * q, i), w0(2 * q + 1, i));
        bW0T[nt][1] = pack_bf16(w0(2 * q + 8, i), w0(2 * q + 9, i));
        // dH = dZo Wo: B[k = out][n = hidden]; outputs 8..15 are padding
        bWoT[nt] = pack_bf16(wo(2 * q, h), wo(2 * q + 1, h));
    }
    // O = H Wo^T: B[k = hidden][n = out]
    bWo[0] = pack_bf16(wo(g, 2 * q), wo(g, 2 * q + 1));
    bWo[1] = pack_bf16(wo(g, 2 * q + 8), wo(g, 2 * q + 9));
    float bb0[2][2];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        bb0[nt][0] = P[K::P_B0 + nt * 8 + 2 * q];
        bb0[nt][1] = P[K::P_B0 + nt * 8 + 2 * q + 1];
    }
    const float bo0 = P[K::P_BO + 0], bo1 = P[K::P_BO + 1], bo2 = P[K::P_BO + 2];
    for (int i = threadIdx.x; i < K::NPARAM; i += blockDim.x) sm.g[i] = 0.f;

    // gradients of the whole kernel (accumulator layouts)
    float gw0[2][4], gwo[2][4], gb0[2][2], gbo[3] = {0.f, 0.f, 0.f}, loss_acc = 0.f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int k = 0; k < 4; ++k) gw0[i][k] = gwo[i][k] = 0.f;
        gb0[i][0] = gb0[i][1] = 0.f;
    }
    __syncthreads();

    ShadeSmallWarp& ws = sm.w[warp];
    const int64_t nchunks = (a.num_pixels + 31) / 32;
    const int64_t cstride = (int64_t)gridDim.x * kShadeSmallWarps;
    // the rast entry of the warp's next chunk is requested one chunk ahead
    float4 r_next = make_float4(0.f, 0.f, 0.f, 0.f);
    {
        const int64_t p0 = ((int64_t)blockIdx.x * kShadeSmallWarps + warp) * 32 + lane;
        if (p0 < a.num_pixels) r_next = reinterpret_cast<const float4*>(a.rast)[p0];
    }
    for (int64_t chunk = (int64_t)blockIdx.x * kShadeSmallWarps + warp; chunk < nchunks; chunk += cstride) {
        // ---------------- pixel front: gather features, view direction ----------
        const int64_t p = chunk * 32 + lane;
        const bool valid = p < a.num_pixels;
        const float4 r = r_next;
        {
            const int64_t pn = p + cstride * 32;
            r_next = make_float4(0.f, 0.f, 0.f, 0.f);
            if (pn < a.num_pixels) r_next = reinterpret_cast<const float4*>(a.rast)[pn];
        }
        float tgt[3] = {0.f, 0.f, 0.f};  // requested here, used after the MLP forward
        if (valid) {
#pragma unroll
            for (int c = 0; c < 3; ++c) tgt[c] = a.target[p * 3 + c];
        }
        const int t = (int)r.w - 1;
        const bool mask = valid && t >= 0;
        float x[IN];
#pragma unroll
        for (int c = 0; c < IN; ++c) x[c] = 0.f;
        uint32_t idx[3] = {0, 0, 0};
        float wgt[3] = {0.f, 0.f, 0.f};
        if (mask) {
            lattice_cell(r.x, r.y, (uint32_t)a.level, idx, wgt);
            const __nv_bfloat16* tf = a.feat + (size_t)t * a.S * 8;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const uint4 u = __ldg(reinterpret_cast<const uint4*>(tf + (size_t)idx[k] * 8));
                const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float2 f = __bfloat1622float2(h2[j]);
                    x[2 * j] = __fmaf_rn(wgt[k], f.x, x[2 * j]);
                    x[2 * j + 1] = __fmaf_rn(wgt[k], f.y, x[2 * j + 1]);
                }
            }
            const int b = view_of_pixel(a.views, a.B, p);
            const ds_view_desc vd = a.views[b];
            const int local = (int)(p - vd.pix_offset);  // < H*W < 2^31: 32-bit division
            const int py = local / vd.W, px = local - py * vd.W;
            float M[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) M[k] = __ldg(a.inv_mvp + (size_t)b * 16 + k);
            float d[3];
            view_direction(pix_ndc(px, vd.W), pix_ndc(py, vd.H), M, d);
            x[8] = d[0]; x[9] = d[1]; x[10] = d[2];
        }
        // a chunk without covered pixels has an all-background colour: no MLP, no gradients
        const bool any = __any_sync(0xffffffffu, mask);
        uint32_t aH[2][4];  // relu(X W0^T + b0) as bf16, A operand of the next products
        if (any) {
            {
                __nv_bfloat16* xr = ws.X + lane * 24;
                *reinterpret_cast<uint4*>(xr) = make_uint4(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]),
                                                           pack_bf16(x[4], x[5]), pack_bf16(x[6], x[7]));
                *reinterpret_cast<uint4*>(xr + 8) = make_uint4(pack_bf16(x[8], x[9]), pack_bf16(x[10], 0.f), 0u, 0u);
            }
            __syncwarp();

            // ---------------- MLP forward (activations in registers) ------------------
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                uint32_t aX[4];
                load_a(aX, ws.X, 24, mt * 16, 0);
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
                    mma_16816(acc, aX, bW0[nt]);
                    aH[mt][2 * nt] = pack_bf16(fmaxf(acc[0] + bb0[nt][0], 0.f), fmaxf(acc[1] + bb0[nt][1], 0.f));
                    aH[mt][2 * nt + 1] = pack_bf16(fmaxf(acc[2] + bb0[nt][0], 0.f), fmaxf(acc[3] + bb0[nt][1], 0.f));
                }
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                mma_16816(acc, aH[mt], bWo);
                if (q < 2) {  // logits of outputs 2q, 2q+1 for rows g, g+8
                    ws.scr[(mt * 16 + g) * 17 + 2 * q] = acc[0];
                    ws.scr[(mt * 16 + g) * 17 + 2 * q + 1] = acc[1];
                    ws.scr[(mt * 16 + g + 8) * 17 + 2 * q] = acc[2];
                    ws.scr[(mt * 16 + g + 8) * 17 + 2 * q + 1] = acc[3];
                }
            }
            __syncwarp();
        }

        // ---------------- blend, loss, dL/dcolour (lane = pixel) ------------------
        float dz[3] = {0.f, 0.f, 0.f};
        float dxd[4] = {0.f, 0.f, 0.f, 0.f};  // direct gradient of x[0..3] through the blend
        if (valid) {
            const float res = x[3];
            const float bo[3] = {bo0, bo1, bo2};
            float l1 = 0.f;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float s = mask ? 1.f / (1.f + expf(-(ws.scr[lane * 17 + c] + bo[c]))) : 0.f;
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
#pragma unroll
        for (int c = 0; c < 3; ++c) gbo[c] += dz[c];
        __syncwarp();  // scr is rewritten below
        if (!any) continue;

        // ---------------- MLP backward --------------------------------------------
        // dZo as an A operand: rows g, g+8 of each m-tile; outputs 2q, 2q+1 (q < 2)
        const uint32_t dz01 = pack_bf16(dz[0], dz[1]), dz2 = pack_bf16(dz[2], 0.f);
        uint32_t aDZo[2][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int src = mt * 16 + g + 8 * h;
                const uint32_t u01 = __shfl_sync(0xffffffffu, dz01, src);
                const uint32_t u2 = __shfl_sync(0xffffffffu, dz2, src);
                aDZo[mt][h] = q == 0 ? u01 : (q == 1 ? u2 : 0u);
            }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            uint32_t aX[4];  // reloaded: cheaper than keeping both m-tiles live
            load_a(aX, ws.X, 24, mt * 16, 0);
            // dZ1 = (dZo Wo) * relu'(H)
            uint32_t aD[4];
            const uint32_t aDZoF[4] = {aDZo[mt][0], aDZo[mt][1], 0u, 0u};
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                const uint32_t bf[2] = {bWoT[nt], 0u};
                mma_16816(acc, aDZoF, bf);
                const __nv_bfloat162 hlo = *reinterpret_cast<const __nv_bfloat162*>(&aH[mt][2 * nt]);
                const __nv_bfloat162 hhi = *reinterpret_cast<const __nv_bfloat162*>(&aH[mt][2 * nt + 1]);
                const float d0 = __low2float(hlo) > 0.f ? acc[0] : 0.f, d1 = __high2float(hlo) > 0.f ? acc[1] : 0.f;
                const float d2 = __low2float(hhi) > 0.f ? acc[2] : 0.f, d3 = __high2float(hhi) > 0.f ? acc[3] : 0.f;
                gb0[nt][0] += d0 + d2;
                gb0[nt][1] += d1 + d3;
                aD[2 * nt] = pack_bf16(d0, d1);
                aD[2 * nt + 1] = pack_bf16(d2, d3);
            }
            // dX = dZ1 W0 -> scr, for the feature scatter
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                mma_16816(acc, aD, bW0T[ni]);
                if (ni == 0) {  // inputs 0..7 are the features
                    ws.scr[(mt * 16 + g) * 17 + 2 * q] = acc[0];
                    ws.scr[(mt * 16 + g) * 17 + 2 * q + 1] = acc[1];
                    ws.scr[(mt * 16 + g + 8) * 17 + 2 * q] = acc[2];
                    ws.scr[(mt * 16 + g + 8) * 17 + 2 * q + 1] = acc[3];
                }
            }
            // dW0 += dZ1^T X: A = dZ1^T (hidden x pixels), B = X (pixels x inputs)
            {
                const uint32_t aT[4] = {movmatrix_t(aD[0]), movmatrix_t(aD[2]), movmatrix_t(aD[1]),
                                        movmatrix_t(aD[3])};
                const uint32_t bx0[2] = {movmatrix_t(aX[0]), movmatrix_t(aX[1])};
                const uint32_t bx1[2] = {movmatrix_t(aX[2]), movmatrix_t(aX[3])};
                mma_16816(gw0[0], aT, bx0);
                mma_16816(gw0[1], aT, bx1);
            }
            // dWo += dZo^T H: A = dZo^T (outputs x pixels), B = H (pixels x hidden)
            {
                const uint32_t aT[4] = {movmatrix_t(aDZo[mt][0]), 0u, movmatrix_t(aDZo[mt][1]), 0u};
                const uint32_t bh0[2] = {movmatrix_t(aH[mt][0]), movmatrix_t(aH[mt][1])};
                const uint32_t bh1[2] = {movmatrix_t(aH[mt][2]), movmatrix_t(aH[mt][3])};
                mma_16816(gwo[0], aT, bh0);
                mma_16816(gwo[1], aT, bh1);
            }
        }
        __syncwarp();

        // ---------------- feature-gradient scatter (lane = pixel) -------------------
        if (mask) {
            float dx[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) dx[c] = ws.scr[lane * 17 + c] + (c < 4 ? dxd[c] : 0.f);
            float* tg = a.grad_feat + (size_t)t * a.S * 8;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float* dst = tg + (size_t)idx[k] * 8;
#pragma unroll
                for (int c = 0; c < 8; c += 4)
                    atomicAdd(reinterpret_cast<float4*>(dst + c),
                              make_float4(wgt[k] * dx[c], wgt[k] * dx[c + 1], wgt[k] * dx[c + 2], wgt[k] * dx[c + 3]));
            }
        }
        __syncwarp();
    }

    // ---- the kernel's gradients into the CTA accumulators ----------------------
    // W0[h][i]: tile ni holds rows h = g (+8), columns i = ni*8 + 2q (+1)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni) {
        const int i0 = ni * 8 + 2 * q;
        if (i0 < IN) {
            atomicAdd(&sm.g[K::P_W0 + g * IN + i0], gw0[ni][0]);
            atomicAdd(&sm.g[K::P_W0 + (g + 8) * IN + i0], gw0[ni][2]);
        }
        if (i0 + 1 < IN) {
            atomicAdd(&sm.g[K::P_W0 + g * IN + i0 + 1], gw0[ni][1]);
            atomicAdd(&sm.g[K::P_W0 + (g + 8) * IN + i0 + 1], gw0[ni][3]);
        }
    }
    // Wo[o][h]: tile nt holds rows o = g (< 3 used), columns h = nt*8 + 2q (+1)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        if (g < 3) {
            atomicAdd(&sm.g[K::P_WO + g * 16 + nt * 8 + 2 * q], gwo[nt][0]);
            atomicAdd(&sm.g[K::P_WO + g * 16 + nt * 8 + 2 * q + 1], gwo[nt][1]);
        }
        float s0 = gb0[nt][0], s1 = gb0[nt][1];
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        }
        if (g == 0) {
            atomicAdd(&sm.g[K::P_B0 + nt * 8 + 2 * q], s0);
            atomicAdd(&sm.g[K::P_B0 + nt * 8 + 2 * q + 1], s1);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float v = gbo[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) atomicAdd(&sm.g[K::P_BO + c], v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o);
    if (lane == 0) sm.loss[warp] = loss_acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kShadeSmallWarps; ++w) s += sm.loss[w];
        atomicAdd(a.loss_sum, s);
    }
    for (int i = threadIdx.x; i < K::NPARAM; i += blockDim.x)
        if (sm.g[i] != 0.f) atomicAdd(a.grad_params + i, sm.g[i]);
}

}  // namespace dsb
