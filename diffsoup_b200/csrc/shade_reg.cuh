// diffsoup_b200/csrc/shade_reg.cuh -- the fused shading step for shading MLPs
// of width 16 (ColorMLP with hidden_dim 16, n_layers 1 or 2, at most 16
// inputs: C features + a 3-D view direction or its 9 SH2 coefficients), with
// the MLP's activations kept in tensor-core fragments.
//
// Same pixel arithmetic as shade_step_kernel (shade.cuh): feature gather
// (multires.cu:224-247), view encoding (encoding.cu:28-118), ColorMLP
// (multires.py:171-207) with the residual blend, MSE loss, MLP backward and
// the feature scatter (multires.cu:268-292).  What differs is where the
// intermediate tiles live.  The m16n8k16 accumulator of two adjacent n-tiles
// has exactly the register layout of the A operand of the next product
// (rows g, g+8; columns 2q, 2q+1 and 2q+8, 2q+9), so hidden activations and
// their gradients pass from one mma to the next in registers, and movmatrix
// (an 8x8 transpose within the warp) turns them, and the input tile X, into
// the transposed operands of the weight-gradient products.  Shared memory
// keeps only the per-pixel rows: X on its way in (one 16-byte store per half
// row, then ldmatrix), the output logits, and dX on its way to the feature
// scatter.  The weights live in registers as fragments (or, for the wider
// variants, in a per-CTA fragment table in shared memory), and the weight
// gradients of the whole kernel accumulate in fragments.
//
// SPLIT: every MLP operand is carried as two bf16 planes, hi = bf16(v) and
// lo = bf16(v - hi), features are gathered from the fp32 table, and each
// product is hi*hi + hi*lo + lo*hi on the BF16 tensor cores with fp32
// accumulation (the precision mode whose gradients agree with the FP64
// oracle to ~1e-5).
#pragma once

#include "shade.cuh"

namespace dsb {

// 8x8 b16 transpose across the warp (fragment layout in, fragment layout out).
__device__ __forceinline__ uint32_t movmatrix_t(uint32_t x) {
    uint32_t y;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;\n" : "=r"(y) : "r"(x));
    return y;
}

#ifndef DSB_SHADE_REG_WARPS
#define DSB_SHADE_REG_WARPS 8
#endif
constexpr int kShadeRegWarps = DSB_SHADE_REG_WARPS;

// C_ features (4..8; the first four feed the residual blend), ENC_ = 3 (view
// direction) or 9 (SH2), NL_ hidden layers of 16.
template <int C_, int ENC_, int NL_, bool SPLIT_>
struct RegCfg {
    static constexpr int C = C_, ENC = ENC_, NL = NL_, HID = 16, OUT = 3;
    static constexpr int IN = C_ + ENC_;
    static constexpr int CP = 8;  // channel stride of the gathered feature tables
    static constexpr bool SPLIT = SPLIT_;
    static constexpr int NS = SPLIT_ ? 2 : 1;
    // packed fp32 parameters (ColorMLP order): W0[16][IN] b0[16] (W1[16][16] b1[16]) Wo[3][16] bo[3]
    static constexpr int P_W0 = 0;
    static constexpr int P_B0 = HID * IN;
    static constexpr int P_W1 = P_B0 + HID;
    static constexpr int P_B1 = P_W1 + HID * HID;
    static constexpr int P_WO = P_B0 + HID + (NL_ - 1) * (HID * HID + HID);
    static constexpr int P_BO = P_WO + OUT * HID;
    static constexpr int NPARAM = P_BO + OUT;
    // weight fragments held in registers for the whole kernel (else read from
    // the CTA's fragment table at each use)
    static constexpr bool WREG = !SPLIT_ && NL_ == 1;
    // resident 8-warp CTAs per SM the register budget is sized for
    static constexpr int MIN_CTAS = 2;
    static_assert(C_ >= 4 && C_ <= 8 && IN <= 16 && (ENC_ == 3 || ENC_ == 9) && (NL_ == 1 || NL_ == 2),
                  "register-resident shading MLP shape");
};

// The weight fragments of one lane, per bf16 plane.
template <class K>
struct RegWeights {
    uint32_t w0[K::NS][2][2];   // Z1 = X W0^T: B[k = in][n = hidden], per hidden n-tile
    uint32_t w0t[K::NS][2];     // dX = dZ1 W0: B[k = hidden][n = in 0..7]
    uint32_t w1[K::NS][2][2];   // Z2 = H1 W1^T (NL == 2)
    uint32_t w1t[K::NS][2][2];  // dH1 = dZ2 W1: B[k = hidden2][n = hidden1], per n-tile
    uint32_t wo[K::NS][2];      // O = H Wo^T: B[k = hidden][n = out 0..7]
    uint32_t wot[K::NS][2];     // dH = dZo Wo: B[k = out 0..7][n = hidden], per hidden n-tile (first k half)
};

template <class K>
struct RegWarpSmem {
    __align__(16) __nv_bfloat16 X[K::NS][32 * 24];  // per-pixel input rows, 16 used (48-byte stride)
    float scr[32 * 17];                             // per-pixel fp32 rows: logits, then dX
    // the hidden activations' A fragments between forward and backward
    // ([plane][layer][m-tile][register][lane]: lane-minor, conflict-free)
    uint32_t H[K::NS][K::NL][2][4][32];
};

template <class K>
struct RegSmem {
    float g[K::NPARAM];  // CTA gradient accumulators (packed like the parameters)
    float loss[kShadeRegWarps];
    uint32_t wtab[K::WREG ? 1 : sizeof(RegWeights<K>) / 4][32];  // fragment table (lane-minor)
    RegWarpSmem<K> w[kShadeRegWarps];
};

// bf16 planes of the pair (v0, v1)
template <int NS>
__device__ __forceinline__ void planes(float v0, float v1, uint32_t* o) {
    if (NS == 2) split_bf16(v0, v1, o[0], o[1]);
    else o[0] = pack_bf16(v0, v1);
}

// acc += A B summed over the planes: hi*hi (+ hi*lo + lo*hi)
template <int NS>
__device__ __forceinline__ void mma3(float acc[4], const uint32_t* ah, const uint32_t* al, const uint32_t* bh,
                                     const uint32_t* bl) {
    mma_16816(acc, ah, bh);
    if (NS == 2) {
        mma_16816(acc, ah, bl);
        mma_16816(acc, al, bh);
    }
}

// relu'(h) applied to an accumulator pair, h one bf16x2 register of the activation's hi plane
__device__ __forceinline__ float2 gate2(uint32_t h, float v0, float v1) {
    const __nv_bfloat162 hv = *reinterpret_cast<const __nv_bfloat162*>(&h);
    return make_float2(__low2float(hv) > 0.f ? v0 : 0.f, __high2float(hv) > 0.f ? v1 : 0.f);
}

template <class K>
__device__ __forceinline__ void reg_weights(RegWeights<K>& f, const float* __restrict__ P, int g, int q) {
    constexpr int NS = K::NS, IN = K::IN;
    auto w0 = [&](int h, int i) { return i < IN ? __ldg(P + K::P_W0 + h * IN + i) : 0.f; };
    auto w1 = [&](int o, int i) { return __ldg(P + K::P_W1 + o * 16 + i); };
    auto wo = [&](int o, int h) { return o < 3 ? __ldg(P + K::P_WO + o * 16 + h) : 0.f; };
    uint32_t t[NS];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        const int h = nt * 8 + g;
#pragma unroll
        for (int hk = 0; hk < 2; ++hk) {
            planes<NS>(w0(h, 2 * q + 8 * hk), w0(h, 2 * q + 1 + 8 * hk), t);
#pragma unroll
            for (int s = 0; s < NS; ++s) f.w0[s][nt][hk] = t[s];
            if (K::NL == 2) {
                planes<NS>(w1(h, 2 * q + 8 * hk), w1(h, 2 * q + 1 + 8 * hk), t);
#pragma unroll
                for (int s = 0; s < NS; ++s) f.w1[s][nt][hk] = t[s];
                planes<NS>(w1(2 * q + 8 * hk, h), w1(2 * q + 1 + 8 * hk, h), t);
#pragma unroll
                for (int s = 0; s < NS; ++s) f.w1t[s][nt][hk] = t[s];
            }
        }
        planes<NS>(wo(2 * q, h), wo(2 * q + 1, h), t);
#pragma unroll
        for (int s = 0; s < NS; ++s) f.wot[s][nt] = t[s];
    }
#pragma unroll
    for (int hk = 0; hk < 2; ++hk) {
        planes<NS>(w0(2 * q + 8 * hk, g), w0(2 * q + 1 + 8 * hk, g), t);
#pragma unroll
        for (int s = 0; s < NS; ++s) f.w0t[s][hk] = t[s];
        planes<NS>(wo(g, 2 * q + 8 * hk), wo(g, 2 * q + 1 + 8 * hk), t);
#pragma unroll
        for (int s = 0; s < NS; ++s) f.wo[s][hk] = t[s];
    }
}

template <class K>
__global__ void __launch_bounds__(kShadeRegWarps * 32, K::MIN_CTAS) shade_reg_kernel(ShadeArgs a) {
    constexpr int NS = K::NS, IN = K::IN, C = K::C, NL = K::NL;
    extern __shared__ __align__(16) unsigned char reg_smem_raw[];  // RegSmem<K> (above the 48 KB static limit)
    RegSmem<K>& sm = *reinterpret_cast<RegSmem<K>*>(reg_smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const float* P = a.params;

    // ---- weights as fragments --------------------------------------------
    RegWeights<K> wreg;
    reg_weights<K>(wreg, P, g, q);
    if (!K::WREG && warp == 0) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&wreg);
#pragma unroll
        for (int i = 0; i < (int)(sizeof(RegWeights<K>) / 4); ++i) sm.wtab[i][lane] = src[i];
    }
    // the lane's fragments, from registers or from the CTA table
    auto W = [&]() -> RegWeights<K> {
        if (K::WREG) return wreg;
        RegWeights<K> f;
        uint32_t* dst = reinterpret_cast<uint32_t*>(&f);
#pragma unroll
        for (int i = 0; i < (int)(sizeof(RegWeights<K>) / 4); ++i) dst[i] = sm.wtab[i][lane];
        return f;
    };
    float bb0[2][2], bb1[2][2];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        bb0[nt][0] = __ldg(P + K::P_B0 + nt * 8 + 2 * q);
        bb0[nt][1] = __ldg(P + K::P_B0 + nt * 8 + 2 * q + 1);
        bb1[nt][0] = NL == 2 ? __ldg(P + K::P_B1 + nt * 8 + 2 * q) : 0.f;
        bb1[nt][1] = NL == 2 ? __ldg(P + K::P_B1 + nt * 8 + 2 * q + 1) : 0.f;
    }
    const float bo0 = __ldg(P + K::P_BO + 0), bo1 = __ldg(P + K::P_BO + 1), bo2 = __ldg(P + K::P_BO + 2);
    for (int i = threadIdx.x; i < K::NPARAM; i += blockDim.x) sm.g[i] = 0.f;

    // gradients of the whole kernel (accumulator layouts)
    float gw0[2][4], gw1[2][4], gwo[2][4], gb0[2][2], gb1[2][2], gbo[3] = {0.f, 0.f, 0.f}, loss_acc = 0.f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int k = 0; k < 4; ++k) gw0[i][k] = gw1[i][k] = gwo[i][k] = 0.f;
        gb0[i][0] = gb0[i][1] = gb1[i][0] = gb1[i][1] = 0.f;
    }
    __syncthreads();

    RegWarpSmem<K>& ws = sm.w[warp];
    const int64_t nchunks = (a.num_pixels + 31) / 32;
    const int64_t cstride = (int64_t)gridDim.x * kShadeRegWarps;
    // the rast entry of the warp's next chunk is requested one chunk ahead
    float4 r_next = make_float4(0.f, 0.f, 0.f, 0.f);
    {
        const int64_t p0 = ((int64_t)blockIdx.x * kShadeRegWarps + warp) * 32 + lane;
        if (p0 < a.num_pixels) r_next = reinterpret_cast<const float4*>(a.rast)[p0];
    }
    for (int64_t chunk = (int64_t)blockIdx.x * kShadeRegWarps + warp; chunk < nchunks; chunk += cstride) {
        // ---------------- pixel front: gather features, view encoding --------------
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
            for (int c = 0; c < 3; ++c) tgt[c] = target_at(a, p, c);
        }
        const int t = (int)r.w - 1;
        const bool mask = valid && t >= 0;
        float x[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) x[c] = 0.f;
        uint32_t idx[3] = {0, 0, 0};
        float wgt[3] = {0.f, 0.f, 0.f};
        if (mask) {
            lattice_cell(r.x, r.y, (uint32_t)a.level, idx, wgt);
            float f[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float v[8];
                if (K::SPLIT) {  // fp32 features
                    const float4* fv = reinterpret_cast<const float4*>(a.feat_f32 + ((size_t)t * a.S + idx[k]) * 8);
                    const float4 u0 = __ldg(fv), u1 = __ldg(fv + 1);
                    v[0] = u0.x; v[1] = u0.y; v[2] = u0.z; v[3] = u0.w;
                    v[4] = u1.x; v[5] = u1.y; v[6] = u1.z; v[7] = u1.w;
                } else {
                    const uint4 u = __ldg(reinterpret_cast<const uint4*>(a.feat + ((size_t)t * a.S + idx[k]) * 8));
                    const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 ff = __bfloat1622float2(h2[j]);
                        v[2 * j] = ff.x;
                        v[2 * j + 1] = ff.y;
                    }
                }
#pragma unroll
                for (int c = 0; c < 8; ++c) f[c] = __fmaf_rn(wgt[k], v[c], f[c]);
            }
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = f[c];
            const int b = view_of_pixel(a.views, a.B, p);
            const ds_view_desc vd = a.views[b];
            const int local = (int)(p - vd.pix_offset);  // < H*W < 2^31: 32-bit division
            const int py = local / vd.W, px = local - py * vd.W;
            float M[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) M[k] = __ldg(a.inv_mvp + (size_t)b * 16 + k);
            float d[3];
            view_direction(pix_ndc(px, vd.W), pix_ndc(py, vd.H), M, d);
            if (K::ENC == 9) {
                float sh[9];
                sh2_basis(d[0], d[1], d[2], sh);
#pragma unroll
                for (int k = 0; k < 9; ++k) x[(C + k) & 15] = sh[k];
            } else {
                x[C] = d[0]; x[(C + 1) & 15] = d[1]; x[(C + 2) & 15] = d[2];
            }
        }
        // a chunk without covered pixels has an all-background colour: no MLP, no gradients
        const bool any = __any_sync(0xffffffffu, mask);
        if (any) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t u[NS][4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    uint32_t t2[NS];
                    planes<NS>(x[8 * h + 2 * j], x[8 * h + 2 * j + 1], t2);
#pragma unroll
                    for (int s = 0; s < NS; ++s) u[s][j] = t2[s];
                }
#pragma unroll
                for (int s = 0; s < NS; ++s)
                    *reinterpret_cast<uint4*>(ws.X[s] + lane * 24 + 8 * h) = make_uint4(u[s][0], u[s][1], u[s][2], u[s][3]);
            }
            __syncwarp();

            // ---------------- MLP forward (activations in registers) ------------------
            const RegWeights<K> f = W();
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                // relu activations as bf16 planes, A operands of the next products: [plane][reg]
                uint32_t aH1[NS][4], aH2[NS][4];
                uint32_t (&HL)[NS][4] = NL == 2 ? aH2 : aH1;  // the last hidden layer
                uint32_t aX[NS][4];
#pragma unroll
                for (int s = 0; s < NS; ++s) load_a(aX[s], ws.X[s], 24, mt * 16, 0);
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
                    mma3<NS>(acc, aX[0], aX[NS - 1], f.w0[0][nt], f.w0[NS - 1][nt]);
                    uint32_t t0[NS], t1[NS];
                    planes<NS>(fmaxf(acc[0] + bb0[nt][0], 0.f), fmaxf(acc[1] + bb0[nt][1], 0.f), t0);
                    planes<NS>(fmaxf(acc[2] + bb0[nt][0], 0.f), fmaxf(acc[3] + bb0[nt][1], 0.f), t1);
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        aH1[s][2 * nt] = t0[s];
                        aH1[s][2 * nt + 1] = t1[s];
                    }
                }
                if constexpr (NL == 2) {
#pragma unroll
                    for (int nt = 0; nt < 2; ++nt) {
                        float acc[4] = {0.f, 0.f, 0.f, 0.f};
                        mma3<NS>(acc, aH1[0], aH1[NS - 1], f.w1[0][nt], f.w1[NS - 1][nt]);
                        uint32_t t0[NS], t1[NS];
                        planes<NS>(fmaxf(acc[0] + bb1[nt][0], 0.f), fmaxf(acc[1] + bb1[nt][1], 0.f), t0);
                        planes<NS>(fmaxf(acc[2] + bb1[nt][0], 0.f), fmaxf(acc[3] + bb1[nt][1], 0.f), t1);
#pragma unroll
                        for (int s = 0; s < NS; ++s) {
                            aH2[s][2 * nt] = t0[s];
                            aH2[s][2 * nt + 1] = t1[s];
                        }
                    }
                }
#pragma unroll
                for (int s = 0; s < NS; ++s)
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        ws.H[s][0][mt][k][lane] = aH1[s][k];
                        if (NL == 2) ws.H[s][NL - 1][mt][k][lane] = aH2[s][k];
                    }
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                mma3<NS>(acc, HL[0], HL[NS - 1], f.wo[0], f.wo[NS - 1]);
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
        const RegWeights<K> f = W();
        // dZo as an A operand: rows g, g+8 of each m-tile; outputs 2q, 2q+1 (q < 2)
        uint32_t dz01[NS], dz2[NS];
        planes<NS>(dz[0], dz[1], dz01);
        planes<NS>(dz[2], 0.f, dz2);
        uint32_t aDZo[NS][2][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int src = mt * 16 + g + 8 * h;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const uint32_t u01 = __shfl_sync(0xffffffffu, dz01[s], src);
                    const uint32_t u2 = __shfl_sync(0xffffffffu, dz2[s], src);
                    aDZo[s][mt][h] = q == 0 ? u01 : (q == 1 ? u2 : 0u);
                }
            }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            // this m-tile's activations, from the forward pass
            uint32_t aH1[NS][4], HL[NS][4];
#pragma unroll
            for (int s = 0; s < NS; ++s)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    HL[s][k] = ws.H[s][NL - 1][mt][k][lane];
                    aH1[s][k] = NL == 2 ? ws.H[s][0][mt][k][lane] : HL[s][k];
                }
            // dZ_last = (dZo Wo) * relu'(H_last)
            uint32_t aDL[NS][4];
            {
                uint32_t aZ[NS][4];
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    aZ[s][0] = aDZo[s][mt][0]; aZ[s][1] = aDZo[s][mt][1]; aZ[s][2] = 0u; aZ[s][3] = 0u;
                }
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
                    const uint32_t bh[2] = {f.wot[0][nt], 0u}, bl[2] = {f.wot[NS - 1][nt], 0u};
                    mma3<NS>(acc, aZ[0], aZ[NS - 1], bh, bl);
                    const float2 lo = gate2(HL[0][2 * nt], acc[0], acc[1]);
                    const float2 hi = gate2(HL[0][2 * nt + 1], acc[2], acc[3]);
                    float (&gb)[2][2] = NL == 2 ? gb1 : gb0;
                    gb[nt][0] += lo.x + hi.x;
                    gb[nt][1] += lo.y + hi.y;
                    uint32_t t0[NS], t1[NS];
                    planes<NS>(lo.x, lo.y, t0);
                    planes<NS>(hi.x, hi.y, t1);
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        aDL[s][2 * nt] = t0[s];
                        aDL[s][2 * nt + 1] = t1[s];
                    }
                }
            }
            // dWo += dZo^T H_last: A = dZo^T (outputs x pixels), B = H_last (pixels x hidden)
            {
                uint32_t aT[NS][4], b0[NS][2], b1[NS][2];
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    aT[s][0] = movmatrix_t(aDZo[s][mt][0]); aT[s][1] = 0u;
                    aT[s][2] = movmatrix_t(aDZo[s][mt][1]); aT[s][3] = 0u;
                    b0[s][0] = movmatrix_t(HL[s][0]); b0[s][1] = movmatrix_t(HL[s][1]);
                    b1[s][0] = movmatrix_t(HL[s][2]); b1[s][1] = movmatrix_t(HL[s][3]);
                }
                mma3<NS>(gwo[0], aT[0], aT[NS - 1], b0[0], b0[NS - 1]);
                mma3<NS>(gwo[1], aT[0], aT[NS - 1], b1[0], b1[NS - 1]);
            }
            uint32_t aD1[NS][4];
            if constexpr (NL == 2) {
                // dW1 += dZ2^T H1
                {
                    uint32_t aT[NS][4], b0[NS][2], b1[NS][2];
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        aT[s][0] = movmatrix_t(aDL[s][0]); aT[s][1] = movmatrix_t(aDL[s][2]);
                        aT[s][2] = movmatrix_t(aDL[s][1]); aT[s][3] = movmatrix_t(aDL[s][3]);
                        b0[s][0] = movmatrix_t(aH1[s][0]); b0[s][1] = movmatrix_t(aH1[s][1]);
                        b1[s][0] = movmatrix_t(aH1[s][2]); b1[s][1] = movmatrix_t(aH1[s][3]);
                    }
                    mma3<NS>(gw1[0], aT[0], aT[NS - 1], b0[0], b0[NS - 1]);
                    mma3<NS>(gw1[1], aT[0], aT[NS - 1], b1[0], b1[NS - 1]);
                }
                // dZ1 = (dZ2 W1) * relu'(H1)
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
                    mma3<NS>(acc, aDL[0], aDL[NS - 1], f.w1t[0][nt], f.w1t[NS - 1][nt]);
                    const float2 lo = gate2(aH1[0][2 * nt], acc[0], acc[1]);
                    const float2 hi = gate2(aH1[0][2 * nt + 1], acc[2], acc[3]);
                    gb0[nt][0] += lo.x + hi.x;
                    gb0[nt][1] += lo.y + hi.y;
                    uint32_t t0[NS], t1[NS];
                    planes<NS>(lo.x, lo.y, t0);
                    planes<NS>(hi.x, hi.y, t1);
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        aD1[s][2 * nt] = t0[s];
                        aD1[s][2 * nt + 1] = t1[s];
                    }
                }
            } else {
#pragma unroll
                for (int s = 0; s < NS; ++s)
#pragma unroll
                    for (int k = 0; k < 4; ++k) aD1[s][k] = aDL[s][k];
            }
            // dW0 += dZ1^T X: A = dZ1^T (hidden x pixels), B = X (pixels x inputs)
            {
                uint32_t aX[NS][4];  // reloaded: cheaper than keeping both m-tiles live
#pragma unroll
                for (int s = 0; s < NS; ++s) load_a(aX[s], ws.X[s], 24, mt * 16, 0);
                uint32_t aT[NS][4], b0[NS][2], b1[NS][2];
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    aT[s][0] = movmatrix_t(aD1[s][0]); aT[s][1] = movmatrix_t(aD1[s][2]);
                    aT[s][2] = movmatrix_t(aD1[s][1]); aT[s][3] = movmatrix_t(aD1[s][3]);
                    b0[s][0] = movmatrix_t(aX[s][0]); b0[s][1] = movmatrix_t(aX[s][1]);
                    b1[s][0] = movmatrix_t(aX[s][2]); b1[s][1] = movmatrix_t(aX[s][3]);
                }
                mma3<NS>(gw0[0], aT[0], aT[NS - 1], b0[0], b0[NS - 1]);
                mma3<NS>(gw0[1], aT[0], aT[NS - 1], b1[0], b1[NS - 1]);
            }
            // dX = dZ1 W0 for inputs 0..7 (the features) -> scr, for the feature scatter
            {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                mma3<NS>(acc, aD1[0], aD1[NS - 1], f.w0t[0], f.w0t[NS - 1]);
                ws.scr[(mt * 16 + g) * 17 + 2 * q] = acc[0];
                ws.scr[(mt * 16 + g) * 17 + 2 * q + 1] = acc[1];
                ws.scr[(mt * 16 + g + 8) * 17 + 2 * q] = acc[2];
                ws.scr[(mt * 16 + g + 8) * 17 + 2 * q + 1] = acc[3];
            }
        }
        __syncwarp();

        // ---------------- feature-gradient scatter (lane = pixel) -------------------
        if (mask) {
            float dx[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) dx[c] = c < C ? ws.scr[lane * 17 + c] + (c < 4 ? dxd[c] : 0.f) : 0.f;
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
    // W0[h][i] (and W1[o][i]): tile ni holds rows g (+8), columns ni*8 + 2q (+1)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni) {
        const int i0 = ni * 8 + 2 * q;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            if (i0 + e < IN) {
                atomicAdd(&sm.g[K::P_W0 + g * IN + i0 + e], gw0[ni][e]);
                atomicAdd(&sm.g[K::P_W0 + (g + 8) * IN + i0 + e], gw0[ni][2 + e]);
            }
            if (NL == 2) {
                atomicAdd(&sm.g[K::P_W1 + g * 16 + i0 + e], gw1[ni][e]);
                atomicAdd(&sm.g[K::P_W1 + (g + 8) * 16 + i0 + e], gw1[ni][2 + e]);
            }
        }
    }
    // Wo[o][h]: tile nt holds rows o = g (< 3 used), columns h = nt*8 + 2q (+1)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        if (g < 3) {
            atomicAdd(&sm.g[K::P_WO + g * 16 + nt * 8 + 2 * q], gwo[nt][0]);
            atomicAdd(&sm.g[K::P_WO + g * 16 + nt * 8 + 2 * q + 1], gwo[nt][1]);
        }
        // hidden biases: sums over the rows g of the lane's columns
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            float s0 = l == 0 ? gb0[nt][0] : gb1[nt][0], s1 = l == 0 ? gb0[nt][1] : gb1[nt][1];
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            }
            const int pb = l == 0 ? K::P_B0 : K::P_B1;
            if (g == 0) {
                atomicAdd(&sm.g[pb + nt * 8 + 2 * q], s0);
                atomicAdd(&sm.g[pb + nt * 8 + 2 * q + 1], s1);
            }
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
        for (int w = 0; w < kShadeRegWarps; ++w) s += sm.loss[w];
        atomicAdd(a.loss_sum, s);
    }
    for (int i = threadIdx.x; i < K::NPARAM; i += blockDim.x)
        if (sm.g[i] != 0.f) atomicAdd(a.grad_params + i, sm.g[i]);
}

}  // namespace dsb
