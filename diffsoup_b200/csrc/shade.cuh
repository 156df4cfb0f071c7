// diffsoup_b200/csrc/shade.cuh -- fused per-pixel shading forward+backward
// of the DiffSoup training step, with the shading MLP on BF16 tensor cores.
//
// For every pixel of the packed batch this kernel does, in one pass:
//   feature gather     multires_triangle_color (multires.cu:224-247), bf16
//                      features, fp32 interpolation
//   view direction     compute_view_direction (encoding.cu:28-53)
//   shading MLP        ColorMLP (multires.py:171-207): Linear/ReLU layers and
//                      a sigmoid output on mma.sync m16n8k16 (bf16 x bf16 ->
//                      fp32), biases added in fp32
//   residual blend     (1 - x3) * x[0:3] + x3 * mlp(x), background 1 where the
//                      pixel is empty (examples/02_synthetic.py:365-368)
//   MSE loss           sum of (c - target)^2 and dL/dc = 2 (c - target) / N
//   MLP backward       dX and dW/db on the tensor cores
//   feature scatter    adjoint of the gather (multires.cu:268-292)
// and writes colour, dL/dcolour and |c - target| summed over channels for the
// edge-gradient and opacity passes.  A warp owns 32 consecutive pixels; its
// activations live in shared memory as row-major bf16 tiles that ldmatrix
// turns into fragments (plain or transposed as each product needs).
#pragma once

#include "geometry.cuh"
#include "mma.cuh"

namespace dsb {

// SPLIT_: every MLP operand is carried as two bf16 planes, hi = bf16(v) and
// lo = bf16(v - hi) (16 significant bits together), features are gathered from
// the fp32 copy, and each product is hi*hi + hi*lo + lo*hi on the BF16 tensor
// cores with fp32 accumulation -- the precision mode whose gradients agree with
// the FP64 oracle to ~1e-5 (the lo*lo term is below 2^-16 of the product).
template <int C_, int IN_PAD_, int HID_, int NL_, bool SPLIT_ = false>
struct ShadeCfg {
    static constexpr int C = C_;             // feature channels
    static constexpr int IN_REAL = C_ + 3;   // features + view direction
    static constexpr int IN_PAD = IN_PAD_;   // multiple of 16
    static constexpr int HID = HID_;         // multiple of 16
    static constexpr int NL = NL_;           // hidden layers
    static constexpr int OUT = 3;
    static constexpr int LDX = IN_PAD + 8;   // padded row strides (bf16): conflict-free ldmatrix
    static constexpr int LDH = HID + 8;
    static constexpr int LDO = 16 + 8;
    static constexpr int LDS = (IN_PAD > 16 ? IN_PAD : 16) + 1;  // fp32 scratch stride
    static constexpr bool SPLIT = SPLIT_;
    static constexpr int NS = SPLIT_ ? 2 : 1;  // bf16 planes per operand
    // warps per CTA: the split planes of the large MLP need twice the shared memory
    static constexpr int WARPS = (SPLIT_ && HID_ > 32) ? 2 : 4;
    static constexpr int NH = NL > 1 ? NL - 1 : 1;  // hidden-to-hidden matrices (at least 1 slot)
    // packed fp32 parameter offsets: W0[HID][IN_REAL] b0[HID] (Wl[HID][HID] bl[HID])* Wo[3][HID] bo[3]
    static constexpr int P_W0 = 0;
    static constexpr int P_B0 = HID * IN_REAL;
    static constexpr int P_WH = P_B0 + HID;
    static constexpr int P_WO = P_WH + (NL - 1) * (HID * HID + HID);
    static constexpr int P_BO = P_WO + OUT * HID;
    static constexpr int NPARAM = P_BO + OUT;
    // Small MLPs keep their weight and bias gradients in registers for the
    // whole kernel (mma accumulators that persist across pixel chunks)
    // instead of adding every chunk's tiles into shared memory.
    static constexpr bool REG_GRADS = NL == 1 && HID * IN_PAD <= 256;
    // Otherwise the weight gradients are computed per round of WARPS chunks:
    // every warp owns some of the weight-gradient tiles and sums them over
    // all the CTA's chunks of the round (no atomics); the dZ_l tiles of a
    // chunk stay in its warp's two DH buffers, which holds for NL <= 2.
    static_assert(REG_GRADS || NL <= 2, "distributed weight gradients need NL <= 2");
    static_assert(IN_PAD % 16 == 0 && IN_PAD >= IN_REAL && HID % 16 == 0, "MLP dims");
    static_assert((LDX * 2) % 16 == 0 && (LDH * 2) % 16 == 0 && (LDO * 2) % 16 == 0, "ldmatrix row alignment");
};

// Every ldmatrix row address must be 16-byte aligned: all tiles start on
// 16-byte boundaries and their row strides are multiples of 8 bf16.
// [plane][...]: plane 0 holds bf16(v), plane 1 (SPLIT only) bf16(v - plane 0).
template <class K>
struct __align__(16) ShadeWarpSmem {
    __align__(16) __nv_bfloat16 X[K::NS][32 * K::LDX];
    __align__(16) __nv_bfloat16 H[K::NL][K::NS][32 * K::LDH];
    __align__(16) __nv_bfloat16 DZO[K::NS][32 * K::LDO];
    __align__(16) __nv_bfloat16 DH[2][K::NS][32 * K::LDH];
    __align__(16) float scr[32 * K::LDS];
};

template <class K>
struct __align__(16) ShadeSmem {
    __align__(16) __nv_bfloat16 W0[K::NS][K::HID * K::LDX];
    __align__(16) __nv_bfloat16 WH[K::NH][K::NS][K::HID * K::LDH];
    __align__(16) __nv_bfloat16 WO[K::NS][16 * K::LDH];
    float b0[K::HID];
    float bh[K::NH][K::HID];
    float bo[4];
    // fp32 gradient accumulators of this CTA (same packing as the parameters)
    float g[K::NPARAM];
    float loss[K::WARPS];
    int ran[K::WARPS];  // per warp: its chunk of the current round left MLP tiles in its shared memory
    __align__(16) ShadeWarpSmem<K> w[K::WARPS];
};

struct ShadeArgs {
    int B;
    const ds_view_desc* views;
    int64_t num_pixels;
    const float* rast;            // [P,4]
    const __nv_bfloat16* feat;    // [T,S,C] sigmoid features, bf16
    const float* feat_f32;        // [T,S,C] the same in fp32 (read by the SPLIT kernels)
    int level, S;
    const float* inv_mvp;         // [B,16]
    const float* target;          // [P,3] fp32, or
    const uint8_t* target_u8;     // [P,3] 8-bit, value / 255 (used when non-null)
    const float* params;          // packed fp32 MLP parameters
    float inv_n;                  // 1 / (P * 3)
    float* color;                 // [P,3]
    float* grad_color;            // [P,3]
    float* l1;                    // [P]
    float* grad_feat;             // [T,S,C] fp32, accumulates
    float* grad_params;           // packed, accumulates
    double* loss_sum;             // [1], accumulates sum of squared errors
    int* status;                  // step status bits (DS_STATUS_*), may be null
};

// bf16 planes of two values: hi = bf16(v), lo = bf16(v - hi).
__device__ __forceinline__ void split_bf16(float v0, float v1, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(v0 - hf.x, v1 - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Stores (v0, v1) at element `off` of an operand tile's planes.
template <class K, class Tile>
__device__ __forceinline__ void put2(Tile& t, int off, float v0, float v1) {
    if (K::SPLIT) {
        uint32_t hi, lo;
        split_bf16(v0, v1, hi, lo);
        *reinterpret_cast<uint32_t*>(&t[0][off]) = hi;
        *reinterpret_cast<uint32_t*>(&t[K::NS - 1][off]) = lo;
    } else {
        *reinterpret_cast<uint32_t*>(&t[0][off]) = pack_bf16(v0, v1);
    }
}

// acc += A B over the planes: hi*hi (+ hi*lo + lo*hi with SPLIT).
template <class K>
__device__ __forceinline__ void mma_planes(float acc[4], const uint32_t a[K::NS][4], const uint32_t b[K::NS][2]) {
    mma_16816(acc, a[0], b[0]);
    if (K::SPLIT) {
        mma_16816(acc, a[0], b[K::NS - 1]);
        mma_16816(acc, a[K::NS - 1], b[0]);
    }
}

// Target channel c of pixel p: fp32, or an 8-bit value / 255 (correctly
// rounded, so that an fp32 target holding the same quotient gives the same
// step).
__device__ __forceinline__ float target_at(const ShadeArgs& a, int64_t p, int c) {
    return a.target_u8 ? __fdiv_rn((float)a.target_u8[p * 3 + c], 255.f) : a.target[p * 3 + c];
}

// Relu mask of an activation element stored as bf16 in smem.
__device__ __forceinline__ float2 relu_gate(const __nv_bfloat16* h, float2 v) {
    const __nv_bfloat162 hv = *reinterpret_cast<const __nv_bfloat162*>(h);
    return make_float2(__low2float(hv) > 0.f ? v.x : 0.f, __high2float(hv) > 0.f ? v.y : 0.f);
}

#ifndef DSB_SHADE_MIN_CTAS
#define DSB_SHADE_MIN_CTAS 5  // resident CTAs per SM the small-MLP register budget is sized for
#endif

template <class K>
__global__ void __launch_bounds__(K::WARPS * 32, K::REG_GRADS ? DSB_SHADE_MIN_CTAS : 1) shade_step_kernel(ShadeArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ShadeSmem<K>& sm = *reinterpret_cast<ShadeSmem<K>*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    constexpr int HID = K::HID, IN_PAD = K::IN_PAD;

    // ---- weights to shared memory (bf16 planes, zero padded), biases fp32 ---
    for (int i = threadIdx.x; i < HID * K::LDX; i += blockDim.x) {
        const int r = i / K::LDX, c = i % K::LDX;
        const float v = c < K::IN_REAL ? a.params[K::P_W0 + r * K::IN_REAL + c] : 0.f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        sm.W0[0][i] = h;
        if (K::SPLIT) sm.W0[K::NS - 1][i] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
    for (int l = 0; l < K::NL - 1; ++l)
        for (int i = threadIdx.x; i < HID * K::LDH; i += blockDim.x) {
            const int r = i / K::LDH, c = i % K::LDH;
            const float v = c < HID ? a.params[K::P_WH + l * (HID * HID + HID) + r * HID + c] : 0.f;
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            sm.WH[l][0][i] = h;
            if (K::SPLIT) sm.WH[l][K::NS - 1][i] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
    for (int i = threadIdx.x; i < 16 * K::LDH; i += blockDim.x) {
        const int r = i / K::LDH, c = i % K::LDH;
        const float v = r < K::OUT && c < HID ? a.params[K::P_WO + r * HID + c] : 0.f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        sm.WO[0][i] = h;
        if (K::SPLIT) sm.WO[K::NS - 1][i] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        sm.b0[i] = a.params[K::P_B0 + i];
        for (int l = 0; l < K::NL - 1; ++l) sm.bh[l][i] = a.params[K::P_WH + l * (HID * HID + HID) + HID * HID + i];
    }
    if (threadIdx.x < 4) sm.bo[threadIdx.x] = threadIdx.x < 3 ? a.params[K::P_BO + threadIdx.x] : 0.f;
    for (int i = threadIdx.x; i < K::NPARAM; i += blockDim.x) sm.g[i] = 0.f;
    __syncthreads();

    ShadeWarpSmem<K>& ws = sm.w[warp];
    float loss_acc = 0.f;
    // REG_GRADS: per-lane partial gradients (mma accumulator layout)
    constexpr int GW0M = K::REG_GRADS ? HID / 16 : 1, GW0N = K::REG_GRADS ? IN_PAD / 8 : 1;
    constexpr int GWO = K::REG_GRADS ? HID / 8 : 1;
    float gw0[GW0M][GW0N][4], gwo[GWO][4], gbh[GWO][2], gbo[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < GW0M; ++i)
#pragma unroll
        for (int j = 0; j < GW0N; ++j)
#pragma unroll
            for (int k = 0; k < 4; ++k) gw0[i][j][k] = 0.f;
#pragma unroll
    for (int i = 0; i < GWO; ++i) {
#pragma unroll
        for (int k = 0; k < 4; ++k) gwo[i][k] = 0.f;
        gbh[i][0] = gbh[i][1] = 0.f;
    }
    const int64_t nchunks = (a.num_pixels + 31) / 32;
    // Every warp runs the same number of rounds (the CTA synchronises once per
    // round for the weight gradients); a warp whose chunk lies past the end
    // takes part with no pixels.
    const int64_t per_round = (int64_t)gridDim.x * K::WARPS;
    const int64_t rounds = (nchunks + per_round - 1) / per_round;
    for (int64_t rd = 0; rd < rounds; ++rd) {
      const int64_t chunk = rd * per_round + (int64_t)blockIdx.x * K::WARPS + warp;
      bool ran = false;  // this warp's chunk ran the MLP: its tiles in shared memory feed the weight gradients
      do {  // one chunk; `continue` leaves it
        // ---------------- pixel front: gather features, view direction ----------
        const int64_t p = chunk * 32 + lane;
        const bool valid = p < a.num_pixels;
        float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
        if (valid) r = reinterpret_cast<const float4*>(a.rast)[p];
        const int t = (int)r.w - 1;
        const bool mask = valid && t >= 0;
        float x[K::IN_REAL];
#pragma unroll
        for (int c = 0; c < K::IN_REAL; ++c) x[c] = 0.f;
        uint32_t idx[3] = {0, 0, 0};
        float wgt[3] = {0.f, 0.f, 0.f};
        if (mask) {
            lattice_cell(r.x, r.y, (uint32_t)a.level, idx, wgt);
            const __nv_bfloat16* tf = a.feat + (size_t)t * a.S * K::C;
            const float* tf32 = a.feat_f32 + (size_t)t * a.S * K::C;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (K::SPLIT) {  // fp32 features
                    const float* fv = tf32 + (size_t)idx[k] * K::C;
#pragma unroll
                    for (int c = 0; c < K::C; c += 4) {
                        const float4 u = __ldg(reinterpret_cast<const float4*>(fv + c));
                        x[c] = __fmaf_rn(wgt[k], u.x, x[c]);
                        x[c + 1] = __fmaf_rn(wgt[k], u.y, x[c + 1]);
                        x[c + 2] = __fmaf_rn(wgt[k], u.z, x[c + 2]);
                        x[c + 3] = __fmaf_rn(wgt[k], u.w, x[c + 3]);
                    }
                    continue;
                }
                const __nv_bfloat16* fv = tf + (size_t)idx[k] * K::C;
#pragma unroll
                for (int c = 0; c < K::C; c += 8) {
                    const uint4 u = __ldg(reinterpret_cast<const uint4*>(fv + c));
                    const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 f = __bfloat1622float2(h2[j]);
                        x[c + 2 * j] = __fmaf_rn(wgt[k], f.x, x[c + 2 * j]);
                        x[c + 2 * j + 1] = __fmaf_rn(wgt[k], f.y, x[c + 2 * j + 1]);
                    }
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
            x[K::C + 0] = d[0]; x[K::C + 1] = d[1]; x[K::C + 2] = d[2];
        }
        if (!__any_sync(0xffffffffu, mask)) {
            // no covered pixel in the chunk: background colour 1, no MLP and no gradients
            if (valid) {
                float l1 = 0.f;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float diff = 1.f - target_at(a, p, c);
                    loss_acc += diff * diff;
                    a.color[p * 3 + c] = 1.f;
                    a.grad_color[p * 3 + c] = 2.f * diff * a.inv_n;
                    l1 += fabsf(diff);
                }
                a.l1[p] = l1;
            }
            continue;
        }
        {
            // 16-byte stores: rows are 16-byte aligned and, at these strides,
            // the 8 lanes of each store phase hit distinct bank groups
#pragma unroll
            for (int c = 0; c < IN_PAD; c += 8) {
                uint32_t u[4], ul[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c0 = c + 2 * j, c1 = c + 2 * j + 1;
                    const float v0 = c0 < K::IN_REAL ? x[c0 < K::IN_REAL ? c0 : 0] : 0.f;
                    const float v1 = c1 < K::IN_REAL ? x[c1 < K::IN_REAL ? c1 : 0] : 0.f;
                    if (K::SPLIT) split_bf16(v0, v1, u[j], ul[j]);
                    else u[j] = pack_bf16(v0, v1);
                }
                *reinterpret_cast<uint4*>(ws.X[0] + lane * K::LDX + c) = make_uint4(u[0], u[1], u[2], u[3]);
                if (K::SPLIT)
                    *reinterpret_cast<uint4*>(ws.X[K::NS - 1] + lane * K::LDX + c) = make_uint4(ul[0], ul[1], ul[2], ul[3]);
            }
        }
        __syncwarp();

        // ---------------- MLP forward -------------------------------------------
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
            for (int nt = 0; nt < HID / 8; ++nt) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int kt = 0; kt < IN_PAD / 16; ++kt) {
                    uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                    for (int s = 0; s < K::NS; ++s) {
                        load_a(af[s], ws.X[s], K::LDX, mt * 16, kt * 16);
                        load_b(bf[s], sm.W0[s], K::LDX, nt * 8, kt * 16);
                    }
                    mma_planes<K>(acc, af, bf);
                }
                const int col = nt * 8 + 2 * q;
                const float b0v = sm.b0[col], b1v = sm.b0[col + 1];
                put2<K>(ws.H[0], (mt * 16 + g) * K::LDH + col, fmaxf(acc[0] + b0v, 0.f), fmaxf(acc[1] + b1v, 0.f));
                put2<K>(ws.H[0], (mt * 16 + g + 8) * K::LDH + col, fmaxf(acc[2] + b0v, 0.f), fmaxf(acc[3] + b1v, 0.f));
            }
        }
        __syncwarp();
#pragma unroll
        for (int l = 1; l < K::NL; ++l) {
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
                for (int nt = 0; nt < HID / 8; ++nt) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                    for (int kt = 0; kt < HID / 16; ++kt) {
                        uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                        for (int s = 0; s < K::NS; ++s) {
                            load_a(af[s], ws.H[l - 1][s], K::LDH, mt * 16, kt * 16);
                            load_b(bf[s], sm.WH[l - 1][s], K::LDH, nt * 8, kt * 16);
                        }
                        mma_planes<K>(acc, af, bf);
                    }
                    const int col = nt * 8 + 2 * q;
                    const float b0v = sm.bh[l - 1][col], b1v = sm.bh[l - 1][col + 1];
                    put2<K>(ws.H[l], (mt * 16 + g) * K::LDH + col, fmaxf(acc[0] + b0v, 0.f), fmaxf(acc[1] + b1v, 0.f));
                    put2<K>(ws.H[l], (mt * 16 + g + 8) * K::LDH + col, fmaxf(acc[2] + b0v, 0.f),
                            fmaxf(acc[3] + b1v, 0.f));
                }
            }
            __syncwarp();
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < HID / 16; ++kt) {
                uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                for (int s = 0; s < K::NS; ++s) {
                    load_a(af[s], ws.H[K::NL - 1][s], K::LDH, mt * 16, kt * 16);
                    load_b(bf[s], sm.WO[s], K::LDH, 0, kt * 16);
                }
                mma_planes<K>(acc, af, bf);
            }
            if (q < 2) {
                const int col = 2 * q;
                ws.scr[(mt * 16 + g) * K::LDS + col] = acc[0];
                ws.scr[(mt * 16 + g) * K::LDS + col + 1] = acc[1];
                ws.scr[(mt * 16 + g + 8) * K::LDS + col] = acc[2];
                ws.scr[(mt * 16 + g + 8) * K::LDS + col + 1] = acc[3];
            }
        }
        __syncwarp();

        // ---------------- blend, loss, dL/dcolour, output-layer gradient ---------
        float dz[3] = {0.f, 0.f, 0.f};
        float dxd[4] = {0.f, 0.f, 0.f, 0.f};  // direct gradient of x[0..3] through the blend
        if (valid) {
            const float res = x[3];
            float s[3], col[3], tg[3];
            float l1 = 0.f;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                s[c] = 1.f / (1.f + expf(-(ws.scr[lane * K::LDS + c] + sm.bo[c])));
                col[c] = mask ? (1.f - res) * x[c] + res * s[c] : 1.f;
                tg[c] = target_at(a, p, c);
                const float diff = col[c] - tg[c];
                loss_acc += diff * diff;
                const float gc = 2.f * diff * a.inv_n;
                a.color[p * 3 + c] = col[c];
                a.grad_color[p * 3 + c] = gc;
                l1 += fabsf(diff);
                if (mask) {
                    dxd[c] = (1.f - res) * gc;
                    dxd[3] += (s[c] - x[c]) * gc;
                    dz[c] = res * gc * s[c] * (1.f - s[c]);
                }
            }
            a.l1[p] = l1;
        }
#pragma unroll
        for (int s = 0; s < K::NS; ++s) {
            uint32_t h01, l01, h2, l2;
            split_bf16(dz[0], dz[1], h01, l01);
            split_bf16(dz[2], 0.f, h2, l2);
            if (!K::SPLIT) { h01 = pack_bf16(dz[0], dz[1]); h2 = pack_bf16(dz[2], 0.f); }
            __nv_bfloat16* dr = ws.DZO[s] + lane * K::LDO;
            *reinterpret_cast<uint4*>(dr) = s == 0 ? make_uint4(h01, h2, 0u, 0u) : make_uint4(l01, l2, 0u, 0u);
            *reinterpret_cast<uint4*>(dr + 8) = make_uint4(0u, 0u, 0u, 0u);
        }
        // output-layer bias gradient: column sums of dz over the warp
        if (K::REG_GRADS) {
#pragma unroll
            for (int c = 0; c < 3; ++c) gbo[c] += dz[c];
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float v = dz[c];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) atomicAdd(&sm.g[K::P_BO + c], v);
            }
        }
        __syncwarp();

        // ---------------- MLP backward ------------------------------------------
        // dWo[o][h] += sum_px dz[px][o] * H_last[px][h]  (REG_GRADS; else per round below)
#pragma unroll
        for (int nt = 0; nt < (K::REG_GRADS ? HID / 8 : 0); ++nt) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            float* d = K::REG_GRADS ? gwo[nt < GWO ? nt : 0] : acc;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt) {
                uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                for (int s = 0; s < K::NS; ++s) {
                    load_a_t(af[s], ws.DZO[s], K::LDO, kt * 16, 0);
                    load_b_t(bf[s], ws.H[K::NL - 1][s], K::LDH, kt * 16, nt * 8);
                }
                mma_planes<K>(d, af, bf);
            }
            if (!K::REG_GRADS && g < K::OUT) {
                atomicAdd(&sm.g[K::P_WO + g * HID + nt * 8 + 2 * q], acc[0]);
                atomicAdd(&sm.g[K::P_WO + g * HID + nt * 8 + 2 * q + 1], acc[1]);
            }
        }
        // dZ_last = (dz . Wo) * relu'(H_last)
        int cur = 0;
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
            for (int nt = 0; nt < HID / 8; ++nt) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                for (int s = 0; s < K::NS; ++s) {
                    load_a(af[s], ws.DZO[s], K::LDO, mt * 16, 0);
                    load_b_t(bf[s], sm.WO[s], K::LDH, 0, nt * 8);
                }
                mma_planes<K>(acc, af, bf);
                const int col = nt * 8 + 2 * q;
                const __nv_bfloat16* h = ws.H[K::NL - 1][0];
                const float2 lo = relu_gate(h + (mt * 16 + g) * K::LDH + col, make_float2(acc[0], acc[1]));
                const float2 hi = relu_gate(h + (mt * 16 + g + 8) * K::LDH + col, make_float2(acc[2], acc[3]));
                put2<K>(ws.DH[cur], (mt * 16 + g) * K::LDH + col, lo.x, lo.y);
                put2<K>(ws.DH[cur], (mt * 16 + g + 8) * K::LDH + col, hi.x, hi.y);
                const int pb = K::NL == 1 ? K::P_B0 : K::P_WH + (K::NL - 2) * (HID * HID + HID) + HID * HID;
                float s0 = lo.x + hi.x, s1 = lo.y + hi.y;
                if (K::REG_GRADS) {
                    gbh[nt < GWO ? nt : 0][0] += s0;
                    gbh[nt < GWO ? nt : 0][1] += s1;
                } else {
#pragma unroll
                    for (int o = 4; o < 32; o <<= 1) {
                        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                    }
                    if (g == 0) {
                        atomicAdd(&sm.g[pb + col], s0);
                        atomicAdd(&sm.g[pb + col + 1], s1);
                    }
                }
            }
        }
        __syncwarp();
        // hidden layers, last to first
#pragma unroll
        for (int l = K::NL - 1; l >= 0; --l) {
            const __nv_bfloat16* ain[K::NS];
            const __nv_bfloat16* wl[K::NS];
#pragma unroll
            for (int s = 0; s < K::NS; ++s) {
                ain[s] = l == 0 ? ws.X[s] : ws.H[l > 0 ? l - 1 : 0][s];
                wl[s] = l == 0 ? sm.W0[s] : sm.WH[l > 0 ? l - 1 : 0][s];
            }
            const int ldin = l == 0 ? K::LDX : K::LDH;
            const int nin = l == 0 ? IN_PAD : HID;
            const int ldw = l == 0 ? K::LDX : K::LDH;
            const int pw = l == 0 ? K::P_W0 : K::P_WH + (l - 1) * (HID * HID + HID);
            const int win = l == 0 ? K::IN_REAL : HID;  // row length of the packed W_l
            // dW_l[h][i] += sum_px dZ_l[px][h] * A_in[px][i]  (REG_GRADS; else per round below)
#pragma unroll
            for (int mh = 0; mh < (K::REG_GRADS ? HID / 16 : 0); ++mh) {
#pragma unroll
                for (int ni = 0; ni < nin / 8; ++ni) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
                    float* d = K::REG_GRADS ? gw0[mh < GW0M ? mh : 0][ni < GW0N ? ni : 0] : acc;
#pragma unroll
                    for (int kt = 0; kt < 2; ++kt) {
                        uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                        for (int s = 0; s < K::NS; ++s) {
                            load_a_t(af[s], ws.DH[cur][s], K::LDH, kt * 16, mh * 16);
                            load_b_t(bf[s], ain[s], ldin, kt * 16, ni * 8);
                        }
                        mma_planes<K>(d, af, bf);
                    }
                    if (K::REG_GRADS) continue;
                    const int i0 = ni * 8 + 2 * q;
                    const int h0 = mh * 16 + g;
                    if (i0 < win) {
                        atomicAdd(&sm.g[pw + h0 * win + i0], acc[0]);
                        atomicAdd(&sm.g[pw + (h0 + 8) * win + i0], acc[2]);
                    }
                    if (i0 + 1 < win) {
                        atomicAdd(&sm.g[pw + h0 * win + i0 + 1], acc[1]);
                        atomicAdd(&sm.g[pw + (h0 + 8) * win + i0 + 1], acc[3]);
                    }
                }
            }
            // dA_in = dZ_l . W_l
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
                for (int ni = 0; ni < nin / 8; ++ni) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                    for (int kt = 0; kt < HID / 16; ++kt) {
                        uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                        for (int s = 0; s < K::NS; ++s) {
                            load_a(af[s], ws.DH[cur][s], K::LDH, mt * 16, kt * 16);
                            load_b_t(bf[s], wl[s], ldw, kt * 16, ni * 8);
                        }
                        mma_planes<K>(acc, af, bf);
                    }
                    const int col = ni * 8 + 2 * q;
                    if (l == 0) {
                        ws.scr[(mt * 16 + g) * K::LDS + col] = acc[0];
                        ws.scr[(mt * 16 + g) * K::LDS + col + 1] = acc[1];
                        ws.scr[(mt * 16 + g + 8) * K::LDS + col] = acc[2];
                        ws.scr[(mt * 16 + g + 8) * K::LDS + col + 1] = acc[3];
                    } else {
                        const __nv_bfloat16* h = ws.H[l > 0 ? l - 1 : 0][0];
                        const float2 lo = relu_gate(h + (mt * 16 + g) * K::LDH + col, make_float2(acc[0], acc[1]));
                        const float2 hi = relu_gate(h + (mt * 16 + g + 8) * K::LDH + col, make_float2(acc[2], acc[3]));
                        put2<K>(ws.DH[cur ^ 1], (mt * 16 + g) * K::LDH + col, lo.x, lo.y);
                        put2<K>(ws.DH[cur ^ 1], (mt * 16 + g + 8) * K::LDH + col, hi.x, hi.y);
                        const int pb = l - 1 == 0 ? K::P_B0 : K::P_WH + (l - 2) * (HID * HID + HID) + HID * HID;
                        float s0 = lo.x + hi.x, s1 = lo.y + hi.y;
#pragma unroll
                        for (int o = 4; o < 32; o <<= 1) {
                            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                        }
                        if (g == 0) {
                            atomicAdd(&sm.g[pb + col], s0);
                            atomicAdd(&sm.g[pb + col + 1], s1);
                        }
                    }
                }
            }
            __syncwarp();
            cur ^= 1;
        }

        // ---------------- feature-gradient scatter --------------------------------
        if (mask) {
            float dx[K::C];
#pragma unroll
            for (int c = 0; c < K::C; ++c) dx[c] = ws.scr[lane * K::LDS + c] + (c < 4 ? dxd[c] : 0.f);
            float* tg = a.grad_feat + (size_t)t * a.S * K::C;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float* dst = tg + (size_t)idx[k] * K::C;
#pragma unroll
                for (int c = 0; c < K::C; c += 4)
                    atomicAdd(reinterpret_cast<float4*>(dst + c),
                              make_float4(wgt[k] * dx[c], wgt[k] * dx[c + 1], wgt[k] * dx[c + 2], wgt[k] * dx[c + 3]));
            }
        }
        __syncwarp();
        ran = true;
      } while (false);
      if (!K::REG_GRADS) {
        // ---------------- weight gradients of the round's chunks ---------------------
        // Warp w owns the hidden-row m-tiles mh = w, w + WARPS, ... of every dW_l and
        // the hidden n-tiles nt = w, w + WARPS, ... of dWo, and sums them over the
        // chunks of all the CTA's warps that ran the MLP; owned entries of sm.g are
        // plain read-modify-writes.
        if (lane == 0) sm.ran[warp] = ran ? 1 : 0;
        __syncthreads();
#pragma unroll
        for (int l = 0; l < K::NL; ++l) {
            const int buf = (K::NL - 1 - l) & 1;  // the DH buffer that holds dZ_l
            const int ldin = l == 0 ? K::LDX : K::LDH;
            const int nin = l == 0 ? IN_PAD : HID;
            const int pw = l == 0 ? K::P_W0 : K::P_WH + (l - 1) * (HID * HID + HID);
            const int win = l == 0 ? K::IN_REAL : HID;
            for (int mh = warp; mh < HID / 16; mh += K::WARPS) {
#pragma unroll
                for (int ni = 0; ni < nin / 8; ++ni) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
                    for (int src = 0; src < K::WARPS; ++src) {
                        if (!sm.ran[src]) continue;  // CTA-uniform
                        const ShadeWarpSmem<K>& os = sm.w[src];
#pragma unroll
                        for (int kt = 0; kt < 2; ++kt) {
                            uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                            for (int s2 = 0; s2 < K::NS; ++s2) {
                                load_a_t(af[s2], os.DH[buf][s2], K::LDH, kt * 16, mh * 16);
                                load_b_t(bf[s2], l == 0 ? os.X[s2] : os.H[l > 0 ? l - 1 : 0][s2], ldin, kt * 16,
                                         ni * 8);
                            }
                            mma_planes<K>(acc, af, bf);
                        }
                    }
                    const int i0 = ni * 8 + 2 * q, h0 = mh * 16 + g;
                    if (i0 < win) {
                        sm.g[pw + h0 * win + i0] += acc[0];
                        sm.g[pw + (h0 + 8) * win + i0] += acc[2];
                    }
                    if (i0 + 1 < win) {
                        sm.g[pw + h0 * win + i0 + 1] += acc[1];
                        sm.g[pw + (h0 + 8) * win + i0 + 1] += acc[3];
                    }
                }
            }
        }
        for (int nt = warp; nt < HID / 8; nt += K::WARPS) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            for (int src = 0; src < K::WARPS; ++src) {
                if (!sm.ran[src]) continue;
                const ShadeWarpSmem<K>& os = sm.w[src];
#pragma unroll
                for (int kt = 0; kt < 2; ++kt) {
                    uint32_t af[K::NS][4], bf[K::NS][2];
#pragma unroll
                    for (int s2 = 0; s2 < K::NS; ++s2) {
                        load_a_t(af[s2], os.DZO[s2], K::LDO, kt * 16, 0);
                        load_b_t(bf[s2], os.H[K::NL - 1][s2], K::LDH, kt * 16, nt * 8);
                    }
                    mma_planes<K>(acc, af, bf);
                }
            }
            if (g < K::OUT) {
                sm.g[K::P_WO + g * HID + nt * 8 + 2 * q] += acc[0];
                sm.g[K::P_WO + g * HID + nt * 8 + 2 * q + 1] += acc[1];
            }
        }
        __syncthreads();  // the warps' tiles are rewritten in the next round
      }
    }

    if (K::REG_GRADS) {
        // W0[h][i]: tile (mh, ni) holds rows h0 = mh*16 + g (+8), columns i0 = ni*8 + 2q (+1)
#pragma unroll
        for (int mh = 0; mh < GW0M; ++mh)
#pragma unroll
            for (int ni = 0; ni < GW0N; ++ni) {
                const int i0 = ni * 8 + 2 * q, h0 = mh * 16 + g;
                if (i0 < K::IN_REAL) {
                    atomicAdd(&sm.g[K::P_W0 + h0 * K::IN_REAL + i0], gw0[mh][ni][0]);
                    atomicAdd(&sm.g[K::P_W0 + (h0 + 8) * K::IN_REAL + i0], gw0[mh][ni][2]);
                }
                if (i0 + 1 < K::IN_REAL) {
                    atomicAdd(&sm.g[K::P_W0 + h0 * K::IN_REAL + i0 + 1], gw0[mh][ni][1]);
                    atomicAdd(&sm.g[K::P_W0 + (h0 + 8) * K::IN_REAL + i0 + 1], gw0[mh][ni][3]);
                }
            }
#pragma unroll
        for (int nt = 0; nt < GWO; ++nt) {
            if (g < K::OUT) {
                atomicAdd(&sm.g[K::P_WO + g * HID + nt * 8 + 2 * q], gwo[nt][0]);
                atomicAdd(&sm.g[K::P_WO + g * HID + nt * 8 + 2 * q + 1], gwo[nt][1]);
            }
            // hidden bias: sum over the rows g of the lane's columns
            float s0 = gbh[nt][0], s1 = gbh[nt][1];
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
    }

    // ---- CTA reduction of the loss and the parameter gradients ----------------
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o);
    if (lane == 0) sm.loss[warp] = loss_acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < K::WARPS; ++w) s += sm.loss[w];
        atomicAdd(a.loss_sum, s);
    }
    for (int i = threadIdx.x; i < K::NPARAM; i += blockDim.x)
        if (sm.g[i] != 0.f) atomicAdd(a.grad_params + i, sm.g[i]);
}

}  // namespace dsb
