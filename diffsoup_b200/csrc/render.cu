// diffsoup_b200/csrc/render.cu -- headless restatement of the viewer's
// deferred shading (viewer/src/viewer.cpp:169-340, one frame of its benchmark
// loop :861-909): the inference render of a trained soup without a window or
// a graphics API.
//
// The viewer draws a frame in two passes.
//   geometry pass (viewer.cpp:169-238): every triangle is rasterized with a
//     depth test; a fragment interpolates two RGBA8 LUTs over the lattice cell
//     of its barycentrics at level uLevel and is discarded when the
//     interpolated opacity b.a is below 0.5, so each pixel keeps the nearest
//     fragment whose opacity is at least 0.5.  Here the tiled rasterizer does
//     that (csrc/tiled.cu, threshold mode 0 with 0.5) on the opacity channel
//     of the LUT, decoded once to FP32 [T,S].
//   post pass (viewer.cpp:241-341): per pixel, the LUT interpolation A (rgba)
//     and B (rgb), the view direction normalize(near - far) through the
//     inverse MVP at the pixel centre, its SH2 encoding, a 16 -> 16 -> 16 -> 3
//     MLP (ReLU, ReLU, sigmoid) on x = [A.rgba, B.rgb, sh0..8] and the blend
//     mix(A.rgb, mlp, A.a); pixels that kept no fragment show the background
//     (the clear colour of buffer A, viewer.cpp:870-871).
// The frame's image is written as FP32 rgb and/or RGBA8 (the viewer's final
// GL_RGBA8 target), rows in framebuffer order (row 0 at NDC y = -1, as
// glReadPixels returns them).  The post pass runs one pixel per lane: the LUT
// interpolation and view encoding in FP32 as the shader, the MLP of a warp's 32
// pixels on the tensor cores in 3xTF32 (FP32 accuracy, below).
#include "geometry.cuh"

namespace dsb {


// UNORM8 decode c / 255, correctly rounded: q = c * (1/255) rounded, then one
// Newton correction with the exact residual c - 255 q (checked exhaustively
// for the 256 codes against the correctly rounded quotient; c * (1/255) alone
// differs from it for 126 of them).
__device__ __forceinline__ float unorm8(unsigned c) {
    const float cf = (float)c, r = 1.f / 255.f;
    const float q = __fmul_rn(cf, r);
    return __fmaf_rn(__fmaf_rn(-q, 255.f, cf), r, q);
}

__device__ __forceinline__ void add_texel(float4& acc, uchar4 t, float w) {
    acc.x = fmaf(unorm8(t.x), w, acc.x);
    acc.y = fmaf(unorm8(t.y), w, acc.y);
    acc.z = fmaf(unorm8(t.z), w, acc.z);
    acc.w = fmaf(unorm8(t.w), w, acc.w);
}

// ---------------------------------------------------------------------------
// The MLP on the tensor cores in 3xTF32: every FP32 operand v is split into
// hi = tf32(v) and lo = tf32(v - hi), and a product is lo*hi + hi*lo + hi*hi
// with FP32 accumulation (the lo*lo term, below 2^-22 of the product, is
// dropped), which keeps the FP32 shader's accuracy at a tenth of the issue
// cost of scalar FMAs.  A warp shades 32 pixels as a 32 x 16 activation tile
// (two m16 tiles) with mma.sync m16n8k8 tf32.  Tiles go through shared memory
// between layers (rows of kActStride floats: the fragment reads of a quarter
// warp fall in distinct banks).
// ---------------------------------------------------------------------------
constexpr int kActStride = 20;
constexpr int kRenderWarps = kThreads / 32;

__device__ __forceinline__ uint32_t to_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r;
}

__device__ __forceinline__ void split_tf32(float v, uint32_t& hi, uint32_t& lo) {
    hi = to_tf32(v);
    lo = to_tf32(v - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Weights as the B operand (k = input, n = output), split once per block:
// hi and lo planes of rows n (outputs) x kActStride (inputs, 16 used).
struct RenderWeights {
    uint32_t hi[40 * kActStride];  // layer 1 rows 0..15, layer 2 rows 16..31, layer 3 rows 32..39 (3 used)
    uint32_t lo[40 * kActStride];
    float bias[40];
};

// One layer, 16 inputs -> NT * 8 outputs, on the warp's activation tile:
// act[32][kActStride] holds the inputs and receives the outputs (ReLU'd when
// RELU), written after every lane has read its fragments.
template <int NT, bool RELU>
__device__ __forceinline__ void mlp_layer(float* act, const RenderWeights& w, int row0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    float d[2][NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
        const float c0 = w.bias[row0 + nt * 8 + 2 * t], c1 = w.bias[row0 + nt * 8 + 2 * t + 1];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            d[mt][nt][0] = c0; d[mt][nt][1] = c1; d[mt][nt][2] = c0; d[mt][nt][3] = c1;
        }
    }
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
        uint32_t ahi[2][4], alo[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                split_tf32(act[(mt * 16 + g + (i & 1) * 8) * kActStride + kt * 8 + t + (i >> 1) * 4], ahi[mt][i],
                           alo[mt][i]);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int wb = (row0 + nt * 8 + g) * kActStride + kt * 8 + t;
            const uint32_t bh0 = w.hi[wb], bh1 = w.hi[wb + 4], bl0 = w.lo[wb], bl1 = w.lo[wb + 4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                mma_tf32(d[mt][nt], alo[mt], bh0, bh1);
                mma_tf32(d[mt][nt], ahi[mt], bl0, bl1);
                mma_tf32(d[mt][nt], ahi[mt], bh0, bh1);
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float2 v = make_float2(d[mt][nt][2 * h], d[mt][nt][2 * h + 1]);
                if (RELU) {
                    v.x = fmaxf(v.x, 0.f);
                    v.y = fmaxf(v.y, 0.f);
                }
                *reinterpret_cast<float2*>(act + (mt * 16 + g + h * 8) * kActStride + nt * 8 + 2 * t) = v;
            }
    __syncwarp();
}

__global__ void __launch_bounds__(kThreads) deferred_shade_kernel(
    int B, const ds_view_desc* __restrict__ views, int64_t num_pixels, const float4* __restrict__ gbuf, int level,
    int S, const uchar4* __restrict__ lut0, const uchar4* __restrict__ lut1, int64_t num_texels,
    const float* __restrict__ inv_mvp, const float* __restrict__ params, float bg_r, float bg_g, float bg_b,
    float* __restrict__ rgb, uchar4* __restrict__ rgba8) {
    __shared__ RenderWeights w;
    __shared__ __align__(16) float act_all[kRenderWarps][32 * kActStride];
    // params: W1 [16,16], b1 [16], W2 [16,16], b2 [16], W3 [3,16], b3 [3]
    for (int i = threadIdx.x; i < 40 * kActStride; i += blockDim.x) {
        const int n = i / kActStride, k = i - n * kActStride;
        float v = 0.f;
        if (k < 16) {
            if (n < 16) v = params[n * 16 + k];
            else if (n < 32) v = params[272 + (n - 16) * 16 + k];
            else if (n < 35) v = params[544 + (n - 32) * 16 + k];
        }
        split_tf32(v, w.hi[i], w.lo[i]);
    }
    for (int i = threadIdx.x; i < 40; i += blockDim.x)
        w.bias[i] = i < 16 ? params[256 + i] : (i < 32 ? params[528 + i - 16] : (i < 35 ? params[592 + i - 32] : 0.f));
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* act = act_all[warp];
    const int64_t stride = (int64_t)gridDim.x * kRenderWarps * 32;
    int64_t base = ((int64_t)blockIdx.x * kRenderWarps + warp) * 32;
    // the G-buffer of the next chunk is loaded one iteration ahead
    float4 r_next = base + lane < num_pixels ? gbuf[base + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    for (; base < num_pixels; base += stride) {
        const int64_t p = base + lane;
        const bool valid = p < num_pixels;
        const float4 r = r_next;
        r_next = base + stride + lane < num_pixels ? gbuf[base + stride + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
        const int id = (int)r.w - 1;
        const bool covered = valid && id >= 0;
        float out[3] = {bg_r, bg_g, bg_b};
        if (__ballot_sync(0xffffffffu, covered)) {  // warps of empty pixels keep the background
            // view direction through the inverse MVP at the pixel centre (the
            // shader's divisions as the fast reciprocal-based division, which
            // GLSL's own division also allows)
            float sh[9];
            {
                const int64_t q = valid ? p : num_pixels - 1;
                const int b = view_of_pixel(views, B, q);
                const int W = __ldg(&views[b].W), H = __ldg(&views[b].H);
                const int local = (int)(q - __ldg(&views[b].pix_offset));
                const int py = local / W, px = local - py * W;
                const float nx = __fdividef((float)px + 0.5f, (float)W) * 2.f - 1.f;
                const float ny = __fdividef((float)py + 0.5f, (float)H) * 2.f - 1.f;
                const float* M = inv_mvp + (size_t)b * 16;
                float wp[2][3];
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const float nz = s == 0 ? -1.f : 1.f;
                    float c[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        c[k] = __ldg(M + k * 4 + 0) * nx + __ldg(M + k * 4 + 1) * ny + __ldg(M + k * 4 + 2) * nz +
                               __ldg(M + k * 4 + 3);
                    const float cw = fabsf(c[3]) < 1e-20f ? 1e-20f : c[3];
                    wp[s][0] = __fdividef(c[0], cw);
                    wp[s][1] = __fdividef(c[1], cw);
                    wp[s][2] = __fdividef(c[2], cw);
                }
                float d[3] = {wp[0][0] - wp[1][0], wp[0][1] - wp[1][1], wp[0][2] - wp[1][2]};
                const float il = rsqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                sh2_basis(d[0] * il, d[1] * il, d[2] * il, sh);
            }
            float4 A = make_float4(0.f, 0.f, 0.f, 0.f), Bv = make_float4(0.f, 0.f, 0.f, 0.f);
            if (covered) {
                // geometry pass: a = sum_k lut0[c_k] w_k, b = sum_k lut1[c_k] w_k
                uint32_t idx[3];
                float wt[3];
                lattice_cell(r.x, r.y, (uint32_t)level, idx, wt);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int64_t tx = (int64_t)id * S + idx[k];
                    if (tx < num_texels) {
                        add_texel(A, __ldg(lut0 + tx), wt[k]);
                        add_texel(Bv, __ldg(lut1 + tx), wt[k]);
                    }
                }
            }
            // MLP input x = [A.rgba, B.rgb, sh0..8], one row per lane
            float4* row = reinterpret_cast<float4*>(act + lane * kActStride);
            row[0] = A;
            row[1] = make_float4(Bv.x, Bv.y, Bv.z, sh[0]);
            row[2] = make_float4(sh[1], sh[2], sh[3], sh[4]);
            row[3] = make_float4(sh[5], sh[6], sh[7], sh[8]);
            __syncwarp();
            mlp_layer<2, true>(act, w, 0, lane);    // 16 -> 16, ReLU
            mlp_layer<2, true>(act, w, 16, lane);   // 16 -> 16, ReLU
            mlp_layer<1, false>(act, w, 32, lane);  // 16 -> 3 (outputs 3..7 are zero rows)
            if (covered) {
                const float alb[3] = {A.x, A.y, A.z};
#pragma unroll
                for (int o = 0; o < 3; ++o) {
                    const float m = __fdividef(1.f, 1.f + __expf(-act[lane * kActStride + o]));
                    out[o] = fmaf(A.w, m - alb[o], alb[o]);  // mix(albedo, mlp, a)
                }
            }
            __syncwarp();
        }
        if (valid) {
            if (rgb) {
                rgb[p * 3 + 0] = out[0];
                rgb[p * 3 + 1] = out[1];
                rgb[p * 3 + 2] = out[2];
            }
            if (rgba8) {
                uchar4 c;
                c.x = (unsigned char)__float2int_rn(fminf(fmaxf(out[0], 0.f), 1.f) * 255.f);
                c.y = (unsigned char)__float2int_rn(fminf(fmaxf(out[1], 0.f), 1.f) * 255.f);
                c.z = (unsigned char)__float2int_rn(fminf(fmaxf(out[2], 0.f), 1.f) * 255.f);
                c.w = 255;
                rgba8[p] = c;
            }
        }
    }
}

// Opacity channel of the LUT as FP32, alpha[t] = lut1[t].a / 255.
__global__ void __launch_bounds__(kThreads) lut_opacity_kernel(int64_t n, const uchar4* __restrict__ lut1,
                                                               float* __restrict__ alpha) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        alpha[i] = __fdiv_rn((float)__ldg(lut1 + i).w, 255.f);
}

static unsigned pixel_grid(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)sm_count() * 8;
    return (unsigned)(b < 1 ? 1 : (b < cap ? b : cap));
}

static int check_post_args(int B, const ds_view_desc* views, int64_t num_pixels, const float* gbuf, int level,
                           const unsigned char* lut0, const unsigned char* lut1, int64_t num_texels,
                           const float* inv_mvp, const float* mlp_params, const float* rgb,
                           const unsigned char* rgba8) {
    DS_CHECK_ARG(B > 0 && num_pixels >= 0 && num_texels >= 0, "render: bad sizes");
    DS_CHECK_ARG(level >= 0 && level <= 12, "render: level %d outside 0..12", level);
    DS_CHECK_ARG(num_pixels == 0 || (views && gbuf && lut0 && lut1 && inv_mvp && mlp_params && (rgb || rgba8)),
                 "render: null pointer");
    DS_CHECK_ARG(((uintptr_t)gbuf & 15) == 0 && (((uintptr_t)lut0 | (uintptr_t)lut1 | (uintptr_t)rgba8) & 3) == 0,
                 "render: misaligned buffer");
    return DS_OK;
}

static int launch_post(int B, const ds_view_desc* views, int64_t num_pixels, const float* gbuf, int level,
                       const unsigned char* lut0, const unsigned char* lut1, int64_t num_texels,
                       const float* inv_mvp, const float* mlp_params, float bg_r, float bg_g, float bg_b, float* rgb,
                       unsigned char* rgba8, cudaStream_t st) {
    if (num_pixels == 0) return DS_OK;
    deferred_shade_kernel<<<pixel_grid(num_pixels), kThreads, 0, st>>>(
        B, views, num_pixels, reinterpret_cast<const float4*>(gbuf), level, (int)feats_at_level((uint32_t)level),
        reinterpret_cast<const uchar4*>(lut0), reinterpret_cast<const uchar4*>(lut1), num_texels, inv_mvp,
        mlp_params, bg_r, bg_g, bg_b, rgb, reinterpret_cast<uchar4*>(rgba8));
    return check_launch("render_deferred");
}

static size_t al256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace dsb

using namespace dsb;

extern "C" {

int ds_render_lut_opacity(int64_t num_texels, const unsigned char* lut1, float* alpha, ds_stream_t stream) {
    DS_CHECK_ARG(num_texels >= 0, "render_lut_opacity: bad size");
    DS_CHECK_ARG(num_texels == 0 || (lut1 && alpha), "render_lut_opacity: null pointer");
    DS_CHECK_ARG(((uintptr_t)lut1 & 3) == 0, "render_lut_opacity: lut1 not 4-byte aligned");
    if (num_texels == 0) return DS_OK;
    lut_opacity_kernel<<<pixel_grid(num_texels), kThreads, 0, (cudaStream_t)stream>>>(
        num_texels, reinterpret_cast<const uchar4*>(lut1), alpha);
    return check_launch("render_lut_opacity");
}

int ds_render_deferred(int B, const ds_view_desc* views, int64_t num_pixels, const float* gbuf, int level,
                       const unsigned char* lut0, const unsigned char* lut1, int64_t num_texels,
                       const float* inv_mvp, const float* mlp_params, float bg_r, float bg_g, float bg_b,
                       float* rgb, unsigned char* rgba8, ds_stream_t stream) {
    const int rc = check_post_args(B, views, num_pixels, gbuf, level, lut0, lut1, num_texels, inv_mvp, mlp_params,
                                   rgb, rgba8);
    if (rc) return rc;
    return launch_post(B, views, num_pixels, gbuf, level, lut0, lut1, num_texels, inv_mvp, mlp_params, bg_r, bg_g,
                       bg_b, rgb, rgba8, (cudaStream_t)stream);
}

size_t ds_render_workspace_size(int B, int V, int T, int num_tiles, int64_t list_capacity) {
    return al256((size_t)B * V * 4 * sizeof(float)) + ds_tiles_workspace_size(B, T, num_tiles, list_capacity);
}

int ds_render_frame(int B, const ds_view_desc* views, int num_tiles, int64_t num_pixels, int V, const float* verts,
                    int T, const int* faces, const float* mvp, const float* inv_mvp, int level,
                    const unsigned char* lut0, const unsigned char* lut1, int64_t num_texels, const float* alpha,
                    const float* mlp_params, float bg_r, float bg_g, float bg_b, float* gbuf, float* rgb,
                    unsigned char* rgba8, void* workspace, size_t workspace_bytes, int64_t list_capacity,
                    int* status, ds_stream_t stream) {
    int rc = check_post_args(B, views, num_pixels, gbuf, level, lut0, lut1, num_texels, inv_mvp, mlp_params, rgb,
                             rgba8);
    if (rc) return rc;
    const int S = (int)feats_at_level((uint32_t)level);
    DS_CHECK_ARG(V >= 0 && T >= 0 && (T == 0 || (verts && faces && mvp && alpha)) && status != nullptr,
                 "render_frame: null pointer");
    DS_CHECK_ARG((int64_t)T * S <= num_texels, "render_frame: LUT of %lld texels is smaller than %d faces x %d",
                 (long long)num_texels, T, S);
    DS_CHECK_ARG(workspace != nullptr && workspace_bytes >= ds_render_workspace_size(B, V, T, num_tiles, list_capacity),
                 "render_frame: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    float* pos = reinterpret_cast<float*>(workspace);
    void* tiles = reinterpret_cast<char*>(workspace) + al256((size_t)B * V * 4 * sizeof(float));
    const size_t tiles_bytes = workspace_bytes - al256((size_t)B * V * 4 * sizeof(float));
    if ((rc = ds_project_vertices(B, V, verts, mvp, pos, stream))) return rc;
    if ((rc = ds_tiles_bin(B, views, num_tiles, V, pos, T, faces, tiles, tiles_bytes, list_capacity, status, stream)))
        return rc;
    if ((rc = ds_tiles_rasterize(B, views, num_tiles, V, pos, T, faces, level, S, alpha, 0, 0.5f, nullptr, gbuf,
                                 tiles, tiles_bytes, list_capacity, stream)))
        return rc;
    return launch_post(B, views, num_pixels, gbuf, level, lut0, lut1, num_texels, inv_mvp, mlp_params, bg_r, bg_g,
                       bg_b, rgb, rgba8, st);
}

}  // extern "C"
