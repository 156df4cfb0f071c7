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
// glReadPixels returns them).  The post pass runs one thread per pixel in FP32
// as the shader does, with the MLP weights in shared memory (every thread reads
// the same weight at the same time, so the reads broadcast).
#include "geometry.cuh"

namespace dsb {

constexpr int kRenderParams = 16 * 16 + 16 + 16 * 16 + 16 + 3 * 16 + 3;  // W1 b1 W2 b2 W3 b3

__device__ __forceinline__ void add_texel(float4& acc, uchar4 t, float w, const float* unorm) {
    acc.x = fmaf(unorm[t.x], w, acc.x);
    acc.y = fmaf(unorm[t.y], w, acc.y);
    acc.z = fmaf(unorm[t.z], w, acc.z);
    acc.w = fmaf(unorm[t.w], w, acc.w);
}

// UNORM8 decode c / 255, correctly rounded (c * (1/255) differs from it for
// 126 of the 256 codes, so it is tabulated once per block).
__device__ __forceinline__ void fill_unorm_table(float* unorm) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) unorm[i] = __fdiv_rn((float)i, 255.f);
}

__global__ void __launch_bounds__(kThreads) deferred_shade_kernel(
    int B, const ds_view_desc* __restrict__ views, int64_t num_pixels, const float4* __restrict__ gbuf, int level,
    int S, const uchar4* __restrict__ lut0, const uchar4* __restrict__ lut1, int64_t num_texels,
    const float* __restrict__ inv_mvp, const float* __restrict__ params, float bg_r, float bg_g, float bg_b,
    float* __restrict__ rgb, uchar4* __restrict__ rgba8) {
    __shared__ float w[kRenderParams];
    __shared__ float unorm[256];
    for (int i = threadIdx.x; i < kRenderParams; i += blockDim.x) w[i] = params[i];
    fill_unorm_table(unorm);
    __syncthreads();
    const float* W1 = w;
    const float* b1 = W1 + 256;
    const float* W2 = b1 + 16;
    const float* b2 = W2 + 256;
    const float* W3 = b2 + 16;
    const float* b3 = W3 + 48;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < num_pixels;
         p += (int64_t)gridDim.x * blockDim.x) {
        const float4 r = gbuf[p];
        const int id = (int)r.w - 1;
        float out[3] = {bg_r, bg_g, bg_b};
        if (id >= 0) {
            // geometry pass: a = sum_k lut0[c_k] w_k, b = sum_k lut1[c_k] w_k
            uint32_t idx[3];
            float wt[3];
            lattice_cell(r.x, r.y, (uint32_t)level, idx, wt);
            float4 A = make_float4(0.f, 0.f, 0.f, 0.f), Bv = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int64_t tx = (int64_t)id * S + idx[k];
                if (tx < num_texels) {
                    add_texel(A, __ldg(lut0 + tx), wt[k], unorm);
                    add_texel(Bv, __ldg(lut1 + tx), wt[k], unorm);
                }
            }
            // post pass: view direction through the inverse MVP at the pixel centre
            const int b = view_of_pixel(views, B, p);
            const int W = __ldg(&views[b].W), H = __ldg(&views[b].H);
            const int local = (int)(p - __ldg(&views[b].pix_offset));
            const int py = local / W, px = local - py * W;
            const float nx = ((float)px + 0.5f) / (float)W * 2.f - 1.f;
            const float ny = ((float)py + 0.5f) / (float)H * 2.f - 1.f;
            const float* M = inv_mvp + (size_t)b * 16;
            float wp[2][3];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const float nz = s == 0 ? -1.f : 1.f;
                float c[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    c[q] = __ldg(M + q * 4 + 0) * nx + __ldg(M + q * 4 + 1) * ny + __ldg(M + q * 4 + 2) * nz +
                           __ldg(M + q * 4 + 3);
                const float cw = fabsf(c[3]) < 1e-20f ? 1e-20f : c[3];
                wp[s][0] = c[0] / cw;
                wp[s][1] = c[1] / cw;
                wp[s][2] = c[2] / cw;
            }
            float d[3] = {wp[0][0] - wp[1][0], wp[0][1] - wp[1][1], wp[0][2] - wp[1][2]};
            const float il = rsqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            d[0] *= il;
            d[1] *= il;
            d[2] *= il;
            float x[16];
            x[0] = A.x; x[1] = A.y; x[2] = A.z; x[3] = A.w;
            x[4] = Bv.x; x[5] = Bv.y; x[6] = Bv.z;
            sh2_basis(d[0], d[1], d[2], x + 7);
            // MLP 16 -> 16 (ReLU) -> 16 (ReLU) -> 3 (sigmoid), W row-major [out, in]
            float y[16], z[16];
#pragma unroll
            for (int o = 0; o < 16; ++o) {
                float acc = b1[o];
#pragma unroll
                for (int i = 0; i < 16; ++i) acc = fmaf(W1[o * 16 + i], x[i], acc);
                y[o] = fmaxf(acc, 0.f);
            }
#pragma unroll
            for (int o = 0; o < 16; ++o) {
                float acc = b2[o];
#pragma unroll
                for (int i = 0; i < 16; ++i) acc = fmaf(W2[o * 16 + i], y[i], acc);
                z[o] = fmaxf(acc, 0.f);
            }
            const float alb[3] = {A.x, A.y, A.z};
#pragma unroll
            for (int o = 0; o < 3; ++o) {
                float acc = b3[o];
#pragma unroll
                for (int i = 0; i < 16; ++i) acc = fmaf(W3[o * 16 + i], z[i], acc);
                const float m = 1.f / (1.f + expf(-acc));
                out[o] = fmaf(A.w, m - alb[o], alb[o]);  // mix(albedo, mlp, a)
            }
        }
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

// Opacity channel of the LUT as FP32, alpha[t] = lut1[t].a / 255.
__global__ void __launch_bounds__(kThreads) lut_opacity_kernel(int64_t n, const uchar4* __restrict__ lut1,
                                                               float* __restrict__ alpha) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        alpha[i] = __fdiv_rn((float)__ldg(lut1 + i).w, 255.f);
}

static unsigned pixel_grid(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)kSMs * 8;
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
