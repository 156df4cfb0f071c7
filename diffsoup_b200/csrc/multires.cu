// diffsoup_b200/csrc/multires.cu -- multi-resolution barycentric features
// (kenji-tojo/diffsoup src/cuda/multires.cu) behind the C ABI.
//
// Forward gathers use 16-byte vector loads when the feature width allows it;
// the scatters use vector atomics (red.global.add.v4.f32, sm_90+) so one
// instruction updates four channels.
#include "geometry.cuh"

namespace dsb {

// multires.cu:130-156: alpha per fragment.
__global__ void __launch_bounds__(kThreads) alpha_kernel(int n, const float* __restrict__ frag_attrs, uint32_t lo,
                                                         uint32_t hi, uint32_t S, const float* __restrict__ alpha_src,
                                                         float* __restrict__ frag_alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = reinterpret_cast<const float4*>(frag_attrs)[i];
    const int t = (int)a.w - 1;
    if (t < 0) return;
    frag_alpha[i] = interp_scalar(a.x, a.y, lo, hi, alpha_src + (size_t)t * S);
}

// multires.cu:178-202
__global__ void __launch_bounds__(kThreads) alpha_backward_kernel(int n, const float* __restrict__ frag_attrs,
                                                                  uint32_t lo, uint32_t hi, uint32_t S,
                                                                  float* __restrict__ grad_alpha_src,
                                                                  const float* __restrict__ grad_frag_alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = reinterpret_cast<const float4*>(frag_attrs)[i];
    const int t = (int)a.w - 1;
    if (t < 0) return;
    const float g = grad_frag_alpha[i];
    float* dst = grad_alpha_src + (size_t)t * S;
    uint32_t off = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; float w[3];
        lattice_cell(a.x, a.y, l, idx, w);
#pragma unroll
        for (int k = 0; k < 3; ++k) atomicAdd(dst + off + idx[k], g * w[k]);
        off += feats_at_level(l);
    }
}

// multires.cu:224-247: features per pixel, accumulated into out.
template <int VEC>
__global__ void __launch_bounds__(kThreads) color_kernel(int64_t n, const float* __restrict__ rast, uint32_t lo,
                                                         uint32_t hi, uint32_t S, int C,
                                                         const float* __restrict__ feat, float* __restrict__ out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 r = reinterpret_cast<const float4*>(rast)[p];
    const int t = (int)r.w - 1;
    if (t < 0) return;
    const float* tf = feat + (size_t)t * S * C;
    float* o = out + (size_t)p * C;
    uint32_t off = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; float w[3];
        lattice_cell(r.x, r.y, l, idx, w);
        if (VEC == 4) {
            for (int c = 0; c < C; c += 4) {
                float4 acc = *reinterpret_cast<float4*>(o + c);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float4 f = __ldg(reinterpret_cast<const float4*>(tf + (size_t)(off + idx[k]) * C + c));
                    acc.x = madd(acc.x, w[k], f.x); acc.y = madd(acc.y, w[k], f.y);
                    acc.z = madd(acc.z, w[k], f.z); acc.w = madd(acc.w, w[k], f.w);
                }
                *reinterpret_cast<float4*>(o + c) = acc;
            }
        } else {
            for (int c = 0; c < C; ++c) {
                float acc = o[c];
#pragma unroll
                for (int k = 0; k < 3; ++k) acc = madd(acc, w[k], __ldg(tf + (size_t)(off + idx[k]) * C + c));
                o[c] = acc;
            }
        }
        off += feats_at_level(l);
    }
}

// multires.cu:268-292: scatter of per-pixel feature gradients.
template <int VEC>
__global__ void __launch_bounds__(kThreads) color_backward_kernel(int64_t n, const float* __restrict__ rast,
                                                                  uint32_t lo, uint32_t hi, uint32_t S, int C,
                                                                  float* __restrict__ grad_feat,
                                                                  const float* __restrict__ grad_out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 r = reinterpret_cast<const float4*>(rast)[p];
    const int t = (int)r.w - 1;
    if (t < 0) return;
    float* tg = grad_feat + (size_t)t * S * C;
    const float* g = grad_out + (size_t)p * C;
    uint32_t off = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; float w[3];
        lattice_cell(r.x, r.y, l, idx, w);
        if (VEC == 4) {
            for (int c = 0; c < C; c += 4) {
                const float4 gv = __ldg(reinterpret_cast<const float4*>(g + c));
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    atomicAdd(reinterpret_cast<float4*>(tg + (size_t)(off + idx[k]) * C + c),
                              make_float4(gv.x * w[k], gv.y * w[k], gv.z * w[k], gv.w * w[k]));
            }
        } else {
            for (int c = 0; c < C; ++c) {
                const float gv = __ldg(g + c);
#pragma unroll
                for (int k = 0; k < 3; ++k) atomicAdd(tg + (size_t)(off + idx[k]) * C + c, gv * w[k]);
            }
        }
        off += feats_at_level(l);
    }
}

// multires.cu:329-369: evaluate levels [lo, hi] at the target lattice vertices.
__global__ void __launch_bounds__(kThreads) accumulate_forward_kernel(int T, uint32_t lo, uint32_t hi, uint32_t target,
                                                                      uint32_t S, uint32_t ST, int C,
                                                                      const float* __restrict__ feat,
                                                                      float* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)T * ST) return;
    const uint32_t t = (uint32_t)(i / ST), k = (uint32_t)(i % ST);
    uint32_t x, y;
    index_to_xy(k, x, y);
    const float R = (float)(1u << target);
    const float b0 = __fdiv_rn((float)x, R), b1 = __fdiv_rn((float)y, R);
    const float* tf = feat + (size_t)t * S * C;
    float* o = out + (size_t)i * C;
    for (int c = 0; c < C; ++c) o[c] = 0.f;
    uint32_t off = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; float w[3];
        lattice_cell(b0, b1, l, idx, w);
        for (int c = 0; c < C; ++c) {
            float acc = o[c];
#pragma unroll
            for (int q = 0; q < 3; ++q) acc = madd(acc, w[q], __ldg(tf + (size_t)(off + idx[q]) * C + c));
            o[c] = acc;
        }
        off += feats_at_level(l);
    }
}

// multires.cu:393-430
__global__ void __launch_bounds__(kThreads) accumulate_backward_kernel(int T, uint32_t lo, uint32_t hi,
                                                                       uint32_t target, uint32_t S, uint32_t ST, int C,
                                                                       float* __restrict__ grad_feat,
                                                                       const float* __restrict__ grad_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)T * ST) return;
    const uint32_t t = (uint32_t)(i / ST), k = (uint32_t)(i % ST);
    uint32_t x, y;
    index_to_xy(k, x, y);
    const float R = (float)(1u << target);
    const float b0 = __fdiv_rn((float)x, R), b1 = __fdiv_rn((float)y, R);
    float* tg = grad_feat + (size_t)t * S * C;
    const float* g = grad_out + (size_t)i * C;
    uint32_t off = 0;
    for (uint32_t l = lo; l <= hi; ++l) {
        uint32_t idx[3]; float w[3];
        lattice_cell(b0, b1, l, idx, w);
        for (int c = 0; c < C; ++c) {
            const float gv = __ldg(g + c);
#pragma unroll
            for (int q = 0; q < 3; ++q) atomicAdd(tg + (size_t)(off + idx[q]) * C + c, gv * w[q]);
        }
        off += feats_at_level(l);
    }
}

static bool levels_ok(int lo, int hi) { return lo >= 0 && hi >= lo && hi <= 12; }
static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

}  // namespace dsb

using namespace dsb;

extern "C" {

int ds_multires_triangle_alpha(int num_frags, const float* frag_attrs, int min_level, int max_level, int S,
                               const float* alpha_src, float* frag_alpha, ds_stream_t stream) {
    DS_CHECK_ARG(num_frags >= 0 && levels_ok(min_level, max_level), "multires_triangle_alpha: bad levels");
    DS_CHECK_ARG((uint32_t)S == total_feats(min_level, max_level), "Invalid feature size.");
    if (num_frags == 0) return DS_OK;
    DS_CHECK_ARG(aligned16(frag_attrs), "multires_triangle_alpha: frag_attrs not 16-byte aligned");
    alpha_kernel<<<blocks_for(num_frags), kThreads, 0, (cudaStream_t)stream>>>(num_frags, frag_attrs, min_level,
                                                                               max_level, S, alpha_src, frag_alpha);
    return check_launch("multires_triangle_alpha");
}

int ds_backward_multires_triangle_alpha(int num_frags, const float* frag_attrs, int min_level, int max_level, int S,
                                        float* grad_alpha_src, const float* grad_frag_alpha, ds_stream_t stream) {
    DS_CHECK_ARG(num_frags >= 0 && levels_ok(min_level, max_level), "backward_multires_triangle_alpha: bad levels");
    DS_CHECK_ARG((uint32_t)S == total_feats(min_level, max_level), "Invalid feature size.");
    if (num_frags == 0) return DS_OK;
    DS_CHECK_ARG(aligned16(frag_attrs), "backward_multires_triangle_alpha: frag_attrs not 16-byte aligned");
    alpha_backward_kernel<<<blocks_for(num_frags), kThreads, 0, (cudaStream_t)stream>>>(
        num_frags, frag_attrs, min_level, max_level, S, grad_alpha_src, grad_frag_alpha);
    return check_launch("backward_multires_triangle_alpha");
}

int ds_multires_triangle_color(int B, int H, int W, const float* rast, int min_level, int max_level, int S, int C,
                               const float* features, float* out, ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H >= 0 && W >= 0 && C > 0 && levels_ok(min_level, max_level),
                 "multires_triangle_color: bad sizes");
    DS_CHECK_ARG((uint32_t)S == total_feats(min_level, max_level), "Invalid feature size.");
    const int64_t n = (int64_t)B * H * W;
    if (n == 0) return DS_OK;
    DS_CHECK_ARG(aligned16(rast), "multires_triangle_color: rast not 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    if (C % 4 == 0 && aligned16(features) && aligned16(out))
        color_kernel<4><<<blocks_for(n), kThreads, 0, st>>>(n, rast, min_level, max_level, S, C, features, out);
    else
        color_kernel<1><<<blocks_for(n), kThreads, 0, st>>>(n, rast, min_level, max_level, S, C, features, out);
    return check_launch("multires_triangle_color");
}

int ds_backward_multires_triangle_color(int B, int H, int W, const float* rast, int min_level, int max_level, int S,
                                        int C, float* grad_features, const float* grad_out, ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H >= 0 && W >= 0 && C > 0 && levels_ok(min_level, max_level),
                 "backward_multires_triangle_color: bad sizes");
    DS_CHECK_ARG((uint32_t)S == total_feats(min_level, max_level), "Invalid feature size.");
    const int64_t n = (int64_t)B * H * W;
    if (n == 0) return DS_OK;
    DS_CHECK_ARG(aligned16(rast), "backward_multires_triangle_color: rast not 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    if (C % 4 == 0 && aligned16(grad_features) && aligned16(grad_out))
        color_backward_kernel<4><<<blocks_for(n), kThreads, 0, st>>>(n, rast, min_level, max_level, S, C,
                                                                     grad_features, grad_out);
    else
        color_backward_kernel<1><<<blocks_for(n), kThreads, 0, st>>>(n, rast, min_level, max_level, S, C,
                                                                     grad_features, grad_out);
    return check_launch("backward_multires_triangle_color");
}

int ds_accumulate_to_level_forward(int T, int min_level, int max_level, int target_level, int S, int S_target, int C,
                                   const float* features, float* out, ds_stream_t stream) {
    DS_CHECK_ARG(T >= 0 && C > 0 && levels_ok(min_level, max_level) && target_level >= 0 && target_level <= 12,
                 "accumulate_to_level_forward: bad sizes");
    DS_CHECK_ARG((uint32_t)S == total_feats(min_level, max_level), "Invalid feature size.");
    DS_CHECK_ARG((uint32_t)S_target == feats_at_level(target_level), "Invalid feature size.");
    const int64_t n = (int64_t)T * S_target;
    if (n == 0) return DS_OK;
    accumulate_forward_kernel<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(
        T, min_level, max_level, target_level, S, S_target, C, features, out);
    return check_launch("accumulate_to_level_forward");
}

int ds_accumulate_to_level_backward(int T, int min_level, int max_level, int target_level, int S, int S_target,
                                    int C, float* grad_features, const float* grad_out, ds_stream_t stream) {
    DS_CHECK_ARG(T >= 0 && C > 0 && levels_ok(min_level, max_level) && target_level >= 0 && target_level <= 12,
                 "accumulate_to_level_backward: bad sizes");
    DS_CHECK_ARG((uint32_t)S == total_feats(min_level, max_level), "Invalid feature size.");
    DS_CHECK_ARG((uint32_t)S_target == feats_at_level(target_level), "Invalid feature size.");
    const int64_t n = (int64_t)T * S_target;
    if (n == 0) return DS_OK;
    accumulate_backward_kernel<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(
        T, min_level, max_level, target_level, S, S_target, C, grad_features, grad_out);
    return check_launch("accumulate_to_level_backward");
}

}  // extern "C"
