// diffsoup_b200/csrc/edge.cu -- silhouette/implicit edge gradients and the
// per-fragment opacity auxiliary gradient (kenji-tojo/diffsoup
// src/cuda/rasterize.cu:489-992) behind the C ABI.
#include "edge_math.cuh"

namespace dsb {

// rasterize.cu:653-903: one thread per pixel, 4 neighbours.
__global__ void __launch_bounds__(kThreads) edge_grad_kernel(int B, int H, int W, int C,
                                                             const float* __restrict__ color,
                                                             const float* __restrict__ grad_color,
                                                             const float* __restrict__ rast, int V,
                                                             const float* __restrict__ pos,
                                                             float* __restrict__ grad_pos,
                                                             const int* __restrict__ tri) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t hw = (int64_t)H * W;
    if (idx >= (int64_t)B * hw) return;
    const int b = (int)(idx / hw);
    const int y0 = (int)((idx % hw) / W), x0 = (int)((idx % hw) % W);
    EdgeAccum acc;
    const int it0 = edge_grad_pixel(b, y0, x0, H, W, C, color, grad_color, rast, pos + (size_t)b * V * 4, tri,
                                    b * hw, acc);
    if (it0 < 0 || !acc.any) return;
    float* gp = grad_pos + (size_t)b * V * 4;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int v = __ldg(tri + it0 * 3 + k);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (acc.g[k * 4 + j] != 0.f) atomicAdd(gp + (size_t)v * 4 + j, acc.g[k * 4 + j]);
    }
}

// rasterize.cu:923-971: one thread per fragment.
__global__ void __launch_bounds__(kThreads) aux_fragment_kernel(int H, int W, int C, const float* __restrict__ color,
                                                                const float* __restrict__ target,
                                                                const float* __restrict__ rast, int n,
                                                                const int* __restrict__ frag_pix,
                                                                const float* __restrict__ frag_attrs,
                                                                const float* __restrict__ frag_alpha,
                                                                float* __restrict__ grad_frag_alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = frag_pix[(size_t)i * 3];
    if (b < 0) return;
    const int64_t p = (int64_t)b * H * W + (int64_t)frag_pix[(size_t)i * 3 + 1] * W + frag_pix[(size_t)i * 3 + 2];
    const float4 fa = reinterpret_cast<const float4*>(frag_attrs)[i];
    const float4 rp = reinterpret_cast<const float4*>(rast)[p];
    const int tf = (int)fa.w - 1, tp = (int)rp.w - 1;
    if (tp >= 0 && fa.z > rp.z) return;
    float loss = 0.f;
    for (int c = 0; c < C; ++c) loss += fabsf(color[p * C + c] - target[p * C + c]);
    grad_frag_alpha[i] += aux_alpha_grad(loss, frag_alpha[i], tp >= 0 && tf == tp);
}

}  // namespace dsb

using namespace dsb;

extern "C" {

int ds_backward_edge_grad(int B, int H, int W, int C, const float* color, const float* grad_color, const float* rast,
                          int V, const float* pos, float* grad_pos, const int* tri, ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H >= 0 && W >= 0 && C > 0 && V >= 0, "backward_edge_grad: bad sizes");
    const int64_t n = (int64_t)B * H * W;
    if (n == 0) return DS_OK;
    DS_CHECK_ARG(((uintptr_t)rast & 15) == 0 && ((uintptr_t)pos & 15) == 0,
                 "backward_edge_grad: rast/pos not 16-byte aligned");
    edge_grad_kernel<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(B, H, W, C, color, grad_color, rast, V, pos,
                                                                          grad_pos, tri);
    return check_launch("backward_edge_grad");
}

int ds_backward_opacity_aux_loss(int B, int H, int W, int C, const float* color, const float* target,
                                 const float* rast, int num_frags, const int* frag_pix, const float* frag_attrs,
                                 const float* frag_alpha, float* grad_frag_alpha, ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H >= 0 && W >= 0 && C > 0 && num_frags >= 0, "backward_opacity_aux_loss: bad sizes");
    if (num_frags == 0) return DS_OK;
    DS_CHECK_ARG(((uintptr_t)rast & 15) == 0 && ((uintptr_t)frag_attrs & 15) == 0,
                 "backward_opacity_aux_loss: rast/frag_attrs not 16-byte aligned");
    aux_fragment_kernel<<<blocks_for(num_frags), kThreads, 0, (cudaStream_t)stream>>>(
        H, W, C, color, target, rast, num_frags, frag_pix, frag_attrs, frag_alpha, grad_frag_alpha);
    return check_launch("backward_opacity_aux_loss");
}

}  // extern "C"
