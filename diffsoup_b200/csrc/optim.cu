// diffsoup_b200/csrc/optim.cu -- the optimiser updates that follow the
// training step: VectorAdam for the soup's vertex positions
// (python/diffsoup/optimize.py:7-68) and Adam for the neural features,
// opacities and MLP (torch.optim.Adam as examples/02_synthetic.py:310-315
// uses it: no weight decay, no amsgrad).  One fused elementwise pass each,
// memory bound: a parameter, its gradient and its moments are read once and
// written once.  The step count lives in device memory and is advanced by the
// call itself, so an update captures into a CUDA graph with the step.
#include <cmath>

#include "common.cuh"

namespace dsb {

// Bias corrections of step t (the count after this update's increment).
struct AdamScale {
    float b1, b2, one_m_b1, one_m_b2, step_size, bc2_sqrt;
};

// The hyperparameters arrive in double, as torch's Python scalars: the
// complements 1 - beta are formed in double and then rounded, like torch's
// alpha / weight arguments.
__device__ __forceinline__ AdamScale adam_scale(const int* step, double lr, double b1, double b2) {
    const double t = (double)(*step + 1);
    const double bc1 = 1.0 - pow(b1, t), bc2 = 1.0 - pow(b2, t);
    AdamScale s;
    s.b1 = (float)b1;
    s.b2 = (float)b2;
    s.one_m_b1 = (float)(1.0 - b1);
    s.one_m_b2 = (float)(1.0 - b2);
    s.step_size = (float)(lr / bc1);
    s.bc2_sqrt = (float)sqrt(bc2);
    return s;
}

// torch.optim.Adam, one element: m <- m + (1-b1)(g - m), v <- b2 v + (1-b2) g^2,
// p <- p - lr/bc1 * m / (sqrt(v)/sqrt(bc2) + eps).
__device__ __forceinline__ void adam_one(float& p, float g, float& m, float& v, const AdamScale& s, float eps) {
    m = fmaf(s.one_m_b1, g - m, m);
    v = fmaf(s.one_m_b2 * g, g, s.b2 * v);
    p = p - s.step_size * m / (sqrtf(v) / s.bc2_sqrt + eps);
}

__global__ void __launch_bounds__(kThreads) adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g,
                                                        float* __restrict__ m, float* __restrict__ v,
                                                        const int* __restrict__ step, double lr, double b1,
                                                        double b2, float eps, int vec4) {
    const AdamScale s = adam_scale(step, lr, b1, b2);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (vec4) {
        const int64_t n4 = n >> 2;
        for (; i < n4; i += stride) {
            float4 pp = reinterpret_cast<float4*>(p)[i];
            const float4 gg = reinterpret_cast<const float4*>(g)[i];
            float4 mm = reinterpret_cast<float4*>(m)[i], vv = reinterpret_cast<float4*>(v)[i];
            adam_one(pp.x, gg.x, mm.x, vv.x, s, eps);
            adam_one(pp.y, gg.y, mm.y, vv.y, s, eps);
            adam_one(pp.z, gg.z, mm.z, vv.z, s, eps);
            adam_one(pp.w, gg.w, mm.w, vv.w, s, eps);
            reinterpret_cast<float4*>(p)[i] = pp;
            reinterpret_cast<float4*>(m)[i] = mm;
            reinterpret_cast<float4*>(v)[i] = vv;
        }
        i = (n4 << 2) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // the n % 4 tail
    }
    for (; i < n; i += stride) {
        float pp = p[i], mm = m[i], vv = v[i];
        adam_one(pp, g[i], mm, vv, s, eps);
        p[i] = pp;
        m[i] = mm;
        v[i] = vv;
    }
}

// VectorAdam, one row of `dim` components sharing one second moment:
// g1 <- b1 g1 + (1-b1) g, g2 <- b2 g2 + (1-b2) |g|^2,
// p <- p - lr * (g1/bc1) / (sqrt(g2/bc2) + 1e-8)   (optimize.py:51-68).
template <int D>
__global__ void __launch_bounds__(kThreads) vector_adam_kernel(int64_t rows, int dim, float* __restrict__ p,
                                                               const float* __restrict__ g, float* __restrict__ g1,
                                                               float* __restrict__ g2, const int* __restrict__ step,
                                                               double lr_d, double b1_d, double b2_d) {
    const double t = (double)(*step + 1);
    const float bc1 = (float)(1.0 - pow(b1_d, t)), bc2 = (float)(1.0 - pow(b2_d, t));
    const float lr = (float)lr_d, b1 = (float)b1_d, b2 = (float)b2_d;
    const float c1 = (float)(1.0 - b1_d), c2 = (float)(1.0 - b2_d);
    const int n = D > 0 ? D : dim;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = r * n;
        float sq = 0.f;
        for (int k = 0; k < n; ++k) {
            const float gk = g[o + k];
            sq = fmaf(gk, gk, sq);
            g1[o + k] = b1 * g1[o + k] + c1 * gk;
        }
        const float m2 = b2 * g2[r] + c2 * sq;
        g2[r] = m2;
        const float denom = sqrtf(m2 / bc2) + 1e-8f;
        for (int k = 0; k < n; ++k) p[o + k] -= lr * (g1[o + k] / bc1) / denom;
    }
}

__global__ void advance_step_kernel(int* step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

static unsigned grid_for(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)sm_count() * 8;
    return (unsigned)(b < 1 ? 1 : (b < cap ? b : cap));
}

}  // namespace dsb

using namespace dsb;

extern "C" {

int ds_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, double lr,
                 double beta1, double beta2, double eps, int* step, ds_stream_t stream) {
    DS_CHECK_ARG(n >= 0, "adam_step: n < 0");
    DS_CHECK_ARG(step != nullptr && (n == 0 || (param && grad && exp_avg && exp_avg_sq)), "adam_step: null pointer");
    DS_CHECK_ARG(beta1 >= 0.0 && beta1 < 1.0 && beta2 >= 0.0 && beta2 < 1.0, "adam_step: betas outside [0, 1)");
    cudaStream_t st = (cudaStream_t)stream;
    if (n > 0) {
        const bool v4 = n >= 4 && (((uintptr_t)param | (uintptr_t)grad | (uintptr_t)exp_avg | (uintptr_t)exp_avg_sq) & 15) == 0;
        adam_kernel<<<grid_for(v4 ? n / 4 : n), kThreads, 0, st>>>(n, param, grad, exp_avg, exp_avg_sq, step, lr,
                                                                   beta1, beta2, (float)eps, v4 ? 1 : 0);
    }
    advance_step_kernel<<<1, 32, 0, st>>>(step);
    return check_launch("adam_step");
}

int ds_vector_adam_step(float* param, const float* grad, float* g1, float* g2, int64_t rows, int dim, double lr,
                        double beta1, double beta2, int* step, ds_stream_t stream) {
    DS_CHECK_ARG(rows >= 0 && dim > 0, "vector_adam_step: bad shape (%lld rows of %d)", (long long)rows, dim);
    DS_CHECK_ARG(step != nullptr && (rows == 0 || (param && grad && g1 && g2)), "vector_adam_step: null pointer");
    DS_CHECK_ARG(beta1 >= 0.0 && beta1 < 1.0 && beta2 >= 0.0 && beta2 < 1.0,
                 "vector_adam_step: betas outside [0, 1)");
    cudaStream_t st = (cudaStream_t)stream;
    if (rows > 0) {
        if (dim == 3)
            vector_adam_kernel<3><<<grid_for(rows), kThreads, 0, st>>>(rows, dim, param, grad, g1, g2, step, lr, beta1,
                                                                       beta2);
        else
            vector_adam_kernel<0><<<grid_for(rows), kThreads, 0, st>>>(rows, dim, param, grad, g1, g2, step, lr, beta1,
                                                                       beta2);
    }
    advance_step_kernel<<<1, 32, 0, st>>>(step);
    return check_launch("vector_adam_step");
}

}  // extern "C"
