// diffsoup_b200/csrc/encoding.cu -- per-pixel view-direction encodings
// (kenji-tojo/diffsoup src/cuda/encoding.cu:9-130).
#include "geometry.cuh"

namespace dsb {

// encoding.cu:89-118 (SH2, 9 coefficients) and the raw direction (3).
template <int K>
__global__ void __launch_bounds__(kThreads) encode_view_kernel(int B, int H, int W, const float* __restrict__ rast,
                                                               const float* __restrict__ inv_mvp,
                                                               float* __restrict__ enc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t hw = (int64_t)H * W;
    if (i >= (int64_t)B * hw) return;
    const int b = (int)(i / hw);
    const int y = (int)((i % hw) / W), x = (int)((i % hw) % W);
    if ((int)reinterpret_cast<const float4*>(rast)[i].w - 1 < 0) return;
    float M[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) M[k] = __ldg(inv_mvp + (size_t)b * 16 + k);
    float d[3];
    view_direction(pix_ndc(x, W), pix_ndc(y, H), M, d);
    float* o = enc + (size_t)i * K;
    if (K == 9) {
        float sh[9];
        sh2_basis(d[0], d[1], d[2], sh);
#pragma unroll
        for (int k = 0; k < 9; ++k) o[k] = sh[k];
    } else {
        o[0] = d[0]; o[1] = d[1]; o[2] = d[2];
    }
}

}  // namespace dsb

using namespace dsb;

extern "C" {

int ds_encode_view_dir_sh2(int B, int H, int W, const float* rast, const float* inv_mvp, float* encoding,
                           ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H >= 0 && W >= 0, "encode_view_dir_sh2: bad sizes");
    const int64_t n = (int64_t)B * H * W;
    if (n == 0) return DS_OK;
    DS_CHECK_ARG(((uintptr_t)rast & 15) == 0, "encode_view_dir_sh2: rast not 16-byte aligned");
    encode_view_kernel<9><<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(B, H, W, rast, inv_mvp, encoding);
    return check_launch("encode_view_dir_sh2");
}

int ds_encode_view_dir(int B, int H, int W, const float* rast, const float* inv_mvp, float* encoding,
                       ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H >= 0 && W >= 0, "encode_view_dir: bad sizes");
    const int64_t n = (int64_t)B * H * W;
    if (n == 0) return DS_OK;
    DS_CHECK_ARG(((uintptr_t)rast & 15) == 0, "encode_view_dir: rast not 16-byte aligned");
    encode_view_kernel<3><<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(B, H, W, rast, inv_mvp, encoding);
    return check_launch("encode_view_dir");
}

}  // extern "C"
