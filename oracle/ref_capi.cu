// oracle/ref_capi.cu -- plain C entry points over the reference's own CUDA
// launchers (kenji-tojo/diffsoup src/cuda/*.cuh), replacing its nanobind
// module (src/main.cpp:30-304, which cannot be built here: nanobind is not
// installed).  TEST INFRASTRUCTURE ONLY: linked with the unmodified reference
// sources into oracle/_ref/ by oracle/Makefile and used as the parity
// reference for the oracle and for the product kernels.
//
// Each wrapper forwards its arguments unchanged, with the shape parameters the
// nanobind lambdas derive from tensor shapes passed explicitly.

#include <cstdint>
#include <cuda_runtime.h>

#include "rasterize.cuh"
#include "multires.cuh"
#include "encoding.cuh"

namespace dc = diffsoup::cuda;

extern "C" {

// main.cpp:30-48
int dsref_compute_triangle_rects(int H, int W, int B, int V, const float* pos, int T, const int* tri,
                                 int* rects, int* prefix) {
    return dc::compute_triangle_rects(H, W, B, V, pos, T, tri, rects, prefix);
}

// main.cpp:50-76
void dsref_compute_fragments(int H, int W, int B, int V, const float* pos, int T, const int* tri,
                             const int* prefix, const int* rects, int num_frags, int* frag_pix, float* frag_attrs) {
    dc::compute_fragments(H, W, V, pos, T, tri, B * T, num_frags, prefix, rects, frag_pix, frag_attrs);
}

// main.cpp:78-94
void dsref_depth_test(int B, int H, int W, int num_frags, const int* frag_pix, const float* frag_attrs,
                      const float* frag_alpha, const float* alpha_thresh, float* rast) {
    dc::depth_test(B, H, W, num_frags, frag_pix, frag_attrs, frag_alpha, alpha_thresh, rast);
}

// main.cpp:96-108
int dsref_filter_valid_fragments(int num_frags, const int* frag_pix, const float* frag_attrs, int* pix_out,
                                 float* attrs_out) {
    return dc::filter_valid_fragments(num_frags, frag_pix, frag_attrs, pix_out, attrs_out);
}

// main.cpp:112-130
void dsref_backward_edge_grad(int B, int H, int W, int C, const float* color, const float* grad_color,
                              const float* rast, int V, const float* pos, float* grad_pos, const int* tri) {
    dc::backward_edge_grad(B, H, W, C, color, grad_color, rast, V, pos, grad_pos, tri);
}

// main.cpp:134-154
void dsref_backward_opacity_aux_loss(int B, int H, int W, int C, const float* color, const float* target,
                                     const float* rast, int num_frags, const int* frag_pix, const float* frag_attrs,
                                     const float* frag_alpha, float* grad_frag_alpha) {
    dc::backward_opacity_aux_loss(B, H, W, C, color, target, rast, num_frags, frag_pix, frag_attrs, frag_alpha,
                                  grad_frag_alpha);
}

// main.cpp:158-170
void dsref_encode_view_dir_sh2(int B, int H, int W, const float* rast, const float* inv_mvp, float* enc) {
    dc::encode_view_dir_sh2(B, H, W, rast, inv_mvp, enc);
}

// main.cpp:174-191
void dsref_multires_triangle_alpha(int num_frags, const float* frag_attrs, int min_level, int max_level,
                                   const float* alpha_src, float* frag_alpha) {
    dc::multires_triangle_alpha(num_frags, frag_attrs, (uint32_t)min_level, (uint32_t)max_level, alpha_src,
                                frag_alpha);
}

// main.cpp:193-210
void dsref_backward_multires_triangle_alpha(int num_frags, const float* frag_attrs, int min_level, int max_level,
                                            float* grad_alpha_src, const float* grad_frag_alpha) {
    dc::backward_multires_triangle_alpha(num_frags, frag_attrs, (uint32_t)min_level, (uint32_t)max_level,
                                         grad_alpha_src, grad_frag_alpha);
}

// main.cpp:212-232
void dsref_multires_triangle_color(int B, int H, int W, const float* rast, int min_level, int max_level, int C,
                                   const float* feat, float* out) {
    dc::multires_triangle_color(B, H, W, rast, (uint32_t)min_level, (uint32_t)max_level, (uint32_t)C, feat, out);
}

// main.cpp:234-254
void dsref_backward_multires_triangle_color(int B, int H, int W, const float* rast, int min_level, int max_level,
                                            int C, float* grad_feat, const float* grad_out) {
    dc::backward_multires_triangle_color(B, H, W, rast, (uint32_t)min_level, (uint32_t)max_level, (uint32_t)C,
                                         grad_feat, grad_out);
}

// main.cpp:258-280
void dsref_accumulate_to_level_forward(int T, int min_level, int max_level, int target_level, int C,
                                       const float* feat, float* out) {
    dc::accumulate_to_level_forward(T, (uint32_t)min_level, (uint32_t)max_level, (uint32_t)target_level,
                                    (uint32_t)C, feat, out);
}

// main.cpp:282-304
void dsref_accumulate_to_level_backward(int T, int min_level, int max_level, int target_level, int C,
                                        float* grad_feat, const float* grad_out) {
    dc::accumulate_to_level_backward(T, (uint32_t)min_level, (uint32_t)max_level, (uint32_t)target_level,
                                     (uint32_t)C, grad_feat, grad_out);
}

int dsref_device_synchronize() { return (int)cudaDeviceSynchronize(); }

}  // extern "C"
