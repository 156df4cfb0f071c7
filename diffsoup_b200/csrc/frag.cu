// diffsoup_b200/csrc/frag.cu -- the reference's fragment-list operators
// (kenji-tojo/diffsoup src/cuda/rasterize.cu:43-487) behind the C ABI.
//
// These keep the reference's `_core` semantics for drop-in callers; the B200
// forward path itself (tiled.cu) never materialises a fragment list.
// Differences from the reference: temporaries come from the caller's
// workspace instead of cudaMalloc per call, work runs on the caller's stream,
// the prefix sums are carried in 64 bits (a total above 2^31-1 is reported as
// DS_ERR_OVERFLOW instead of wrapping), and compaction preserves fragment
// order, so results are deterministic.
#include "geometry.cuh"
#include "scan.cuh"

namespace dsb {

// rasterize.cu:43-137: one thread per (view, triangle).
__global__ void __launch_bounds__(kThreads) rects_kernel(int H, int W, int B, int V, const float* __restrict__ pos,
                                                         int T, const int* __restrict__ tri, int* __restrict__ rects,
                                                         int* __restrict__ counts) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * T) return;
    const int b = (int)(i / T), t = (int)(i % T);
    const float* P = pos + (size_t)b * V * 4;
    const float4 p0 = load_vertex(P, tri[t * 3 + 0]);
    const float4 p1 = load_vertex(P, tri[t * 3 + 1]);
    const float4 p2 = load_vertex(P, tri[t * 3 + 2]);
    int h0, hl, w0, wl;
    triangle_rect(H, W, p0, p1, p2, h0, hl, w0, wl);
    reinterpret_cast<int4*>(rects)[i] = make_int4(h0, hl, w0, wl);
    counts[i] = hl * wl;
}

// rasterize.cu:208-277: one thread per bbox pixel; the owning triangle is
// found by binary search over the inclusive prefix.
__global__ void __launch_bounds__(kThreads) fragments_kernel(int H, int W, int V, const float* __restrict__ pos,
                                                             int T, const int* __restrict__ tri, int num_tris,
                                                             int num_frags, const int* __restrict__ prefix,
                                                             const int* __restrict__ rects, int* __restrict__ frag_pix,
                                                             float* __restrict__ frag_attrs) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= num_frags) return;
    int lo = 0, hi = num_tris;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= idx) lo = mid + 1; else hi = mid;
    }
    const int ti = lo;
    if (ti >= num_tris) return;
    const int4 r = __ldg(reinterpret_cast<const int4*>(rects) + ti);
    if (r.w <= 0 || r.y <= 0) return;
    const int local = idx - (ti == 0 ? 0 : __ldg(prefix + ti - 1));
    const int y = r.x + local / r.w;
    const int x = r.z + local % r.w;
    if (x < 0 || x >= W || y < 0 || y >= H) return;
    const int b = ti / T, t = ti % T;
    const float* P = pos + (size_t)b * V * 4;
    const float4 p0 = load_vertex(P, tri[t * 3 + 0]);
    const float4 p1 = load_vertex(P, tri[t * 3 + 1]);
    const float4 p2 = load_vertex(P, tri[t * 3 + 2]);
    float b0, b1, depth;
    if (!fragment_at(pix_ndc(y, H), pix_ndc(x, W), p0, p1, p2, b0, b1, depth)) return;
    frag_pix[(size_t)idx * 3 + 0] = b;
    frag_pix[(size_t)idx * 3 + 1] = y;
    frag_pix[(size_t)idx * 3 + 2] = x;
    reinterpret_cast<float4*>(frag_attrs)[idx] = make_float4(b0, b1, depth, (float)(t + 1));
}

__global__ void __launch_bounds__(kThreads) valid_flags_kernel(int n, const int* __restrict__ frag_pix,
                                                               int* __restrict__ flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = frag_pix[(size_t)i * 3] >= 0 ? 1 : 0;
}

__global__ void __launch_bounds__(kThreads) compact_kernel(int n, const int* __restrict__ flags,
                                                           const int* __restrict__ dst, const int* __restrict__ frag_pix,
                                                           const float* __restrict__ frag_attrs,
                                                           int* __restrict__ pix_out, float* __restrict__ attrs_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flags[i]) return;
    const int k = dst[i];
    pix_out[(size_t)k * 3 + 0] = frag_pix[(size_t)i * 3 + 0];
    pix_out[(size_t)k * 3 + 1] = frag_pix[(size_t)i * 3 + 1];
    pix_out[(size_t)k * 3 + 2] = frag_pix[(size_t)i * 3 + 2];
    reinterpret_cast<float4*>(attrs_out)[k] = reinterpret_cast<const float4*>(frag_attrs)[i];
}

__global__ void fill_u64_kernel(unsigned long long* p, int64_t n, unsigned long long v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// rasterize.cu:319-345
__global__ void __launch_bounds__(kThreads) depth_test_kernel(int H, int W, int num_frags,
                                                              const int* __restrict__ frag_pix,
                                                              const float* __restrict__ frag_attrs,
                                                              const float* __restrict__ frag_alpha,
                                                              const float* __restrict__ thresh,
                                                              unsigned long long* __restrict__ zbuf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num_frags) return;
    const int b = frag_pix[(size_t)i * 3];
    if (b < 0) return;
    const int64_t p = (int64_t)b * H * W + (int64_t)frag_pix[(size_t)i * 3 + 1] * W + frag_pix[(size_t)i * 3 + 2];
    if (frag_alpha[i] < thresh[i]) return;
    const float z = frag_attrs[(size_t)i * 4 + 2];
    if (z <= -1.f || !isfinite(z)) return;
    atomicMin(zbuf + p, depth_key(z, (uint32_t)i));
}

// rasterize.cu:347-365
__global__ void __launch_bounds__(kThreads) depth_gather_kernel(int64_t n, const unsigned long long* __restrict__ zbuf,
                                                                const float* __restrict__ frag_attrs,
                                                                float* __restrict__ rast) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const unsigned long long k = zbuf[p];
    if (k == ~0ull) return;
    const uint32_t f = (uint32_t)(k & 0xffffffffu);
    reinterpret_cast<float4*>(rast)[p] = reinterpret_cast<const float4*>(frag_attrs)[f];
}

}  // namespace dsb

using namespace dsb;

extern "C" {

size_t ds_compute_triangle_rects_workspace(int B, int T) {
    const int64_t n = (int64_t)B * T;
    return (size_t)n * sizeof(int) + scan_workspace_bytes(n) + 256;
}

int ds_compute_triangle_rects(int H, int W, int B, int V, const float* pos, int T, const int* tri, int* rects,
                              int* prefix, int* num_frags_host, void* workspace, size_t workspace_bytes,
                              ds_stream_t stream) {
    DS_CHECK_ARG(H > 0 && W > 0 && B >= 0 && V >= 0 && T >= 0, "compute_triangle_rects: bad sizes");
    const int64_t n = (int64_t)B * T;
    if (num_frags_host) *num_frags_host = 0;
    if (n == 0) return DS_OK;
    if (workspace_bytes < ds_compute_triangle_rects_workspace(B, T))
        return set_error(DS_ERR_WORKSPACE, "compute_triangle_rects: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    int* counts = reinterpret_cast<int*>(workspace);
    void* scan_ws = reinterpret_cast<char*>(workspace) + (((size_t)n * sizeof(int) + 255) & ~(size_t)255);
    rects_kernel<<<blocks_for(n), kThreads, 0, st>>>(H, W, B, V, pos, T, tri, rects, counts);
    int64_t* total_dev = nullptr;
    int rc = device_scan<int, int>(counts, n, prefix, true, scan_ws, st, &total_dev);
    if (rc) return rc;
    int64_t total = 0;
    DS_CUDA(cudaMemcpyAsync(&total, total_dev, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    DS_CUDA(cudaStreamSynchronize(st));
    if (total > 0x7fffffff)
        return set_error(DS_ERR_OVERFLOW, "compute_triangle_rects: %lld bbox pixels exceed the int32 fragment layout",
                         (long long)total);
    if (num_frags_host) *num_frags_host = (int)total;
    return DS_OK;
}

int ds_compute_fragments(int H, int W, int B, int V, const float* pos, int T, const int* tri, const int* prefix,
                         const int* rects, int num_frags, int* frag_pix, float* frag_attrs, ds_stream_t stream) {
    DS_CHECK_ARG(H > 0 && W > 0 && B >= 0 && T >= 0 && num_frags >= 0, "compute_fragments: bad sizes");
    if (num_frags == 0 || (int64_t)B * T == 0) return DS_OK;
    DS_CHECK_ARG((int64_t)B * T <= 0x7fffffff, "compute_fragments: B*T exceeds int32");
    fragments_kernel<<<blocks_for(num_frags), kThreads, 0, (cudaStream_t)stream>>>(
        H, W, V, pos, T, tri, B * T, num_frags, prefix, rects, frag_pix, frag_attrs);
    return check_launch("compute_fragments");
}

size_t ds_filter_valid_fragments_workspace(int num_frags) {
    const size_t flags = (((size_t)num_frags * sizeof(int)) + 255) & ~(size_t)255;
    return 2 * flags + scan_workspace_bytes(num_frags) + 256;
}

int ds_filter_valid_fragments(int num_frags, const int* frag_pix, const float* frag_attrs, int* frag_pix_out,
                              float* frag_attrs_out, int* count_host, void* workspace, size_t workspace_bytes,
                              ds_stream_t stream) {
    DS_CHECK_ARG(num_frags >= 0, "filter_valid_fragments: bad size");
    if (count_host) *count_host = 0;
    if (num_frags == 0) return DS_OK;
    if (workspace_bytes < ds_filter_valid_fragments_workspace(num_frags))
        return set_error(DS_ERR_WORKSPACE, "filter_valid_fragments: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t fb = (((size_t)num_frags * sizeof(int)) + 255) & ~(size_t)255;
    int* flags = reinterpret_cast<int*>(workspace);
    int* dst = reinterpret_cast<int*>(reinterpret_cast<char*>(workspace) + fb);
    void* scan_ws = reinterpret_cast<char*>(workspace) + 2 * fb;
    valid_flags_kernel<<<blocks_for(num_frags), kThreads, 0, st>>>(num_frags, frag_pix, flags);
    int64_t* total_dev = nullptr;
    int rc = device_scan<int, int>(flags, num_frags, dst, false, scan_ws, st, &total_dev);
    if (rc) return rc;
    compact_kernel<<<blocks_for(num_frags), kThreads, 0, st>>>(num_frags, flags, dst, frag_pix, frag_attrs,
                                                                frag_pix_out, frag_attrs_out);
    rc = check_launch("filter_valid_fragments");
    if (rc) return rc;
    int64_t total = 0;
    DS_CUDA(cudaMemcpyAsync(&total, total_dev, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    DS_CUDA(cudaStreamSynchronize(st));
    if (count_host) *count_host = (int)total;
    return DS_OK;
}

size_t ds_depth_test_workspace(int B, int H, int W) { return (size_t)B * H * W * sizeof(unsigned long long); }

int ds_depth_test(int B, int H, int W, int num_frags, const int* frag_pix, const float* frag_attrs,
                  const float* frag_alpha, const float* alpha_thresh, float* rast, void* workspace,
                  size_t workspace_bytes, ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H > 0 && W > 0 && num_frags >= 0, "depth_test: bad sizes");
    if (num_frags == 0) return DS_OK;
    const int64_t npix = (int64_t)B * H * W;
    if (workspace_bytes < ds_depth_test_workspace(B, H, W))
        return set_error(DS_ERR_WORKSPACE, "depth_test: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long* zbuf = reinterpret_cast<unsigned long long*>(workspace);
    fill_u64_kernel<<<sm_count() * 4, kThreads, 0, st>>>(zbuf, npix, ~0ull);
    depth_test_kernel<<<blocks_for(num_frags), kThreads, 0, st>>>(H, W, num_frags, frag_pix, frag_attrs, frag_alpha,
                                                                  alpha_thresh, zbuf);
    depth_gather_kernel<<<blocks_for(npix), kThreads, 0, st>>>(npix, zbuf, frag_attrs, rast);
    return check_launch("depth_test");
}

}  // extern "C"
