// diffsoup_b200/csrc/noalloc.cu -- a depth test that needs no caller memory.
//
// ds_depth_test needs a temporary depth-key buffer of 8 bytes per pixel,
// which the caller allocates and passes as workspace.  Some callers cannot do
// that: code that runs inside a host application whose allocator owns all
// device memory and forbids direct cudaMalloc, callers working under a fixed
// memory budget that must not grow mid-run, and latency-sensitive loops that
// cannot afford cudaMalloc/cudaFree (cudaFree synchronises the whole device).
// ds_depth_test_noalloc serves them with a depth-key buffer that lives in
// this library's own device memory: a file-scope __device__ array of fixed
// size, reserved on every GPU that loads the library until the process exits.
//
// Limits and sharing:
//   * at most kNoAllocMaxPixels = 2^21 pixels (B*H*W) per call, e.g. two
//     1024x1024 views or three 800x800 views; larger batches are rejected
//     with DS_ERR_ARG before any GPU work;
//   * every call on a device uses the same buffer, which keeps the previous
//     call's keys; each call clears the part it uses before the depth test.
//     Two calls whose GPU work overlaps (different streams, or threads without
//     ordering between them) race on the buffer and corrupt each other;
//   * host code cannot use the array's name as a device address, so the
//     first call on each device looks the address up with
//     cudaGetSymbolAddress (with that device current) and caches it.  Make
//     that first call before any stream capture.  The cached address belongs
//     to the device's current (primary) context: do not call this entry point
//     again after cudaDeviceReset or after that context was destroyed and
//     re-created, where the library's module may be loaded at another address;
//   * fragments whose (batch, row, column) lies outside [0,B) x [0,H) x [0,W)
//     are skipped, so a bad fragment cannot write into the shared buffer
//     beyond its own batch (the workspace version leaves that to the caller).
#include <mutex>

#include "geometry.cuh"

namespace dsb {

constexpr int64_t kNoAllocMaxPixels = int64_t(1) << 21;  // 16 MiB of 64-bit depth keys

// The depth-key buffer (file scope, one per device that loads the library).
static __device__ __align__(256) unsigned long long g_depth_keys[kNoAllocMaxPixels];

namespace {

constexpr int kMaxDevices = 64;

std::mutex g_addr_mutex;
unsigned long long* g_addr[kMaxDevices] = {};

// Device address of g_depth_keys on the current device (looked up once).
int depth_keys_address(unsigned long long** out) {
    int dev = 0;
    DS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(DS_ERR_ARG, "depth_test_noalloc: device %d beyond the %d supported", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (g_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_depth_keys);
        if (e != cudaSuccess || p == nullptr)
            return set_error(DS_ERR_CUDA, "depth_test_noalloc: cudaGetSymbolAddress failed: %s",
                             cudaGetErrorString(e));
        g_addr[dev] = reinterpret_cast<unsigned long long*>(p);
    }
    *out = g_addr[dev];
    return DS_OK;
}

__global__ void noalloc_clear_kernel(unsigned long long* keys, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        keys[i] = ~0ull;
}

// Same test as the workspace version (rasterize.cu:319-345).
__global__ void __launch_bounds__(kThreads) noalloc_depth_kernel(int B, int H, int W, int num_frags,
                                                                 const int* __restrict__ frag_pix,
                                                                 const float* __restrict__ frag_attrs,
                                                                 const float* __restrict__ frag_alpha,
                                                                 const float* __restrict__ thresh,
                                                                 unsigned long long* __restrict__ keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num_frags) return;
    const int b = frag_pix[(size_t)i * 3];
    const int y = frag_pix[(size_t)i * 3 + 1], x = frag_pix[(size_t)i * 3 + 2];
    // b < 0 marks a rejected fragment; anything else outside the batch is skipped too
    if (b < 0 || b >= B || y < 0 || y >= H || x < 0 || x >= W) return;
    const int64_t p = ((int64_t)b * H + y) * W + x;
    if (frag_alpha[i] < thresh[i]) return;
    const float z = frag_attrs[(size_t)i * 4 + 2];
    if (z <= -1.f || !isfinite(z)) return;
    atomicMin(keys + p, depth_key(z, (uint32_t)i));
}

// rasterize.cu:347-365
__global__ void __launch_bounds__(kThreads) noalloc_gather_kernel(int64_t n, const unsigned long long* __restrict__ keys,
                                                                  const float* __restrict__ frag_attrs,
                                                                  float* __restrict__ rast) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const unsigned long long k = keys[p];
    if (k == ~0ull) return;
    reinterpret_cast<float4*>(rast)[p] = reinterpret_cast<const float4*>(frag_attrs)[(uint32_t)(k & 0xffffffffu)];
}

}  // namespace
}  // namespace dsb

using namespace dsb;

extern "C" int ds_depth_test_noalloc(int B, int H, int W, int num_frags, const int* frag_pix, const float* frag_attrs,
                                     const float* frag_alpha, const float* alpha_thresh, float* rast,
                                     ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && H > 0 && W > 0 && num_frags >= 0, "depth_test_noalloc: bad sizes");
    const int64_t npix = (int64_t)B * H * W;
    if (npix > kNoAllocMaxPixels)
        return set_error(DS_ERR_ARG,
                         "depth_test_noalloc: %lld pixels exceed its fixed %lld-pixel depth buffer; "
                         "split the batch or use ds_depth_test with a workspace",
                         (long long)npix, (long long)kNoAllocMaxPixels);
    if (num_frags == 0) return DS_OK;
    DS_CHECK_ARG(((uintptr_t)frag_attrs & 15) == 0 && ((uintptr_t)rast & 15) == 0,
                 "depth_test_noalloc: frag_attrs/rast not 16-byte aligned");
    unsigned long long* keys = nullptr;
    const int rc = depth_keys_address(&keys);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    noalloc_clear_kernel<<<sm_count() * 4, kThreads, 0, st>>>(keys, npix);
    noalloc_depth_kernel<<<blocks_for(num_frags), kThreads, 0, st>>>(B, H, W, num_frags, frag_pix, frag_attrs,
                                                                     frag_alpha, alpha_thresh, keys);
    noalloc_gather_kernel<<<blocks_for(npix), kThreads, 0, st>>>(npix, keys, frag_attrs, rast);
    return check_launch("depth_test_noalloc");
}
