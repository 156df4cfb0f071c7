// diffsoup_b200/csrc/scan.cuh -- device-wide prefix sum of int32 counts.
//
// Three launches, no host synchronisation (graph-capturable): block sums,
// one-block scan of the block sums, and a rescan that adds each block's
// offset; short scans in one launch (scan_one_cta_kernel).  Sums are carried
// in int64 so totals never wrap.
#pragma once

#include "common.cuh"

namespace dsb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048 items per block

static inline int64_t scan_num_blocks(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

// Workspace bytes: one int64 per block plus the grand total.
inline size_t scan_workspace_bytes(int64_t n) { return (size_t)(scan_num_blocks(n) + 1) * sizeof(int64_t); }

// Exclusive block-wide scan of one int64 per thread; returns the block total.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t& excl) {
    __shared__ int64_t warp_tot[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    int64_t base = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w) {
        const int64_t t = warp_tot[w];
        if (w < warp) base += t;
        total += t;
    }
    __syncthreads();
    excl = base + x - v;
    return total;
}

template <typename In>
__global__ void __launch_bounds__(kScanThreads) scan_block_sums_kernel(const In* __restrict__ in, int64_t n,
                                                                        int64_t* __restrict__ partials) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) s += (int64_t)in[base + i];
    int64_t excl;
    const int64_t tot = block_exclusive_scan(s, excl);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// Exclusive scan of nb block sums in place; partials[nb] receives the total.
static __global__ void __launch_bounds__(kScanThreads) scan_partials_kernel(int64_t* __restrict__ partials, int64_t nb) {
    int64_t carry = 0;
    for (int64_t start = 0; start < nb; start += kScanThreads) {
        const int64_t i = start + threadIdx.x;
        const int64_t v = i < nb ? partials[i] : 0;
        int64_t excl;
        const int64_t tot = block_exclusive_scan(v, excl);
        if (i < nb) partials[i] = carry + excl;
        carry += tot;
    }
    if (threadIdx.x == 0) partials[nb] = carry;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const In* __restrict__ in, int64_t n,
                                                                   const int64_t* __restrict__ partials,
                                                                   Out* __restrict__ out, bool inclusive) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? (int64_t)in[base + i] : 0;
        s += v[i];
    }
    int64_t excl;
    block_exclusive_scan(s, excl);
    int64_t run = partials[blockIdx.x] + excl;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (inclusive) run += v[i];
        if (base + i < n) out[base + i] = (Out)run;
        if (!inclusive) run += v[i];
    }
}

// out[i] = sum of in[0..i] (inclusive) or in[0..i) (exclusive); the total is
// left at ((int64_t*)ws)[num_blocks] on the device.
template <typename In, typename Out>
int device_scan(const In* in, int64_t n, Out* out, bool inclusive, void* ws, cudaStream_t st,
                int64_t** total_dev = nullptr) {
    int64_t* partials = reinterpret_cast<int64_t*>(ws);
    const int64_t nb = scan_num_blocks(n);
    if (total_dev) *total_dev = partials + nb;
    if (n == 0) {
        DS_CUDA(cudaMemsetAsync(partials, 0, sizeof(int64_t), st));
        return DS_OK;
    }
    scan_block_sums_kernel<In><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, partials);
    scan_partials_kernel<<<1, kScanThreads, 0, st>>>(partials, nb);
    scan_apply_kernel<In, Out><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, partials, out, inclusive);
    return check_launch("device_scan");
}

// Short scans in one launch: a single CTA of kScanOneThreads threads, each
// summing up to kScanOneItems consecutive counts, then re-reading them (from
// L1) to write their offsets.  Up to 4 items a thread this beats the three
// launches (the 2,500 tiles of one 800x800 view); at 20 (8 such views) the
// threads' serial loads make it slower than them.
constexpr int kScanOneThreads = 1024;
constexpr int kScanOneItems = 4;
constexpr int64_t kScanOneMax = (int64_t)kScanOneThreads * kScanOneItems;

// out[i] = sum of in[0..i) for i < n and out[n] = the total (n <= kScanOneMax);
// zero[0..n) is cleared on the way (a per-item cursor of the next pass; may
// be null).
static __global__ void __launch_bounds__(kScanOneThreads) scan_one_cta_kernel(const int* __restrict__ in, int n,
                                                                              int64_t* __restrict__ out,
                                                                              int* __restrict__ zero) {
    __shared__ int64_t warp_tot[kScanOneThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per = (n + kScanOneThreads - 1) / kScanOneThreads;  // <= kScanOneItems
    const int i0 = threadIdx.x * per, i1 = min(i0 + per, n);
    int64_t s = 0;
    for (int i = i0; i < i1; ++i) s += in[i];
    int64_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    int64_t base = 0, total = 0;
#pragma unroll 8
    for (int w = 0; w < kScanOneThreads / 32; ++w) {
        const int64_t t = warp_tot[w];
        if (w < warp) base += t;
        total += t;
    }
    int64_t run = base + x - s;
    for (int i = i0; i < i1; ++i) {
        out[i] = run;
        run += in[i];
        if (zero) zero[i] = 0;
    }
    if (threadIdx.x == 0) out[n] = total;
}

}  // namespace dsb
