// diffsoup_b200/csrc/count.cu -- per-triangle pixel counts of an ID buffer
// (count_triangle_ids, python/diffsoup/rasterize.py:348-366, which the
// reference computes with torch.bincount), the visibility statistic of
// resampling (examples/utils.py:445-482).  One thread per pixel; neighbouring
// pixels mostly show the same triangle, so lanes holding equal IDs are
// grouped with __match_any_sync and one of them adds the group's size.
#include "common.cuh"

namespace dsb {

__global__ void __launch_bounds__(kThreads) count_ids_kernel(int64_t n, const float4* __restrict__ rast, int num_tris,
                                                             unsigned long long* __restrict__ counts,
                                                             int* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const int id = i < n ? (int)rast[i].w - 1 : -1;
        const bool in = id >= 0 && id < num_tris;
        if (id >= num_tris && bad) atomicOr(bad, 1);
        const unsigned active = __ballot_sync(0xffffffffu, in);
        if (in) {
            const unsigned peers = __match_any_sync(active, id);
            if (lane == __ffs(peers) - 1) atomicAdd(counts + id, (unsigned long long)__popc(peers));
        }
    }
}

}  // namespace dsb

using namespace dsb;

extern "C" {

int ds_count_triangle_ids(int64_t num_pixels, const float* rast, int num_tris, int64_t* counts, int* status,
                          ds_stream_t stream) {
    DS_CHECK_ARG(num_pixels >= 0 && num_tris >= 0, "count_triangle_ids: bad sizes");
    DS_CHECK_ARG(num_pixels == 0 || (rast != nullptr && counts != nullptr), "count_triangle_ids: null pointer");
    DS_CHECK_ARG(((uintptr_t)rast & 15) == 0, "count_triangle_ids: rast not 16-byte aligned");
    if (num_pixels == 0) return DS_OK;
    const int64_t blocks = (num_pixels + kThreads - 1) / kThreads;
    const unsigned grid = (unsigned)(blocks < (int64_t)sm_count() * 16 ? blocks : (int64_t)sm_count() * 16);
    count_ids_kernel<<<grid, kThreads, 0, (cudaStream_t)stream>>>(
        num_pixels, reinterpret_cast<const float4*>(rast), num_tris, reinterpret_cast<unsigned long long*>(counts),
        status);
    return check_launch("count_triangle_ids");
}

}  // extern "C"
