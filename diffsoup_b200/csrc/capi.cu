// diffsoup_b200/csrc/capi.cu -- error reporting, version and view tables of
// the C ABI (include/diffsoup_b200.h).
#include <cstdarg>
#include <cstdio>

#include "common.cuh"

namespace dsb {

static thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int sm_count() {
    constexpr int kMaxDevices = 64;
    static int cache[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 1;
    if (dev < kMaxDevices && cache[dev] > 0) return cache[dev];
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 1;
    if (dev < kMaxDevices) cache[dev] = n;
    return n;
}

int check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(DS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return DS_OK;
}

}  // namespace dsb

extern "C" {

const char* ds_last_error(void) { return dsb::g_err; }

const char* ds_version(void) { return "diffsoup_b200 0.1.0 (sm_100a)"; }

int ds_make_view_table(int B, const int* H_host, const int* W_host, ds_view_desc* desc_host,
                       int64_t* num_pixels_host) {
    if (B < 0) return dsb::set_error(DS_ERR_ARG, "ds_make_view_table: B < 0");
    int64_t pix = 0;
    int64_t tiles = 0;
    for (int b = 0; b < B; ++b) {
        const int H = H_host[b], W = W_host[b];
        if (H <= 0 || W <= 0) return dsb::set_error(DS_ERR_ARG, "ds_make_view_table: view %d has size %dx%d", b, H, W);
        ds_view_desc& d = desc_host[b];
        d.H = H;
        d.W = W;
        d.tiles_x = (W + DS_TILE - 1) / DS_TILE;
        d.tiles_y = (H + DS_TILE - 1) / DS_TILE;
        d.pix_offset = pix;
        d.tile_base = (int32_t)tiles;
        d.pad = 0;
        pix += (int64_t)H * W;
        tiles += (int64_t)d.tiles_x * d.tiles_y;
        if (tiles > (int64_t)1 << 30) return dsb::set_error(DS_ERR_OVERFLOW, "ds_make_view_table: too many tiles");
    }
    if (num_pixels_host) *num_pixels_host = pix;
    return (int)tiles;
}

}  // extern "C"
