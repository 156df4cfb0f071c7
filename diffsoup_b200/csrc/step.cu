// diffsoup_b200/csrc/step.cu -- the batched training step of DiffSoup
// (examples/02_synthetic.py:354-388 with an MSE photometric loss) as one
// graph-capturable sequence of sm_100a kernels:
//
//   accumulate_to_level(...).sigmoid() for opacity and features   (prep)
//   project_vertices (examples/utils.py:412-426)                   (prep)
//   screen-tile binning + tiled stochastic-opacity rasterizer      (tiled.cu)
//   fused shading forward + backward, BF16 MLP on tensor cores     (shade.cuh)
//   opacity auxiliary gradient, recomputed tile by tile            (tiled.cu)
//   edge gradients to clip-space vertices                          (edge)
//   adjoints of the sigmoid, the level accumulation and projection (finish)
//
// Views may differ in resolution; their pixels are packed back to back.
#include <cmath>
#include <cstdio>

#include "edge_math.cuh"
#include "shade.cuh"
#include "shade_reg.cuh"
#include "shade_tc.cuh"
#include "tiled.cuh"

namespace dsb {

// ---------------------------------------------------------------------------
// Level accumulation + sigmoid, one warp per triangle (multires.cu:329-369).
// The triangle's source samples are staged in shared memory; outputs are
// sigmoid(sum over levels of the lattice interpolation at each target vertex).
// ---------------------------------------------------------------------------
constexpr int kPrepWarps = 4;
constexpr int kMaxSrc = 2048;  // floats of one triangle's samples per warp (S*C)

// Outputs have a channel stride of CP >= C (padding channels written as zero).
template <bool BF16OUT>
__global__ void __launch_bounds__(kPrepWarps * 32) accum_sigmoid_kernel(int T, int lo, int hi, int target, int S,
                                                                       int ST, int C, int CP,
                                                                       const float* __restrict__ src,
                                                                       float* __restrict__ out_f32,
                                                                       __nv_bfloat16* __restrict__ out_bf16) {
    __shared__ float s_src[kPrepWarps][kMaxSrc];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * kPrepWarps + warp;
    if (t >= T) return;
    const int n = S * C;
    const float* ts = src + (size_t)t * n;
    for (int i = lane; i < n; i += 32) s_src[warp][i] = ts[i];
    __syncwarp();
    const float R = (float)(1u << target);
    for (int e = lane; e < ST * CP; e += 32) {
        const int k = e / CP, c = e % CP;
        if (c >= C) {
            out_f32[(size_t)t * ST * CP + e] = 0.f;
            if (BF16OUT) out_bf16[(size_t)t * ST * CP + e] = __float2bfloat16_rn(0.f);
            continue;
        }
        uint32_t x, y;
        index_to_xy((uint32_t)k, x, y);
        const float b0 = __fdiv_rn((float)x, R), b1 = __fdiv_rn((float)y, R);
        float acc = 0.f;
        uint32_t off = 0;
        for (int l = lo; l <= hi; ++l) {
            uint32_t idx[3]; float w[3];
            lattice_cell(b0, b1, (uint32_t)l, idx, w);
#pragma unroll
            for (int j = 0; j < 3; ++j) acc = madd(acc, w[j], s_src[warp][(off + idx[j]) * C + c]);
            off += feats_at_level((uint32_t)l);
        }
        const float s = 1.f / (1.f + expf(-acc));
        out_f32[(size_t)t * ST * CP + e] = s;
        if (BF16OUT) out_bf16[(size_t)t * ST * CP + e] = __float2bfloat16_rn(s);
    }
}

// Adjoint of accum_sigmoid: grad_src[t] = sum_k lattice^T (grad_out * s (1-s)).
// Accumulated per warp in shared memory, written once (no global atomics).
// sig and grad_out have the channel stride CP, grad_src the stride C.
__global__ void __launch_bounds__(kPrepWarps * 32) accum_sigmoid_backward_kernel(
    int T, int lo, int hi, int target, int S, int ST, int C, int CP, const float* __restrict__ sig,
    const float* __restrict__ grad_out, float* __restrict__ grad_src) {
    __shared__ float s_acc[kPrepWarps][kMaxSrc];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * kPrepWarps + warp;
    if (t >= T) return;
    const int n = S * C;
    for (int i = lane; i < n; i += 32) s_acc[warp][i] = 0.f;
    __syncwarp();
    const float R = (float)(1u << target);
    for (int e = lane; e < ST * C; e += 32) {
        const int k = e / C, c = e % C;
        const size_t o = ((size_t)t * ST + k) * CP + c;
        const float s = sig[o];
        const float gz = grad_out[o] * s * (1.f - s);
        if (gz == 0.f) continue;
        uint32_t x, y;
        index_to_xy((uint32_t)k, x, y);
        const float b0 = __fdiv_rn((float)x, R), b1 = __fdiv_rn((float)y, R);
        uint32_t off = 0;
        for (int l = lo; l <= hi; ++l) {
            uint32_t idx[3]; float w[3];
            lattice_cell(b0, b1, (uint32_t)l, idx, w);
#pragma unroll
            for (int j = 0; j < 3; ++j) atomicAdd(&s_acc[warp][(off + idx[j]) * C + c], gz * w[j]);
            off += feats_at_level((uint32_t)l);
        }
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) grad_src[(size_t)t * n + i] = s_acc[warp][i];
}

// ---------------------------------------------------------------------------
// Table-driven level accumulation.  The interpolation from the levels'
// lattices to the target lattice is the same sparse map for every triangle,
// so each CTA of the forward kernel builds it in shared memory (the grid is
// one wave of persistent CTAs) and the adjoint copies the forward's: the
// forward table lists, per
// target sample, its (source sample, weight) pairs in level-then-corner
// order (the summation order of accum_sigmoid_kernel), and the backward
// table is the same map grouped by source sample, which turns the adjoint
// into a gather without atomics.  Pairs of weight zero are left out (a
// target sample that is a lattice vertex of a level takes one corner there):
// about half of them, and adding 0 * x leaves a finite sum unchanged.
//
// The kernels run a warp over G = 32 / CP triangles at a time, lane (g, c)
// taking channel c of triangle g: every lane walks the same table row, so
// the table reads are broadcasts and the loops lane-uniform; the sources (or
// the target gradients) of the G triangles sit in shared memory as
// [sample][lane].  The opacities of the G triangles go through the same
// table with lane (g, j) taking the target (or source) samples j, j + CP, ...
// ---------------------------------------------------------------------------
constexpr int kTabMax = 1024;  // (target sample, level, corner) entries
constexpr int kTabWarps = 8;
constexpr size_t kTabSmemMax = 100 * 1024;  // two CTAs per SM at most this size

// The tables in dynamic shared memory (room for N nonzero pairs), followed
// by each warp's staging buffer.
struct LatticeTab {
    int2* fent;  // per target sample (rows frow): {source sample, weight bits}
    int* frow;   // [ST + 1]
    int2* bent;  // per source sample (rows brow): {target sample, weight bits}
    int* brow;   // [S + 1]
};

__host__ __device__ inline size_t lattice_tab_bytes(int N, int S, int ST) {
    return ((size_t)N * 16 + (size_t)(S + ST + 2) * 4 + 15) & ~(size_t)15;
}

__device__ inline LatticeTab lattice_tab_at(unsigned char* base, int N, int S, int ST) {
    LatticeTab L;
    L.fent = reinterpret_cast<int2*>(base);
    L.bent = reinterpret_cast<int2*>(base + (size_t)N * 8);
    L.frow = reinterpret_cast<int*>(base + (size_t)N * 16);
    L.brow = L.frow + ST + 1;
    return L;
}

// Per-warp staging floats: a [rows][32] sample-by-lane buffer and the G
// triangles' opacity rows (rows = S sources forward, ST targets backward).
__host__ __device__ inline int tab_stage_floats(int rows, int CP) { return 32 * rows + (32 / CP) * (rows + 1); }

// Exclusive prefix of rows[1..n] into rows[0..n] (rows[0] = 0), one warp.
__device__ inline void tab_scan(int* rows, int n) {
    const int lane = threadIdx.x & 31;
    int carry = 0;
    if (lane == 0) rows[0] = 0;
    for (int d0 = 0; d0 < n; d0 += 32) {
        const int d = d0 + lane;
        int v = d < n ? rows[d + 1] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        if (d < n) rows[d + 1] = carry + v;
        carry += __shfl_sync(0xffffffffu, v, 31);
    }
}

// Builds the tables; `scratch` holds N ints, N floats and S ints during the build.
__device__ void build_lattice_tab(const LatticeTab& L, int lo, int hi, int ST, int S, unsigned char* scratch) {
    const int NL = hi - lo + 1, NE = NL * 3, N = ST * NE;
    int* fidx = reinterpret_cast<int*>(scratch);
    float* fw = reinterpret_cast<float*>(scratch + (size_t)N * 4);
    const float inv_r = 1.f / (float)(1u << hi);  // a power of two: x * inv_r == x / 2^hi exactly
    for (int u = threadIdx.x; u < ST * NL; u += blockDim.x) {
        const int k = u / NL, li = u - (u / NL) * NL, l = lo + li;
        uint32_t x, y;
        index_to_xy((uint32_t)k, x, y);
        uint32_t idx[3];
        float w[3];
        lattice_cell(__fmul_rn((float)x, inv_r), __fmul_rn((float)y, inv_r), (uint32_t)l, idx, w);
        uint32_t off = 0;
        for (int m = lo; m < l; ++m) off += feats_at_level((uint32_t)m);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            fidx[k * NE + li * 3 + j] = (int)(off + idx[j]);
            fw[k * NE + li * 3 + j] = w[j];
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < ST; k += blockDim.x) {  // forward row lengths
        int cnt = 0;
        for (int n = 0; n < NE; ++n) cnt += fw[k * NE + n] != 0.f;
        L.frow[k + 1] = cnt;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int d = threadIdx.x; d < S; d += blockDim.x) L.brow[d + 1] = 0;  // backward row lengths
    __syncthreads();
    for (int e = threadIdx.x; e < N; e += blockDim.x)
        if (fw[e] != 0.f) atomicAdd(&L.brow[fidx[e] + 1], 1);
    __syncthreads();
    if (warp == 0) tab_scan(L.frow, ST);
    if (warp == 1 % nw) tab_scan(L.brow, S);
    __syncthreads();
    for (int k = threadIdx.x; k < ST; k += blockDim.x) {  // forward rows, in (level, corner) order
        int at = L.frow[k];
        for (int n = 0; n < NE; ++n)
            if (fw[k * NE + n] != 0.f) L.fent[at++] = make_int2(fidx[k * NE + n], __float_as_int(fw[k * NE + n]));
    }
    if (warp == nw - 1) {  // backward rows, in (target, level, corner) order: one warp walks the pairs
        int* cursor = reinterpret_cast<int*>(fw + N);  // per source: the next free slot of its row
        for (int d = lane; d < S; d += 32) cursor[d] = L.brow[d];
        __syncwarp();
        for (int e0 = 0; e0 < N; e0 += 32) {
            const int e = e0 + lane;
            const bool hit = e < N && fw[e] != 0.f;
            const int d = hit ? fidx[e] : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, d);  // the lanes with this source
            const int leader = __ffs(peers) - 1;
            int base = 0;
            if (hit && lane == leader) {
                base = cursor[d];
                cursor[d] = base + __popc(peers);
            }
            base = __shfl_sync(0xffffffffu, base, leader);
            if (hit) L.bent[base + __popc(peers & ((1u << lane) - 1u))] = make_int2(e / NE, __float_as_int(fw[e]));
            __syncwarp();
        }
    }
    __syncthreads();
}

__device__ __forceinline__ float sigmoid_ref(float x) { return 1.f / (1.f + expf(-x)); }

// 4-byte global -> shared copy that bypasses registers (cp.async), and the wait for all of a thread's.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// alpha_out[t] = sigmoid(accumulate(alpha_src[t])), feat_out[t] likewise
// per channel (+ a bf16 copy; both with the channel stride CP >= C, padding
// channels zero).
template <int C, int CP>
__global__ void __launch_bounds__(kTabWarps * 32) accum_tab_kernel(int T, int lo, int hi, int S, int ST,
                                                                   const float* __restrict__ alpha_src,
                                                                   const float* __restrict__ feat_src,
                                                                   float* __restrict__ alpha_out,
                                                                   float* __restrict__ feat_out,
                                                                   __nv_bfloat16* __restrict__ feat_bf16,
                                                                   uint4* __restrict__ tab_out) {
    constexpr int G = 32 / CP;
    static_assert(CP == 8 || CP == 16, "channel stride of the accumulated tables");
    extern __shared__ __align__(16) unsigned char tab_smem[];
    const int N = ST * (hi - lo + 1) * 3;
    const size_t tab_bytes = lattice_tab_bytes(N, S, ST);
    const LatticeTab L = lattice_tab_at(tab_smem, N, S, ST);
    build_lattice_tab(L, lo, hi, ST, S, tab_smem + tab_bytes);  // the scratch is the staging area
    if (blockIdx.x == 0) {  // the tables for the adjoint kernel of this step
        const uint4* src = reinterpret_cast<const uint4*>(tab_smem);
        for (int i = threadIdx.x; i < (int)(tab_bytes / 16); i += blockDim.x) tab_out[i] = src[i];
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / CP, c = lane % CP;
    const int M = S;
    float* sf = reinterpret_cast<float*>(tab_smem + tab_bytes) + (size_t)warp * tab_stage_floats(M, CP);
    float* sa = sf + 32 * M;  // [G][M + 1]
    for (int t0 = (blockIdx.x * kTabWarps + warp) * G; t0 < T; t0 += gridDim.x * kTabWarps * G) {
        const int t = t0 + g;
        const bool tv = t < T;
        // every sample copied without registers (cp.async), then one wait: one round trip a pass
        for (int s = 0; s < S; ++s) {
            float* dst = sf + s * 32 + lane;
            if (tv && c < C) cp_async4(dst, feat_src + ((size_t)t * S + s) * C + c);
            else *dst = 0.f;
        }
        for (int i = lane; i < G * S; i += 32) {
            const int gi = i / S;
            float* dst = sa + gi * (M + 1) + (i - gi * S);
            if (t0 + gi < T) cp_async4(dst, alpha_src + (size_t)t0 * S + i);
            else *dst = 0.f;
        }
        cp_async_wait_all();
        __syncwarp();
        // opacity: lane (g, j) takes targets j, j + CP, ...
        for (int k = c; k < ST; k += CP) {
            float acc = 0.f;
            for (int n = L.frow[k]; n < L.frow[k + 1]; ++n) {
                const int2 e = L.fent[n];
                acc = madd(acc, __int_as_float(e.y), sa[g * (M + 1) + e.x]);
            }
            if (tv) alpha_out[(size_t)t * ST + k] = sigmoid_ref(acc);
        }
        // features: lane (g, c) takes channel c of every target
        for (int k = 0; k < ST; ++k) {
            float acc = 0.f;
#pragma unroll 4
            for (int n = L.frow[k]; n < L.frow[k + 1]; ++n) {
                const int2 e = L.fent[n];
                acc = madd(acc, __int_as_float(e.y), sf[e.x * 32 + lane]);
            }
            const float v = c < C ? sigmoid_ref(acc) : 0.f;
            if (tv) {
                feat_out[((size_t)t * ST + k) * CP + c] = v;
                feat_bf16[((size_t)t * ST + k) * CP + c] = __float2bfloat16_rn(v);
            }
        }
        __syncwarp();
    }
}

// Adjoint of accum_tab_kernel: grad_src[t][d] = sum over the targets k that
// read d of w * grad_out[t][k] * s (1 - s); a gather, written once.  feat_sig and
// feat_grad have the channel stride CP, feat_src_grad the stride C.
template <int C, int CP>
__global__ void __launch_bounds__(kTabWarps * 32) accum_tab_backward_kernel(
    int T, int lo, int hi, int S, int ST, const float* __restrict__ alpha_sig, const float* __restrict__ alpha_grad,
    const float* __restrict__ feat_sig, const float* __restrict__ feat_grad, float* __restrict__ alpha_src_grad,
    float* __restrict__ feat_src_grad, const uint4* __restrict__ tab_in) {
    constexpr int G = 32 / CP;
    extern __shared__ __align__(16) unsigned char tab_smem[];
    const int N = ST * (hi - lo + 1) * 3;
    const size_t tab_bytes = lattice_tab_bytes(N, S, ST);
    const LatticeTab L = lattice_tab_at(tab_smem, N, S, ST);
    {
        uint4* dst = reinterpret_cast<uint4*>(tab_smem);
        for (int i = threadIdx.x; i < (int)(tab_bytes / 16); i += blockDim.x) dst[i] = tab_in[i];
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / CP, c = lane % CP;
    const int M = ST;
    float* gf = reinterpret_cast<float*>(tab_smem + tab_bytes) + (size_t)warp * tab_stage_floats(M, CP);
    float* ga = gf + 32 * M;  // [G][M + 1]
    for (int t0 = (blockIdx.x * kTabWarps + warp) * G; t0 < T; t0 += gridDim.x * kTabWarps * G) {
        const int t = t0 + g;
        const bool tv = t < T;
        // sixteen (sigmoid, gradient) pairs in flight per lane before their stores
        for (int k0 = 0; k0 < ST; k0 += 16) {
            float sg[16], gr[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const bool in = k0 + j < ST && tv && c < C;
                const size_t o = ((size_t)t * ST + k0 + j) * CP + c;
                sg[j] = in ? __ldg(feat_sig + o) : 0.f;
                gr[j] = in ? __ldg(feat_grad + o) : 0.f;
            }
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (k0 + j < ST) gf[(k0 + j) * 32 + lane] = gr[j] * sg[j] * (1.f - sg[j]);
        }
        for (int i0 = 0; i0 < G * ST; i0 += 128) {
            float sg[4], gr[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int i = i0 + j * 32 + lane, gi = i / ST;
                const bool in = i < G * ST && t0 + gi < T;
                sg[j] = in ? __ldg(alpha_sig + (size_t)t0 * ST + i) : 0.f;
                gr[j] = in ? __ldg(alpha_grad + (size_t)t0 * ST + i) : 0.f;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int i = i0 + j * 32 + lane, gi = i / ST;
                if (i < G * ST) ga[gi * (M + 1) + (i - gi * ST)] = gr[j] * sg[j] * (1.f - sg[j]);
            }
        }
        __syncwarp();
        for (int d = c; d < S; d += CP) {  // opacity: lane (g, j) takes sources j, j + CP, ...
            float v = 0.f;
            for (int n = L.brow[d]; n < L.brow[d + 1]; ++n) {
                const int2 e = L.bent[n];
                v = fmaf(__int_as_float(e.y), ga[g * (M + 1) + e.x], v);
            }
            if (tv) alpha_src_grad[(size_t)t * S + d] = v;
        }
        for (int d = 0; d < S; ++d) {  // features: lane (g, c) takes channel c of every source
            float v = 0.f;
#pragma unroll 4
            for (int n = L.brow[d]; n < L.brow[d + 1]; ++n) {
                const int2 e = L.bent[n];
                v = fmaf(__int_as_float(e.y), gf[e.x * 32 + lane], v);
            }
            if (tv && c < C) feat_src_grad[((size_t)t * S + d) * C + c] = v;
        }
        __syncwarp();
    }
}

// Dynamic shared memory of the table kernels: tables + per-warp staging of
// the sources (forward) or of the
// target gradients (backward).
static size_t lattice_tab_smem(int lo, int hi, int S, int ST, int CP, bool backward) {
    const int N = ST * (hi - lo + 1) * 3;
    return lattice_tab_bytes(N, S, ST) + (size_t)kTabWarps * tab_stage_floats(backward ? ST : S, CP) * 4;
}

// Whether the table kernels cover this configuration.
static bool lattice_tab_fits(int lo, int hi, int S, int ST, int CP) {
    return ST * (hi - lo + 1) * 3 <= kTabMax && (CP == 8 || CP == 16) &&
           lattice_tab_smem(lo, hi, S, ST, CP, false) <= kTabSmemMax;
}

// The table kernels' dynamic shared memory above the 48 KB default, and
// the CTAs of that size one SM holds (one record per kernel: the template
// argument is the kernel itself).
template <auto Kernel>
static int tab_smem_attr(size_t smem, int* per_sm = nullptr) {
    static size_t set = 0;
    static int fit = 1;
    if (smem != set) {
        DS_CUDA(cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, Kernel, kTabWarps * 32, smem));
        if (fit < 1) fit = 1;
        set = smem;
    }
    if (per_sm) *per_sm = fit;
    return DS_OK;
}

// clip[b][v] = mvp[b] . (verts[v], 1)  (examples/utils.py:412-426)
__global__ void __launch_bounds__(kThreads) project_kernel(int B, int V, const float* __restrict__ verts,
                                                           const float* __restrict__ mvp, float* __restrict__ pos) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * V) return;
    const int b = (int)(i / V), v = (int)(i % V);
    const float* M = mvp + (size_t)b * 16;
    const float x = verts[(size_t)v * 3], y = verts[(size_t)v * 3 + 1], z = verts[(size_t)v * 3 + 2];
    // fixed evaluation order: ((M[r][3] + M[r][0] x) + M[r][1] y) + M[r][2] z, fused
    float4 o;
    o.x = __fmaf_rn(M[2], z, __fmaf_rn(M[1], y, __fmaf_rn(M[0], x, M[3])));
    o.y = __fmaf_rn(M[6], z, __fmaf_rn(M[5], y, __fmaf_rn(M[4], x, M[7])));
    o.z = __fmaf_rn(M[10], z, __fmaf_rn(M[9], y, __fmaf_rn(M[8], x, M[11])));
    o.w = __fmaf_rn(M[14], z, __fmaf_rn(M[13], y, __fmaf_rn(M[12], x, M[15])));
    reinterpret_cast<float4*>(pos)[i] = o;
}

// grad_verts[v] = sum_b mvp[b][:, :3]^T grad_pos[b][v]
__global__ void __launch_bounds__(kThreads) project_backward_kernel(int B, int V, const float* __restrict__ mvp,
                                                                    const double* __restrict__ grad_pos,
                                                                    float* __restrict__ grad_verts) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int b = 0; b < B; ++b) {
        const float* M = mvp + (size_t)b * 16;
        const double* gp = grad_pos + ((size_t)b * V + v) * 4;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            gx += (double)M[r * 4 + 0] * gp[r];
            gy += (double)M[r * 4 + 1] * gp[r];
            gz += (double)M[r * 4 + 2] * gp[r];
        }
    }
    grad_verts[(size_t)v * 3] = (float)gx;
    grad_verts[(size_t)v * 3 + 1] = (float)gy;
    grad_verts[(size_t)v * 3 + 2] = (float)gz;
}

// Edge gradients over packed views (rasterize.cu:653-903): one CTA per
// 16x16 screen tile, one thread per pixel.  The tile and its one-pixel
// border are staged in shared memory first (triangle, depth, colour,
// dL/dcolour and the triangle's far depth bound), so the four neighbours of
// every pixel are shared-memory reads.  Pixels of a warp (two rows of 16)
// mostly share a triangle along a row: a segmented warp reduction sums runs
// of equal triangles before one FP64 atomic per vertex component.  Only
// covered pixels have a contribution, so after staging the tile's covered
// pixels are compacted (row-major order kept) onto the CTA's first threads:
// warps run full of covered pixels and the warps left without one exit.
constexpr int kEdgeThreads = DS_TILE * DS_TILE;
#ifndef DSB_EDGE_MIN_CTAS
#define DSB_EDGE_MIN_CTAS 4  // resident 8-warp CTAs per SM the register budget is sized for (64 registers)
#endif

__device__ __forceinline__ int tile_view(const ds_view_desc* __restrict__ views, int B, int tile) {
    int lo = 0, hi = B - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&views[mid].tile_base) <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kEdgeThreads, DSB_EDGE_MIN_CTAS) edge_step_kernel(
    int B, const ds_view_desc* __restrict__ views, int V, int T, TileTables tab, const int* __restrict__ tri,
    const float* __restrict__ color, const float* __restrict__ grad_color, const float* __restrict__ rast,
    double* __restrict__ grad_pos) {
    __shared__ EdgeHalo h;
    const int tile = blockIdx.x;
    // no triangle may cover a pixel centre of the tile (its list is empty): every pixel is background,
    // and background pixels contribute nothing as the centre of a pair
    if (tab.offsets[tile] == tab.offsets[tile + 1]) return;
    const int b = tile_view(views, B, tile);
    const ds_view_desc vd = views[b];
    const int tl = tile - vd.tile_base;
    const int tx0 = (tl % vd.tiles_x) * DS_TILE, ty0 = (tl / vd.tiles_x) * DS_TILE;
    const TriBox* __restrict__ boxes = tab.boxes + (size_t)b * T;
    for (int i = threadIdx.x; i < kHaloN; i += kEdgeThreads) {
        const int hy = i / kHaloW, hx = i - (i / kHaloW) * kHaloW;
        const int y = ty0 + hy - 1, x = tx0 + hx - 1;
        int it = kOutside;
        float dep = 0.f, zh = 0.f, cc[3] = {0.f, 0.f, 0.f}, gg[3] = {0.f, 0.f, 0.f};
        if (y >= 0 && y < vd.H && x >= 0 && x < vd.W) {
            const int64_t p = vd.pix_offset + (int64_t)y * vd.W + x;
            const float4 r = reinterpret_cast<const float4*>(rast)[p];
            it = (int)r.w - 1;
            dep = r.z;
#pragma unroll
            for (int k = 0; k < 3; ++k) { cc[k] = color[p * 3 + k]; gg[k] = grad_color[p * 3 + k]; }
            if (it >= 0) zh = boxes[it].zhi;
        }
        h.it[i] = it;
        h.dep[i] = dep;
        h.zhi[i] = zh;
#pragma unroll
        for (int k = 0; k < 3; ++k) { h.c[k][i] = cc[k]; h.g[k][i] = gg[k]; }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ short s_pix[kEdgeThreads];
    __shared__ int s_warp_n[kEdgeThreads / 32];
    int n = 0;
    {
        const int cy = threadIdx.x / DS_TILE, cx = threadIdx.x % DS_TILE;
        const bool cov = h.it[(cy + 1) * kHaloW + cx + 1] >= 0;  // a triangle (not background, not outside)
        const unsigned m = __ballot_sync(0xffffffffu, cov);
        if (lane == 0) s_warp_n[warp] = __popc(m);
        __syncthreads();
        int off = 0;
#pragma unroll
        for (int w = 0; w < kEdgeThreads / 32; ++w) {
            off += w < warp ? s_warp_n[w] : 0;
            n += s_warp_n[w];
        }
        if (cov) s_pix[off + __popc(m & ((1u << lane) - 1u))] = (short)threadIdx.x;
        __syncthreads();
    }
    if (warp * 32 >= n) return;  // warp-uniform: no covered pixel left for this warp
    const bool active = (int)threadIdx.x < n;
    const int src = active ? s_pix[threadIdx.x] : 0;
    const int ly = src / DS_TILE, lx = src % DS_TILE;
    const int y = ty0 + ly, x = tx0 + lx;
    EdgeAccum acc;
    __shared__ float s_adj[4 * kEdgeLanes];  // per thread and neighbour: the marked pairs' adjoints
    static_assert(kEdgeLanes == kEdgeThreads, "one thread per pixel of the tile");
    // every lane of the warp takes part (warp-wide reductions inside); lanes past the covered
    // pixels contribute nothing
    const int it0 = edge_grad_pixel_staged(h, (ly + 1) * kHaloW + lx + 1, y, x, vd.H, vd.W,
                                           tab.verts + (size_t)b * T, acc, s_adj + threadIdx.x, active);
    const int key = (it0 >= 0 && acc.any) ? it0 : -1 - lane;
    if (__ballot_sync(0xffffffffu, key >= 0) == 0) return;  // no lane of the warp has a contribution
    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || prev != key);
    const int seg = __popc(heads & ((2u << lane) - 1u));
    int oseg[5];
#pragma unroll
    for (int s = 0; s < 5; ++s) oseg[s] = __shfl_down_sync(0xffffffffu, seg, 1 << s);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        float v = acc.g[k];
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const float ov = __shfl_down_sync(0xffffffffu, v, 1 << s);
            if (lane + (1 << s) < 32 && oseg[s] == seg) v += ov;
        }
        acc.g[k] = v;
    }
    const bool head = (heads >> lane) & 1u;
    if (head && key >= 0) {
        double* gp = grad_pos + (size_t)b * V * 4;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int v = __ldg(tri + it0 * 3 + k);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (acc.g[k * 4 + j] != 0.f) atomicAdd(gp + (size_t)v * 4 + j, (double)acc.g[k * 4 + j]);
        }
    }
}

__global__ void finish_kernel(const double* __restrict__ loss_sum, float inv_n, float* __restrict__ loss,
                              uint64_t* __restrict__ rng, const int* __restrict__ rec_counters,
                              int* __restrict__ status) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *loss = (float)(*loss_sum * (double)inv_n);
        if (rng) rng[1] += 1;  // next iteration of the opacity-threshold RNG
        if (status && rec_counters[1] > 0) atomicOr(status, DS_STATUS_RECORD_FALLBACK);
    }
}

template <class K>
static int launch_shade(const ShadeArgs& a, cudaStream_t st) {
    const size_t smem = sizeof(ShadeSmem<K>);
    static int per_sm = 0;  // set on the first (eager) call, before any graph capture
    if (per_sm == 0) {
        DS_CUDA(cudaFuncSetAttribute(shade_step_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shade_step_kernel<K>, K::WARPS * 32, smem));
        if (per_sm <= 0) return set_error(DS_ERR_CUDA, "shade_step: kernel does not fit on an SM");
    }
    const int64_t chunks = (a.num_pixels + 31) / 32;
    const int64_t want = (chunks + K::WARPS - 1) / K::WARPS;
    const int64_t cap = (int64_t)sm_count() * (per_sm > 0 ? per_sm : 1);
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
    shade_step_kernel<K><<<grid, K::WARPS * 32, smem, st>>>(a);
    return check_launch("shade_step");
}

// The register-resident kernels of the width-16 MLPs.
template <class K>
static int launch_shade_reg(const ShadeArgs& a, cudaStream_t st) {
    const size_t smem = sizeof(RegSmem<K>);
    static int per_sm = 0;  // set on the first (eager) call, before any graph capture
    if (per_sm == 0) {
        DS_CUDA(cudaFuncSetAttribute(shade_reg_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shade_reg_kernel<K>, kShadeRegWarps * 32, smem));
        if (per_sm <= 0) return set_error(DS_ERR_CUDA, "shade_reg: kernel does not fit on an SM");
    }
    const int64_t chunks = (a.num_pixels + 31) / 32;
    const int64_t want = (chunks + kShadeRegWarps - 1) / kShadeRegWarps;
    const int64_t cap = (int64_t)sm_count() * per_sm;
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
    shade_reg_kernel<K><<<grid, kShadeRegWarps * 32, smem, st>>>(a);
    return check_launch("shade_reg");
}

// The tcgen05 kernel of the wide BF16 MLP: persistent over 128-pixel tiles.
static int launch_shade_tc(const ShadeArgs& a, cudaStream_t st) {
    const size_t smem = sizeof(TcSmem);
    static int per_sm = 0;  // set on the first (eager) call, before any graph capture
    if (per_sm == 0) {
        DS_CUDA(cudaFuncSetAttribute(shade_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DS_CUDA(cudaFuncSetAttribute(shade_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
        DS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shade_tc_kernel, kTcThreads, smem));
        // The query answers 1 for this kernel's 105 KB, while two CTAs fit the SM's shared memory and
        // registers (and run together: measured 1.6x the throughput of one).  Take the count those two
        // limits allow.
        int dev = 0, smem_sm = 0, reserved = 0;
        cudaFuncAttributes fa;
        DS_CUDA(cudaGetDevice(&dev));
        DS_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        DS_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
        DS_CUDA(cudaFuncGetAttributes(&fa, shade_tc_kernel));
        const int by_smem = smem_sm / (int)(smem + (size_t)reserved);
        const int regs = (fa.numRegs + 7) / 8 * 8;  // allocation granularity per thread
        const int by_regs = regs > 0 ? 65536 / (regs * kTcThreads) : 1;
        const int fit = by_smem < by_regs ? by_smem : by_regs;
        if (fit > per_sm) per_sm = fit;
        if (per_sm <= 0) return set_error(DS_ERR_CUDA, "shade_tc: kernel does not fit on an SM");
        if (per_sm > 2) per_sm = 2;  // 256 TMEM columns per CTA: two CTAs fill an SM's 512
    }
    const int64_t tiles = (a.num_pixels + kTcThreads - 1) / kTcThreads;
    const int64_t cap = (int64_t)sm_count() * per_sm;
    const unsigned grid = (unsigned)(tiles < 1 ? 1 : (tiles < cap ? tiles : cap));
    shade_tc_kernel<<<grid, kTcThreads, smem, st>>>(a);
    return check_launch("shade_tc");
}

static inline size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

// Optional phase events (profiling): recorded on the step's stream at the
// boundaries prep | bin | raster | shade | aux | edge | finish.
constexpr int kStepEvents = 8;
static cudaEvent_t g_step_events[kStepEvents];
static int g_step_nevents = 0;

static int mark(int i, cudaStream_t st) {
    if (i < g_step_nevents) DS_CUDA(cudaEventRecord(g_step_events[i], st));
    return DS_OK;
}

// A second stream per device for the parts of the step that do not depend on
// each other (level accumulation beside projection and binning; the opacity
// auxiliary gradient beside the edge gradients).  The caller's stream forks
// to it through an event and joins it back before the dependent kernels, so
// the step stays one ordered unit on the caller's stream and captures into a
// CUDA graph as parallel branches.  Created on a device's first step.
constexpr int kMaxDevices = 64;
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork[2] = {nullptr, nullptr}, join[2] = {nullptr, nullptr};
};
static SideStream g_side[kMaxDevices];

static SideStream* side_stream() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    SideStream& x = g_side[dev];
    if (x.s == nullptr) {
        SideStream n;
        if (cudaStreamCreateWithFlags(&n.s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        for (int i = 0; i < 2; ++i)
            if (cudaEventCreateWithFlags(&n.fork[i], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&n.join[i], cudaEventDisableTiming) != cudaSuccess)
                return nullptr;
        x = n;
    }
    return &x;
}

// The side stream starts after everything issued so far on st.
static int fork_to(SideStream* x, int i, cudaStream_t st) {
    DS_CUDA(cudaEventRecord(x->fork[i], st));
    DS_CUDA(cudaStreamWaitEvent(x->s, x->fork[i], 0));
    return DS_OK;
}

// Work issued on st from now on starts after the side stream's work.
static int join_from(SideStream* x, int i, cudaStream_t st) {
    DS_CUDA(cudaEventRecord(x->join[i], x->s));
    DS_CUDA(cudaStreamWaitEvent(st, x->join[i], 0));
    return DS_OK;
}

struct StepWs {
    float* pos;
    float* alpha_acc;
    float* feat_acc;
    __nv_bfloat16* feat_bf16;
    float* rast;
    float* color;
    float* grad_color;
    float* l1;
    uint4* tab;         // lattice tables of the level accumulation, from its forward kernel
    double* grad_pos;
    float* grad_alpha_acc;
    float* grad_feat_acc;
    double* loss_sum;
    int* rec_counters;  // [2], zeroed with the accumulators
    void* tiles;
    size_t tiles_bytes;
    RecordStore rec;    // rec.capacity == 0: no records
};

// Fragment records reserved for P pixels: frag_records per pixel plus one
// chunk for every warp of the rasterizer's grid (each warp's last chunk is
// partly filled), a multiple of the chunk size.
static int64_t record_capacity(const ds_step_config& c, int num_tiles, int64_t P) {
    if (!(c.frag_records > 0.f)) return 0;
    const double n = std::ceil((double)P * (double)c.frag_records / kRecChunk);
    const int64_t items = (int64_t)num_tiles * 8;
    const int64_t warps = max_resident_warps();
    return ((int64_t)n + (items < warps ? items : warps)) * kRecChunk;
}

// Channel stride of the step's accumulated feature tables (and their
// gradients): C rounded up to a multiple of 8, so that a lattice sample is
// one or more 16-byte (bf16) / 32-byte (fp32) vectors.
static int feat_stride(const ds_step_config& c) { return (c.C + 7) & ~7; }

static StepWs carve_step(void* ws, const ds_step_config& c, int num_tiles, int64_t P, int64_t cap, size_t* total) {
    char* base = reinterpret_cast<char*>(ws);
    const int ST = (int)feats_at_level((uint32_t)c.max_level);
    size_t o = 0;
    StepWs w;
    w.pos = reinterpret_cast<float*>(base + o); o += al((size_t)c.B * c.V * 16);
    w.alpha_acc = reinterpret_cast<float*>(base + o); o += al((size_t)c.T * ST * 4);
    const int CP = feat_stride(c);
    w.feat_acc = reinterpret_cast<float*>(base + o); o += al((size_t)c.T * ST * CP * 4);
    w.feat_bf16 = reinterpret_cast<__nv_bfloat16*>(base + o); o += al((size_t)c.T * ST * CP * 2);
    w.rast = reinterpret_cast<float*>(base + o); o += al((size_t)P * 16);
    w.color = reinterpret_cast<float*>(base + o); o += al((size_t)P * 12);
    w.grad_color = reinterpret_cast<float*>(base + o); o += al((size_t)P * 12);
    w.l1 = reinterpret_cast<float*>(base + o); o += al((size_t)P * 4);
    w.tab = reinterpret_cast<uint4*>(base + o);
    o += al(lattice_tab_bytes(ST * (c.max_level - c.min_level + 1) * 3,
                              (int)total_feats((uint32_t)c.min_level, (uint32_t)c.max_level), ST));
    // zeroed together each step: grad_pos .. loss_sum
    w.grad_pos = reinterpret_cast<double*>(base + o); o += al((size_t)c.B * c.V * 32);
    w.grad_alpha_acc = reinterpret_cast<float*>(base + o); o += al((size_t)c.T * ST * 4);
    w.grad_feat_acc = reinterpret_cast<float*>(base + o); o += al((size_t)c.T * ST * CP * 4);
    w.loss_sum = reinterpret_cast<double*>(base + o);
    w.rec_counters = reinterpret_cast<int*>(base + o + 64);
    o += 256;
    w.tiles = base + o;
    w.tiles_bytes = ds_tiles_workspace_size(c.B, c.T, num_tiles, cap);
    o += al(w.tiles_bytes);
    const int64_t rcap = record_capacity(c, num_tiles, P);
    w.rec.capacity = rcap;
    w.rec.counters = w.rec_counters;
    w.rec.rec = reinterpret_cast<int4*>(base + o); o += al((size_t)rcap * sizeof(int4));
    w.rec.chunk_fill = reinterpret_cast<int*>(base + o); o += al((size_t)(rcap / kRecChunk) * sizeof(int));
    w.rec.fallback = reinterpret_cast<int*>(base + o); o += al(rcap > 0 ? (size_t)num_tiles * 8 * sizeof(int) : 0);
    if (total) *total = o;
    return w;
}

// log2 of the width of the tiled kernels' pixel blocks for ds_step_config.block_shape
static int block_shape_log2(const ds_step_config& c) {
    return c.block_shape == 1 ? 4 : (c.block_shape == 2 ? 2 : kDefaultBlockShape);
}

// The fused shading kernels a step can run, by MLP shape.
enum ShadeShape {
    kShadeUnsupported = 0,
    kShadeC8Dir16 = 1,     // 8 features + view direction -> 16 -> 3 (the benchmark configurations 1-3)
    kShadeC7Sh2_16x2 = 2,  // 7 features + SH2 -> 16 -> 16 -> 3 (the reference's own model)
    kShadeC16Dir64x2 = 3,  // 16 features + view direction -> 64 -> 64 -> 3 (configurations 4-5)
};

static int shade_shape(const ds_step_config& c) {
    if (c.hidden == 16 && c.n_layers == 1 && c.C == 8 && c.view_enc == 0) return kShadeC8Dir16;
    if (c.hidden == 16 && c.n_layers == 2 && c.C == 7 && c.view_enc == 1) return kShadeC7Sh2_16x2;
    if (c.hidden == 64 && c.n_layers == 2 && c.C == 16 && c.view_enc == 0) return kShadeC16Dir64x2;
    return kShadeUnsupported;
}

}  // namespace dsb

using namespace dsb;

using ShadeC8Dir16 = RegCfg<8, 3, 1, false>;        // 8 features + 3 view dir -> 16 -> 3
using ShadeC8Dir16Split = RegCfg<8, 3, 1, true>;
using ShadeC7Sh2_16x2 = RegCfg<7, 9, 2, false>;     // 7 features + 9 SH2 -> 16 -> 16 -> 3
using ShadeC7Sh2_16x2Split = RegCfg<7, 9, 2, true>;
using ShadeC16H64 = ShadeCfg<16, 32, 64, 2>;        // 16 + 3 -> 64 -> 64 -> 3
using ShadeC16H64Split = ShadeCfg<16, 32, 64, 2, true>;

extern "C" {

size_t ds_train_step_workspace_size(const ds_step_config* cfg, int num_tiles, int64_t num_pixels,
                                    int64_t list_capacity) {
    size_t total = 0;
    carve_step(nullptr, *cfg, num_tiles, num_pixels, list_capacity, &total);
    return total;
}

int ds_train_step_set_events(void* const* events, int n) {
    DS_CHECK_ARG(n >= 0 && n <= kStepEvents && (n == 0 || events != nullptr), "train_step_set_events: bad count");
    for (int i = 0; i < n; ++i) g_step_events[i] = (cudaEvent_t)events[i];
    g_step_nevents = n;
    return DS_OK;
}

int ds_train_step_layout(const ds_step_config* cfg, int num_tiles, int64_t num_pixels, int64_t list_capacity,
                         int64_t* offsets) {
    DS_CHECK_ARG(cfg != nullptr && offsets != nullptr, "train_step_layout: null argument");
    StepWs w = carve_step(nullptr, *cfg, num_tiles, num_pixels, list_capacity, nullptr);
    const void* ptrs[15] = {w.pos, w.alpha_acc, w.feat_acc, w.feat_bf16, w.rast, w.color, w.grad_color, w.l1,
                            w.grad_pos, w.grad_alpha_acc, w.grad_feat_acc, w.rec.rec, w.rec.chunk_fill,
                            w.rec_counters, w.rec.fallback};
    for (int i = 0; i < 15; ++i) offsets[i] = (int64_t)(reinterpret_cast<const char*>(ptrs[i]) - (const char*)nullptr);
    offsets[15] = w.rec.capacity;
    return DS_OK;
}

int ds_project_vertices(int B, int V, const float* verts, const float* mvp, float* pos, ds_stream_t stream) {
    DS_CHECK_ARG(B >= 0 && V >= 0 && (int64_t)B * V <= 0x7fffffff, "project_vertices: bad sizes");
    DS_CHECK_ARG((int64_t)B * V == 0 || (verts && mvp && pos), "project_vertices: null pointer");
    DS_CHECK_ARG(((uintptr_t)pos & 15) == 0, "project_vertices: pos not 16-byte aligned");
    if ((int64_t)B * V == 0) return DS_OK;
    project_kernel<<<blocks_for((int64_t)B * V), kThreads, 0, (cudaStream_t)stream>>>(B, V, verts, mvp, pos);
    return check_launch("project_vertices");
}

int ds_mlp_param_count(int C, int hidden, int n_layers) {
    const int in = C + 3;
    return hidden * in + hidden + (n_layers - 1) * (hidden * hidden + hidden) + 3 * hidden + 3;
}

int ds_step_mlp_param_count(const ds_step_config* cfg) {
    if (cfg == nullptr) return set_error(DS_ERR_ARG, "step_mlp_param_count: null config"), -1;
    // C + 9 inputs with SH2: the count for C + 6 features and a 3-D direction
    return ds_mlp_param_count(cfg->C + (cfg->view_enc ? 6 : 0), cfg->hidden, cfg->n_layers);
}

int ds_train_step(const ds_step_config* cfg, const ds_view_desc* views, int num_tiles, int64_t num_pixels,
                  const float* verts, const int* tri, const float* mvp, const float* inv_mvp, const float* feat_src,
                  const float* alpha_src, const float* mlp_params, const void* target, uint64_t* rng,
                  float* loss, float* grad_verts, float* grad_feat_src, float* grad_alpha_src,
                  float* grad_mlp_params, float* rast_out, float* color_out, void* workspace, size_t workspace_bytes,
                  int64_t list_capacity, int* status, ds_stream_t stream) {
    DS_CHECK_ARG(cfg != nullptr, "train_step: null config");
    const ds_step_config c = *cfg;
    DS_CHECK_ARG(c.B > 0 && c.T >= 0 && c.V >= 0 && num_tiles > 0 && num_pixels > 0, "train_step: bad sizes");
    DS_CHECK_ARG(c.min_level >= 0 && c.max_level >= c.min_level && c.max_level <= 8, "train_step: bad levels");
    DS_CHECK_ARG(c.stochastic == 0 || rng != nullptr, "train_step: stochastic opacity needs the rng state");
    DS_CHECK_ARG(c.precision == 0 || c.precision == 1, "train_step: precision must be 0 (bf16) or 1 (split bf16)");
    DS_CHECK_ARG(c.block_shape >= 0 && c.block_shape <= 2, "train_step: block_shape must be 0 (8x4), 1 (16x2) or 2 (4x8)");
    DS_CHECK_ARG(c.view_enc == 0 || c.view_enc == 1, "train_step: view_enc must be 0 (direction) or 1 (SH2)");
    DS_CHECK_ARG(c.target_u8 == 0 || c.target_u8 == 1, "train_step: target_u8 must be 0 (fp32) or 1 (8-bit)");
    DS_CHECK_ARG(c.shade_mode == 0 || c.shade_mode == 1, "train_step: shade_mode must be 0 (mma.sync) or 1 (tcgen05)");
    const int shape = shade_shape(c);
    DS_CHECK_ARG(shape != kShadeUnsupported,
                 "train_step: unsupported MLP (C=%d, %s, hidden=%d, layers=%d); built: 8+dir->16->3, "
                 "7+SH2->16->16->3, 16+dir->64->64->3", c.C, c.view_enc ? "SH2" : "dir", c.hidden, c.n_layers);
    const int CP = feat_stride(c);
    const int S = (int)total_feats((uint32_t)c.min_level, (uint32_t)c.max_level);
    const int ST = (int)feats_at_level((uint32_t)c.max_level);
    DS_CHECK_ARG(S * c.C <= kMaxSrc, "train_step: %d samples x %d channels exceed the per-triangle limit", S, c.C);
    DS_CHECK_ARG(num_pixels <= 0xffffffffLL, "train_step: more than 2^32 pixels");
    DS_CHECK_ARG(c.frag_records >= 0.f && record_capacity(c, num_tiles, num_pixels) <= 0x7fffffffLL - max_resident_warps() * kRecChunk,
                 "train_step: frag_records %g gives too many records", (double)c.frag_records);
    size_t need = 0;
    StepWs w = carve_step(workspace, c, num_tiles, num_pixels, list_capacity, &need);
    const RecordStore* rs = w.rec.capacity > 0 ? &w.rec : nullptr;
    if (workspace_bytes < need) return set_error(DS_ERR_WORKSPACE, "train_step: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;

    int rc = mark(0, st);
    if (rc) return rc;
    // zero the accumulators of this step
    DS_CUDA(cudaMemsetAsync(w.grad_pos, 0,
                            reinterpret_cast<char*>(w.rec_counters + 2) - reinterpret_cast<char*>(w.grad_pos), st));
    DS_CUDA(cudaMemsetAsync(grad_mlp_params, 0, sizeof(float) * ds_step_mlp_param_count(&c), st));

    // Side stream for independent parts; the phase events (profiling) time
    // the phases one after another on st instead.
    SideStream* side = g_step_nevents == 0 ? side_stream() : nullptr;
    const cudaStream_t sst = side ? side->s : st;
    if (side && (rc = fork_to(side, 0, st))) return rc;

    // prep: opacity and feature accumulation + sigmoid (side), projection (st)
    const unsigned tb = (unsigned)((c.T + kPrepWarps - 1) / kPrepWarps);
    const bool tab = lattice_tab_fits(c.min_level, c.max_level, S, ST, CP);
    const size_t tsm = lattice_tab_smem(c.min_level, c.max_level, S, ST, CP, false);
    const size_t tsm_bwd = lattice_tab_smem(c.min_level, c.max_level, S, ST, CP, true);
    const int64_t tw = ((int64_t)c.T + (32 / CP) * kTabWarps - 1) / ((32 / CP) * kTabWarps);  // CTAs of 32/CP triangles a warp
    const int64_t nsm = sm_count();
    // the adjoint: persistent CTAs, each copying the forward's tables once
    const unsigned tgrid_bwd = (unsigned)(tw < nsm * 8 ? tw : nsm * 8);
    if (c.T > 0 && tab) {
#define DSB_ACCUM_TAB(CC, CPP)                                                                                     \
    do {                                                                                                           \
        int per_sm = 1;                                                                                            \
        if ((rc = tab_smem_attr<accum_tab_kernel<CC, CPP>>(tsm, &per_sm))) return rc;                              \
        /* one wave of persistent CTAs, each building the tables once */                                           \
        const unsigned tgrid = (unsigned)(tw < nsm * per_sm ? tw : nsm * per_sm);                                  \
        accum_tab_kernel<CC, CPP><<<tgrid, kTabWarps * 32, tsm, sst>>>(c.T, c.min_level, c.max_level, S, ST,       \
                                                                       alpha_src, feat_src, w.alpha_acc,           \
                                                                       w.feat_acc, w.feat_bf16, w.tab);            \
    } while (0)
        if (c.C == 8) DSB_ACCUM_TAB(8, 8);
        else if (c.C == 7) DSB_ACCUM_TAB(7, 8);
        else DSB_ACCUM_TAB(16, 16);
#undef DSB_ACCUM_TAB
    } else if (c.T > 0) {
        accum_sigmoid_kernel<false><<<tb, kPrepWarps * 32, 0, sst>>>(c.T, c.min_level, c.max_level, c.max_level, S, ST,
                                                                    1, 1, alpha_src, w.alpha_acc, nullptr);
        accum_sigmoid_kernel<true><<<tb, kPrepWarps * 32, 0, sst>>>(c.T, c.min_level, c.max_level, c.max_level, S, ST,
                                                                   c.C, CP, feat_src, w.feat_acc, w.feat_bf16);
    }
    if ((int64_t)c.B * c.V > 0)
        project_kernel<<<blocks_for((int64_t)c.B * c.V), kThreads, 0, st>>>(c.B, c.V, verts, mvp, w.pos);
    rc = check_launch("train_step prep");
    if (rc || (rc = mark(1, st))) return rc;

    // forward rasterization
    float* rast = rast_out ? rast_out : w.rast;
    rc = ds_tiles_bin(c.B, views, num_tiles, c.V, w.pos, c.T, tri, w.tiles, w.tiles_bytes, list_capacity, status,
                      stream);
    if (rc || (rc = mark(2, st))) return rc;
    if (side && (rc = join_from(side, 0, st))) return rc;  // the rasterizer reads the accumulated opacities
    rc = tiles_rasterize_impl(c.B, views, num_tiles, c.T, c.max_level, ST, w.alpha_acc, c.stochastic ? 1 : 0,
                              c.thr_const, rng, rast, w.tiles, list_capacity, rs, st, block_shape_log2(c));
    if (rc || (rc = mark(3, st))) return rc;

    // fused shading forward + backward
    ShadeArgs a;
    a.B = c.B; a.views = views; a.num_pixels = num_pixels; a.rast = rast; a.feat = w.feat_bf16;
    a.feat_f32 = w.feat_acc;
    a.level = c.max_level; a.S = ST; a.inv_mvp = inv_mvp; a.params = mlp_params;
    a.target = c.target_u8 ? nullptr : reinterpret_cast<const float*>(target);
    a.target_u8 = c.target_u8 ? reinterpret_cast<const uint8_t*>(target) : nullptr;
    a.inv_n = (float)(1.0 / ((double)num_pixels * 3.0));
    a.color = color_out ? color_out : w.color; a.grad_color = w.grad_color; a.l1 = w.l1;
    a.grad_feat = w.grad_feat_acc; a.grad_params = grad_mlp_params; a.loss_sum = w.loss_sum; a.status = status;
    const bool split = c.precision == 1;
    switch (shape) {
        case kShadeC8Dir16:
            rc = split ? launch_shade_reg<ShadeC8Dir16Split>(a, st) : launch_shade_reg<ShadeC8Dir16>(a, st);
            break;
        case kShadeC7Sh2_16x2:
            rc = split ? launch_shade_reg<ShadeC7Sh2_16x2Split>(a, st) : launch_shade_reg<ShadeC7Sh2_16x2>(a, st);
            break;
        default:
            if (split) rc = launch_shade<ShadeC16H64Split>(a, st);
            else rc = c.shade_mode == 1 ? launch_shade_tc(a, st) : launch_shade<ShadeC16H64>(a, st);
    }
    if (rc || (rc = mark(4, st))) return rc;

    // adjoints of sigmoid + level accumulation: they read the opacity and feature gradients, not the
    // vertex gradients, so with a side stream they run there after the opacity pass, beside the edge
    // gradients
    auto accum_backward = [&](cudaStream_t s) -> int {
        int r = DS_OK;
        if (c.T > 0 && tab) {
#define DSB_ACCUM_TAB_BWD(CC, CPP)                                                                                 \
    do {                                                                                                           \
        if ((r = tab_smem_attr<accum_tab_backward_kernel<CC, CPP>>(tsm_bwd))) return r;                            \
        accum_tab_backward_kernel<CC, CPP><<<tgrid_bwd, kTabWarps * 32, tsm_bwd, s>>>(                             \
            c.T, c.min_level, c.max_level, S, ST, w.alpha_acc, w.grad_alpha_acc, w.feat_acc, w.grad_feat_acc,      \
            grad_alpha_src, grad_feat_src, w.tab);                                                                 \
    } while (0)
            if (c.C == 8) DSB_ACCUM_TAB_BWD(8, 8);
            else if (c.C == 7) DSB_ACCUM_TAB_BWD(7, 8);
            else DSB_ACCUM_TAB_BWD(16, 16);
#undef DSB_ACCUM_TAB_BWD
        } else if (c.T > 0) {
            accum_sigmoid_backward_kernel<<<tb, kPrepWarps * 32, 0, s>>>(c.T, c.min_level, c.max_level, c.max_level,
                                                                         S, ST, 1, 1, w.alpha_acc, w.grad_alpha_acc,
                                                                         grad_alpha_src);
            accum_sigmoid_backward_kernel<<<tb, kPrepWarps * 32, 0, s>>>(c.T, c.min_level, c.max_level, c.max_level,
                                                                         S, ST, c.C, CP, w.feat_acc,
                                                                         w.grad_feat_acc, grad_feat_src);
        }
        return r;
    };

    // opacity auxiliary gradient (scaled by 1/numel(colour), rasterize.py:183-195), on the side
    // stream beside the edge gradients
    if (side && (rc = fork_to(side, 1, st))) return rc;
    rc = tiles_aux_impl(c.B, views, num_tiles, c.T, c.max_level, ST, w.alpha_acc, w.l1, rast, a.inv_n,
                        w.grad_alpha_acc, w.tiles, list_capacity, rs, sst, block_shape_log2(c));
    if (rc) return rc;
    if (side && (rc = accum_backward(sst))) return rc;
    if ((rc = mark(5, st))) return rc;

    // edge gradients to clip-space positions
    edge_step_kernel<<<(unsigned)num_tiles, kEdgeThreads, 0, st>>>(
        c.B, views, c.V, c.T, tiles_tables(w.tiles, c.B, c.T, num_tiles, list_capacity), tri, a.color, w.grad_color,
        rast, w.grad_pos);
    if ((rc = mark(6, st))) return rc;
    if (side && (rc = join_from(side, 1, st))) return rc;
    // (one stream: the phases in order, so that the profiling events time each alone)
    if (!side && (rc = accum_backward(st))) return rc;
    // adjoint of the projection
    if (c.V > 0) project_backward_kernel<<<blocks_for(c.V), kThreads, 0, st>>>(c.B, c.V, mvp, w.grad_pos, grad_verts);
    finish_kernel<<<1, 32, 0, st>>>(w.loss_sum, a.inv_n, loss, c.stochastic ? rng : nullptr, w.rec_counters, status);
    if ((rc = mark(7, st))) return rc;
    return check_launch("train_step");
}

}  // extern "C"
