// Batched reductions of a dense column-major batched matrix along any set of
// axes (rows, columns, batches), with the kernel picked per shape by timing.
//
// Replaces the reference's reductions over axis combinations
// (cuMat/src/ReductionOps.h, the sum / prod / minCoeff / maxCoeff plugins of
// ReductionOpsPlugin.inl) and their dynamic algorithm selection, whose
// thresholds were measured on an RTX 2070 (ReductionAlgorithmSelection.h:40-112).
//
// Layout: input [batches][cols][rows] (rows fastest, the reference's
// ColumnMajor), output the kept axes in the same order. Any reduction of the
// three axes is one of five views after merging neighbouring axes of the same
// role, all covered by one index form over four levels, outer to inner,
//     in[((o2 * K2 + k2) * O1 + o1) * K1 + k1]  ->  out[o2 * O1 + o1]
// (k: reduced, o: kept). Kernels:
//   thread   one thread per output, o1 across the threads (coalesced when the
//            reduction is not along rows, K1 == 1), k in order
//   warp     one warp per output, lanes over k1 (contiguous), shuffle combine
//   block    one CTA per output, threads over (k2, k1), shuffles + one shared
//            combine
//   split    outputs' reductions cut into S chunks over S CTAs (few outputs,
//            long reductions), partials in context scratch, then one warp per
//            output adds its S partials (lanes over the partials in order,
//            then the shuffle tree)
//   tile     reductions along an outer axis (K1 == 1, the kept innermost axis
//            O1 contiguous): a CTA covers 32 V consecutive outputs of one o2
//            (16-byte loads, V = 16 / sizeof(T), where O1 and the address
//            allow) and a chunk of k2 split over its 8 warps; the warps'
//            partials are added in warp order, and with S chunks per output
//            the chunks' partials are combined as for split
// The warp kernel reads the contiguous reduced run with 16-byte loads where
// K1 and the address allow; block and split do so wherever the reduced range
// of an output is one contiguous run (K2 == 1).
// Each kernel combines in a fixed order, so a given kernel is deterministic;
// MIN / MAX do not depend on the kernel at all, SUM / PROD do at the rounding
// level. The first reduction of a shape times every applicable kernel (one
// warm-up and three timed launches on the context stream) and keeps the
// fastest, in memory and in the tuning cache file of the SpMV autotuner
// (CUMAT_TUNE_CACHE), so later processes on the same GPU model reuse it;
// CUMAT_REDUCE_KERNEL=thread|warp|block|split|tile forces one.

#include <sys/stat.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "common.cuh"
#include "objects.h"

namespace cmcg {
namespace {

enum Kern { K_THREAD = 0, K_WARP = 1, K_BLOCK = 2, K_SPLIT = 3, K_TILE = 4, K_COUNT = 5 };
const char* const kKernName[K_COUNT] = {"thread", "warp", "block", "split", "tile"};

struct View {
    int64_t K1, O1, K2, O2;
    __host__ __device__ int64_t outputs() const { return O1 * O2; }
    __host__ __device__ int64_t length() const { return K1 * K2; }
};

template <typename T, int OP>
struct RedOp;
template <typename T>
struct RedOp<T, CMCG_REDUCE_SUM> {
    __device__ __forceinline__ static T id() { return T(0); }
    __device__ __forceinline__ static T f(T a, T b) { return a + b; }
};
template <typename T>
struct RedOp<T, CMCG_REDUCE_PROD> {
    __device__ __forceinline__ static T id() { return T(1); }
    __device__ __forceinline__ static T f(T a, T b) { return a * b; }
};
template <typename T>
struct RedOp<T, CMCG_REDUCE_MIN> {
    __device__ __forceinline__ static T id() { return static_cast<T>(INFINITY); }
    __device__ __forceinline__ static T f(T a, T b) { return b < a ? b : a; }
};
template <typename T>
struct RedOp<T, CMCG_REDUCE_MAX> {
    __device__ __forceinline__ static T id() { return -static_cast<T>(INFINITY); }
    __device__ __forceinline__ static T f(T a, T b) { return b > a ? b : a; }
};

template <typename T, int OP>
__device__ __forceinline__ T warp_red(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = RedOp<T, OP>::f(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

template <typename T>
__device__ __forceinline__ int64_t at(const View& v, int64_t o1, int64_t o2, int64_t k1, int64_t k2) {
    return ((o2 * v.K2 + k2) * v.O1 + o1) * v.K1 + k1;
}

// reduction of output o over the k range [kb, ke) of the flattened (k2, k1)
// index, by one thread, in order
template <typename T, int OP>
__device__ __forceinline__ T serial(const T* __restrict__ in, const View& v, int64_t o1, int64_t o2) {
    T acc = RedOp<T, OP>::id();
    for (int64_t k2 = 0; k2 < v.K2; ++k2) {
        const T* row = in + at<T>(v, o1, o2, 0, k2);
        for (int64_t k1 = 0; k1 < v.K1; ++k1) acc = RedOp<T, OP>::f(acc, row[k1]);
    }
    return acc;
}

// f over the flattened reduced index k in [kb, ke), k = k2 * K1 + k1, taking
// every blockDim.x-th element from kb + threadIdx.x; (k2, k1) advance by a
// precomputed step instead of a division per element
template <typename T, int OP>
__device__ __forceinline__ T strided(const T* __restrict__ in, const View& v, int64_t o1, int64_t o2, int64_t kb,
                                     int64_t ke) {
    T acc = RedOp<T, OP>::id();
    int64_t k = kb + threadIdx.x;
    if (k >= ke) return acc;
    int64_t k2 = k / v.K1, k1 = k - k2 * v.K1;
    const int64_t s2 = blockDim.x / v.K1, s1 = blockDim.x - s2 * v.K1;
    for (; k < ke; k += blockDim.x) {
        acc = RedOp<T, OP>::f(acc, in[at<T>(v, o1, o2, k1, k2)]);
        k1 += s1;
        k2 += s2;
        if (k1 >= v.K1) {
            k1 -= v.K1;
            ++k2;
        }
    }
    return acc;
}

template <typename T, int OP>
__global__ void __launch_bounds__(256) k_red_thread(const T* __restrict__ in, T* __restrict__ out, View v) {
    const int64_t n = v.outputs();
    for (int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; o < n;
         o += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t o2 = o / v.O1, o1 = o - o2 * v.O1;
        out[o] = serial<T, OP>(in, v, o1, o2);
    }
}

// V consecutive values from p (16-byte aligned when V > 1)
template <typename T, int V>
__device__ __forceinline__ void load_vec(const T* __restrict__ p, T (&x)[V]) {
    if constexpr (V == 1) {
        x[0] = __ldg(p);
    } else if constexpr (sizeof(T) == 4 && V == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(p));
        x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
    } else {
        static_assert(sizeof(T) == 8 && V == 2, "16-byte vectors of float or double");
        const double2 q = __ldg(reinterpret_cast<const double2*>(p));
        x[0] = q.x; x[1] = q.y;
    }
}

// V > 1: K1 is a multiple of V and the input 16-byte aligned, so every
// reduced run starts on a 16-byte boundary
template <typename T, int OP, int V>
__global__ void __launch_bounds__(256) k_red_warp(const T* __restrict__ in, T* __restrict__ out, View v) {
    const int lane = threadIdx.x & 31;
    const int64_t n = v.outputs();
    const int64_t w0 = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t o = w0; o < n; o += nw) {   // uniform per warp
        const int64_t o2 = o / v.O1, o1 = o - o2 * v.O1;
        T acc = RedOp<T, OP>::id();
        for (int64_t k2 = 0; k2 < v.K2; ++k2) {
            const T* __restrict__ row = in + at<T>(v, o1, o2, 0, k2);
#pragma unroll 4
            for (int64_t k1 = lane * V; k1 < v.K1; k1 += 32 * V) {
                T x[V];
                load_vec<T, V>(row + k1, x);
#pragma unroll
                for (int j = 0; j < V; ++j) acc = RedOp<T, OP>::f(acc, x[j]);
            }
        }
        acc = warp_red<T, OP>(acc);
        if (lane == 0) out[o] = acc;
    }
}

// tile (K1 == 1): item (tile t of 32 V outputs along o1 within o2, chunk s of
// k2); dst = out when S == 1, else the partials [output][S]. V > 1: O1 is a
// multiple of V and the input 16-byte aligned.
template <typename T, int OP, int V>
__global__ void __launch_bounds__(256) k_red_tile(const T* __restrict__ in, T* __restrict__ dst, View v, int32_t S,
                                                  int64_t tiles_o1) {
    __shared__ T sh[8][32 * V];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t items = tiles_o1 * v.O2 * S;
    const int64_t chunk = (v.K2 + S - 1) / S;
    for (int64_t item = blockIdx.x; item < items; item += gridDim.x) {
        const int64_t t = item / S, s = item - t * S;
        const int64_t o2 = t / tiles_o1, tile = t - o2 * tiles_o1;
        const int64_t o1 = (tile * 32 + lane) * V;
        const int64_t kb = s * chunk, ke = min(v.K2, kb + chunk);
        T acc[V];
#pragma unroll
        for (int j = 0; j < V; ++j) acc[j] = RedOp<T, OP>::id();
        if (o1 < v.O1) {
            const T* __restrict__ col = in + (o2 * v.K2) * v.O1 + o1;
            int64_t k2 = kb + warp;
            // four rows of the chunk in flight per thread, added in row order
            for (; k2 + 24 < ke; k2 += 32) {
                T x[4][V];
#pragma unroll
                for (int u = 0; u < 4; ++u) load_vec<T, V>(col + (k2 + 8 * u) * v.O1, x[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int j = 0; j < V; ++j) acc[j] = RedOp<T, OP>::f(acc[j], x[u][j]);
            }
            for (; k2 < ke; k2 += 8) {
                T x[V];
                load_vec<T, V>(col + k2 * v.O1, x);
#pragma unroll
                for (int j = 0; j < V; ++j) acc[j] = RedOp<T, OP>::f(acc[j], x[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < V; ++j) sh[warp][lane * V + j] = acc[j];
        __syncthreads();
        for (int c = threadIdx.x; c < 32 * V; c += blockDim.x) {
            T r = sh[0][c];
#pragma unroll
            for (int w = 1; w < 8; ++w) r = RedOp<T, OP>::f(r, sh[w][c]);
            const int64_t oo = tile * 32 * V + c;
            if (oo < v.O1) {
                const int64_t o = o2 * v.O1 + oo;
                if (S == 1) dst[o] = r;
                else dst[o * S + s] = r;
            }
        }
        __syncthreads();
    }
}

// block-wide combine: warp shuffles, then the warps' values in order
template <typename T, int OP>
__device__ __forceinline__ T block_red(T acc, T* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    acc = warp_red<T, OP>(acc);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    T t = lane < nw ? red[lane] : RedOp<T, OP>::id();
    t = warp_red<T, OP>(t);
    __syncthreads();
    return t;
}

// f over the contiguous run p[kb, ke) by the CTA's threads (the reduced range
// of one output when K2 == 1): scalar loads up to the first 16-byte boundary
// and after the last one, 16-byte loads in between, four of them in flight
// per thread; each thread adds its elements in a fixed order
template <typename T, int OP>
__device__ __forceinline__ T run_reduce(const T* __restrict__ p, int64_t kb, int64_t ke) {
    constexpr int V = 16 / static_cast<int>(sizeof(T));
    T acc = RedOp<T, OP>::id();
    const int64_t mis = static_cast<int64_t>((reinterpret_cast<uintptr_t>(p + kb) & 15) / sizeof(T));
    const int64_t hb = min(ke, kb + (mis ? V - mis : 0));
    for (int64_t k = kb + threadIdx.x; k < hb; k += blockDim.x) acc = RedOp<T, OP>::f(acc, p[k]);
    const int64_t nv = (ke - hb) / V;
    const T* __restrict__ q = p + hb;
    const int64_t bd = blockDim.x;
    int64_t i = threadIdx.x;
    for (; i + 3 * bd < nv; i += 4 * bd) {
        T x[4][V];
#pragma unroll
        for (int u = 0; u < 4; ++u) load_vec<T, V>(q + (i + u * bd) * V, x[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int j = 0; j < V; ++j) acc = RedOp<T, OP>::f(acc, x[u][j]);
    }
    for (; i < nv; i += bd) {
        T x[V];
        load_vec<T, V>(q + i * V, x);
#pragma unroll
        for (int j = 0; j < V; ++j) acc = RedOp<T, OP>::f(acc, x[j]);
    }
    for (int64_t k = hb + nv * V + threadIdx.x; k < ke; k += bd) acc = RedOp<T, OP>::f(acc, p[k]);
    return acc;
}

template <typename T, int OP>
__global__ void __launch_bounds__(256) k_red_block(const T* __restrict__ in, T* __restrict__ out, View v) {
    __shared__ T red[8];
    const int64_t n = v.outputs(), len = v.length();
    for (int64_t o = blockIdx.x; o < n; o += gridDim.x) {
        const int64_t o2 = o / v.O1, o1 = o - o2 * v.O1;
        T acc = v.K2 == 1 ? run_reduce<T, OP>(in + at<T>(v, o1, o2, 0, 0), 0, len)
                          : strided<T, OP>(in, v, o1, o2, 0, len);
        acc = block_red<T, OP>(acc, red);
        if (threadIdx.x == 0) out[o] = acc;
    }
}

// split: CTA (o, s) reduces chunk s of output o into part[o * S + s]
template <typename T, int OP>
__global__ void __launch_bounds__(256) k_red_split(const T* __restrict__ in, T* __restrict__ part, View v, int32_t S) {
    __shared__ T red[8];
    const int64_t n = v.outputs(), len = v.length();
    const int64_t chunk = (len + S - 1) / S;
    for (int64_t item = blockIdx.x; item < n * S; item += gridDim.x) {
        const int64_t o = item / S, s = item - o * S;
        const int64_t o2 = o / v.O1, o1 = o - o2 * v.O1;
        const int64_t kb = s * chunk, ke = min(len, kb + chunk);
        T acc = v.K2 == 1 ? run_reduce<T, OP>(in + at<T>(v, o1, o2, 0, 0), kb, ke)
                          : strided<T, OP>(in, v, o1, o2, kb, ke);
        acc = block_red<T, OP>(acc, red);
        if (threadIdx.x == 0) part[item] = acc;
    }
}

// the S partials of each output added by one warp: lane l takes partials
// l, l + 32, ... in order, then the lanes are combined by the shuffle tree
// (a fixed order for a given S)
template <typename T, int OP>
__global__ void __launch_bounds__(256) k_red_split_combine(const T* __restrict__ part, T* __restrict__ out, int64_t n,
                                                           int32_t S) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t o = w0; o < n; o += nw) {   // uniform per warp
        T acc = RedOp<T, OP>::id();
        for (int s = lane; s < S; s += 32) acc = RedOp<T, OP>::f(acc, part[o * S + s]);
        acc = warp_red<T, OP>(acc);
        if (lane == 0) out[o] = acc;
    }
}

// Merges the three axes (rows, cols, batches; sizes R, C, B) into the view.
View make_view(int64_t R, int64_t C, int64_t B, int32_t axes) {
    const int64_t sz[3] = {R, C, B};
    const bool red[3] = {(axes & CMCG_AXIS_ROW) != 0, (axes & CMCG_AXIS_COLUMN) != 0, (axes & CMCG_AXIS_BATCH) != 0};
    // runs of equal role from the innermost axis fill the levels K1, O1, K2,
    // O2 in turn (a kept innermost axis leaves K1 = 1); three axes need at
    // most four levels
    int64_t run[4] = {1, 1, 1, 1};
    int level = red[0] ? 0 : 1;
    for (int a = 0; a < 3; ++a) {
        if (a > 0 && red[a] != red[a - 1]) ++level;
        run[level] *= sz[a];
    }
    return View{run[0], run[1], run[2], run[3]};
}

// elements per 16-byte vector
template <typename T>
constexpr int kVec = 16 / static_cast<int>(sizeof(T));

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename T, int OP>
cmcg_status launch_kern(cmcg_ctx ctx, int kern, const View& v, const T* in, T* out) {
    const int64_t n = v.outputs(), len = v.length();
    const int sms = ctx->sm_count;
    cudaStream_t st = ctx->stream;
    if (kern == K_THREAD) {
        const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sms * 16)));
        k_red_thread<T, OP><<<grid, 256, 0, st>>>(in, out, v);
    } else if (kern == K_WARP) {
        const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, sms * 16)));
        if (v.K1 % kVec<T> == 0 && aligned16(in)) k_red_warp<T, OP, kVec<T>><<<grid, 256, 0, st>>>(in, out, v);
        else k_red_warp<T, OP, 1><<<grid, 256, 0, st>>>(in, out, v);
    } else if (kern == K_TILE) {
        const bool vec = v.O1 % kVec<T> == 0 && aligned16(in);
        const int64_t per = 32 * (vec ? kVec<T> : 1);
        const int64_t tiles_o1 = (v.O1 + per - 1) / per;
        const int64_t tiles = tiles_o1 * v.O2;
        // S chunks of k2 per tile so that about 8 CTAs per SM have work, each
        // chunk at least 64 rows of the tile
        const int64_t want = std::max<int64_t>(1, (static_cast<int64_t>(sms) * 8 + tiles - 1) / tiles);
        const int32_t S = static_cast<int32_t>(std::max<int64_t>(1, std::min<int64_t>(want, (v.K2 + 63) / 64)));
        T* dst = out;
        if (S > 1) {
            CMCG_TRY(ensure_buffer(&ctx->red_partial, &ctx->red_partial_bytes, sizeof(T) * static_cast<size_t>(n) * S));
            dst = static_cast<T*>(ctx->red_partial);
        }
        const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(tiles * S, sms * 8)));
        if (vec) k_red_tile<T, OP, kVec<T>><<<grid, 256, 0, st>>>(in, dst, v, S, tiles_o1);
        else k_red_tile<T, OP, 1><<<grid, 256, 0, st>>>(in, dst, v, S, tiles_o1);
        if (S > 1) {
            const int g2 = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, sms * 16)));
            k_red_split_combine<T, OP><<<g2, 256, 0, st>>>(dst, out, n, S);
            count_launch();
        }
    } else if (kern == K_BLOCK) {
        const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(n, sms * 8)));
        k_red_block<T, OP><<<grid, 256, 0, st>>>(in, out, v);
    } else {
        // S chunks per output so that about 8 CTAs per SM have work, each
        // chunk at least 4096 elements
        const int64_t want = std::max<int64_t>(1, (static_cast<int64_t>(sms) * 8 + n - 1) / n);
        const int32_t S = static_cast<int32_t>(std::max<int64_t>(1, std::min<int64_t>(want, (len + 4095) / 4096)));
        const size_t need = sizeof(T) * static_cast<size_t>(n) * S;
        CMCG_TRY(ensure_buffer(&ctx->red_partial, &ctx->red_partial_bytes, need));
        T* part = static_cast<T*>(ctx->red_partial);
        const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(n * S, sms * 8)));
        k_red_split<T, OP><<<grid, 256, 0, st>>>(in, part, v, S);
        const int g2 = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, sms * 16)));
        k_red_split_combine<T, OP><<<g2, 256, 0, st>>>(part, out, n, S);
        count_launch();
    }
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

std::mutex g_red_mu;

// the device's name for the cache keys (' ' and '|' replaced), queried once
// per device: the property query costs far more than a reduction
std::string gpu_name(int device) {
    static std::map<int, std::string> names;
    std::lock_guard<std::mutex> lk(g_red_mu);
    auto it = names.find(device);
    if (it != names.end()) return it->second;
    cudaDeviceProp prop{};
    std::string gpu = cudaGetDeviceProperties(&prop, device) == cudaSuccess ? prop.name : "unknown";
    for (char& ch : gpu)
        if (ch == ' ' || ch == '|') ch = '_';
    names[device] = gpu;
    return gpu;
}

std::map<std::string, int>& red_choices() {
    static std::map<std::string, int> m;
    return m;
}

std::string red_cache_path() {
    if (const char* e = std::getenv("CUMAT_TUNE_CACHE")) return e;
    const char* h = std::getenv("HOME");
    return h ? std::string(h) + "/.cache/cumat_b200/spmv_tune.txt" : std::string();
}

int red_cache_lookup(const std::string& key) {
    const std::string path = red_cache_path();
    if (path.empty()) return -1;
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return -1;
    char line[512];
    int found = -1;
    while (std::fgets(line, sizeof(line), f)) {
        const char* sp = std::strrchr(line, ' ');
        if (sp && std::string(line, sp - line) == key) found = std::atoi(sp + 1);
    }
    std::fclose(f);
    return found;
}

void red_cache_store(const std::string& key, int kern) {
    const std::string path = red_cache_path();
    if (path.empty()) return;
    for (size_t i = path.find('/', 1); i != std::string::npos; i = path.find('/', i + 1))
        ::mkdir(path.substr(0, i).c_str(), 0755);
    if (FILE* f = std::fopen(path.c_str(), "a")) {
        std::fprintf(f, "%s %d\n", key.c_str(), kern);
        std::fclose(f);
    }
}

// The kernels that apply to a view: warp needs a contiguous reduced run
// (K1 > 1), tile an outer reduced axis with the innermost kept (K1 == 1);
// block and split need a reduction long enough to share.
int candidates(const View& v, int (&c)[K_COUNT]) {
    int n = 0;
    c[n++] = K_THREAD;
    if (v.K1 > 1) c[n++] = K_WARP;
    if (v.K1 == 1 && v.K2 > 1) c[n++] = K_TILE;
    if (v.length() >= 512) c[n++] = K_BLOCK;
    if (v.length() >= 8192 && v.outputs() < 4096) c[n++] = K_SPLIT;
    return n;
}

template <typename T, int OP>
cmcg_status reduce_t(cmcg_ctx ctx, const View& v, const void* in_, void* out_) {
    const T* in = static_cast<const T*>(in_);
    T* out = static_cast<T*>(out_);
    // (a forced tile kernel applies only with the innermost axis kept)
    if (const char* e = std::getenv("CUMAT_REDUCE_KERNEL")) {
        for (int k = 0; k < K_COUNT; ++k)
            if (std::strcmp(e, kKernName[k]) == 0 && (k != K_TILE || v.K1 == 1))
                return launch_kern<T, OP>(ctx, k, v, in, out);
    }
    int cand[K_COUNT];
    const int nc = candidates(v, cand);
    if (nc == 1) return launch_kern<T, OP>(ctx, cand[0], v, in, out);
    const std::string key = gpu_name(ctx->device) + "|reduce|" + std::to_string(sizeof(T)) + "|" + std::to_string(OP) + "|" +
                            std::to_string(v.K1) + "|" + std::to_string(v.O1) + "|" + std::to_string(v.K2) + "|" +
                            std::to_string(v.O2);
    {
        std::lock_guard<std::mutex> lk(g_red_mu);
        auto it = red_choices().find(key);
        int k = it != red_choices().end() ? it->second : red_cache_lookup(key);
        if (k >= 0 && k < K_COUNT) {
            red_choices()[key] = k;
            return launch_kern<T, OP>(ctx, k, v, in, out);
        }
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
        return launch_kern<T, OP>(ctx, cand[0], v, in, out);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CMCG_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(CMCG_ERR_CUDA, "reduce autotune: event creation failed");
    }
    float best = 0.0f;
    int pick = cand[0];
    cmcg_status rc = CMCG_OK;
    for (int j = 0; j < nc && rc == CMCG_OK; ++j) {
        rc = launch_kern<T, OP>(ctx, cand[j], v, in, out);
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < 3 && rc == CMCG_OK; ++r) rc = launch_kern<T, OP>(ctx, cand[j], v, in, out);
        cudaEventRecord(e1, ctx->stream);
        float ms = 0.0f;
        if (rc == CMCG_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
            rc = fail(CMCG_ERR_CUDA, "reduce autotune: timing failed");
        if (rc == CMCG_OK && (j == 0 || ms < best)) {
            best = ms;
            pick = cand[j];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != CMCG_OK) return rc;
    {
        std::lock_guard<std::mutex> lk(g_red_mu);
        red_choices()[key] = pick;
        red_cache_store(key, pick);
    }
    log_msg(1, "reduction %s: %s kernel timed fastest (%.3f ms for 3 calls)", key.c_str(), kKernName[pick], best);
    // the last candidate's result is in out; rerun the pick if it was another one
    return pick == cand[nc - 1] ? CMCG_OK : launch_kern<T, OP>(ctx, pick, v, in, out);
}

template <typename T>
cmcg_status reduce_op(cmcg_ctx ctx, int32_t op, const View& v, const void* in, void* out) {
    switch (op) {
        case CMCG_REDUCE_SUM: return reduce_t<T, CMCG_REDUCE_SUM>(ctx, v, in, out);
        case CMCG_REDUCE_PROD: return reduce_t<T, CMCG_REDUCE_PROD>(ctx, v, in, out);
        case CMCG_REDUCE_MIN: return reduce_t<T, CMCG_REDUCE_MIN>(ctx, v, in, out);
        case CMCG_REDUCE_MAX: return reduce_t<T, CMCG_REDUCE_MAX>(ctx, v, in, out);
    }
    return fail(CMCG_ERR_INVALID_ARGUMENT, "cmcg_reduce: op must be SUM, PROD, MIN or MAX");
}

}  // namespace
}  // namespace cmcg

using namespace cmcg;

extern "C" {

cmcg_status cmcg_reduce(cmcg_ctx ctx, int32_t dtype, int32_t op, int64_t rows, int64_t cols, int64_t batches,
                        int32_t axes, const void* in, void* out) {
    NvtxRange nvtx_("cmcg_reduce");
    CMCG_REQUIRE(ctx && in && out, "cmcg_reduce: NULL argument");
    CMCG_REQUIRE(rows > 0 && cols > 0 && batches > 0, "cmcg_reduce: sizes must be positive");
    CMCG_REQUIRE((axes & ~7) == 0, "cmcg_reduce: axes is a mask of CMCG_AXIS_ROW | COLUMN | BATCH");
    CMCG_REQUIRE(dtype == CMCG_F32 || dtype == CMCG_F64, "cmcg_reduce: dtype must be F32 or F64");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    const View v = make_view(rows, cols, batches, axes);
    return dtype == CMCG_F32 ? reduce_op<float>(ctx, op, v, in, out) : reduce_op<double>(ctx, op, v, in, out);
}

}  // extern "C"
