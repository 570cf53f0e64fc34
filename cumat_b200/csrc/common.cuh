// Shared definitions of the sm_100a batched sparse CG library.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/cumat_cg.h"

namespace cmcg {

// ---- errors -----------------------------------------------------------------
// Errors never cross the C ABI as exceptions: every entry point returns a
// status code and records a message retrievable with cmcg_last_error_string()
// (per host thread, like the reference's per-thread Context,
// cuMat/src/Context.h:204-214).
void set_error(const std::string& msg);
cmcg_status fail(cmcg_status code, const std::string& msg);
cmcg_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define CMCG_CUDA(call)                                                          \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) return ::cmcg::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

#define CMCG_CHECK_LAUNCH() CMCG_CUDA(cudaGetLastError())

#define CMCG_REQUIRE(cond, msg)                                                  \
    do {                                                                         \
        if (!(cond)) return ::cmcg::fail(CMCG_ERR_INVALID_ARGUMENT, msg);         \
    } while (0)

#define CMCG_TRY(expr)                                                           \
    do {                                                                         \
        cmcg_status s_ = (expr);                                                 \
        if (s_ != CMCG_OK) return s_;                                            \
    } while (0)

// Log hook (cmcg_set_log_callback / CUMAT_LOG): level 0 = error, 1 = info,
// 2 = detail. log_on tells whether a message of that level goes anywhere, so
// callers skip formatting otherwise.
bool log_on(int level);
void log_msg(int level, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

// NVTX range over an entry point (a no-op unless a tool listens)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Number of kernel launches issued by this library on the current host thread
// (a test hook in the spirit of the reference's CUMAT_PROFILING counters,
// cuMat/src/Profiling.h:23-145).
void count_launch(int n = 1);

// ---- dtype helpers ------------------------------------------------------------
inline size_t dtype_size(int dt) {
    switch (dt) {
        case CMCG_F32: return 4;
        case CMCG_F64: return 8;
        case CMCG_BF16: return 2;
        default: return 0;
    }
}

template <typename T> struct DT;
template <> struct DT<float> { static constexpr int id = CMCG_F32; };
template <> struct DT<double> { static constexpr int id = CMCG_F64; };
template <> struct DT<__nv_bfloat16> { static constexpr int id = CMCG_BF16; };

__device__ __forceinline__ float to_f32(float v) { return v; }
__device__ __forceinline__ float to_f32(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ double to_f64(float v) { return static_cast<double>(v); }
__device__ __forceinline__ double to_f64(double v) { return v; }
__device__ __forceinline__ double to_f64(__nv_bfloat16 v) { return static_cast<double>(__bfloat162float(v)); }

// Converts a stored matrix value to the arithmetic type VT.
template <typename VT, typename MT> __device__ __forceinline__ VT mval(MT v);
template <> __device__ __forceinline__ float mval<float, float>(float v) { return v; }
template <> __device__ __forceinline__ float mval<float, __nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float mval<float, double>(double v) { return static_cast<float>(v); }
template <> __device__ __forceinline__ double mval<double, float>(float v) { return static_cast<double>(v); }
template <> __device__ __forceinline__ double mval<double, double>(double v) { return v; }
template <> __device__ __forceinline__ double mval<double, __nv_bfloat16>(__nv_bfloat16 v) { return static_cast<double>(__bfloat162float(v)); }

// Rounds an FP64 value to the storage type T.
template <typename T> __device__ __forceinline__ T from_f64(double v);
template <> __device__ __forceinline__ float from_f64<float>(double v) { return static_cast<float>(v); }
template <> __device__ __forceinline__ double from_f64<double>(double v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f64<__nv_bfloat16>(double v) { return __double2bfloat16(v); }

// Four consecutive stored values starting at a 4-entry aligned index.
template <typename MT> struct Vals4;
template <> struct Vals4<float> {
    float v[4];
    __device__ __forceinline__ void load(const float* p) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
};
template <> struct Vals4<double> {
    double v[4];
    __device__ __forceinline__ void load(const double* p) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
};
template <> struct Vals4<__nv_bfloat16> {
    __nv_bfloat16 v[4];
    __device__ __forceinline__ void load(const __nv_bfloat16* p) {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
        const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&t.x);
        const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&t.y);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
};

// ---- warp / block reductions ---------------------------------------------------
constexpr unsigned FULL = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Block-wide sum of NV values; every thread gets the totals. `red` is shared
// scratch of at least NV * (blockDim.x / 32) elements. Two __syncthreads.
// The combine order is fixed, so results are deterministic.
template <typename T, int NV>
__device__ __forceinline__ void block_sum(T (&v)[NV], T* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) red[j * nw + warp] = v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        T s = (lane < nw) ? red[j * nw + lane] : T(0);
        v[j] = warp_sum(s);
    }
    __syncthreads();
}

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

}  // namespace cmcg
