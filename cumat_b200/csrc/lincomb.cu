// Fused linear combination out (mode)= sum_t c_t v_t of up to kMaxTerms
// vectors, every batch, in one streaming pass.
//
// Replaces the reference's cwise evaluation of `v0 * f0 + v1 * f1 + ...`
// (cuMat/src/CwiseOp.h:66-85: one fused kernel per expression tree, as timed
// by benchmarks/linear_combination/Implementation_cuMat.cu:52-66), which a
// BLAS caller would run as a chain of axpy calls, each re-reading the output.
// Here the coefficients and vector pointers travel in the kernel parameters;
// every thread loads one 16-byte vector of every term before the first
// multiply, so a launch keeps k loads per thread in flight, and the sum is
// formed in term order (c_0 v_0 + c_1 v_1 + ...).

#include <algorithm>

#include "common.cuh"
#include "objects.h"

namespace cmcg {
namespace {

constexpr int kMaxTerms = 16;
constexpr int kLcThreads = 256;

template <typename VT>
struct LcArgs {
    const VT* v[kMaxTerms];
    int64_t vstride[kMaxTerms];   // 0: one batch broadcast to all
    VT c[kMaxTerms];
    int32_t k;
    int64_t n;
    int32_t ob;
    VT* out;
    int32_t mode;
};

template <typename VT> struct Vec16;
template <> struct Vec16<float> {
    using T = float4;
    static constexpr int N = 4;
    __device__ static void unpack(const T& t, float (&o)[4]) { o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w; }
    __device__ static T pack(const float (&o)[4]) { return make_float4(o[0], o[1], o[2], o[3]); }
};
template <> struct Vec16<double> {
    using T = double2;
    static constexpr int N = 2;
    __device__ static void unpack(const T& t, double (&o)[2]) { o[0] = t.x; o[1] = t.y; }
    __device__ static T pack(const double (&o)[2]) { return make_double2(o[0], o[1]); }
};

template <int MODE, typename VT>
__device__ __forceinline__ VT lc_out(VT old, VT v) {
    return MODE == CMCG_ASSIGN ? v : MODE == CMCG_ADD ? old + v : old - v;
}

// 16-byte path: n a multiple of the vector width, every pointer 16-byte aligned;
// KM >= k bounds the unrolled term loop (and the registers it holds)
template <typename VT, int MODE, int KM>
__global__ void __launch_bounds__(kLcThreads) k_lincomb_vec(LcArgs<VT> a) {
    using V = Vec16<VT>;
    constexpr int W = V::N;
    const int64_t nv = a.n / W, total = nv * a.ob;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(kLcThreads) + threadIdx.x; it < total;
         it += static_cast<int64_t>(gridDim.x) * kLcThreads) {
        const int64_t b = it / nv, e = it - b * nv;
        typename V::T t[KM];
#pragma unroll
        for (int j = 0; j < KM; ++j)
            if (j < a.k) t[j] = __ldg(reinterpret_cast<const typename V::T*>(a.v[j] + b * a.vstride[j]) + e);
        VT acc[W];
#pragma unroll
        for (int q = 0; q < W; ++q) acc[q] = VT(0);
#pragma unroll
        for (int j = 0; j < KM; ++j) {
            if (j < a.k) {
                VT x[W];
                V::unpack(t[j], x);
#pragma unroll
                for (int q = 0; q < W; ++q) acc[q] = j == 0 ? a.c[0] * x[q] : fma(a.c[j], x[q], acc[q]);
            }
        }
        typename V::T* o = reinterpret_cast<typename V::T*>(a.out + b * a.n) + e;
        if (MODE != CMCG_ASSIGN) {
            VT old[W];
            V::unpack(*o, old);
#pragma unroll
            for (int q = 0; q < W; ++q) acc[q] = lc_out<MODE>(old[q], acc[q]);
        }
        *o = V::pack(acc);
    }
}

// any n and alignment: one element per thread and step
template <typename VT, int MODE, int KM>
__global__ void __launch_bounds__(kLcThreads) k_lincomb_scalar(LcArgs<VT> a) {
    const int64_t total = a.n * a.ob;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(kLcThreads) + threadIdx.x; it < total;
         it += static_cast<int64_t>(gridDim.x) * kLcThreads) {
        const int64_t b = it / a.n, e = it - b * a.n;
        VT t[KM];
#pragma unroll
        for (int j = 0; j < KM; ++j)
            if (j < a.k) t[j] = __ldg(a.v[j] + b * a.vstride[j] + e);
        VT acc = VT(0);
#pragma unroll
        for (int j = 0; j < KM; ++j)
            if (j < a.k) acc = j == 0 ? a.c[0] * t[0] : fma(a.c[j], t[j], acc);
        VT* o = a.out + b * a.n + e;
        *o = lc_out<MODE>(MODE == CMCG_ASSIGN ? VT(0) : *o, acc);
    }
}

template <typename VT>
cmcg_status launch_lincomb(cmcg_ctx ctx, int64_t n, int32_t k, const double* coeffs, const void* const* vectors,
                           const int32_t* vb, void* out, int32_t ob, int32_t mode) {
    LcArgs<VT> a{};
    bool aligned = n % Vec16<VT>::N == 0 && reinterpret_cast<uintptr_t>(out) % 16 == 0;
    for (int j = 0; j < k; ++j) {
        a.v[j] = static_cast<const VT*>(vectors[j]);
        a.vstride[j] = vb[j] == 1 ? 0 : n;
        a.c[j] = static_cast<VT>(coeffs[j]);
        aligned = aligned && reinterpret_cast<uintptr_t>(vectors[j]) % 16 == 0;
    }
    a.k = k;
    a.n = n;
    a.ob = ob;
    a.out = static_cast<VT*>(out);
    a.mode = mode;
    const int64_t items = aligned ? n / Vec16<VT>::N * ob : n * ob;
    const int blocks = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>((items + kLcThreads - 1) / kLcThreads, static_cast<int64_t>(ctx->sm_count) * 8)));
#define CMCG_LC_KM(KERN, M, KM) KERN<VT, M, KM><<<blocks, kLcThreads, 0, ctx->stream>>>(a)
#define CMCG_LC(KERN, M)                     \
    if (k <= 2) CMCG_LC_KM(KERN, M, 2);      \
    else if (k <= 4) CMCG_LC_KM(KERN, M, 4); \
    else if (k <= 8) CMCG_LC_KM(KERN, M, 8); \
    else CMCG_LC_KM(KERN, M, kMaxTerms)
    if (aligned) {
        if (mode == CMCG_ASSIGN) { CMCG_LC(k_lincomb_vec, CMCG_ASSIGN); }
        else if (mode == CMCG_ADD) { CMCG_LC(k_lincomb_vec, CMCG_ADD); }
        else { CMCG_LC(k_lincomb_vec, CMCG_SUB); }
    } else {
        if (mode == CMCG_ASSIGN) { CMCG_LC(k_lincomb_scalar, CMCG_ASSIGN); }
        else if (mode == CMCG_ADD) { CMCG_LC(k_lincomb_scalar, CMCG_ADD); }
        else { CMCG_LC(k_lincomb_scalar, CMCG_SUB); }
    }
#undef CMCG_LC
#undef CMCG_LC_KM
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

}  // namespace
}  // namespace cmcg

using namespace cmcg;

extern "C" cmcg_status cmcg_lincomb(cmcg_ctx ctx, int32_t dtype, int64_t n, int32_t n_terms, const double* coeffs,
                                    const void* const* vectors, const int32_t* v_batches, void* out,
                                    int32_t out_batches, int32_t mode) {
    NvtxRange nvtx_("cmcg_lincomb");
    CMCG_REQUIRE(ctx && coeffs && vectors && v_batches && out, "cmcg_lincomb: NULL argument");
    CMCG_REQUIRE(dtype == CMCG_F32 || dtype == CMCG_F64, "cmcg_lincomb: dtype must be F32 or F64");
    CMCG_REQUIRE(n_terms >= 1 && n_terms <= kMaxTerms, "cmcg_lincomb: 1 to 16 terms");
    CMCG_REQUIRE(n >= 0 && out_batches >= 1, "cmcg_lincomb: bad size");
    CMCG_REQUIRE(mode == CMCG_ASSIGN || mode == CMCG_ADD || mode == CMCG_SUB, "cmcg_lincomb: bad mode");
    for (int j = 0; j < n_terms; ++j) {
        CMCG_REQUIRE(vectors[j], "cmcg_lincomb: NULL vector");
        CMCG_REQUIRE(v_batches[j] == 1 || v_batches[j] == out_batches,
                     "cmcg_lincomb: every vector has one batch or out_batches batches");
    }
    if (n == 0) return CMCG_OK;
    CMCG_CUDA(cudaSetDevice(ctx->device));
    return dtype == CMCG_F32 ? launch_lincomb<float>(ctx, n, n_terms, coeffs, vectors, v_batches, out, out_batches, mode)
                             : launch_lincomb<double>(ctx, n, n_terms, coeffs, vectors, v_batches, out, out_batches, mode);
}
