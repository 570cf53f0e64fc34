// Shared-memory-resident persistent CG kernels (one 1024-thread CTA per system).
//
// For systems of up to kSmemMaxRows rows the whole FP32 working set of an
// iteration stays on the SM: the search direction p, the residual r and the
// solution (or its FP32 increments) live in shared memory (p is gathered by
// the product from shared memory), each thread keeps q = A p for its own rows
// (rows t, t + 1024, ...) in registers, and the inverse diagonal is read
// through the read-only cache. Global memory is read for the matrix and the
// diagonal only. Per iteration: one product (thread per row over the 32-row
// slices, one 128-byte load per warp and entry), three block reductions, no
// grid synchronisation, no host round trip.
#pragma once

#include "cg_dev.cuh"

namespace cmcg {

constexpr int kSmemThreads = 1024;
constexpr int kSmemNK = 16;                                // rows per thread
constexpr int kSmemMaxRows = kSmemThreads * kSmemNK;       // 16384

// x[c] gathered from a shared-memory copy of a system's rows [r0, r0 + n)
struct SmemX {
    const float* p;
    int r0;
    __device__ __forceinline__ float operator()(int c) const { return p[c - r0]; }
};

// q[k] = (A xf)[local row tid + k * 1024] for the rows this thread owns
// (thread-per-row over the sliced layout; a warp's rows form one slice).
template <typename MT, int FMT, typename XF>
__device__ __forceinline__ void smem_product(const InstMatrix<MT, FMT>& A, int s, int r0, int n, const XF& xf,
                                             float (&q)[kSmemNK]) {
#pragma unroll
    for (int k = 0; k < kSmemNK; ++k) {
        const int i = threadIdx.x + k * kSmemThreads;
        q[k] = (i < n) ? row_product<float>(A.rm, s, r0, i, xf) : 0.0f;
    }
}

struct SmemLayout {
    float* p;   // search direction (gathered by the product)
    float* r;   // residual
    float* x;   // solution (plain) / FP32 increments since the last FP64 fold (mixed)
};

__device__ __forceinline__ SmemLayout smem_layout(float* sm, int nmax) {
    SmemLayout L;
    L.p = sm;
    L.r = sm + nmax;
    L.x = sm + 2 * nmax;
    return L;
}

inline size_t smem_bytes(int nmax) { return static_cast<size_t>(nmax) * 3 * sizeof(float); }

}  // namespace cmcg
