// Device routines of the conjugate-gradient solver.
//
// Algorithm per system (reference cuMat/src/ConjugateGradient.h:123-206, the
// Eigen PCG loop): r = b - A x0; stop early when |b|^2 < tol^2 (x = 0) or
// |r|^2 < tol^2 |b|^2; p = M^-1 r; rz = r.p; then repeat
//   q = A p; alpha = rz / p.q; x += alpha p; r -= alpha q;
//   if |r|^2 < tol^2 |b|^2: stop (iterations = i)
//   z = M^-1 r; beta = r.z / rz; rz = r.z; p = z + beta p; ++i
// with M^-1 = identity or the inverse diagonal (1 where a_ii == 0).
// Unlike the reference, which iterates all batches until all converge, each
// system stops on its own; breakdown (p.q <= 0, r.z <= 0) and non-finite
// scalars stop a system with a status instead of propagating NaNs.
#pragma once

#include "common.cuh"
#include "spmv_dev.cuh"

namespace cmcg {

enum : int32_t { ST_RUNNING = -1 };

template <typename VT>
__device__ __forceinline__ bool finite_(VT v) { return isfinite(v); }

template <typename MT> struct RowMat;

// Matrix of one instance (batch) in either format.
template <typename MT, int FMT>
struct InstMatrix;

// Row-major access for thread-per-row products. CSR patterns are read through
// their sliced ELLPACK copy (32-row slices, column-major inside a slice,
// padding = own column with value 0); ELLPACK patterns directly (stride
// rows_pad, padding index -1). Rows of a warp must be the 32 rows of one slice
// (row i of a system handled by lane i % 32), which makes every load of the
// warp one 128-byte access.
template <typename MT>
struct RowMat {
    const int32_t* __restrict__ col;
    const MT* __restrict__ val;
    const int64_t* __restrict__ slice_off;   // null: ELLPACK
    const int32_t* __restrict__ slice_w;
    const int32_t* __restrict__ sys_slice0;
    int32_t ell_stride, ell_w;
};

constexpr int kRowUnroll = 4;

// (A x)[row] for row i (local) of system s starting at global row r0.
template <typename VT, typename MT, typename XF>
__device__ __forceinline__ VT row_product(const RowMat<MT>& A, int s, int r0, int i, const XF& xf) {
    int64_t base;
    int stride, w;
    if (A.slice_off) {
        const int sl = __ldg(A.sys_slice0 + s) + (i >> 5);
        base = __ldg(A.slice_off + sl) + (i & 31);
        stride = 32;
        w = __ldg(A.slice_w + sl);
    } else {
        base = r0 + i;
        stride = A.ell_stride;
        w = A.ell_w;
    }
    VT acc = VT(0);
    int j0 = 0;
    for (; j0 < w; j0 += kRowUnroll) {
        int c[kRowUnroll];
        MT v[kRowUnroll];
#pragma unroll
        for (int j = 0; j < kRowUnroll; ++j) {
            if (j0 + j < w) {
                const int64_t o = base + static_cast<int64_t>(j0 + j) * stride;
                c[j] = __ldg(A.col + o);
                v[j] = A.val[o];
            }
        }
#pragma unroll
        for (int j = 0; j < kRowUnroll; ++j) {
            if (j0 + j < w) {
                if (A.slice_off) acc += mval<VT>(v[j]) * xf(c[j]);
                else if (c[j] >= 0) acc += mval<VT>(v[j]) * xf(c[j]);
            }
        }
    }
    return acc;
}

template <typename MT, int FMT>
struct InstMatrix {
    CsrView<MT> csr;
    EllView<MT> ell;
    RowMat<MT> rm;
};

// Thread-per-row product over the local rows [i0, i0 + n) of system s (first
// global row r0) with the whole CTA: thread t takes rows i0 + t, i0 + t +
// blockDim.x, ... (i0 a multiple of 32); f(global row, value).
template <typename VT, typename MT, int FMT, typename XF, typename F>
__device__ __forceinline__ void cta_rows(const InstMatrix<MT, FMT>& A, int s, int r0, int i0, int n, const XF& xf,
                                         F&& f) {
    for (int i = i0 + threadIdx.x; i < i0 + n; i += blockDim.x) f(r0 + i, row_product<VT>(A.rm, s, r0, i, xf));
}

constexpr int kRowsInFlight = 4;   // rows per thread whose loads are interleaved

// (A x) for K rows i[k] (local, ok[k] = row exists) of system s at once: the
// slice descriptors, then two entries of every row, are loaded before any of
// them is used, so a thread has K times the independent loads of
// row_product in flight. Per row the entries are added in the same order as
// row_product.
template <typename VT, int K, typename MT, typename XF>
__device__ __forceinline__ void row_products(const RowMat<MT>& A, int s, int r0, const int (&i)[K], const bool (&ok)[K],
                                             const XF& xf, VT (&out)[K]) {
    int64_t base[K];
    int w[K];
    int stride;
    if (A.slice_off) {
        const int sl0 = __ldg(A.sys_slice0 + s);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int sl = sl0 + (i[k] >> 5);
            base[k] = ok[k] ? __ldg(A.slice_off + sl) + (i[k] & 31) : 0;
            w[k] = ok[k] ? __ldg(A.slice_w + sl) : 0;
        }
        stride = 32;
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            base[k] = r0 + i[k];
            w[k] = ok[k] ? A.ell_w : 0;
        }
        stride = A.ell_stride;
    }
    int wmax = w[0];
#pragma unroll
    for (int k = 1; k < K; ++k) wmax = max(wmax, w[k]);
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = VT(0);
    for (int j0 = 0; j0 < wmax; j0 += 2) {
        int c[K][2];
        MT v[K][2];
#pragma unroll
        for (int k = 0; k < K; ++k) {
#pragma unroll
            for (int jj = 0; jj < 2; ++jj) {
                const bool in = j0 + jj < w[k];
                const int64_t o = base[k] + static_cast<int64_t>(j0 + jj) * stride;
                c[k][jj] = in ? __ldg(A.col + o) : -1;
                v[k][jj] = in ? A.val[o] : MT{};
            }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
                if (c[k][jj] >= 0) out[k] += mval<VT>(v[k][jj]) * xf(c[k][jj]);
        }
    }
}

// cta_rows with kRowsInFlight rows per thread in flight: thread t takes rows
// i0 + t + k * blockDim.x, k = 0, 1, ... in groups of kRowsInFlight (i0 a
// multiple of 32); f(global row, value) is called in increasing row order per
// thread, as in cta_rows.
template <typename VT, typename MT, int FMT, typename XF, typename F>
__device__ __forceinline__ void cta_rows_seg(const InstMatrix<MT, FMT>& A, int s, int r0, int i0, int n, const XF& xf,
                                             F&& f) {
    // FP64 vectors or values: two rows (register budget of 1024-thread CTAs)
    constexpr int K = sizeof(VT) + sizeof(MT) > 8 ? 2 : kRowsInFlight;
    const int T = blockDim.x, end = i0 + n;
    for (int ib = i0 + threadIdx.x; ib < end; ib += K * T) {
        int ii[K];
        bool ok[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            ii[k] = ib + k * T;
            ok[k] = ii[k] < end;
        }
        VT v[K];
        row_products<VT, K>(A.rm, s, r0, ii, ok, xf, v);
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (ok[k]) f(r0 + ii[k], v[k]);
    }
}

// (A x) for the four consecutive rows i .. i+3 (local, i a multiple of 4) of
// one slice of the sliced layout: per entry slot one 16-byte index load and
// one 4-value load cover the four rows (a warp's eight lanes per slice read
// whole 128-byte lines), and the slots of a step are all loaded before the
// first gather. Rows sum their entries in entry order.
template <typename VT, typename MT, typename XF>
__device__ __forceinline__ void sell_rows4(const RowMat<MT>& A, int s, int i, const XF& xf, VT (&out)[4]) {
    // slots per step: fewer for 8-byte values (register budget)
    constexpr int S = sizeof(MT) == 8 ? 2 : 4;
    const int sl = __ldg(A.sys_slice0 + s) + (i >> 5);
    const int64_t base = __ldg(A.slice_off + sl) + (i & 31);
    const int w = __ldg(A.slice_w + sl);
#pragma unroll
    for (int q = 0; q < 4; ++q) out[q] = VT(0);
    for (int j0 = 0; j0 < w; j0 += S) {
        int4 c[S];
        Vals4<MT> v[S];
#pragma unroll
        for (int jj = 0; jj < S; ++jj) {
            if (j0 + jj < w) {
                const int64_t o = base + static_cast<int64_t>(j0 + jj) * 32;
                c[jj] = __ldg(reinterpret_cast<const int4*>(A.col + o));
                v[jj].load(A.val + o);
            }
        }
#pragma unroll
        for (int jj = 0; jj < S; ++jj) {
            if (j0 + jj < w) {
                out[0] += mval<VT>(v[jj].v[0]) * xf(c[jj].x);
                out[1] += mval<VT>(v[jj].v[1]) * xf(c[jj].y);
                out[2] += mval<VT>(v[jj].v[2]) * xf(c[jj].z);
                out[3] += mval<VT>(v[jj].v[3]) * xf(c[jj].w);
            }
        }
    }
}

// Thread-per-4-rows product over the local rows [i0, i0 + n) of system s (i0 a
// multiple of 32; the range ends at a multiple of 4 or at the system's end):
// thread t takes rows i0 + 4 t .. + 3, then i0 + 4 (t + blockDim.x) ...;
// f(global row, value) per row in increasing order per thread. The sliced
// layout (CSR patterns) only; ELLPACK patterns take cta_rows_seg.
template <typename VT, typename MT, int FMT, typename XF, typename F>
__device__ __forceinline__ void cta_rows4_seg(const InstMatrix<MT, FMT>& A, int s, int r0, int i0, int n, const XF& xf,
                                              F&& f) {
    if (!A.rm.slice_off) {
        cta_rows_seg<VT>(A, s, r0, i0, n, xf, f);
        return;
    }
    const int end = i0 + n;
    for (int ib = i0 + 4 * threadIdx.x; ib < end; ib += 4 * blockDim.x) {
        VT v[4];
        sell_rows4<VT>(A.rm, s, ib, xf, v);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (ib + q < end) f(r0 + ib + q, v[q]);
    }
}

// Applies the product to the rows [r0, r0 + n) of one system with the whole
// CTA: warp w takes the 32-row blocks w, w + W, ... so thread t always owns
// rows r0 + t + k * blockDim.x. f(row, value) is called on the owning lane.
template <typename VT, typename MT, int FMT, typename XF, typename F>
__device__ __forceinline__ void cta_rows_product(const InstMatrix<MT, FMT>& A, int r0, int n, const XF& xf,
                                                 WarpStage<VT>* stage, F&& f) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int blk = warp; blk * 32 < n; blk += nw) {
        const int rb = r0 + blk * 32;
        const int nr = min(32, n - blk * 32);
        if (FMT == CMCG_CSR) {
            const VT v = warp_csr_rows<VT>(A.csr, rb, nr, xf, stage[warp]);
            if (lane < nr) f(rb + lane, v);
        } else {
            if (lane < nr) f(rb + lane, ell_row<VT>(A.ell, rb + lane, xf));
        }
    }
}

}  // namespace cmcg
