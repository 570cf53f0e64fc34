// Device-side building blocks of the sparse products, shared by the stand-alone
// SpMV kernels and the fused CG kernels.
#pragma once

#include "common.cuh"

namespace cmcg {

// One batch of a CSR matrix: the reference's JA (row_ptr) / IA (col) / data
// (cuMat/src/SparseMatrixBase.h:89-147). `val` and `ci` are 16-byte aligned and
// padded to a multiple of 4 entries.
template <typename MT>
struct CsrView {
    const int32_t* __restrict__ rp;
    const int32_t* __restrict__ ci;
    const MT* __restrict__ val;
};

// One batch of a column-major ELLPACK matrix with rows padded to rows_pad
// (entry (row, slot) at row + slot * rows_pad; index -1 = padding).
template <typename MT>
struct EllView {
    const int32_t* __restrict__ idx;
    const MT* __restrict__ val;
    int32_t width;
    int32_t rows_pad;
};

// Per-warp staging buffer of the CSR row-block product: 128 products.
template <typename VT>
struct alignas(16) WarpStage {
    VT p[128];
};

template <typename VT>
__device__ __forceinline__ void stage_store4(WarpStage<VT>& st, int lane, const VT (&v)[4]);
template <>
__device__ __forceinline__ void stage_store4<float>(WarpStage<float>& st, int lane, const float (&v)[4]) {
    reinterpret_cast<float4*>(st.p)[lane] = make_float4(v[0], v[1], v[2], v[3]);
}
template <>
__device__ __forceinline__ void stage_store4<double>(WarpStage<double>& st, int lane, const double (&v)[4]) {
    reinterpret_cast<double2*>(st.p)[2 * lane] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(st.p)[2 * lane + 1] = make_double2(v[2], v[3]);
}

// Row-block CSR product of one warp: rows [r0, r0 + nr), nr in [1, 32]. The
// warp streams the block's contiguous entry range in chunks of 128 entries
// with one 16-byte column load and one 4-value load per lane, multiplies by the
// gathered x (xf(col) -> VT), stages the products in shared memory, and each
// lane then sums the products of its own row in entry order. Returns the row
// sum on lane < nr (0 on the others). Summation order per row is the entry
// order, as in the reference's thread-per-row loop
// (cuMat/src/SparseProductEvaluation.h:55-87).
template <typename VT, typename MT, typename XF>
__device__ __forceinline__ VT warp_csr_rows(const CsrView<MT>& A, int r0, int nr, const XF& xf, WarpStage<VT>& st) {
    const int lane = threadIdx.x & 31;
    int my_lo = 0, my_hi = 0;
    if (lane < nr) {
        my_lo = __ldg(A.rp + r0 + lane);
        my_hi = __ldg(A.rp + r0 + lane + 1);
    }
    const int lo = __shfl_sync(FULL, my_lo, 0);
    const int hi = __shfl_sync(FULL, my_hi, nr - 1);
    VT acc = VT(0);
    for (int c = lo & ~3; c < hi; c += 128) {
        const int k0 = c + 4 * lane;
        VT prod[4];
        if (k0 >= lo && k0 + 4 <= hi) {
            const int4 cc = __ldg(reinterpret_cast<const int4*>(A.ci + k0));
            Vals4<MT> v;
            v.load(A.val + k0);
            prod[0] = mval<VT>(v.v[0]) * xf(cc.x);
            prod[1] = mval<VT>(v.v[1]) * xf(cc.y);
            prod[2] = mval<VT>(v.v[2]) * xf(cc.z);
            prod[3] = mval<VT>(v.v[3]) * xf(cc.w);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int k = k0 + j;
                prod[j] = (k >= lo && k < hi) ? mval<VT>(A.val[k]) * xf(__ldg(A.ci + k)) : VT(0);
            }
        }
        stage_store4<VT>(st, lane, prod);
        __syncwarp();
        const int a = max(my_lo, c), e = min(my_hi, c + 128);
        for (int k = a; k < e; ++k) acc += st.p[k - c];
        __syncwarp();
    }
    return acc;
}

// ELLPACK product of one row, thread per row: coalesced across the rows of a
// warp because of the column-major layout; padding (index < 0) is skipped
// (reference ELLPACKMVKernel_StaticBatches, SparseProductEvaluation.h:206-224).
template <typename VT, typename MT, typename XF>
__device__ __forceinline__ VT ell_row(const EllView<MT>& A, int r, const XF& xf) {
    VT acc = VT(0);
    for (int j = 0; j < A.width; ++j) {
        const int64_t o = r + static_cast<int64_t>(j) * A.rows_pad;
        const int c = __ldg(A.idx + o);
        if (c >= 0) acc += mval<VT>(A.val[o]) * xf(c);
    }
    return acc;
}

// Gathers x[c] through the read-only cache.
template <typename VT>
struct GlobalX {
    const VT* __restrict__ x;
    __device__ __forceinline__ VT operator()(int c) const { return __ldg(x + c); }
};

// Gathers x[c] through the read-only cache with a column offset (systems whose
// columns are global indices into a packed vector).
template <typename VT>
struct OffsetX {
    const VT* __restrict__ x;  // already shifted by -col_base
    __device__ __forceinline__ VT operator()(int c) const { return x[c]; }
};

}  // namespace cmcg
