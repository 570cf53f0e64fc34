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

// Matrix of one instance (batch) in either format.
template <typename MT, int FMT>
struct InstMatrix {
    CsrView<MT> csr;
    EllView<MT> ell;
};

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
