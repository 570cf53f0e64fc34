// Plain FP64 batched PCG on the diagonal layout, in CTA tiers.
//
// The reference's algorithm and stopping rule (cuMat/src/ConjugateGradient.h:123-206,
// the Eigen PCG loop with the Jacobi preconditioner, DiagonalPreconditioner
// :218-246) for many independent stencil-shaped systems, one CTA per system
// instance from an atomic work counter, with the same launch machinery as the
// mixed-precision kernel: the matrix's own values (unscaled) in the diagonal
// block layout (no column indices, one value pointer per thread, immediate
// offsets), thread t owning the rows t + T k, and three CTA sizes by system
// size (T = 1024 / 512 / 256, one / two / four CTAs per SM) on their own
// priority streams. p lives in shared memory with a zero halo as wide as the
// largest offset, so the product needs no row tests; r, x and q = A p are FP64
// vectors in global memory read and written by the owning thread (coalesced,
// L2-resident while the system runs); the inverse diagonal is read through the
// read-only path.
#include <cuda_bf16.h>

#include "cg_compact.cuh"
#include "cg_plain.cuh"
#include "objects.h"

namespace cmcg {
namespace {

// Index of the value of diagonal d for row slot k of a T-thread CTA, relative
// to the thread's first row (blocks of kDiaBlockRows rows, ND diagonals each).
template <int T, int ND>
__device__ __forceinline__ constexpr int plain_vidx(int k, int d) {
    return ((k * T) / kDiaBlockRows * ND + d) * kDiaBlockRows + (k * T) % kDiaBlockRows;
}

// CALL with the compile-time slot count NK = nk (1 .. kSmemNK, uniform)
#define CMCG_PLAIN_SLOTS(nk, CALL)                        \
    switch (nk) {                                         \
        case 1: { constexpr int NK = 1; CALL; } break;    \
        case 2: { constexpr int NK = 2; CALL; } break;    \
        case 3: { constexpr int NK = 3; CALL; } break;    \
        case 4: { constexpr int NK = 4; CALL; } break;    \
        case 5: { constexpr int NK = 5; CALL; } break;    \
        case 6: { constexpr int NK = 6; CALL; } break;    \
        case 7: { constexpr int NK = 7; CALL; } break;    \
        case 8: { constexpr int NK = 8; CALL; } break;    \
        case 9: { constexpr int NK = 9; CALL; } break;    \
        case 10: { constexpr int NK = 10; CALL; } break;  \
        case 11: { constexpr int NK = 11; CALL; } break;  \
        case 12: { constexpr int NK = 12; CALL; } break;  \
        case 13: { constexpr int NK = 13; CALL; } break;  \
        case 14: { constexpr int NK = 14; CALL; } break;  \
        case 15: { constexpr int NK = 15; CALL; } break;  \
        default: { constexpr int NK = 16; CALL; } break;  \
    }
static_assert(kSmemNK == 16, "CMCG_PLAIN_SLOTS covers 16 row slots");

// q_i = (A p)_i for the NK row slots (entries in ascending offset order, the
// row's CSR order, fused multiply-adds; absent entries are zeros and the p
// halo is zero), written to Q; pq += p_i q_i over the rows of the system.
template <int NK, int ND, int T, typename MT>
__device__ __forceinline__ void plain_spmv(const MT* __restrict__ vt, const int (&po)[ND], const double* P,
                                           double* __restrict__ Q, int tid, int n, double& pq) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < ND; ++d) acc = fma(mval<double>(__ldg(vt + plain_vidx<T, ND>(k, d))), P[po[d] + k * T], acc);
        const int i = tid + k * T;
        if (i < n) {
            Q[i] = acc;
            pq += P[i] * acc;
        }
    }
}

template <typename MT, int ND, int T>
__global__ void __launch_bounds__(T, kDiaBlockRows / T) k_plain_dia(PlainDiaArgs<MT> a, int nmax) {
    extern __shared__ __align__(16) double smd[];
    __shared__ double red[2 * (T / 32)];
    __shared__ int slot;
    const int M = a.margin;
    double* P = smd + M;
    const int tid = threadIdx.x;
    const double tol = a.tol;
    for (;;) {
        const int item = a.item_begin + fetch_item(a.next, &slot);
        if (item >= a.item_end) return;
        const int s = a.order[item / a.ob], bi = item % a.ob, inst = bi * a.n_sys + s;
        const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0;
        const int64_t vo = static_cast<int64_t>(bi) * a.rows;
        const double* bv = a.b + (a.b_b == 1 ? 0 : vo) + r0;
        double* X = a.x + vo + r0;
        double* R = a.r + vo + r0;
        double* Q = a.q + vo + r0;
        const double* dg = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) + r0 : nullptr;
        const MT* vt = a.vals + (a.mb == 1 ? 0 : static_cast<int64_t>(bi) * a.vstride) + __ldg(a.base + s) + tid;
        int po[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) po[d] = tid + __ldg(a.off + s * kDiaMax + d);
        const int nk = (n + T - 1) / T;
        // zero p's halos and the rows of the last slot past the system's end
        for (int t = tid; t < M; t += T) P[-1 - t] = 0.0;
        for (int i = n + tid; i < nk * T + M; i += T) P[i] = 0.0;
        double acc[2] = {0.0, 0.0};
#pragma unroll
        for (int k = 0; k < kSmemNK; ++k) {
            if (k * T >= n) break;   // uniform: skip row slots past the system
            const int i = tid + k * T;
            if (i < n) {
                const double b_i = bv[i];
                R[i] = b_i;
                X[i] = 0.0;
                acc[0] += b_i * b_i;
            }
        }
        block_sum<double, 2>(acc, red);
        const double bb = acc[0];
        double rr = bb;
        const double thr = tol * tol * bb;
        int32_t status = ST_RUNNING, it = 0;
        if ((a.abs_zero_test && bb < tol * tol) || bb == 0.0) {
            status = CMCG_SOLVE_ZERO_RHS;
        } else if (!finite_(bb)) {
            status = CMCG_SOLVE_NON_FINITE;
        } else if (rr < thr) {
            status = CMCG_SOLVE_CONVERGED;
        } else {
            double rz1[1] = {0.0};
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * T >= n) break;
                const int i = tid + k * T;
                if (i < n) {
                    const double ri = R[i], zi = (dg ? __ldg(dg + i) : 1.0) * ri;
                    P[i] = zi;
                    rz1[0] += ri * zi;
                }
            }
            block_sum<double, 1>(rz1, red);
            double rz = rz1[0];
            if (!finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
            else if (!(rz > 0.0)) status = CMCG_SOLVE_BREAKDOWN;
            const int64_t maxit = sys_max_iter(a.max_iter, n);
            while (status == ST_RUNNING) {
                if (it >= maxit) { status = CMCG_SOLVE_MAX_ITER; break; }
                double pq[1] = {0.0};
                CMCG_PLAIN_SLOTS(nk, (plain_spmv<NK, ND, T>(vt, po, P, Q, tid, n, pq[0])))
                block_sum<double, 1>(pq, red);
                const double alpha = rz / pq[0];
                if (!finite_(pq[0]) || !finite_(alpha)) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (!(pq[0] > 0.0)) { status = CMCG_SOLVE_BREAKDOWN; break; }
                double s2[2] = {0.0, 0.0};
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * T >= n) break;
                    const int i = tid + k * T;
                    if (i < n) {
                        X[i] += alpha * P[i];
                        const double ri = R[i] - alpha * Q[i];
                        R[i] = ri;
                        s2[0] += ri * ri;
                        s2[1] += ri * ((dg ? __ldg(dg + i) : 1.0) * ri);
                    }
                }
                block_sum<double, 2>(s2, red);
                rr = s2[0];
                if (!finite_(rr) || !finite_(s2[1])) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (rr < thr) { status = CMCG_SOLVE_CONVERGED; break; }
                if (!(s2[1] > 0.0)) { status = CMCG_SOLVE_BREAKDOWN; break; }
                const double beta = s2[1] / rz;
                rz = s2[1];
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * T >= n) break;
                    const int i = tid + k * T;
                    if (i < n) P[i] = (dg ? __ldg(dg + i) : 1.0) * R[i] + beta * P[i];
                }
                __syncthreads();
                ++it;
            }
        }
        if (tid == 0) {
            a.st.it[inst] = it;
            a.st.status[inst] = status;
            a.st.rr[inst] = rr;
            a.st.bb[inst] = bb;
            a.st.outer[inst] = 0;
            a.st.err[inst] = (status == CMCG_SOLVE_ZERO_RHS) ? 0.0 : sqrt(rr / bb);
        }
        __syncthreads();
    }
}

template <typename K>
cmcg_status plain_smem_once(K kern, size_t bytes) {
    CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    return CMCG_OK;
}

template <typename MT, int T>
cmcg_status launch_plain_t(const PlainDiaArgs<MT>& a, int nmax, size_t smem, int nd, int grid, cudaStream_t stream) {
    switch (nd) {
        case 5:
            CMCG_TRY(plain_smem_once(k_plain_dia<MT, 5, T>, smem));
            k_plain_dia<MT, 5, T><<<grid, T, smem, stream>>>(a, nmax);
            break;
        case 7:
            CMCG_TRY(plain_smem_once(k_plain_dia<MT, 7, T>, smem));
            k_plain_dia<MT, 7, T><<<grid, T, smem, stream>>>(a, nmax);
            break;
        default:
            return fail(CMCG_ERR_INVALID_ARGUMENT, "unsupported number of diagonals");
    }
    return CMCG_OK;
}

}  // namespace

template <typename MT>
cmcg_status launch_plain_dia(const PlainDiaArgs<MT>& a, int threads, int nmax, size_t smem, int nd, int grid,
                             cudaStream_t stream) {
    if (threads == 256) return launch_plain_t<MT, 256>(a, nmax, smem, nd, grid, stream);
    if (threads == 512) return launch_plain_t<MT, 512>(a, nmax, smem, nd, grid, stream);
    if (threads == kSmemThreads) return launch_plain_t<MT, kSmemThreads>(a, nmax, smem, nd, grid, stream);
    return fail(CMCG_ERR_INVALID_ARGUMENT, "unsupported CTA size");
}

template cmcg_status launch_plain_dia<double>(const PlainDiaArgs<double>&, int, int, size_t, int, int, cudaStream_t);
template cmcg_status launch_plain_dia<float>(const PlainDiaArgs<float>&, int, int, size_t, int, int, cudaStream_t);

}  // namespace cmcg
