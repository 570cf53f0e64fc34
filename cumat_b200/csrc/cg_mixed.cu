// Mixed-precision persistent CG kernel over the compact sliced layout or the
// diagonal layout (one 1024-thread CTA per system instance, reliable updates).
#include <cuda_bf16.h>

#include <type_traits>

#include "cg_compact.cuh"
#include "objects.h"

namespace cmcg {
namespace {

// Diagonal layout in row-slot blocks: the scaled values of a system's row
// slot k (local rows 1024 k .. 1024 k + 1023, the rows tid + 1024 k of the
// CTA) and diagonal d form the block that starts 1024 (k ND + d) values past
// the system's base, so one per-thread pointer reaches every value through an
// immediate offset. Rows past the system's end hold zero values; their p, r
// and xh are zeroed when the system starts and stay zero, so each phase runs
// all NK = ceil(n / 1024) slots with no row test.
static_assert(kDiaBlockRows == kSmemThreads, "diagonal blocks hold one row per thread of a 1024-thread CTA");

// Index of the value of diagonal d for row slot k of a T-thread CTA (thread
// t's row t + T k), relative to the thread's first row: slot k lies in block
// (k T) / 1024 at offset (k T) % 1024, a compile-time constant per (k, d).
template <int T, int ND>
__device__ __forceinline__ constexpr int dia_vidx(int k, int d) {
    return ((k * T) / kDiaBlockRows * ND + d) * kDiaBlockRows + (k * T) % kDiaBlockRows;
}

// q[k] = (S A S p)[tid + 1024 k] for the NK row slots, entries added in
// ascending offset order (the row's CSR order) with fused multiply-adds;
// pq += p_i q_i in slot order. po[d]: p index of the thread's first row plus
// the offset of diagonal d. UNIT: the middle diagonal is offset 0 with every
// value exactly 1 (Jacobi scaling of a positive diagonal), so its values are
// not loaded; fmaf(1, p, acc) rounds as the loaded form did.
template <int NK, int ND, bool UNIT, int T, typename MI>
__device__ __forceinline__ void dia_spmv(const MI* __restrict__ vt, const int (&po)[ND], const float* P, int tid,
                                         float (&q)[kSmemNK], float& pq) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        float acc = 0.0f;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            if (UNIT && d == ND / 2)   // offset 0: the row's own p, read once for both uses
                acc = fmaf(1.0f, P[tid + k * T], acc);
            else
                acc = fmaf(mval<float>(vt[dia_vidx<T, ND>(k, d)]), P[po[d] + k * T], acc);
        }
        q[k] = acc;
        pq += P[tid + k * T] * acc;
    }
}

// r -= alpha q over the NK slots; s1 += r_i^2 in slot order. q[k] then holds
// the new r_i (q is not needed again), for the p update.
template <int NK, int T>
__device__ __forceinline__ void dia_update(float* R, int tid, float alpha, float (&q)[kSmemNK], float& s1) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const int i = tid + k * T;
        const float ri = R[i] - alpha * q[k];
        R[i] = ri;
        s1 += ri * ri;
        q[k] = ri;
    }
}

// p = r + beta p over the NK slots, and with STEP (an iteration without a
// residual replacement) xh += alpha p, the iteration's x increment, from the
// same read of p, with r from the registers dia_update left it in; after a
// replacement the fold took the increment and r comes from shared memory.
template <int NK, bool STEP, int T>
__device__ __forceinline__ void dia_pupdate(float* P, const float* R, float* XH, int tid, float alpha, float beta,
                                            const float (&rr)[kSmemNK]) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const int i = tid + k * T;
        const float pi = P[i];
        if (STEP) XH[i] += alpha * pi;
        P[i] = (STEP ? rr[k] : R[i]) + beta * pi;
    }
}

// xh += alpha p over the NK slots (the pending increment before a fold)
template <int NK, int T>
__device__ __forceinline__ void dia_xinc(const float* P, float* XH, int tid, float alpha) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const int i = tid + k * T;
        XH[i] += alpha * P[i];
    }
}

// CALL with the compile-time slot count NK = nk (1 .. kSmemNK, uniform)
#define CMCG_DIA_SLOTS(nk, CALL)                          \
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
static_assert(kSmemNK == 16, "CMCG_DIA_SLOTS covers 16 row slots");

// Mixed precision with reliable updates on the compact layout. The inner FP32
// CG runs on the symmetrically Jacobi-scaled system S A S (S = diag(s)), which
// is Jacobi PCG in exact arithmetic but needs no diagonal inside the loop; the
// FP64 parts use the unscaled values: x += S xh at every fold and the inner
// residual is S (b - A x). Residual replacement as in k_reliable_smem, the
// trigger compared in the scaled norm.
// ND > 0: the inner iteration reads the scaled values in the diagonal layout
// (ND diagonals per system, row-slot blocks): row i sums v_d[i] * p[i +
// offset_d] over the diagonals in ascending offset order (the row's CSR
// order; absent entries are zeros), with no column index loads and no row
// tests; p carries a zero halo of `margin` entries on both sides in shared
// memory, and nmax is a multiple of 1024. The FP64 residual keeps the compact
// sliced layout.
template <typename MI, typename MO, int ND, int T>
// (1024 / T CTAs per SM: 64 registers per thread for both CTA sizes)
__global__ void __launch_bounds__(T, kDiaBlockRows / T) k_mixed_fast(MixArgs<MI, MO> a, int nmax) {
    extern __shared__ __align__(16) float smf[];
    __shared__ SliceEnt tab[32][kSmemNK];
    __shared__ float red[2 * (T / 32)];
    __shared__ double red64[2 * (T / 32)];
    __shared__ int slot;
    __shared__ int guard[3];
    const int M = ND > 0 ? a.margin : 0;
    float* P = smf + M;
    float* R = smf + nmax + 2 * M;
    float* XH = R + nmax;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const float d2 = a.delta * a.delta;
    for (;;) {
        const int item = a.item_begin + fetch_item(a.next, &slot);
        if (item >= a.item_end) return;
        const int s = a.order[item / a.ob], bi = item % a.ob, inst = bi * a.n_sys + s;
        const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0;
        const int sl0 = __ldg(a.c.sys_slice0 + s), nsl = __ldg(a.c.sys_slice0 + s + 1) - sl0;
        load_slice_table<T>(tab, a.c.off32, a.c.sw, sl0, nsl);
        const int64_t vo = static_cast<int64_t>(bi) * a.rows;
        const MI* vin = a.vin + (a.mb == 1 ? 0 : static_cast<int64_t>(bi) * a.vin_stride);
        const MO* vout = a.vout + (a.mb == 1 ? 0 : static_cast<int64_t>(bi) * a.vout_stride);
        const double* sv = a.s + (a.mb == 1 ? 0 : vo) + r0;
        const double* bv = a.b + (a.b_b == 1 ? 0 : vo) + r0;
        double* x = a.x + vo + r0;
        // diagonal layout: the thread's value pointer (first row), the p index
        // of its first row plus each offset, and zero p, r, xh past the
        // system's end (to the end of its last slot, and the halos of p)
        const int nk = (n + T - 1) / T;
        const MI* vt = nullptr;
        int po[ND > 0 ? ND : 1] = {};
        bool unit = false;
        if constexpr (ND > 0) {
            unit = __ldg(a.dia_unit + (a.mb == 1 ? 0 : bi) * a.n_sys + s) != 0;
            vt = a.vdia + (a.mb == 1 ? 0 : static_cast<int64_t>(bi) * a.vdia_stride) + __ldg(a.dia_base + s) + tid;
#pragma unroll
            for (int d = 0; d < ND; ++d) po[d] = tid + __ldg(a.dia_off + s * kDiaMax + d);
            const int nend = nk * T;
            for (int t = tid; t < M; t += T) P[-1 - t] = 0.0f;
            for (int i = n + tid; i < nend + M; i += T) P[i] = 0.0f;
            for (int i = n + tid; i < nend; i += T) {
                R[i] = 0.0f;
                XH[i] = 0.0f;
            }
        }
        __syncthreads();   // slice table ready
        float q[kSmemNK];
        double acc[1] = {0.0};
        float rz1[1] = {0.0f};
#pragma unroll
        for (int k = 0; k < kSmemNK; ++k) {
            if (k * T >= n) break;
            const int i = tid + k * T;
            if (i < n) {
                const double b_i = bv[i];
                x[i] = 0.0;
                const float rh = static_cast<float>(__ldg(sv + i) * b_i);
                R[i] = rh;
                P[i] = rh;
                XH[i] = 0.0f;
                acc[0] += b_i * b_i;
                rz1[0] += rh * rh;
            }
        }
        block_sum<double, 1>(acc, red64);
        block_sum<float, 1>(rz1, red);
        const double bb = acc[0];
        const double thr = a.outer_tol * a.outer_tol * bb;
        double rr64 = bb;
        float rz = rz1[0];
        float rmax = rz;            // scaled |r|^2 at the last replacement
        float goal = static_cast<float>(thr / rr64) * rmax;   // scaled |r|^2 that would meet the target
        int32_t status = ST_RUNNING, it = 0, updates = 0;
        if (bb == 0.0) status = CMCG_SOLVE_ZERO_RHS;
        else if (!finite_(bb)) status = CMCG_SOLVE_NON_FINITE;
        else if (rr64 < thr) status = CMCG_SOLVE_CONVERGED;
        else if (!(rz > 0.0f)) status = CMCG_SOLVE_BREAKDOWN;
        const int64_t maxit = sys_max_iter(a.max_inner, n);
        // progress guard (stall_len), for BF16 inner values (FP32 values keep
        // the unguarded loop; their cycles stall only past condition ~1e7), in
        // shared memory, so that the iteration loop keeps its registers:
        // guard[0] = iteration that forces the next replacement, [1] = first
        // cycle's length, [2] = stalls in a row; written by thread 0 inside a
        // replacement, between barriers
        constexpr bool kGuard = std::is_same<MI, __nv_bfloat16>::value;
        if (kGuard && tid == 0) {
            guard[0] = stall_len(0, 0, a.delta);
            guard[1] = 0;
            guard[2] = 0;
        }
        __syncthreads();
        bool folded = true;
        // diagonal layout: alpha of the x increment not yet added to xh
        bool pend = false;
        float alpha_pend = 0.0f;
        while (status == ST_RUNNING) {
            if (it >= maxit || updates >= a.max_updates) { status = CMCG_SOLVE_MAX_ITER; break; }
            float pq[1] = {0.0f};
            if constexpr (ND > 0) {
                if (unit) {
                    CMCG_DIA_SLOTS(nk, (dia_spmv<NK, ND, true, T>(vt, po, P, tid, q, pq[0])))
                } else {
                    CMCG_DIA_SLOTS(nk, (dia_spmv<NK, ND, false, T>(vt, po, P, tid, q, pq[0])))
                }
            } else {
                // two row slots at a time (slices past the system have width 0)
#pragma unroll
                for (int k = 0; k < kSmemNK; k += 2) {
                    if (k * T >= n) break;   // uniform: skip row slots past the system
                    const int i0 = tid + k * T, i1 = i0 + T;
                    float q0 = 0.0f, q1 = 0.0f;
                    fast_rows2<float>(a.c.col16, vin, tab[warp][k], tab[warp][k + 1], lane, LocalX<float>{P}, q0, q1);
                    q[k] = i0 < n ? q0 : 0.0f;
                    q[k + 1] = i1 < n ? q1 : 0.0f;
                    if (i0 < n) pq[0] += P[i0] * q[k];
                    if (i1 < n) pq[0] += P[i1] * q[k + 1];
                }
            }
            block_sum<float, 1>(pq, red);
            const float alpha = rz / pq[0];
            if (!finite_(pq[0]) || !finite_(alpha)) { status = CMCG_SOLVE_NON_FINITE; break; }
            if (!(pq[0] > 0.0f)) { status = CMCG_SOLVE_BREAKDOWN; break; }
            float s1[1] = {0.0f};
            if constexpr (ND > 0) {
                // the x increment alpha p is added by the p update (or before a fold)
                CMCG_DIA_SLOTS(nk, (dia_update<NK, T>(R, tid, alpha, q, s1[0])))
                alpha_pend = alpha;
                pend = true;
            } else {
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * T >= n) break;   // uniform: skip row slots past the system
                    const int i = tid + k * T;
                    if (i < n) {
                        XH[i] += alpha * P[i];
                        const float ri = R[i] - alpha * q[k];
                        R[i] = ri;
                        s1[0] += ri * ri;
                    }
                }
            }
            block_sum<float, 1>(s1, red);
            ++it;
            folded = false;
            float rzn = s1[0];
            if (!finite_(rzn)) { status = CMCG_SOLVE_NON_FINITE; break; }
            // replace the residual when it dropped by delta, or when it suggests
            // that the FP64 residual may have reached the target, or when the
            // cycle has run too long (progress guard)
            if (rzn < d2 * rmax || rzn < goal || (kGuard && it >= guard[0])) {
                if (ND > 0 && pend) {
                    CMCG_DIA_SLOTS(nk, (dia_xinc<NK, T>(P, XH, tid, alpha_pend)))
                    pend = false;
                }
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * T >= n) break;
                    const int i = tid + k * T;
                    if (i < n) {
                        x[i] += __ldg(sv + i) * static_cast<double>(XH[i]);
                        XH[i] = 0.0f;
                    }
                }
                __syncthreads();
                double t2[2] = {0.0, 0.0};
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * T >= n) break;
                    const int i = tid + k * T;
                    if (i < n) {
                        const double r64 = bv[i] - fast_row<double>(a.c.col16, vout, tab[warp][k], lane, LocalX<double>{x});
                        const float rh = static_cast<float>(__ldg(sv + i) * r64);
                        R[i] = rh;
                        t2[0] += r64 * r64;
                        t2[1] += static_cast<double>(rh) * static_cast<double>(rh);
                    }
                }
                block_sum<double, 2>(t2, red64);
                ++updates;
                folded = true;
                // (every thread has read guard[] for this iteration: block_sum synchronised)
                int stalls = 0;
                if constexpr (kGuard) {
                    stalls = t2[0] > kStallRatio * rr64 ? guard[2] + 1 : 0;
                    const int cyc0 = updates == 1 ? it : guard[1];
                    __syncthreads();
                    if (tid == 0) {
                        guard[0] = it + stall_len(updates, cyc0, a.delta);
                        guard[1] = cyc0;
                        guard[2] = stalls;
                    }
                }
                rr64 = t2[0];
                rzn = static_cast<float>(t2[1]);
                rmax = rzn;
                goal = static_cast<float>(thr / rr64) * rmax;
                if (!finite_(rr64)) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (rr64 < thr) { status = CMCG_SOLVE_CONVERGED; break; }
                if (kGuard && stalls >= kStallMax) { status = CMCG_SOLVE_BREAKDOWN; break; }
            }
            if (!(rzn > 0.0f)) { status = CMCG_SOLVE_BREAKDOWN; break; }
            const float beta = rzn / rz;
            rz = rzn;
            if constexpr (ND > 0) {
                // pend: no replacement this iteration (the fold clears it)
                if (pend) {
                    CMCG_DIA_SLOTS(nk, (dia_pupdate<NK, true, T>(P, R, XH, tid, alpha_pend, beta, q)))
                } else {
                    CMCG_DIA_SLOTS(nk, (dia_pupdate<NK, false, T>(P, R, XH, tid, alpha_pend, beta, q)))
                }
                pend = false;
            } else {
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * T >= n) break;   // uniform: skip row slots past the system
                    const int i = tid + k * T;
                    if (i < n) P[i] = R[i] + beta * P[i];
                }
            }
            __syncthreads();
        }
        if (!folded) {
            // fold the pending increments and report the true residual
            if (ND > 0 && pend) CMCG_DIA_SLOTS(nk, (dia_xinc<NK, T>(P, XH, tid, alpha_pend)))
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * T >= n) break;   // uniform: skip row slots past the system
                const int i = tid + k * T;
                if (i < n) x[i] += __ldg(sv + i) * static_cast<double>(XH[i]);
            }
            __syncthreads();
            double t1[1] = {0.0};
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * T >= n) break;   // uniform: skip row slots past the system
                const int i = tid + k * T;
                if (i < n) {
                    const double r64 = bv[i] - fast_row<double>(a.c.col16, vout, tab[warp][k], lane, LocalX<double>{x});
                    t1[0] += r64 * r64;
                }
            }
            block_sum<double, 1>(t1, red64);
            rr64 = t1[0];
        }
        if (tid == 0) {
            a.st.it[inst] = it;
            a.st.status[inst] = status;
            a.st.rr[inst] = rr64;
            a.st.bb[inst] = bb;
            a.st.outer[inst] = updates;
            a.st.err[inst] = (status == CMCG_SOLVE_ZERO_RHS) ? 0.0 : sqrt(rr64 / bb);
        }
        __syncthreads();
    }
}


template <typename K>
cmcg_status allow_smem_once(K kern, size_t bytes) {
    CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    // the largest shared-memory carveout, so that two 512-thread or four
    // 256-thread CTAs fit
    CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    return CMCG_OK;
}

}  // namespace

template <typename MI, typename MO, int T>
cmcg_status launch_mixed_t(const MixArgs<MI, MO>& m, int nmax, size_t smem, int nd, int grid, cudaStream_t stream) {
    switch (nd) {
        case 0:
            CMCG_TRY(allow_smem_once(k_mixed_fast<MI, MO, 0, T>, smem));
            k_mixed_fast<MI, MO, 0, T><<<grid, T, smem, stream>>>(m, nmax);
            break;
        case 5:
            CMCG_TRY(allow_smem_once(k_mixed_fast<MI, MO, 5, T>, smem));
            k_mixed_fast<MI, MO, 5, T><<<grid, T, smem, stream>>>(m, nmax);
            break;
        case 7:
            CMCG_TRY(allow_smem_once(k_mixed_fast<MI, MO, 7, T>, smem));
            k_mixed_fast<MI, MO, 7, T><<<grid, T, smem, stream>>>(m, nmax);
            break;
        default:
            return fail(CMCG_ERR_INVALID_ARGUMENT, "unsupported number of diagonals");
    }
    return CMCG_OK;
}

template <typename MI, typename MO>
cmcg_status launch_mixed_fast(const MixArgs<MI, MO>& m, int threads, int nmax, size_t smem, int nd, int grid,
                              cudaStream_t stream) {
    if (threads == 256) return launch_mixed_t<MI, MO, 256>(m, nmax, smem, nd, grid, stream);
    if (threads == 512) return launch_mixed_t<MI, MO, 512>(m, nmax, smem, nd, grid, stream);
    if (threads == kSmemThreads) return launch_mixed_t<MI, MO, kSmemThreads>(m, nmax, smem, nd, grid, stream);
    return fail(CMCG_ERR_INVALID_ARGUMENT, "unsupported CTA size");
}

template cmcg_status launch_mixed_fast<float, float>(const MixArgs<float, float>&, int, int, size_t, int, int,
                                                     cudaStream_t);
template cmcg_status launch_mixed_fast<float, double>(const MixArgs<float, double>&, int, int, size_t, int, int,
                                                      cudaStream_t);
template cmcg_status launch_mixed_fast<__nv_bfloat16, float>(const MixArgs<__nv_bfloat16, float>&, int, int, size_t,
                                                             int, int, cudaStream_t);
template cmcg_status launch_mixed_fast<__nv_bfloat16, double>(const MixArgs<__nv_bfloat16, double>&, int, int, size_t,
                                                              int, int, cudaStream_t);

}  // namespace cmcg
