// Conjugate-gradient solver behind the C ABI.
//
// Replaces cuMat's ConjugateGradient / IterativeSolverBase / DiagonalPreconditioner
// / IdentityPreconditioner (cuMat/src/ConjugateGradient.h:66-265,
// IterativeSolverBase.h:10-135) for sparse matrices. The reference runs each
// iteration as ~11 kernel launches (SpMV, 4 cwise kernels, 3 two-pass CUB
// reductions) plus a blocking device-to-host copy of |r|^2
// (ConjugateGradient.h:180-203). Here:
//
//  * PERSISTENT path: one launch for the whole solve. Each CTA pulls a
//    (system, batch) instance from an atomic work counter (largest systems
//    first) and runs the complete PCG loop for it with CTA-level reductions
//    only (__syncthreads, no grid synchronisation, no host round trip).
//  * GRID path (large systems): three fused kernels per iteration over 256-row
//    tiles - SpMV + p.q, x/r update + |r|^2 + r.z, p update - with the per-system
//    reductions finished by the last tile of each system (ticket counter, fixed
//    combine order, deterministic). Scalars stay on the device; the loop is a
//    CUDA graph with a conditional WHILE node whose condition a one-thread
//    kernel sets from the device-side count of running systems.
//  * REFINED solve (mixed precision): FP64 outer residual / update / norms
//    around the FP32 (F32 or BF16 values) inner PCG, fused into the persistent
//    kernel per system, or driven from the host over the grid path.

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include <type_traits>

#include "cg_cluster.cuh"
#include "cg_compact.cuh"
#include "cg_dev.cuh"
#include "cg_smem.cuh"
#include "common.cuh"
#include "cg_grid.cuh"
#include "cg_plain.cuh"
#include "objects.h"

namespace cmcg {
cmcg_status spmv_dispatch(cmcg_matrix A, int32_t vec_dtype, const void* x, int32_t xb, void* y, int32_t mode);
cmcg_status dot_dispatch(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t xb, const void* y, int32_t yb,
                         void* out, int32_t ob);
cmcg_status sddmm_dispatch(cmcg_matrix M, int32_t dt, double alpha, const void* u, int32_t ub, const void* v,
                           int32_t vb, void* out, int32_t ob);
}  // namespace cmcg

using namespace cmcg;

namespace {


// ---------------------------------------------------------------------------
// One system, one CTA (shared by the persistent plain and refined kernels)
// ---------------------------------------------------------------------------

// PCG of one system with the whole CTA. Vectors are batch slices indexed by
// global row. Returns the status; writes iterations / |r|^2 / |b|^2.
template <typename VT, typename MT, int FMT>
__device__ int32_t cta_pcg(const InstMatrix<MT, FMT>& A, int sys, int r0, int n, const VT* __restrict__ bv,
                           const VT* __restrict__ g, VT* __restrict__ x, VT* __restrict__ r, VT* __restrict__ p,
                           VT* __restrict__ q, const VT* __restrict__ dinv, VT tol, int64_t maxit,
                           VT* red, int32_t& it_out, VT& rr_out, VT& bb_out, bool abs_zero_test = true) {
    const int tid = threadIdx.x, T = blockDim.x;
    const int r1 = r0 + n;
    VT acc[2] = {VT(0), VT(0)};
    if (g) {
        cta_rows<VT>(A, sys, r0, 0, n, GlobalX<VT>{g}, [&](int row, VT v) {
            const VT bi = bv[row];
            const VT ri = bi - v;
            r[row] = ri;
            x[row] = g[row];
            acc[0] += bi * bi;
            acc[1] += ri * ri;
        });
    } else {
        for (int i = r0 + tid; i < r1; i += T) {
            const VT bi = bv[i];
            r[i] = bi;
            x[i] = VT(0);
            acc[0] += bi * bi;
        }
        acc[1] = acc[0];
    }
    block_sum<VT, 2>(acc, red);
    const VT bb = acc[0];
    VT rr = acc[1];
    const VT thr = tol * tol * bb;
    int32_t status = ST_RUNNING;
    int32_t it = 0;
    if ((abs_zero_test && bb < tol * tol) || bb == VT(0)) {
        for (int i = r0 + tid; i < r1; i += T) x[i] = VT(0);
        status = CMCG_SOLVE_ZERO_RHS;
    } else if (!finite_(rr) || !finite_(bb)) {
        status = CMCG_SOLVE_NON_FINITE;
    } else if (rr < thr) {
        status = CMCG_SOLVE_CONVERGED;
    } else {
        VT rzv[1] = {VT(0)};
        for (int i = r0 + tid; i < r1; i += T) {
            const VT ri = r[i];
            const VT zi = dinv ? dinv[i] * ri : ri;
            p[i] = zi;
            rzv[0] += ri * zi;
        }
        block_sum<VT, 1>(rzv, red);
        VT rz = rzv[0];
        if (!finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
        else if (!(rz > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
        while (status == ST_RUNNING) {
            if (it >= maxit) { status = CMCG_SOLVE_MAX_ITER; break; }
            VT pq[1] = {VT(0)};
            cta_rows<VT>(A, sys, r0, 0, n, GlobalX<VT>{p}, [&](int row, VT v) {
                q[row] = v;
                pq[0] += p[row] * v;
            });
            block_sum<VT, 1>(pq, red);
            const VT alpha = rz / pq[0];
            if (!finite_(pq[0]) || !finite_(alpha)) { status = CMCG_SOLVE_NON_FINITE; break; }
            if (!(pq[0] > VT(0))) { status = CMCG_SOLVE_BREAKDOWN; break; }
            VT s2[2] = {VT(0), VT(0)};
            for (int i = r0 + tid; i < r1; i += T) {
                x[i] += alpha * p[i];
                const VT ri = r[i] - alpha * q[i];
                r[i] = ri;
                const VT zi = dinv ? dinv[i] * ri : ri;
                s2[0] += ri * ri;
                s2[1] += ri * zi;
            }
            block_sum<VT, 2>(s2, red);
            rr = s2[0];
            if (!finite_(rr) || !finite_(s2[1])) { status = CMCG_SOLVE_NON_FINITE; break; }
            if (rr < thr) { status = CMCG_SOLVE_CONVERGED; break; }
            const VT rzn = s2[1];
            if (!(rzn > VT(0))) { status = CMCG_SOLVE_BREAKDOWN; break; }
            const VT beta = rzn / rz;
            rz = rzn;
            for (int i = r0 + tid; i < r1; i += T) {
                const VT ri = r[i];
                const VT zi = dinv ? dinv[i] * ri : ri;
                p[i] = zi + beta * p[i];
            }
            __syncthreads();
            ++it;
        }
    }
    __syncthreads();
    it_out = it;
    rr_out = rr;
    bb_out = bb;
    return status;
}


template <typename VT, typename MT, int FMT>
__global__ void __launch_bounds__(kPersistThreads) k_persistent_cg(SolveArgs<VT, MT> a) {
    __shared__ VT red[2 * (kPersistThreads / 32)];
    __shared__ int slot;
    const int n_inst = a.n_sys * a.ob;
    for (;;) {
        const int item = fetch_item(a.next, &slot);
        if (item >= n_inst) return;
        const int s = a.order[item / a.ob], b = item % a.ob, inst = b * a.n_sys + s;
        const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0;
        const auto A = inst_matrix<MT, FMT>(a.m, b);
        const int64_t vo = static_cast<int64_t>(b) * a.rows;
        int32_t it;
        VT rr, bb;
        const int32_t status = cta_pcg<VT, MT, FMT>(
            A, s, r0, n, a.b + (a.b_b == 1 ? 0 : vo), a.guess ? a.guess + (a.g_b == 1 ? 0 : vo) : nullptr, a.x + vo,
            a.r + vo, a.p + vo, a.q + vo, a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr, static_cast<VT>(a.tol),
            sys_max_iter(a.max_iter, n), red, it, rr, bb, a.abs_zero_test != 0);
        if (threadIdx.x == 0) {
            a.st.it[inst] = it;
            a.st.status[inst] = status;
            a.st.rr[inst] = static_cast<double>(rr);
            a.st.bb[inst] = static_cast<double>(bb);
            a.st.outer[inst] = 0;
            a.st.err[inst] = (status == CMCG_SOLVE_ZERO_RHS) ? 0.0 : sqrt(static_cast<double>(rr) / static_cast<double>(bb));
        }
    }
}

// ---------------------------------------------------------------------------
// Refined (mixed precision) persistent kernel
// ---------------------------------------------------------------------------

template <typename MI, typename MO>
struct RefineArgs {
    MatArgs<MI> inner;      // F32 / BF16 values, FP32 arithmetic
    MatArgs<MO> outer;      // F32 / F64 values, FP64 arithmetic
    int32_t rows, n_sys, ob;
    const int32_t* row_off;
    const int32_t* order;
    int32_t* next;
    const float* dinv;
    int32_t dinv_b;
    const double* b;
    int32_t b_b;
    double* x;
    float* r32;   // inner rhs = rounded outer residual
    float* d32;   // inner solution
    float* r;     // inner CG vectors
    float* p;
    float* q;
    double inner_tol, outer_tol;
    int64_t max_inner;
    int32_t max_outer;
    InstState st;
};

template <typename MI, typename MO, int FMT>
__global__ void __launch_bounds__(kPersistThreads) k_persistent_refined(RefineArgs<MI, MO> a) {
    __shared__ double red64[2 * (kPersistThreads / 32)];
    __shared__ float red32[2 * (kPersistThreads / 32)];
    __shared__ int slot;
    const int tid = threadIdx.x, T = blockDim.x;
    const int n_inst = a.n_sys * a.ob;
    for (;;) {
        const int item = fetch_item(a.next, &slot);
        if (item >= n_inst) return;
        const int s = a.order[item / a.ob], bi = item % a.ob, inst = bi * a.n_sys + s;
        const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0, r1 = r0 + n;
        const auto Ai = inst_matrix<MI, FMT>(a.inner, bi);
        const auto Ao = inst_matrix<MO, FMT>(a.outer, bi);
        const int64_t vo = static_cast<int64_t>(bi) * a.rows;
        const double* bv = a.b + (a.b_b == 1 ? 0 : vo);
        double* x = a.x + vo;
        float* r32 = a.r32 + vo;
        float* d32 = a.d32 + vo;
        const float* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
        // x = 0, r = b
        double acc[1] = {0.0};
        for (int i = r0 + tid; i < r1; i += T) {
            const double b_i = bv[i];
            x[i] = 0.0;
            r32[i] = static_cast<float>(b_i);
            acc[0] += b_i * b_i;
        }
        block_sum<double, 1>(acc, red64);
        const double bb = acc[0];
        double rr = bb;
        int32_t status = ST_RUNNING, outer = 0;
        int64_t inner_total = 0;
        const double thr = a.outer_tol * a.outer_tol * bb;
        if (bb == 0.0) status = CMCG_SOLVE_ZERO_RHS;
        else if (!finite_(bb)) status = CMCG_SOLVE_NON_FINITE;
        while (status == ST_RUNNING) {
            if (rr < thr) { status = CMCG_SOLVE_CONVERGED; break; }
            if (outer >= a.max_outer) { status = CMCG_SOLVE_MAX_ITER; break; }
            int32_t it;
            float rr_in, bb_in;
            const int32_t st_in = cta_pcg<float, MI, FMT>(Ai, s, r0, n, r32, nullptr, d32, a.r + vo, a.p + vo, a.q + vo,
                                                          dinv, static_cast<float>(a.inner_tol),
                                                          sys_max_iter(a.max_inner, n), red32, it, rr_in, bb_in,
                                                          /*abs_zero_test=*/false);
            inner_total += it;
            if (st_in == CMCG_SOLVE_NON_FINITE || (st_in == CMCG_SOLVE_BREAKDOWN && it == 0)) { status = st_in; break; }
            for (int i = r0 + tid; i < r1; i += T) x[i] += static_cast<double>(d32[i]);
            __syncthreads();
            // FP64 residual with the outer values, rounded into the next inner rhs
            double rv[1] = {0.0};
            cta_rows<double>(Ao, s, r0, 0, n, GlobalX<double>{x}, [&](int row, double v) {
                const double ri = bv[row] - v;
                r32[row] = static_cast<float>(ri);
                rv[0] += ri * ri;
            });
            block_sum<double, 1>(rv, red64);
            rr = rv[0];
            ++outer;
            if (!finite_(rr)) { status = CMCG_SOLVE_NON_FINITE; break; }
        }
        if (tid == 0) {
            a.st.it[inst] = static_cast<int32_t>(inner_total < INT32_MAX ? inner_total : INT32_MAX);
            a.st.status[inst] = status;
            a.st.rr[inst] = rr;
            a.st.bb[inst] = bb;
            a.st.outer[inst] = outer;
            a.st.err[inst] = (status == CMCG_SOLVE_ZERO_RHS) ? 0.0 : sqrt(rr / bb);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Shared-memory-resident kernels (systems of at most kSmemMaxRows rows)
// ---------------------------------------------------------------------------

// FP32 PCG with the reference's algorithm and stopping rule.
template <typename MT, int FMT>
__global__ void __launch_bounds__(kSmemThreads, 1) k_cg_smem(SolveArgs<float, MT> a, int nmax) {
    extern __shared__ __align__(16) float sm[];
    __shared__ float red[2 * (kSmemThreads / 32)];
    __shared__ int slot;
    const SmemLayout L = smem_layout(sm, nmax);
    const int tid = threadIdx.x;
    const int n_inst = a.n_sys * a.ob;
    const float tol = static_cast<float>(a.tol);
    for (;;) {
        const int item = fetch_item(a.next, &slot);
        if (item >= n_inst) return;
        const int s = a.order[item / a.ob], b = item % a.ob, inst = b * a.n_sys + s;
        const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0;
        const auto A = inst_matrix<MT, FMT>(a.m, b);
        const int64_t vo = static_cast<int64_t>(b) * a.rows;
        const float* bv = a.b + (a.b_b == 1 ? 0 : vo) + r0;
        float* xg = a.x + vo + r0;
        const float* dg = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) + r0 : nullptr;
        float q[kSmemNK];
        float acc[2] = {0.0f, 0.0f};
        // inverse diagonal through the read-only cache (1 for the identity preconditioner)
        auto dv = [&](int i) { return dg ? __ldg(dg + i) : 1.0f; };
        if (a.guess) {
            const float* g = a.guess + (a.g_b == 1 ? 0 : vo);
            smem_product<MT, FMT>(A, s, r0, n, GlobalX<float>{g}, q);
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    const float bi = bv[i];
                    const float ri = bi - q[k];
                    L.x[i] = g[r0 + i];
                    L.r[i] = ri;
                    acc[0] += bi * bi;
                    acc[1] += ri * ri;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    const float bi = bv[i];
                    L.r[i] = bi;
                    L.x[i] = 0.0f;
                    acc[0] += bi * bi;
                }
            }
            acc[1] = acc[0];
        }
        block_sum<float, 2>(acc, red);
        const float bb = acc[0];
        float rr = acc[1];
        const float thr = tol * tol * bb;
        int32_t status = ST_RUNNING, it = 0;
        if ((a.abs_zero_test && bb < tol * tol) || bb == 0.0f) {
            status = CMCG_SOLVE_ZERO_RHS;
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) L.x[i] = 0.0f;
            }
        } else if (!finite_(rr) || !finite_(bb)) {
            status = CMCG_SOLVE_NON_FINITE;
        } else if (rr < thr) {
            status = CMCG_SOLVE_CONVERGED;
        } else {
            float rz1[1] = {0.0f};
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    const float ri = L.r[i];
                    const float zi = dv(i) * ri;
                    L.p[i] = zi;
                    rz1[0] += ri * zi;
                }
            }
            block_sum<float, 1>(rz1, red);
            float rz = rz1[0];
            if (!finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
            else if (!(rz > 0.0f)) status = CMCG_SOLVE_BREAKDOWN;
            const int64_t maxit = sys_max_iter(a.max_iter, n);
            while (status == ST_RUNNING) {
                if (it >= maxit) { status = CMCG_SOLVE_MAX_ITER; break; }
                smem_product<MT, FMT>(A, s, r0, n, SmemX{L.p, r0}, q);
                float pq[1] = {0.0f};
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    const int i = tid + k * kSmemThreads;
                    if (i < n) pq[0] += L.p[i] * q[k];
                }
                block_sum<float, 1>(pq, red);
                const float alpha = rz / pq[0];
                if (!finite_(pq[0]) || !finite_(alpha)) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (!(pq[0] > 0.0f)) { status = CMCG_SOLVE_BREAKDOWN; break; }
                float s2[2] = {0.0f, 0.0f};
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    const int i = tid + k * kSmemThreads;
                    if (i < n) {
                        L.x[i] += alpha * L.p[i];
                        const float ri = L.r[i] - alpha * q[k];
                        L.r[i] = ri;
                        s2[0] += ri * ri;
                        s2[1] += ri * (dv(i) * ri);
                    }
                }
                block_sum<float, 2>(s2, red);
                rr = s2[0];
                if (!finite_(rr) || !finite_(s2[1])) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (rr < thr) { status = CMCG_SOLVE_CONVERGED; break; }
                if (!(s2[1] > 0.0f)) { status = CMCG_SOLVE_BREAKDOWN; break; }
                const float beta = s2[1] / rz;
                rz = s2[1];
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    const int i = tid + k * kSmemThreads;
                    if (i < n) L.p[i] = dv(i) * L.r[i] + beta * L.p[i];
                }
                __syncthreads();
                ++it;
            }
        }
#pragma unroll
        for (int k = 0; k < kSmemNK; ++k) {
            const int i = tid + k * kSmemThreads;
            if (i < n) xg[i] = L.x[i];
        }
        if (tid == 0) {
            a.st.it[inst] = it;
            a.st.status[inst] = status;
            a.st.rr[inst] = rr;
            a.st.bb[inst] = bb;
            a.st.outer[inst] = 0;
            a.st.err[inst] = (status == CMCG_SOLVE_ZERO_RHS) ? 0.0 : sqrt(static_cast<double>(rr) / static_cast<double>(bb));
        }
        __syncthreads();
    }
}

// Mixed precision with reliable updates: FP32 PCG (values MI) whose solution
// increments are folded into the FP64 solution, and whose recursive residual is
// replaced by the true FP64 residual b - A x (values MO) whenever it has dropped
// by `delta` since the last replacement or looks converged (residual
// replacement, van der Vorst & Ye 2000; reliable updates as in Clark et al.
// 2010). The Krylov direction p is kept across replacements, so the iteration
// count stays close to plain CG's. Convergence is decided on the FP64 residual:
// |b - A x| < outer_tol |b|.
template <typename MI, typename MO, int FMT>
__global__ void __launch_bounds__(kSmemThreads, 1) k_reliable_smem(RefineArgs<MI, MO> a, int nmax, float delta) {
    extern __shared__ __align__(16) float sm[];
    __shared__ float red[2 * (kSmemThreads / 32)];
    __shared__ double red64[2 * (kSmemThreads / 32)];
    __shared__ int slot;
    const SmemLayout L = smem_layout(sm, nmax);
    const int tid = threadIdx.x;
    const int n_inst = a.n_sys * a.ob;
    for (;;) {
        const int item = fetch_item(a.next, &slot);
        if (item >= n_inst) return;
        const int s = a.order[item / a.ob], bi = item % a.ob, inst = bi * a.n_sys + s;
        const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0;
        const auto Ai = inst_matrix<MI, FMT>(a.inner, bi);
        const auto Ao = inst_matrix<MO, FMT>(a.outer, bi);
        const int64_t vo = static_cast<int64_t>(bi) * a.rows;
        const double* bv = a.b + (a.b_b == 1 ? 0 : vo);
        double* x = a.x + vo;
        const float* dg = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
        float q[kSmemNK];
        auto dv = [&](int i) { return dg ? __ldg(dg + r0 + i) : 1.0f; };
        double acc[1] = {0.0};
        float rz1[1] = {0.0f};
#pragma unroll
        for (int k = 0; k < kSmemNK; ++k) {
            const int i = tid + k * kSmemThreads;
            if (i < n) {
                const double b_i = bv[r0 + i];
                x[r0 + i] = 0.0;
                const float ri = static_cast<float>(b_i);
                const float di = dv(i);
                L.r[i] = ri;
                L.x[i] = 0.0f;
                L.p[i] = di * ri;
                acc[0] += b_i * b_i;
                rz1[0] += ri * (di * ri);
            }
        }
        block_sum<double, 1>(acc, red64);
        block_sum<float, 1>(rz1, red);
        const double bb = acc[0];
        const double thr = a.outer_tol * a.outer_tol * bb;
        double rr64 = bb;
        double rmax2 = bb;                      // |r|^2 at the last replacement
        const float thr32 = static_cast<float>(thr);
        float rz = rz1[0];
        int32_t status = ST_RUNNING, it = 0, updates = 0;
        if (bb == 0.0) status = CMCG_SOLVE_ZERO_RHS;
        else if (!finite_(bb)) status = CMCG_SOLVE_NON_FINITE;
        else if (rr64 < thr) status = CMCG_SOLVE_CONVERGED;
        else if (!(rz > 0.0f)) status = CMCG_SOLVE_BREAKDOWN;
        const int64_t maxit = sys_max_iter(a.max_inner, n);
        const float d2 = delta * delta;
        while (status == ST_RUNNING) {
            if (it >= maxit || updates >= a.max_outer) { status = CMCG_SOLVE_MAX_ITER; break; }
            smem_product<MI, FMT>(Ai, s, r0, n, SmemX{L.p, r0}, q);
            float pq[1] = {0.0f};
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) pq[0] += L.p[i] * q[k];
            }
            block_sum<float, 1>(pq, red);
            const float alpha = rz / pq[0];
            if (!finite_(pq[0]) || !finite_(alpha)) { status = CMCG_SOLVE_NON_FINITE; break; }
            if (!(pq[0] > 0.0f)) { status = CMCG_SOLVE_BREAKDOWN; break; }
            float s2[2] = {0.0f, 0.0f};
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    L.x[i] += alpha * L.p[i];
                    const float ri = L.r[i] - alpha * q[k];
                    L.r[i] = ri;
                    s2[0] += ri * ri;
                    s2[1] += ri * (dv(i) * ri);
                }
            }
            block_sum<float, 2>(s2, red);
            ++it;
            if (!finite_(s2[0]) || !finite_(s2[1])) { status = CMCG_SOLVE_NON_FINITE; break; }
            float rzn = s2[1];
            if (s2[0] < d2 * static_cast<float>(rmax2) || s2[0] < thr32) {
                // reliable update: fold the FP32 increments into x, replace r
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    const int i = tid + k * kSmemThreads;
                    if (i < n) {
                        x[r0 + i] += static_cast<double>(L.x[i]);
                        L.x[i] = 0.0f;
                    }
                }
                __syncthreads();
                double t2[2] = {0.0, 0.0};
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    const int i = tid + k * kSmemThreads;
                    if (i < n) {
                        const double r64 = bv[r0 + i] - row_product<double>(Ao.rm, s, r0, i, GlobalX<double>{x});
                        const float ri = static_cast<float>(r64);
                        L.r[i] = ri;
                        t2[0] += r64 * r64;
                        t2[1] += static_cast<double>(ri) * static_cast<double>(dv(i) * ri);
                    }
                }
                block_sum<double, 2>(t2, red64);
                ++updates;
                rr64 = t2[0];
                rmax2 = rr64;
                rzn = static_cast<float>(t2[1]);
                if (!finite_(rr64)) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (rr64 < thr) { status = CMCG_SOLVE_CONVERGED; break; }
            }
            if (!(rzn > 0.0f)) { status = CMCG_SOLVE_BREAKDOWN; break; }
            const float beta = rzn / rz;
            rz = rzn;
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) L.p[i] = dv(i) * L.r[i] + beta * L.p[i];
            }
            __syncthreads();
        }
        // fold any pending increments (iteration limit / breakdown exits)
        bool pending = false;
#pragma unroll
        for (int k = 0; k < kSmemNK; ++k) {
            const int i = tid + k * kSmemThreads;
            if (i < n && L.x[i] != 0.0f) { x[r0 + i] += static_cast<double>(L.x[i]); pending = true; }
        }
        if (__syncthreads_or(pending)) {
            double t1[1] = {0.0};
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    const double r64 = bv[r0 + i] - row_product<double>(Ao.rm, s, r0, i, GlobalX<double>{x});
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

// ---------------------------------------------------------------------------
// Fast shared-memory kernels over the compact sliced layout (cg_compact.cuh;
// the mixed-precision one is in cg_mixed.cu)
// ---------------------------------------------------------------------------

// Plain PCG (the reference's algorithm and stopping rule) on the compact layout.
// p always lives in shared memory (it is gathered); r and x live there too when
// RX_SMEM, else in global memory (coalesced, one access per row and pass).
template <typename VT, typename MT, bool RX_SMEM>
__global__ void __launch_bounds__(kSmemThreads, 1) k_cg_fast(SolveArgs<VT, MT> a, CompactArgs c, int nmax) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ SliceEnt tab[32][kSmemNK];
    __shared__ VT red[2 * (kSmemThreads / 32)];
    __shared__ int slot;
    VT* P = reinterpret_cast<VT*>(smraw);
    VT* Rs = P + nmax;
    VT* Xs = P + 2 * nmax;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n_inst = a.n_sys * a.ob;
    const VT tol = static_cast<VT>(a.tol);
    for (;;) {
        const int item = fetch_item(a.next, &slot);
        if (item >= n_inst) return;
        const int s = a.order[item / a.ob], b = item % a.ob, inst = b * a.n_sys + s;
        const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0;
        const int sl0 = __ldg(c.sys_slice0 + s), nsl = __ldg(c.sys_slice0 + s + 1) - sl0;
        load_slice_table(tab, c.off32, c.sw, sl0, nsl);
        const int64_t vo = static_cast<int64_t>(b) * a.rows;
        const MT* vals = a.m.sell_vals + (a.m.mb == 1 ? 0 : static_cast<int64_t>(b) * a.m.sell_vstride);
        const VT* bv = a.b + (a.b_b == 1 ? 0 : vo) + r0;
        VT* xg = a.x + vo + r0;
        VT* R = RX_SMEM ? Rs : a.r + vo + r0;
        VT* X = RX_SMEM ? Xs : xg;
        const VT* dg = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) + r0 : nullptr;
        auto dv = [&](int i) { return dg ? __ldg(dg + i) : VT(1); };
        __syncthreads();   // slice table ready
        // q = A p: registers for FP32; for FP64 (twice the registers) a global
        // buffer written and read back by the same thread (L1 / L2 resident)
        constexpr bool kQReg = sizeof(VT) == 4;
        VT* Qg = a.q + vo + r0;
        VT q[kQReg ? kSmemNK : 1];
        VT acc[2] = {VT(0), VT(0)};
        if (a.guess) {
            const VT* g = a.guess + (a.g_b == 1 ? 0 : vo) + r0;
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * kSmemThreads >= n) break;   // uniform: skip row slots past the system
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    const VT ag = fast_row<VT>(c.col16, vals, tab[warp][k], lane, LocalX<VT>{g});
                    const VT bi = bv[i], ri = bi - ag;
                    X[i] = g[i];
                    R[i] = ri;
                    acc[0] += bi * bi;
                    acc[1] += ri * ri;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * kSmemThreads >= n) break;   // uniform: skip row slots past the system
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    const VT bi = bv[i];
                    R[i] = bi;
                    X[i] = VT(0);
                    acc[0] += bi * bi;
                }
            }
            acc[1] = acc[0];
        }
        block_sum<VT, 2>(acc, red);
        const VT bb = acc[0];
        VT rr = acc[1];
        const VT thr = tol * tol * bb;
        int32_t status = ST_RUNNING, it = 0;
        if ((a.abs_zero_test && bb < tol * tol) || bb == VT(0)) {
            status = CMCG_SOLVE_ZERO_RHS;
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * kSmemThreads >= n) break;   // uniform: skip row slots past the system
                const int i = tid + k * kSmemThreads;
                if (i < n) X[i] = VT(0);
            }
        } else if (!finite_(rr) || !finite_(bb)) {
            status = CMCG_SOLVE_NON_FINITE;
        } else if (rr < thr) {
            status = CMCG_SOLVE_CONVERGED;
        } else {
            VT rz1[1] = {VT(0)};
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * kSmemThreads >= n) break;   // uniform: skip row slots past the system
                const int i = tid + k * kSmemThreads;
                if (i < n) {
                    const VT ri = R[i], zi = dv(i) * ri;
                    P[i] = zi;
                    rz1[0] += ri * zi;
                }
            }
            block_sum<VT, 1>(rz1, red);
            VT rz = rz1[0];
            if (!finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
            else if (!(rz > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
            const int64_t maxit = sys_max_iter(a.max_iter, n);
            while (status == ST_RUNNING) {
                if (it >= maxit) { status = CMCG_SOLVE_MAX_ITER; break; }
                VT pq[1] = {VT(0)};
                // two row slots at a time (slices past the system have width 0)
#pragma unroll
                for (int k = 0; k < kSmemNK; k += 2) {
                    if (k * kSmemThreads >= n) break;
                    const int i0 = tid + k * kSmemThreads, i1 = i0 + kSmemThreads;
                    VT q0, q1;
                    fast_rows2<VT>(c.col16, vals, tab[warp][k], tab[warp][k + 1], lane, LocalX<VT>{P}, q0, q1);
                    if (i0 < n) {
                        if constexpr (kQReg) q[k] = q0; else Qg[i0] = q0;
                        pq[0] += P[i0] * q0;
                    }
                    if (i1 < n) {
                        if constexpr (kQReg) q[k + 1] = q1; else Qg[i1] = q1;
                        pq[0] += P[i1] * q1;
                    }
                }
                block_sum<VT, 1>(pq, red);
                const VT alpha = rz / pq[0];
                if (!finite_(pq[0]) || !finite_(alpha)) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (!(pq[0] > VT(0))) { status = CMCG_SOLVE_BREAKDOWN; break; }
                VT s2[2] = {VT(0), VT(0)};
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * kSmemThreads >= n) break;
                    const int i = tid + k * kSmemThreads;
                    if (i < n) {
                        X[i] += alpha * P[i];
                        VT qi;
                        if constexpr (kQReg) qi = q[kQReg ? k : 0]; else qi = Qg[i];
                        const VT ri = R[i] - alpha * qi;
                        R[i] = ri;
                        s2[0] += ri * ri;
                        s2[1] += ri * (dv(i) * ri);
                    }
                }
                block_sum<VT, 2>(s2, red);
                rr = s2[0];
                if (!finite_(rr) || !finite_(s2[1])) { status = CMCG_SOLVE_NON_FINITE; break; }
                if (rr < thr) { status = CMCG_SOLVE_CONVERGED; break; }
                if (!(s2[1] > VT(0))) { status = CMCG_SOLVE_BREAKDOWN; break; }
                const VT beta = s2[1] / rz;
                rz = s2[1];
#pragma unroll
                for (int k = 0; k < kSmemNK; ++k) {
                    if (k * kSmemThreads >= n) break;
                    const int i = tid + k * kSmemThreads;
                    if (i < n) P[i] = dv(i) * R[i] + beta * P[i];
                }
                __syncthreads();
                ++it;
            }
        }
        if (RX_SMEM) {
#pragma unroll
            for (int k = 0; k < kSmemNK; ++k) {
                if (k * kSmemThreads >= n) break;   // uniform: skip row slots past the system
                const int i = tid + k * kSmemThreads;
                if (i < n) xg[i] = X[i];
            }
        }
        if (tid == 0) {
            a.st.it[inst] = it;
            a.st.status[inst] = status;
            a.st.rr[inst] = static_cast<double>(rr);
            a.st.bb[inst] = static_cast<double>(bb);
            a.st.outer[inst] = 0;
            a.st.err[inst] = (status == CMCG_SOLVE_ZERO_RHS) ? 0.0 : sqrt(static_cast<double>(rr) / static_cast<double>(bb));
        }
        __syncthreads();
    }
}

// s = 1/sqrt(a_ii) where a_ii > 0 (Jacobi), else 1; [mb][rows]
template <typename MT>
__global__ void k_jacobi_scale(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const MT* __restrict__ vals,
                               int64_t vstride, int32_t rows, int32_t mb, int32_t jacobi, double* __restrict__ out) {
    const int64_t items = static_cast<int64_t>(rows) * mb;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(it / rows);
        const int r = static_cast<int>(it - static_cast<int64_t>(b) * rows);
        double d = 0.0;
        if (jacobi)
            for (int k = rp[r]; k < rp[r + 1]; ++k)
                if (ci[k] == r) { d = mval<double>(vals[b * vstride + k]); break; }
        out[it] = d > 0.0 ? 1.0 / sqrt(d) : 1.0;
    }
}

// Scaled values in the diagonal layout: dst[b][pos[k]] = a_k * s_row * s_col for
// every CSR entry k (thread per row); slots without an entry stay zero.
template <typename MT>
__global__ void k_scale_dia(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const MT* __restrict__ vals,
                            int64_t vstride, const int32_t* __restrict__ pos, const double* __restrict__ sc, int32_t rows,
                            int32_t mb, MT* __restrict__ dst, int64_t dstride) {
    const int64_t items = static_cast<int64_t>(rows) * mb;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(it / rows);
        const int r = static_cast<int>(it - static_cast<int64_t>(b) * rows);
        const double* sb = sc + static_cast<int64_t>(b) * rows;
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            dst[b * dstride + pos[k]] = from_f64<MT>(mval<double>(vals[b * vstride + k]) * sb[r] * sb[ci[k]]);
    }
}

// flag[b][s] = 1 when diagonal nd / 2 of system s is offset 0 and its values on
// the system's rows are all exactly 1 (Jacobi scaling of a positive diagonal
// gives 1 after rounding), else 0; one CTA per (batch, system).
template <typename MT>
__global__ void k_dia_unit(const MT* __restrict__ vals, int64_t vstride, const int64_t* __restrict__ base,
                           const int32_t* __restrict__ off, const int32_t* __restrict__ row_off, int32_t n_sys,
                           int32_t mb, int32_t nd, int32_t* __restrict__ flag) {
    for (int64_t item = blockIdx.x; item < static_cast<int64_t>(n_sys) * mb; item += gridDim.x) {
        const int b = static_cast<int>(item / n_sys), s = static_cast<int>(item - static_cast<int64_t>(b) * n_sys);
        const int n = row_off[s + 1] - row_off[s];
        const MT* v = vals + b * vstride + base[s];
        int ok = off[s * kDiaMax + nd / 2] == 0;
        for (int i = threadIdx.x; ok && i < n; i += blockDim.x)
            ok = mval<double>(v[kDiaBlockRows * ((i / kDiaBlockRows) * nd + nd / 2) + i % kDiaBlockRows]) == 1.0;
        ok = __syncthreads_and(ok);
        if (threadIdx.x == 0) flag[item] = ok;
    }
}

// out[b][slot] = a * s_row * s_col for every slot of the sliced layout (warp per slice)
template <typename MS, typename MD>
__global__ void k_scale_sell(const int32_t* __restrict__ col, const int64_t* __restrict__ off64,
                             const int32_t* __restrict__ sw, const int32_t* __restrict__ row0, int32_t n_slices,
                             const MS* __restrict__ src, int64_t sstride, const double* __restrict__ sc, int32_t rows,
                             int32_t mb, MD* __restrict__ dst, int64_t dstride) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t item = wid; item < static_cast<int64_t>(n_slices) * mb; item += nw) {
        const int b = static_cast<int>(item / n_slices);
        const int sl = static_cast<int>(item - static_cast<int64_t>(b) * n_slices);
        const int row = row0[sl] + lane, w = sw[sl];
        const int64_t off = off64[sl];
        const double* sb = sc + static_cast<int64_t>(b) * rows;
        for (int j = 0; j < w; ++j) {
            const int64_t o = off + 32 * j + lane;
            const double v = mval<double>(src[b * sstride + o]);
            double out = 0.0;
            if (v != 0.0 && row < rows) out = v * sb[row] * sb[col[o]];
            dst[b * dstride + o] = from_f64<MD>(out);
        }
    }
}

// ---------------------------------------------------------------------------
// Diagonal-layout products of the grid path (stencil-shaped CSR patterns)
// ---------------------------------------------------------------------------

// The four values of a diagonal for four consecutive rows, loaded as streaming
// data (ld.global.cs: evict-first in L1 and L2). A grid-path product reads each
// value once per iteration while the p entries it gathers at offsets of up to
// a grid plane are read again by later rows; evicting the values first keeps
// those p entries in L2 on systems whose vectors exceed it.
__device__ __forceinline__ void load_stream(Vals4<float>& w, const float* p) {
    const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
    w.v[0] = t.x; w.v[1] = t.y; w.v[2] = t.z; w.v[3] = t.w;
}
__device__ __forceinline__ void load_stream(Vals4<double>& w, const double* p) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    w.v[0] = a.x; w.v[1] = a.y; w.v[2] = b.x; w.v[3] = b.y;
}
__device__ __forceinline__ void load_stream(Vals4<__nv_bfloat16>& w, const __nv_bfloat16* p) {
    const uint2 t = __ldcs(reinterpret_cast<const uint2*>(p));
    const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&t.x);
    const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&t.y);
    w.v[0] = a.x; w.v[1] = a.y; w.v[2] = b.x; w.v[3] = b.y;
}

// p[c .. c + 3] with each index clamped into [lo, hi]: one or two 16-byte loads
// where the four entries lie inside and start on a 16-byte boundary, else four
// clamped scalar loads (the same entries either way).
template <typename VT>
__device__ __forceinline__ void p_quad(const VT* __restrict__ p, int c, int lo, int hi, VT (&o)[4]) {
    if (c >= lo && c + 3 <= hi && (reinterpret_cast<uintptr_t>(p + c) & 15) == 0) {
        if constexpr (sizeof(VT) == 4) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(p + c));
            o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
        } else {
            const double2 a = __ldg(reinterpret_cast<const double2*>(p + c));
            const double2 b = __ldg(reinterpret_cast<const double2*>(p + c) + 1);
            o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = __ldg(p + min(max(c + q, lo), hi));
    }
}

// p_k of the grid path, formed where it is read: p_k[j] = z_j + beta p_{k-1}[j]
// with z = M^-1 r (r and beta of iteration k, p_{k-1} the other p buffer), the
// expression of the former p-update kernel; the product forms it for its own
// rows (and stores them) and for every entry it gathers, so the iteration needs
// no p-update launch. Iteration 0 reads beta = 0 and a zeroed p_{-1}.
template <typename VT>
struct PNext {
    const VT* __restrict__ r;
    const VT* __restrict__ dinv;   // null: identity
    const VT* __restrict__ pin;    // p_{k-1}
    VT beta;
    // (one explicit fused multiply-add, as in the separate p-update kernels,
    // so that both forms round alike)
    __device__ __forceinline__ VT form(VT d, VT ri, VT pi) const {
        const VT z = dinv ? d * ri : ri;
        return fma(beta, pi, z);
    }
    __device__ __forceinline__ VT operator()(int c) const {
        return form(dinv ? __ldg(dinv + c) : VT(1), __ldg(r + c), __ldg(pin + c));
    }
    // entries c .. c + 3, indices clamped into [lo, hi] (see p_quad)
    __device__ __forceinline__ void quad(int c, int lo, int hi, VT (&o)[4]) const {
        VT rq[4], pq[4], dq[4] = {VT(1), VT(1), VT(1), VT(1)};
        p_quad(r, c, lo, hi, rq);
        p_quad(pin, c, lo, hi, pq);
        if (dinv) p_quad(dinv, c, lo, hi, dq);
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = form(dq[q], rq[q], pq[q]);
    }
};

// p_k read as stored (the separate p-update kernel formed it): the product's
// source when the vectors do not stay in L2 (see fuse_p_update)
template <typename VT>
struct PDirect {
    const VT* __restrict__ p;
    __device__ __forceinline__ VT operator()(int c) const { return __ldg(p + c); }
    __device__ __forceinline__ void quad(int c, int lo, int hi, VT (&o)[4]) const { p_quad(p, c, lo, hi, o); }
};

// q[i] = sum_d v_d[i] p[i + off_d] for the rows [r0, r1) of one system (global
// rows sr0 .. send - 1, r0 - sr0 a multiple of 4; v points at the system's
// first value), diagonals in ascending offset order, the row's CSR order, with
// fused multiply-adds: absent entries hold 0 and add 0 * p exactly, so each
// sum equals the sliced layout's. Thread t takes the four rows r0 + 4 t ..
// r0 + 4 t + 3, then r0 + 4 (t + kTile) ..., the rows the sliced path gives
// it, and emits them in the same order, so partial sums over the emitted
// rows match too; the values of a diagonal for its four rows are one 16-byte
// (8-byte for BF16) streaming load. p indices are clamped into the system,
// where a zero value (or, past the system's end, a row that is not emitted)
// meets them. p is p_k: formed from r, M^-1 and p_{k-1} (PNext) or read as
// stored (PDirect). The gathers:
// a thread forms its own four p entries (offset 0) from one quad of each
// input; offsets -1 and +1 take three of them and one entry from the
// neighbouring lane (formed from scalar loads at the warp's edges); other
// offsets form a quad each. The entries are the clamped ones in every case,
// so the sums do not depend on how they were loaded.
// UNIT: the middle diagonal is offset 0 with every value 1 and is not loaded.
// emit(global row, value, p[row]).
template <typename VT, typename MT, int ND, bool UNIT, typename PS, typename F>
__device__ __forceinline__ void dia_rows_seg(const MT* __restrict__ v, const int (&off)[ND], int sr0, int send, int r0,
                                             int r1, const PS& p, F&& emit) {
    const int lane = threadIdx.x & 31;
    // the loop bound is the same for the whole CTA, so every lane takes part
    // in the shuffles
    for (int base = r0; base < r1; base += 4 * kTile) {
        const int ib = base + 4 * threadIdx.x;
        VT own[4];
        p.quad(ib, sr0, send - 1, own);   // (ib >= sr0: only the upper clamp acts)
        const VT from_prev = __shfl_up_sync(FULL, own[3], 1);     // p[ib - 1] of lane - 1's quad
        const VT from_next = __shfl_down_sync(FULL, own[0], 1);   // p[ib + 4] of lane + 1's quad
        if (ib >= r1) continue;
        const int li = ib - sr0;
        const MT* vr = v + (static_cast<int64_t>(li / kDiaBlockRows) * ND * kDiaBlockRows) + li % kDiaBlockRows;
        // The value loads (the streamed bytes) of all diagonals are issued
        // before the first use, so that one diagonal's DRAM latency does not
        // follow another's behind the offset branches below; 8-byte values
        // keep the per-diagonal order (ND quads of them would not fit the
        // 64-register budget of four CTAs per SM).
        constexpr bool kHoist = sizeof(MT) <= 4;
        Vals4<MT> w[kHoist ? ND : 1];
        if constexpr (kHoist) {
#pragma unroll
            for (int d = 0; d < ND; ++d)
                if (!(UNIT && d == ND / 2)) load_stream(w[d], vr + d * kDiaBlockRows);
        }
        VT acc[4] = {VT(0), VT(0), VT(0), VT(0)};
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const int o = off[d];
            VT pv[4];
            if (o == 0) {
#pragma unroll
                for (int q = 0; q < 4; ++q) pv[q] = own[q];
            } else if (o == -1) {
                // lane >= 1: lane - 1's quad starts at ib - 4 >= r0, so its last
                // entry is p[ib - 1] itself
                pv[0] = lane ? from_prev : p(max(ib - 1, sr0));
                pv[1] = own[0]; pv[2] = own[1]; pv[3] = own[2];
            } else if (o == 1) {
                pv[0] = own[1]; pv[1] = own[2]; pv[2] = own[3];
                pv[3] = lane != 31 ? from_next : p(min(ib + 4, send - 1));
            } else {
                p.quad(ib + o, sr0, send - 1, pv);
            }
            if (UNIT && d == ND / 2) {
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] = fma(VT(1), pv[q], acc[q]);
            } else {
                Vals4<MT> wd;
                if constexpr (kHoist) wd = w[d];
                else load_stream(wd, vr + d * kDiaBlockRows);
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] = fma(mval<VT>(wd.v[q]), pv[q], acc[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (ib + q < r1) emit(ib + q, acc[q], own[q]);
    }
}

// The segment's system values and offsets in the diagonal layout.
template <typename MT, int ND>
__device__ __forceinline__ const MT* dia_system(const DiaArgs<MT>& d, int b, int s, int (&off)[ND]) {
#pragma unroll
    for (int j = 0; j < ND; ++j) off[j] = __ldg(d.off + s * kDiaMax + j);
    return d.vals + (d.mb == 1 ? 0 : static_cast<int64_t>(b) * d.vstride) + __ldg(d.base + s);
}

// Values of a CSR matrix in the pattern's diagonal layout, unscaled:
// dst[b][pos[k]] = vals[b][k] (thread per entry; other slots stay zero).
template <typename MT>
__global__ void k_dia_gather(const int32_t* __restrict__ pos, int64_t nnz, const MT* __restrict__ vals, int64_t vstride,
                             int32_t mb, MT* __restrict__ dst, int64_t dstride) {
    const int64_t items = nnz * mb;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = it / nnz, k = it - b * nnz;
        dst[b * dstride + pos[k]] = vals[b * vstride + k];
    }
}

// ---------------------------------------------------------------------------
// Grid path kernels
// ---------------------------------------------------------------------------


// init A: x = guess or 0, r = b - A x, |b|^2, |r|^2 -> status
template <typename VT, typename MT, int FMT>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_grid_init(SolveArgs<VT, MT> a) {
    __shared__ VT red[2 * (kTile / 32)];
    __shared__ bool last_s;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const VT* bv = a.b + (a.b_b == 1 ? 0 : vo);
        VT* x = a.x + vo;
        VT* r = a.r + vo;
        VT acc[2] = {VT(0), VT(0)};
        const auto A = inst_matrix<MT, FMT>(a.m, b_);
        const VT* gv = a.guess ? a.guess + (a.g_b == 1 ? 0 : vo) : nullptr;
        if (gv) {
            cta_rows4_seg<VT>(A, g.s, g.sr0, g.r0 - g.sr0, g.r1 - g.r0, GlobalX<VT>{gv}, [&](int row, VT v) {
                const VT bi = bv[row];
                const VT ri = bi - v;
                r[row] = ri;
                x[row] = gv[row];
                acc[0] += bi * bi;
                acc[1] += ri * ri;
            });
        } else {
#pragma unroll 4
            for (int i = g.r0 + threadIdx.x; i < g.r1; i += kTile) {
                const VT bi = bv[i];
                r[i] = bi;
                x[i] = VT(0);
                acc[0] += bi * bi;
                acc[1] += bi * bi;
            }
        }
        block_sum<VT, 2>(acc, red);
        VT tot[2];
        VT* const parts[2] = {a.part1, a.part2};
        if (tile_ticket<VT, 2>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk1, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            const VT bb = tot[0], rr = tot[1], tol = static_cast<VT>(a.tol);
            a.st.bb[g.inst] = bb;
            a.st.rr[g.inst] = rr;
            a.st.it[g.inst] = 0;
            a.st.outer[g.inst] = 0;
            int32_t status = ST_RUNNING;
            if ((a.abs_zero_test && bb < tol * tol) || bb == VT(0)) status = CMCG_SOLVE_ZERO_RHS;
            else if (!finite_(bb) || !finite_(rr)) status = CMCG_SOLVE_NON_FINITE;
            else if (rr < tol * tol * bb) status = CMCG_SOLVE_CONVERGED;
            a.st.status[g.inst] = status;
            if (status == ST_RUNNING) atomicAdd(a.active, 1);
        }
    }
}

// init B: zero x of zero-rhs systems; r.z, beta = 0 and p_{-1} = 0 (or, when
// the product reads p as stored, p_0 = M^-1 r) of running systems
template <typename VT, typename MT, int FMT>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_grid_init2(SolveArgs<VT, MT> a) {
    __shared__ VT red[2 * (kTile / 32)];
    __shared__ bool last_s;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        const int32_t st = ld_status(a.st.status + g.inst);
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        if (st == CMCG_SOLVE_ZERO_RHS) {
#pragma unroll 4
            for (int i = g.r0 + threadIdx.x; i < g.r1; i += kTile) a.x[vo + i] = VT(0);
            continue;
        }
        if (st != ST_RUNNING) continue;
        const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
        VT acc[1] = {VT(0)};
#pragma unroll 4
        for (int i = g.r0 + threadIdx.x; i < g.r1; i += kTile) {
            const VT ri = a.r[vo + i];
            const VT zi = dinv ? dinv[i] * ri : ri;
            if (a.p2 != a.p) a.p2[vo + i] = VT(0);   // p_{-1}: iteration 0's product forms p_0 = z
            else a.p[vo + i] = zi;                    // p_0 (the product reads p as stored)
            acc[0] += ri * zi;
        }
        block_sum<VT, 1>(acc, red);
        VT tot[1];
        VT* const parts[1] = {a.part1};
        if (tile_ticket<VT, 1>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk2, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            const VT rz = tot[0];
            a.st.rz[g.inst] = rz;
            a.st.beta[g.inst] = 0.0;
            int32_t status = ST_RUNNING;
            if (!finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
            else if (!(rz > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
            if (status != ST_RUNNING) {
                a.st.status[g.inst] = status;
                atomicSub(a.active, 1);
            }
        }
    }
}

// p_k of iteration k (the loop's count of finished iterations) lives in p for
// even k and in p2 for odd k
template <typename VT, typename MT>
__device__ __forceinline__ VT* grid_pk(const SolveArgs<VT, MT>& a, int k) { return (k & 1) ? a.p2 : a.p; }

// iteration kernel 1: p_k = M^-1 r + beta p_{k-1} (formed inside the product),
// q = A p_k, p_k.q -> alpha (ND > 0: the values in the pattern's diagonal
// layout, ND diagonals per system)
template <typename VT, typename MT, int FMT, int ND, bool FUSED>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_grid_spmv_pq(SolveArgs<VT, MT> a) {
    __shared__ VT red[kTile / 32];
    __shared__ bool last_s;
    const int k = __ldcg(a.loops);
    VT* const pk = grid_pk(a, k);
    const VT* const pprev = grid_pk(a, k + 1);
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        if (ld_status(a.st.status + g.inst) != ST_RUNNING) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        using PS = std::conditional_t<FUSED, PNext<VT>, PDirect<VT>>;
        PS pn;
        if constexpr (FUSED)
            pn = PS{a.r + vo, a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr, pprev + vo,
                    static_cast<VT>(a.st.beta[g.inst])};
        else
            pn = PS{pk + vo};
        VT* pout = pk + vo;
        VT* q = a.q + vo;
        VT acc[1] = {VT(0)};
        // q is read once, by the update kernel
        const auto emit3 = [&](int row, VT qv, VT prow) {
            if constexpr (FUSED) pout[row] = prow;
            __stcs(q + row, qv);
            acc[0] += prow * qv;
        };
        if constexpr (ND > 0) {
            int off[ND];
            const MT* v = dia_system<MT, ND>(a.dia, b_, g.s, off);
            dia_rows_seg<VT, MT, ND, false>(v, off, g.sr0, g.send, g.r0, g.r1, pn, emit3);
        } else {
            const auto A = inst_matrix<MT, FMT>(a.m, b_);
            cta_rows4_seg<VT>(A, g.s, g.sr0, g.r0 - g.sr0, g.r1 - g.r0, pn,
                              [&](int row, VT qv) { emit3(row, qv, pn(row)); });
        }
        block_sum<VT, 1>(acc, red);
        VT tot[1];
        VT* const parts[1] = {a.part1};
        if (tile_ticket<VT, 1>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk1, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            const VT pq = tot[0];
            const VT alpha = static_cast<VT>(a.st.rz[g.inst]) / pq;
            int32_t status = ST_RUNNING;
            if (!finite_(pq) || !finite_(alpha)) status = CMCG_SOLVE_NON_FINITE;
            else if (!(pq > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
            if (status != ST_RUNNING) {
                a.st.status[g.inst] = status;
                atomicSub(a.active, 1);
            } else {
                a.st.alpha[g.inst] = alpha;
            }
        }
    }
}

// iteration kernel 2: x += alpha p_k, r -= alpha q, |r|^2, r.z -> convergence, beta
template <typename VT, typename MT, int FMT>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_grid_update(SolveArgs<VT, MT> a) {
    __shared__ VT red[2 * (kTile / 32)];
    __shared__ bool last_s;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        if (ld_status(a.st.status + g.inst) != ST_RUNNING) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const VT alpha = static_cast<VT>(a.st.alpha[g.inst]);
        const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
        VT acc[2] = {VT(0), VT(0)};
        VT* x = a.x + vo;
        const VT* p = grid_pk(a, __ldcg(a.loops)) + vo;
        VT* r = a.r + vo;
        const VT* q = a.q + vo;
        const void* const ptrs[5] = {x + g.r0, p + g.r0, r + g.r0, q + g.r0, dinv ? dinv + g.r0 : nullptr};
        seg_rows_vec<5>(
            g.r0, g.r1, ptrs,
            [&](int i) {
                V4<VT> X, P, R, Q, D;
                X.load(x + i);
                P.load(p + i);
                R.load(r + i);
                Q.load(q + i);
                if (dinv) D.load(dinv + i);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    X.v[k] += alpha * P.v[k];
                    const VT ri = R.v[k] - alpha * Q.v[k];
                    R.v[k] = ri;
                    const VT zi = dinv ? D.v[k] * ri : ri;
                    acc[0] += ri * ri;
                    acc[1] += ri * zi;
                }
                X.store(x + i);
                R.store(r + i);
            },
            [&](int i) {
                x[i] += alpha * p[i];
                const VT ri = r[i] - alpha * q[i];
                r[i] = ri;
                const VT zi = dinv ? dinv[i] * ri : ri;
                acc[0] += ri * ri;
                acc[1] += ri * zi;
            });
        block_sum<VT, 2>(acc, red);
        VT tot[2];
        VT* const parts[2] = {a.part1, a.part2};
        if (tile_ticket<VT, 2>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk2, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            const VT rr = tot[0], rzn = tot[1];
            const VT tol = static_cast<VT>(a.tol);
            const VT bb = static_cast<VT>(a.st.bb[g.inst]);
            a.st.rr[g.inst] = rr;
            int32_t status = ST_RUNNING;
            const int n = g.send - g.sr0;
            if (!finite_(rr) || !finite_(rzn)) status = CMCG_SOLVE_NON_FINITE;
            else if (rr < tol * tol * bb) status = CMCG_SOLVE_CONVERGED;
            else if (!(rzn > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
            else {
                const VT rz = static_cast<VT>(a.st.rz[g.inst]);
                a.st.beta[g.inst] = rzn / rz;
                a.st.rz[g.inst] = rzn;
                const int32_t it = a.st.it[g.inst] + 1;
                a.st.it[g.inst] = it;
                if (it >= sys_max_iter(a.max_iter, n)) status = CMCG_SOLVE_MAX_ITER;
            }
            if (status != ST_RUNNING) {
                a.st.status[g.inst] = status;
                atomicSub(a.active, 1);
            }
        }
    }
}

// iteration kernel 3 where the product does not form p (p2 == p): p = M^-1 r + beta p
template <typename VT, typename MT, int FMT>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_grid_pupdate(SolveArgs<VT, MT> a) {
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        if (ld_status(a.st.status + g.inst) != ST_RUNNING) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const VT beta = static_cast<VT>(a.st.beta[g.inst]);
        const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
        const VT* r = a.r + vo;
        VT* p = a.p + vo;
        const void* const ptrs[3] = {r + g.r0, p + g.r0, dinv ? dinv + g.r0 : nullptr};
        seg_rows_vec<3>(
            g.r0, g.r1, ptrs,
            [&](int i) {
                V4<VT> R, P, D;
                R.load(r + i);
                P.load(p + i);
                if (dinv) D.load(dinv + i);
#pragma unroll
                for (int k = 0; k < 4; ++k) P.v[k] = fma(beta, P.v[k], dinv ? D.v[k] * R.v[k] : R.v[k]);
                P.store(p + i);
            },
            [&](int i) {
                const VT ri = r[i];
                const VT zi = dinv ? dinv[i] * ri : ri;
                p[i] = fma(beta, p[i], zi);
            });
    }
}

// ---------------------------------------------------------------------------
// Grid path, mixed precision with reliable updates (large systems)
//
// The same method as k_mixed_fast, spread over the whole GPU: FP32 CG on the
// Jacobi-scaled system S A S (scaled copy of the values in the sliced
// layout), FP32 increments xh folded into the FP64 solution x with x += S xh,
// and the recursive residual replaced by S (b - A x) computed in FP64 with the
// unscaled outer values whenever it dropped by delta (or looks converged).
// Per iteration the CUDA graph runs: p update + product + p.q, update + |r|^2
// (decides whether to replace), fold, FP64 residual (both no-ops unless a
// replacement is due), loop condition.
// ---------------------------------------------------------------------------

template <typename MI, typename MO>
struct GMixArgs {
    SolveArgs<float, MI> g;   // plan, segments, inner vectors r/p/q (FP32), state; g.m = scaled inner values
    MatArgs<MO> mo;           // outer values (unscaled) in the sliced layout
    const double* s;          // [mb][rows]
    const double* b64;
    double* x64;
    float* xh;
    double* p1;               // FP64 partials of the residual replacement
    double* p2;
    double outer_tol;
    int32_t max_updates;
    float delta;
};

template <typename MI, typename MO>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_gmix_init(GMixArgs<MI, MO> m) {
    const SolveArgs<float, MI>& a = m.g;
    __shared__ double red[2 * (kTile / 32)];
    __shared__ bool last_s;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const double* bv = m.b64 + (a.b_b == 1 ? 0 : vo);
        const double* sv = m.s + (a.m.mb == 1 ? 0 : vo);
        double acc[2] = {0.0, 0.0};
#pragma unroll 4
        for (int i = g.r0 + threadIdx.x; i < g.r1; i += kTile) {
            const double bi = bv[i];
            const float rh = static_cast<float>(sv[i] * bi);
            m.x64[vo + i] = 0.0;
            m.xh[vo + i] = 0.0f;
            a.r[vo + i] = rh;
            if (a.p2 != a.p) a.p2[vo + i] = 0.0f;   // p_{-1}: iteration 0's product forms p_0 = r
            else a.p[vo + i] = rh;                   // p_0 (the product reads p as stored)
            acc[0] += bi * bi;
            acc[1] += static_cast<double>(rh) * static_cast<double>(rh);
        }
        block_sum<double, 2>(acc, red);
        double tot[2];
        double* const parts[2] = {m.p1, m.p2};
        if (tile_ticket<double, 2>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk1, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            const double bb = tot[0];
            const float rz = static_cast<float>(tot[1]);
            const double thr = m.outer_tol * m.outer_tol * bb;
            a.st.bb[g.inst] = bb;
            a.st.rr[g.inst] = bb;
            a.st.rz[g.inst] = rz;
            a.st.beta[g.inst] = 0.0;
            a.st.rmax[g.inst] = rz;
            a.st.goal[g.inst] = static_cast<double>(static_cast<float>(thr / bb) * rz);
            a.st.it[g.inst] = 0;
            a.st.outer[g.inst] = 0;
            a.st.flag[g.inst] = 0;
            a.st.rep_it[g.inst] = 0;
            a.st.cyc0[g.inst] = 0;
            a.st.stall[g.inst] = 0;
            int32_t status = ST_RUNNING;
            if (bb == 0.0) status = CMCG_SOLVE_ZERO_RHS;
            else if (!finite_(bb) || !finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
            else if (bb < thr) status = CMCG_SOLVE_CONVERGED;
            else if (!(rz > 0.0f)) status = CMCG_SOLVE_BREAKDOWN;
            a.st.status[g.inst] = status;
            if (status == ST_RUNNING) atomicAdd(a.active, 1);
        }
    }
}

// Instances that stopped without a final replacement (breakdown, non-finite
// values, loop cap) still hold FP32 increments: the closing fold + FP64
// residual runs for them.
__device__ __forceinline__ bool gmix_tail_status(int32_t st) {
    return st == ST_RUNNING || st == CMCG_SOLVE_BREAKDOWN || st == CMCG_SOLVE_NON_FINITE;
}

// p_k = r + beta p_{k-1} (formed inside the product), q = (S A S) p_k and
// p_k.q -> alpha (ND > 0: the scaled values in the
// pattern's diagonal layout, the unit middle diagonal not loaded where the
// system's flag says so)
template <typename MI, typename MO, int ND, bool FUSED>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_gmix_spmv(GMixArgs<MI, MO> m) {
    const SolveArgs<float, MI>& a = m.g;
    __shared__ float red[kTile / 32];
    __shared__ bool last_s;
    const int k = __ldcg(a.loops);
    float* const pk = grid_pk(a, k);
    const float* const pprev = grid_pk(a, k + 1);
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        if (ld_status(a.st.status + g.inst) != ST_RUNNING) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        // the scaled system needs no preconditioner: p_k = r + beta p_{k-1}
        using PS = std::conditional_t<FUSED, PNext<float>, PDirect<float>>;
        PS pn;
        if constexpr (FUSED) pn = PS{a.r + vo, nullptr, pprev + vo, static_cast<float>(a.st.beta[g.inst])};
        else pn = PS{pk + vo};
        float* pout = pk + vo;
        float* q = a.q + vo;
        float acc[1] = {0.0f};
        // q is read once, by the update kernel
        const auto emit3 = [&](int row, float qv, float prow) {
            if constexpr (FUSED) pout[row] = prow;
            __stcs(q + row, qv);
            acc[0] += prow * qv;
        };
        if constexpr (ND > 0) {
            int off[ND];
            const MI* v = dia_system<MI, ND>(a.dia, b_, g.s, off);
            const bool unit = a.dia.unit && __ldg(a.dia.unit + (a.dia.mb == 1 ? 0 : b_ * a.n_sys) + g.s);
            if (unit) dia_rows_seg<float, MI, ND, true>(v, off, g.sr0, g.send, g.r0, g.r1, pn, emit3);
            else dia_rows_seg<float, MI, ND, false>(v, off, g.sr0, g.send, g.r0, g.r1, pn, emit3);
        } else {
            const auto A = inst_matrix<MI, CMCG_CSR>(a.m, b_);
            cta_rows4_seg<float>(A, g.s, g.sr0, g.r0 - g.sr0, g.r1 - g.r0, pn,
                                 [&](int row, float qv) { emit3(row, qv, pn(row)); });
        }
        block_sum<float, 1>(acc, red);
        float tot[1];
        float* const parts[1] = {a.part1};
        if (tile_ticket<float, 1>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk1, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            const float pq = tot[0];
            const float alpha = static_cast<float>(a.st.rz[g.inst]) / pq;
            int32_t status = ST_RUNNING;
            if (!finite_(pq) || !finite_(alpha)) status = CMCG_SOLVE_NON_FINITE;
            else if (!(pq > 0.0f)) status = CMCG_SOLVE_BREAKDOWN;
            if (status != ST_RUNNING) {
                a.st.status[g.inst] = status;
                atomicSub(a.active, 1);
            } else {
                a.st.alpha[g.inst] = alpha;
            }
        }
    }
}

// Condition probe of BF16 inner values (grid path). CG's residual contracts
// at least as fast as its bound for the scaled system's condition number
// kappa, so the rate rho observed over the first kCondProbe iterations gives
// a lower estimate kappa >= ((1 + rho) / (1 - rho))^2. Refinement through an
// inner system rounded to BF16 (unit roundoff 2^-8) needs kappa * 2^-8 well
// below 1; above kBf16CondLimit the instance stops with BREAKDOWN, and the
// FP32 fallback solves it, instead of the progress guard's thousands of
// iterations later. ratio = |r_k|^2 / |r_0|^2 of the first cycle.
constexpr int32_t kCondProbe = 64;
constexpr float kBf16CondLimit = 256.0f;
// The same decision at every replacement: the inner recursion claimed |r|^2
// down by delta^2 since the last one, the true FP64 residual is down by about
// (delta + u kappa)^2; a true ratio above kBf16Lag delta^2 means the BF16
// rounding term dominates, and the cycles to come will crawl.
constexpr double kBf16Lag = 10.0;
__device__ __forceinline__ bool bf16_condition_ok(float ratio, int32_t k) {
    if (!(ratio < 1.0f)) return false;   // no contraction at all (or NaN)
    const float rho = powf(ratio, 0.5f / static_cast<float>(k));
    const float s = (1.0f + rho) / (1.0f - rho);
    return s * s <= kBf16CondLimit;
}

// xh += alpha p_k, r -= alpha q, |r|^2 -> replacement decision or beta
template <typename MI, typename MO>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_gmix_update(GMixArgs<MI, MO> m) {
    const SolveArgs<float, MI>& a = m.g;
    __shared__ float red[kTile / 32];
    __shared__ bool last_s;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        if (ld_status(a.st.status + g.inst) != ST_RUNNING) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const float alpha = static_cast<float>(a.st.alpha[g.inst]);
        float acc[1] = {0.0f};
        float* xh = m.xh + vo;
        const float* p = grid_pk(a, __ldcg(a.loops)) + vo;
        float* r = a.r + vo;
        const float* q = a.q + vo;
        const void* const ptrs[4] = {xh + g.r0, p + g.r0, r + g.r0, q + g.r0};
        seg_rows_vec<4>(
            g.r0, g.r1, ptrs,
            [&](int i) {
                V4<float> X, P, R, Q;
                X.load(xh + i);
                P.load(p + i);
                R.load(r + i);
                Q.load(q + i);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    X.v[k] += alpha * P.v[k];
                    R.v[k] -= alpha * Q.v[k];
                    acc[0] += R.v[k] * R.v[k];
                }
                X.store(xh + i);
                R.store(r + i);
            },
            [&](int i) {
                xh[i] += alpha * p[i];
                const float ri = r[i] - alpha * q[i];
                r[i] = ri;
                acc[0] += ri * ri;
            });
        block_sum<float, 1>(acc, red);
        float tot[1];
        float* const parts[1] = {a.part2};
        if (tile_ticket<float, 1>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk2, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            const float rzn = tot[0];
            const int32_t it = a.st.it[g.inst] + 1;
            a.st.it[g.inst] = it;
            const float d2 = m.delta * m.delta;
            const int n = g.send - g.sr0;
            if (!finite_(rzn)) {
                a.st.status[g.inst] = CMCG_SOLVE_NON_FINITE;
                atomicSub(a.active, 1);
            } else if (std::is_same<MI, __nv_bfloat16>::value && it == kCondProbe && a.st.outer[g.inst] == 0 &&
                       !bf16_condition_ok(rzn / static_cast<float>(a.st.rmax[g.inst]), it)) {
                a.st.status[g.inst] = CMCG_SOLVE_BREAKDOWN;
                atomicSub(a.active, 1);
            } else if (rzn < d2 * static_cast<float>(a.st.rmax[g.inst]) || rzn < static_cast<float>(a.st.goal[g.inst]) ||
                       it >= sys_max_iter(a.max_iter, n) ||
                       it - a.st.rep_it[g.inst] >= stall_len(a.st.outer[g.inst], a.st.cyc0[g.inst], m.delta)) {
                a.st.flag[g.inst] = 1;   // fold and replace in this iteration
            } else if (!(rzn > 0.0f)) {
                a.st.status[g.inst] = CMCG_SOLVE_BREAKDOWN;
                atomicSub(a.active, 1);
            } else {
                a.st.beta[g.inst] = rzn / static_cast<float>(a.st.rz[g.inst]);
                a.st.rz[g.inst] = rzn;
            }
        }
    }
}

// x += S xh where a replacement is due (TAIL: where the solve stopped unfolded)
template <typename MI, typename MO, bool TAIL>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_gmix_fold(GMixArgs<MI, MO> m) {
    const SolveArgs<float, MI>& a = m.g;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        const int32_t st = ld_status(a.st.status + g.inst);
        if (TAIL ? !gmix_tail_status(st) : (st != ST_RUNNING || !ld_status(a.st.flag + g.inst))) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const double* sv = m.s + (a.m.mb == 1 ? 0 : vo);
#pragma unroll 4
        for (int i = g.r0 + threadIdx.x; i < g.r1; i += kTile) {
            m.x64[vo + i] += sv[i] * static_cast<double>(m.xh[vo + i]);
            m.xh[vo + i] = 0.0f;
        }
    }
}

// r = S (b - A x) in FP64 where a replacement is due -> convergence, beta
// (TAIL: only the final |b - A x|^2 of the instances folded by the tail)
template <typename MI, typename MO, bool TAIL>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_gmix_residual(GMixArgs<MI, MO> m) {
    const SolveArgs<float, MI>& a = m.g;
    __shared__ double red[2 * (kTile / 32)];
    __shared__ bool last_s;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        const int32_t st = ld_status(a.st.status + g.inst);
        if (TAIL ? !gmix_tail_status(st) : (st != ST_RUNNING || !ld_status(a.st.flag + g.inst))) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const double* bv = m.b64 + (a.b_b == 1 ? 0 : vo);
        const double* sv = m.s + (a.m.mb == 1 ? 0 : vo);
        const double* xv = m.x64 + vo;
        const auto Ao = inst_matrix<MO, CMCG_CSR>(m.mo, b_);
        double acc[2] = {0.0, 0.0};
        cta_rows4_seg<double>(Ao, g.s, g.sr0, g.r0 - g.sr0, g.r1 - g.r0, GlobalX<double>{xv}, [&](int row, double v) {
            const double r64 = bv[row] - v;
            const float rh = static_cast<float>(sv[row] * r64);
            if (!TAIL) a.r[vo + row] = rh;
            acc[0] += r64 * r64;
            acc[1] += static_cast<double>(rh) * static_cast<double>(rh);
        });
        block_sum<double, 2>(acc, red);
        double tot[2];
        double* const parts[2] = {m.p1, m.p2};
        if (tile_ticket<double, 2>(acc, parts, g.pbase, 0, g.count, g.pidx, a.st.tk1, g.inst, tot, red, &last_s) &&
            threadIdx.x == 0) {
            if (TAIL) {
                a.st.rr[g.inst] = tot[0];
                continue;
            }
            const double rr64 = tot[0], bb = a.st.bb[g.inst];
            const float rzn = static_cast<float>(tot[1]);
            const double thr = m.outer_tol * m.outer_tol * bb;
            const int32_t outer = a.st.outer[g.inst] + 1;
            a.st.outer[g.inst] = outer;
            // progress guard: the true residual against the last replacement's
            const double rr_prev = a.st.rr[g.inst];
            const int32_t stall = rr64 > kStallRatio * rr_prev ? a.st.stall[g.inst] + 1 : 0;
            a.st.stall[g.inst] = stall;
            if (outer == 1) a.st.cyc0[g.inst] = a.st.it[g.inst];
            a.st.rep_it[g.inst] = a.st.it[g.inst];
            a.st.rr[g.inst] = rr64;
            a.st.rmax[g.inst] = rzn;
            a.st.goal[g.inst] = static_cast<double>(static_cast<float>(thr / rr64) * rzn);
            a.st.flag[g.inst] = 0;
            const int n = g.send - g.sr0;
            int32_t status = ST_RUNNING;
            const double d2 = static_cast<double>(m.delta) * m.delta;
            if (!finite_(rr64)) status = CMCG_SOLVE_NON_FINITE;
            else if (rr64 < thr) status = CMCG_SOLVE_CONVERGED;
            else if (std::is_same<MI, __nv_bfloat16>::value && rr64 > kBf16Lag * d2 * rr_prev)
                status = CMCG_SOLVE_BREAKDOWN;   // BF16 values too coarse for this system
            else if (a.st.it[g.inst] >= sys_max_iter(a.max_iter, n) || outer >= m.max_updates) status = CMCG_SOLVE_MAX_ITER;
            else if (!(rzn > 0.0f) || stall >= kStallMax) status = CMCG_SOLVE_BREAKDOWN;
            if (status != ST_RUNNING) {
                a.st.status[g.inst] = status;
                atomicSub(a.active, 1);
            } else {
                a.st.beta[g.inst] = rzn / static_cast<float>(a.st.rz[g.inst]);
                a.st.rz[g.inst] = rzn;
            }
        }
    }
}


// p = r + beta p, where the product does not form p (p2 == p)
template <typename MI, typename MO>
__global__ void __launch_bounds__(kTile, kGridCtasPerSm) k_gmix_pupdate(GMixArgs<MI, MO> m) {
    const SolveArgs<float, MI>& a = m.g;
    CMCG_FOR_SEGMENTS(a) {
        const SegInfo g = seg_info(a, b_, seg_);
        if (ld_status(a.st.status + g.inst) != ST_RUNNING) continue;
        const int64_t vo = static_cast<int64_t>(b_) * a.rows;
        const float beta = static_cast<float>(a.st.beta[g.inst]);
        const float* r = a.r + vo;
        float* p = a.p + vo;
        const void* const ptrs[2] = {r + g.r0, p + g.r0};
        seg_rows_vec<2>(
            g.r0, g.r1, ptrs,
            [&](int i) {
                V4<float> R, P;
                R.load(r + i);
                P.load(p + i);
#pragma unroll
                for (int k = 0; k < 4; ++k) P.v[k] = fmaf(beta, P.v[k], R.v[k]);
                P.store(p + i);
            },
            [&](int i) { p[i] = fmaf(beta, p[i], r[i]); });
    }
}
// the host-driven loop's count of finished iterations (the graph's condition
// kernel keeps it there; the products read its parity)
__global__ void k_loop_step(int32_t* loops) { ++*loops; }

// loop condition of the graph's WHILE node (one thread); counts the finished
// iterations
__global__ void k_grid_cond(const int32_t* active, int32_t* loops, int32_t cap, cudaGraphConditionalHandle h) {
    const int32_t l = ++(*loops);
    const unsigned go = (*reinterpret_cast<const volatile int32_t*>(active) > 0 && l < cap) ? 1u : 0u;
    cudaGraphSetConditional(h, go);
}

__global__ void k_finalize(InstState st, int32_t n_inst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_inst) return;
    int32_t s = st.status[i];
    if (s == ST_RUNNING) { s = CMCG_SOLVE_MAX_ITER; st.status[i] = s; }
    st.err[i] = (s == CMCG_SOLVE_ZERO_RHS) ? 0.0 : sqrt(st.rr[i] / st.bb[i]);
}

// The grid path's iteration loop without a graph: `body` launches one
// iteration's kernels on `st`; the count of running instances is read back
// every kHostLoopPoll iterations and the loop ends at 0 or after cap - 1
// iterations, as the graph's WHILE node does (k_grid_cond). Iterations run
// after the last instance finished change nothing: the kernels skip finished
// instances.
constexpr int32_t kHostLoopPoll = 16;
template <typename F>
cmcg_status host_loop(cudaStream_t st, const int32_t* active, int32_t cap, int per_iter, F&& body) {
    for (int32_t l = 1;; ++l) {
        body();
        count_launch(per_iter);
        CMCG_CHECK_LAUNCH();
        if (l >= cap) break;
        if (l % kHostLoopPoll == 0) {
            int32_t running = 0;
            CMCG_CUDA(cudaMemcpyAsync(&running, active, sizeof(running), cudaMemcpyDeviceToHost, st));
            CMCG_CUDA(cudaStreamSynchronize(st));
            if (running <= 0) break;
        }
    }
    return CMCG_OK;
}

// ---------------------------------------------------------------------------
// Jacobi: inverse diagonal per batch of values, 1 where a_ii is 0 or absent
// (reference DiagonalPreconditioner + cwiseInverseCheck, ConjugateGradient.h:228-230,
// UnaryOps.h:177; diagonal lookup as coeff(i, i), SparseMatrixBase.h:258-271)
// ---------------------------------------------------------------------------
template <typename VT, typename MT, int FMT>
__global__ void k_inv_diag(MatArgs<MT> m, int32_t rows, VT* __restrict__ out) {
    const int64_t items = static_cast<int64_t>(rows) * m.mb;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(it / rows);
        const int r = static_cast<int>(it - static_cast<int64_t>(b) * rows);
        const MT* v = m.vals + static_cast<int64_t>(b) * m.vstride;
        VT d = VT(0);
        if (FMT == CMCG_CSR) {
            for (int k = m.rp[r]; k < m.rp[r + 1]; ++k)
                if (m.ci[k] == r) { d = mval<VT>(v[k]); break; }
        } else {
            for (int j = 0; j < m.width; ++j) {
                const int64_t o = r + static_cast<int64_t>(j) * m.rows_pad;
                if (m.ell[o] == r) { d = mval<VT>(v[o]); break; }
            }
        }
        out[it] = (d != VT(0)) ? VT(1) / d : VT(1);
    }
}

// Kernel view of a matrix; for CSR the sliced ELLPACK copy must be current
// (ensure_sell_values) before the arguments are taken.
template <typename MT>
MatArgs<MT> mat_args(cmcg_matrix A) {
    cmcg_pattern p = A->pat;
    const SellPlan& S = p->sell;
    return MatArgs<MT>{p->d_row_ptr, p->d_col, p->d_ell, p->width, p->rows_pad, static_cast<const MT*>(A->d_vals),
                       A->stride, A->batches, S.d_col, static_cast<const MT*>(A->d_sell_vals), A->sell_stride,
                       S.d_slice_off, S.d_slice_w, S.d_sys_slice0};
}

}  // namespace

// ---------------------------------------------------------------------------
// Solver object
// ---------------------------------------------------------------------------

struct cmcg_solver_s {
    cmcg_matrix A = nullptr;
    int32_t precond = CMCG_PRECOND_JACOBI;
    double tol = 0.0;
    int64_t max_iter = -1;
    int32_t path = CMCG_PATH_AUTO;
    int32_t refine_method = CMCG_REFINE_RELIABLE;
    double refine_delta = 0.0;   // 0: by the inner value type (refine_delta_for)
    // mixed kernel: systems at order positions >= mix_split on 512-thread CTAs
    // (CUMAT_CG_SMALL=0 keeps every system on 1024-thread CTAs)
    int32_t mix_split = 0, mix_split2 = 0;   // and >= mix_split2 on 256-thread CTAs
    bool mix_small = true;
    cudaStream_t aux_stream[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    bool use_smem = true;     // shared-memory-resident kernels where the systems fit
    bool inner_solve = false; // set while the solver runs the inner solves of a refinement
    bool fast_kernels = true; // compact-layout kernels where available (CUMAT_CG_FAST=0 disables)
    // cooperative one-launch grid solve: 0 never, 1 where it applies (systems up
    // to kCoopMaxRows rows), 2 also for larger systems (CUMAT_CG_COOP)
    int coop = 1;
    // cluster solve of the grid path where it applies (CUMAT_CG_CLUSTER=0 disables)
    bool cluster = true;
    // grid path: the product forms p_k (-1: by the batch's vector bytes against
    // L2, see fuse_p_update; 0 / 1: CUMAT_CG_FUSE)
    int fuse_p = -1;
    // grid path iteration loop: true = one CUDA graph with a device-side WHILE
    // node; false = the same kernels launched from the host, polling the count
    // of running instances (CUMAT_CG_GRAPH=0; kernel profilers do not replay
    // kernels inside conditional graph nodes)
    bool graph_loop = true;
    int64_t systems_version = -1;  // pattern systems the plan was built for
    // plan
    int32_t n_sys = 0, max_sys_rows = 0, n_tiles = 0;
    int32_t* d_order = nullptr;
    int32_t* d_tile_row0 = nullptr;
    // grid path segment plan (see SegInfo)
    int32_t grid_ctas = 1, n_seg = 0;
    int32_t* d_seg_t0 = nullptr;
    int32_t* d_seg_t1 = nullptr;
    int32_t* d_seg_sys = nullptr;
    int32_t* d_cta_seg0 = nullptr;
    int32_t* d_sys_seg0 = nullptr;
    // the same for the cooperative launch (one CTA per SM)
    int32_t coop_ctas = 0, coop_n_seg = 0, coop_max_segs = 0;
    int32_t* d_cseg_t0 = nullptr;
    int32_t* d_cseg_t1 = nullptr;
    int32_t* d_cseg_sys = nullptr;
    int32_t* d_ccta_seg0 = nullptr;
    int32_t* d_csys_seg0 = nullptr;
    // Jacobi inverse diagonal per vector type (F32, F64), [matrix batches][rows]
    void* dinv[2] = {nullptr, nullptr};
    // workspace
    void* vec_ws = nullptr;   size_t vec_ws_bytes = 0;
    void* ref_ws = nullptr;   size_t ref_ws_bytes = 0;
    void* part_ws = nullptr;  size_t part_ws_bytes = 0;
    void* st_ws = nullptr;    size_t st_ws_bytes = 0;
    int32_t* counters = nullptr;  // next, active, loops
    void* host_io = nullptr;  size_t host_io_bytes = 0;
    // mixed solver, fast path: Jacobi-scaled copy of the inner values in the
    // sliced layout ([batch][mix_stride]) and the scale s = 1/sqrt(a_ii)
    // ([batch][rows], FP64); rebuilt when the values or the systems change
    void* mix_vals = nullptr;
    int64_t mix_stride = 0;
    double* mix_s = nullptr;
    int64_t mix_version = -1, mix_plan_id = -1;
    int32_t mix_dtype = -1;
    // the same scaled values in the pattern's diagonal layout, when it has one
    bool dia_kernels = true;  // CUMAT_CG_DIA=0 keeps the sliced layout
    void* dia_vals = nullptr;      // diagonal-layout values, then the unit-diagonal flags
    int32_t* dia_unit = nullptr;   // inside dia_vals
    // the matrix's own (unscaled) values in the diagonal layout, for the plain
    // grid-path product
    void* dia_plain = nullptr;
    int64_t dia_plain_stride = 0;
    int64_t dia_plain_version = -1, dia_plain_plan_id = -1;
    int32_t dia_plain_dtype = -1;
    int64_t dia_stride = 0;
    int64_t dia_version = -1, dia_plan_id = -1;
    int32_t dia_dtype = -1;
    InstState st{};
    int32_t st_inst = 0;
    // graph cache of the grid path
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    std::vector<char> gkey;
    // graph cache of the grid path's mixed solve (keyed by its kernel arguments)
    cudaGraphExec_t gexec_mix = nullptr;
    cudaGraph_t graph_mix = nullptr;
    std::vector<char> gkey_mix;
    // last solve
    int32_t last_inst = 0;
    bool last_refined = false;
    // BF16 inner values: systems the BF16 solve left unconverged are solved
    // again with FP32 values (CUMAT_CG_BF16_FALLBACK=0 disables); fb_* are the
    // FP32 matrix (when the outer one is FP64) and solver used for that
    bool bf16_fallback = true;
    cmcg_matrix fb_mat = nullptr;
    cmcg_solver fb = nullptr;
    double* fb_x = nullptr;
    size_t fb_x_bytes = 0;
    int32_t* fb_list = nullptr;
    size_t fb_list_bytes = 0;
    std::vector<int32_t> fallback;   // per instance of the last refined solve: 1 = re-solved with FP32 values
};

namespace {

cmcg_status build_plan(cmcg_solver s) {
    cmcg_pattern p = s->A->pat;
    const auto& ro = p->row_off;
    const int32_t n_sys = static_cast<int32_t>(ro.size() - 1);
    std::vector<int64_t> nnz(n_sys);
    int32_t maxr = 0;
    for (int32_t i = 0; i < n_sys; ++i) {
        const int64_t a = ro[i], e = ro[i + 1];
        maxr = std::max<int32_t>(maxr, static_cast<int32_t>(e - a));
        nnz[i] = (p->format == CMCG_CSR) ? (p->h_row_ptr[e] - p->h_row_ptr[a]) : (e - a) * p->width;
    }
    std::vector<int32_t> order(n_sys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return nnz[x] > nnz[y]; });
    std::vector<int32_t> t_row0, t_sys, t_begin(n_sys + 1);
    for (int32_t i = 0; i < n_sys; ++i) {
        t_begin[i] = static_cast<int32_t>(t_row0.size());
        for (int64_t r = ro[i]; r < ro[i + 1]; r += kTile) {
            t_row0.push_back(static_cast<int32_t>(r));
            t_sys.push_back(i);
        }
    }
    t_begin[n_sys] = static_cast<int32_t>(t_row0.size());
    s->n_sys = n_sys;
    s->max_sys_rows = maxr;
    // last position of the size order with a system above kMixSmallRows rows
    s->mix_split = s->mix_split2 = 0;
    for (int32_t i = 0; i < n_sys; ++i) {
        const int64_t r = ro[order[i] + 1] - ro[order[i]];
        if (r > kMixSmallRows) s->mix_split = i + 1;
        if (r > kMixTinyRows) s->mix_split2 = i + 1;
    }
    s->n_tiles = static_cast<int32_t>(t_row0.size());
    s->systems_version = p->systems_version;
    // grid path: contiguous tile ranges per CTA, cut into segments at system
    // boundaries (segment ids of one system are consecutive); one plan for the
    // graph kernels, one for the cooperative launch
    struct SegPlan {
        std::vector<int32_t> t0, t1, sys, cta0, sys0;
    };
    auto make_plan = [&](int32_t G) {
        SegPlan P;
        P.cta0.assign(G + 1, 0);
        P.sys0.assign(n_sys + 1, -1);
        for (int32_t c = 0; c < G; ++c) {
            P.cta0[c] = static_cast<int32_t>(P.t0.size());
            const int32_t a = static_cast<int32_t>(static_cast<int64_t>(c) * s->n_tiles / G);
            const int32_t e = static_cast<int32_t>(static_cast<int64_t>(c + 1) * s->n_tiles / G);
            for (int32_t t = a; t < e;) {
                const int32_t sys = t_sys[t];
                int32_t u = t;
                while (u < e && t_sys[u] == sys) ++u;
                if (P.sys0[sys] < 0) P.sys0[sys] = static_cast<int32_t>(P.t0.size());
                P.t0.push_back(t);
                P.t1.push_back(u);
                P.sys.push_back(sys);
                t = u;
            }
        }
        P.cta0[G] = static_cast<int32_t>(P.t0.size());
        P.sys0[n_sys] = static_cast<int32_t>(P.t0.size());
        for (int32_t i = n_sys - 1; i >= 0; --i)
            if (P.sys0[i] < 0) P.sys0[i] = P.sys0[i + 1];   // (every system has at least one tile)
        return P;
    };
    const int32_t G = std::max<int32_t>(1, std::min<int32_t>(s->n_tiles, p->ctx->sm_count * kGridCtasPerSm));
    const int32_t Gc = std::max<int32_t>(1, std::min<int32_t>(s->n_tiles, p->ctx->sm_count));
    const SegPlan pg = make_plan(G), pc = make_plan(Gc);
    s->grid_ctas = G;
    s->n_seg = static_cast<int32_t>(pg.t0.size());
    s->coop_ctas = Gc;
    s->coop_n_seg = static_cast<int32_t>(pc.t0.size());
    s->coop_max_segs = 0;
    for (int32_t c = 0; c < Gc; ++c) s->coop_max_segs = std::max(s->coop_max_segs, pc.cta0[c + 1] - pc.cta0[c]);
    cudaStream_t st = p->ctx->stream;
    int32_t** bufs[] = {&s->d_order, &s->d_tile_row0, &s->d_seg_t0, &s->d_seg_t1, &s->d_seg_sys, &s->d_cta_seg0,
                        &s->d_sys_seg0, &s->d_cseg_t0, &s->d_cseg_t1, &s->d_cseg_sys, &s->d_ccta_seg0, &s->d_csys_seg0};
    const std::vector<int32_t>* src[] = {&order, &t_row0, &pg.t0, &pg.t1, &pg.sys, &pg.cta0, &pg.sys0,
                                         &pc.t0, &pc.t1, &pc.sys, &pc.cta0, &pc.sys0};
    for (int k = 0; k < 12; ++k) {
        dev_free(*bufs[k]);
        *bufs[k] = nullptr;
        CMCG_TRY(dev_alloc(reinterpret_cast<void**>(bufs[k]), std::max<size_t>(src[k]->size(), 1) * 4));
        if (!src[k]->empty())
            CMCG_CUDA(cudaMemcpyAsync(*bufs[k], src[k]->data(), src[k]->size() * 4, cudaMemcpyHostToDevice, st));
    }
    CMCG_CUDA(cudaStreamSynchronize(st));
    return CMCG_OK;
}

// Rebuilds the work plan when the pattern's systems changed since it was made.
cmcg_status refresh_plan(cmcg_solver s) {
    if (s->systems_version == s->A->pat->systems_version) return CMCG_OK;
    CMCG_CUDA(cudaStreamSynchronize(s->A->pat->ctx->stream));
    CMCG_TRY(build_plan(s));
    s->st_inst = 0;   // per-instance state is re-sized on the next solve
    return CMCG_OK;
}

template <typename VT, typename MT>
cmcg_status compute_dinv_t(cmcg_solver s, VT* out) {
    cmcg_matrix A = s->A;
    cmcg_pattern p = A->pat;
    const MatArgs<MT> m = mat_args<MT>(A);
    const int64_t n = static_cast<int64_t>(p->rows) * A->batches;
    const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, p->ctx->sm_count * 8));
    if (p->format == CMCG_CSR) k_inv_diag<VT, MT, CMCG_CSR><<<blocks, 256, 0, p->ctx->stream>>>(m, p->rows, out);
    else k_inv_diag<VT, MT, CMCG_ELLPACK><<<blocks, 256, 0, p->ctx->stream>>>(m, p->rows, out);
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

// Returns the inverse diagonal for vector type vdt (computed on first use).
cmcg_status get_dinv(cmcg_solver s, int32_t vdt, const void** out) {
    *out = nullptr;
    if (s->precond != CMCG_PRECOND_JACOBI) return CMCG_OK;
    const int k = (vdt == CMCG_F64) ? 1 : 0;
    if (!s->dinv[k]) {
        const size_t es = (vdt == CMCG_F64) ? 8 : 4;
        CMCG_TRY(dev_alloc(&s->dinv[k], es * s->A->pat->rows * s->A->batches));
        cmcg_status st;
        if (vdt == CMCG_F64) {
            double* o = static_cast<double*>(s->dinv[k]);
            st = s->A->dtype == CMCG_F32 ? compute_dinv_t<double, float>(s, o)
               : s->A->dtype == CMCG_F64 ? compute_dinv_t<double, double>(s, o)
                                         : compute_dinv_t<double, __nv_bfloat16>(s, o);
        } else {
            float* o = static_cast<float*>(s->dinv[k]);
            st = s->A->dtype == CMCG_F32 ? compute_dinv_t<float, float>(s, o)
               : s->A->dtype == CMCG_F64 ? compute_dinv_t<float, double>(s, o)
                                         : compute_dinv_t<float, __nv_bfloat16>(s, o);
        }
        if (st != CMCG_OK) return st;
    }
    *out = s->dinv[k];
    return CMCG_OK;
}

cmcg_status ensure_state(cmcg_solver s, int32_t n_inst) {
    const size_t per = 8 * sizeof(double) + 7 * sizeof(int32_t) + 2 * sizeof(unsigned);
    const size_t need = per * static_cast<size_t>(n_inst) + 256;
    if (s->st_inst >= n_inst && s->st_ws) return CMCG_OK;
    dev_free(s->st_ws);
    s->st_ws = nullptr;
    s->st_ws_bytes = 0;
    CMCG_TRY(dev_alloc(&s->st_ws, need));
    s->st_ws_bytes = need;
    char* b = static_cast<char*>(s->st_ws);
    const size_t n = static_cast<size_t>(n_inst);
    s->st.bb = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.rr = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.rz = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.alpha = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.beta = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.err = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.rmax = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.goal = reinterpret_cast<double*>(b); b += 8 * n;
    s->st.flag = reinterpret_cast<int32_t*>(b); b += 4 * n;
    s->st.it = reinterpret_cast<int32_t*>(b); b += 4 * n;
    s->st.status = reinterpret_cast<int32_t*>(b); b += 4 * n;
    s->st.outer = reinterpret_cast<int32_t*>(b); b += 4 * n;
    s->st.rep_it = reinterpret_cast<int32_t*>(b); b += 4 * n;
    s->st.cyc0 = reinterpret_cast<int32_t*>(b); b += 4 * n;
    s->st.stall = reinterpret_cast<int32_t*>(b); b += 4 * n;
    s->st.tk1 = reinterpret_cast<unsigned*>(b); b += 4 * n;
    s->st.tk2 = reinterpret_cast<unsigned*>(b); b += 4 * n;
    CMCG_CUDA(cudaMemsetAsync(s->st_ws, 0, need, s->A->pat->ctx->stream));
    s->st_inst = n_inst;
    // the cached graph points at the old state
    if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
    if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
    s->gkey.clear();
    return CMCG_OK;
}

// smem_ok: a shared-memory-resident persistent kernel exists for the solve
// systems above this size are solved faster by a cluster of CTAs than by one
// CTA, when there are few of them
constexpr int32_t kClusterMinRows = 4096;

// cluster_ok: the solve has a cluster form (plain solves; refined solves do not)
int32_t choose_path(cmcg_solver s, int32_t n_inst, bool smem_ok, bool cluster_ok = false) {
    if (s->path != CMCG_PATH_AUTO) return s->path;
    const int sms = s->A->pat->ctx->sm_count;
    // many independent systems of moderate size: one CTA per system
    if (s->max_sys_rows <= 65536 && n_inst >= sms) return CMCG_PATH_PERSISTENT;
    // a few systems above kClusterMinRows rows: one thread-block cluster each
    // (the grid path's cluster solve, which falls back to the other grid loops
    // where it does not apply)
    if (cluster_ok && s->cluster && s->max_sys_rows > kClusterMinRows && n_inst <= sms / kClusterMaxCtas)
        return CMCG_PATH_GRID;
    // a few systems that fit in shared memory: one CTA each still beats the
    // grid path's per-iteration launches (2D Poisson 100^2, one system:
    // 9.5 us vs 18.7 us per iteration on the B200)
    if (smem_ok && s->max_sys_rows <= kSmemMaxRows) return CMCG_PATH_PERSISTENT;
    return CMCG_PATH_GRID;
}

template <typename VT, typename MT>
SolveArgs<VT, MT> base_args(cmcg_solver s, int32_t ob) {
    cmcg_pattern p = s->A->pat;
    SolveArgs<VT, MT> a{};
    a.m = mat_args<MT>(s->A);
    a.rows = p->rows;
    a.n_sys = s->n_sys;
    a.ob = ob;
    a.row_off = p->d_row_off;
    a.order = s->d_order;
    a.next = s->counters;
    a.active = s->counters + 1;
    a.loops = s->counters + 2;
    a.n_tiles = s->n_tiles;
    a.tile_row0 = s->d_tile_row0;
    a.n_seg = s->n_seg;
    a.seg_t0 = s->d_seg_t0;
    a.seg_t1 = s->d_seg_t1;
    a.seg_sys = s->d_seg_sys;
    a.cta_seg0 = s->d_cta_seg0;
    a.sys_seg0 = s->d_sys_seg0;
    a.tol = s->tol;
    a.max_iter = s->max_iter;
    a.abs_zero_test = s->inner_solve ? 0 : 1;
    a.st = s->st;
    return a;
}

// Sets the dynamic shared memory limit of a kernel once per process.
template <typename K>
cmcg_status allow_smem(K kern, size_t bytes) {
    CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    return CMCG_OK;
}

inline int smem_rows(int32_t max_rows) { return (max_rows + 3) / 4 * 4; }

// dynamic shared memory of a 512-thread (256-thread) mixed-kernel CTA such
// that two (four) fit on an SM next to their static arrays
constexpr size_t kMixSmallSmemLimit = 104 * 1024;
constexpr size_t kMixTinySmemLimit = 50 * 1024;

// Streams of the highest and the next priority, and fork / join events, for
// running the CTA tiers of the mixed kernel side by side (created on first use).
// The five handles are created into locals and kept only when every creation
// succeeded (a partial set is destroyed), so a failure leaves the solver
// without any and the next call tries again.
cmcg_status ensure_aux_stream(cmcg_solver s) {
    if (s->aux_stream[0] && s->aux_stream[1] && s->ev_fork && s->ev_join[0] && s->ev_join[1]) return CMCG_OK;
    int least = 0, greatest = 0;
    CMCG_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    cudaStream_t st[2] = {nullptr, nullptr};
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    cudaError_t e = cudaStreamCreateWithPriority(&st[0], cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithPriority(&st[1], cudaStreamNonBlocking, std::min(least, greatest + 1));
    for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        for (auto x : st)
            if (x) cudaStreamDestroy(x);
        for (auto x : ev)
            if (x) cudaEventDestroy(x);
        cudaGetLastError();
        return fail(CMCG_ERR_CUDA, std::string("creating the tier streams: ") + cudaGetErrorString(e));
    }
    s->aux_stream[0] = st[0];
    s->aux_stream[1] = st[1];
    s->ev_fork = ev[0];
    s->ev_join[0] = ev[1];
    s->ev_join[1] = ev[2];
    return CMCG_OK;
}

// Residual-replacement threshold of the reliable updates: the one set, else
// 0.01 for FP32 inner values (the FP32 recurrence stays within ~eps_f32 / 0.01
// of the true residual between replacements) and 0.1 for BF16 inner values
// (an operator perturbed by ~2^-9 needs the FP64 residual more often).
inline float refine_delta_for(cmcg_solver s) {
    if (s->refine_delta > 0.0) return static_cast<float>(s->refine_delta);
    return s->A->dtype == CMCG_BF16 ? 0.1f : 0.01f;
}

// dynamic shared memory the diagonal-layout kernel may use (the opt-in
// maximum per CTA minus the kernel's static arrays, with room to spare)
constexpr size_t kDiaSmemLimit = 216 * 1024;

// Compact sliced layout available for the fast shared-memory kernels?
inline bool compact_ok(cmcg_solver s) {
    const cmcg_pattern p = s->A->pat;
    return p->format == CMCG_CSR && p->sell.d_col16 != nullptr && s->max_sys_rows <= kSmemMaxRows && s->use_smem &&
           s->fast_kernels;
}

inline CompactArgs compact_args(cmcg_pattern p) {
    return CompactArgs{p->sell.d_col16, p->sell.d_slice_off32, p->sell.d_slice_w, p->sell.d_sys_slice0};
}

template <typename MT>
cmcg_status build_mix(cmcg_solver s) {
    cmcg_matrix A = s->A;
    cmcg_pattern p = A->pat;
    cmcg_ctx ctx = p->ctx;
    const SellPlan& S = p->sell;
    const int blocks = ctx->sm_count * 8;
    k_jacobi_scale<MT><<<blocks, 256, 0, ctx->stream>>>(p->d_row_ptr, p->d_col, static_cast<const MT*>(A->d_vals), A->stride,
                                                      p->rows, A->batches, s->precond == CMCG_PRECOND_JACOBI ? 1 : 0, s->mix_s);
    k_scale_sell<MT, MT><<<blocks, 256, 0, ctx->stream>>>(S.d_col, S.d_slice_off, S.d_slice_w, S.d_slice_row0, S.n_slices,
                                                         static_cast<const MT*>(A->d_sell_vals), A->sell_stride, s->mix_s,
                                                         p->rows, A->batches, static_cast<MT*>(s->mix_vals), s->mix_stride);
    count_launch(2);
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

// Jacobi-scaled inner values and the scale vector of the mixed solver's fast
// path, rebuilt when the matrix values or the systems changed.
cmcg_status ensure_mix(cmcg_solver s) {
    cmcg_matrix A = s->A;
    cmcg_pattern p = A->pat;
    CMCG_TRY(ensure_sell_values(A));
    const SellPlan& S = p->sell;
    if (s->mix_vals && s->mix_version == A->version && s->mix_plan_id == S.plan_id && s->mix_dtype == A->dtype)
        return CMCG_OK;
    dev_free(s->mix_vals);
    dev_free(s->mix_s);
    s->mix_vals = nullptr;
    s->mix_s = nullptr;
    s->mix_stride = A->sell_stride;
    CMCG_TRY(dev_alloc(&s->mix_vals, static_cast<size_t>(s->mix_stride) * A->batches * dtype_size(A->dtype)));
    CMCG_TRY(dev_alloc(reinterpret_cast<void**>(&s->mix_s), static_cast<size_t>(p->rows) * A->batches * sizeof(double)));
    cmcg_status st = A->dtype == CMCG_F32 ? build_mix<float>(s) : A->dtype == CMCG_BF16 ? build_mix<__nv_bfloat16>(s)
                                                                                        : build_mix<double>(s);
    if (st != CMCG_OK) return st;
    s->mix_version = A->version;
    s->mix_plan_id = S.plan_id;
    s->mix_dtype = A->dtype;
    return CMCG_OK;
}

// Scaled inner values in the pattern's diagonal layout (after ensure_mix);
// false when the pattern has no diagonal plan.
cmcg_status ensure_dia_vals(cmcg_solver s, bool* ok) {
    *ok = false;
    cmcg_matrix A = s->A;
    cmcg_pattern p = A->pat;
    CMCG_TRY(ensure_dia(p));
    const DiaPlan& D = p->dia;
    if (!D.ok) return CMCG_OK;
    if (!(s->dia_vals && s->dia_version == A->version && s->dia_plan_id == D.plan_id && s->dia_dtype == A->dtype)) {
        cmcg_ctx ctx = p->ctx;
        dev_free(s->dia_vals);
        s->dia_vals = nullptr;
        s->dia_stride = (D.n_slots + 7) / 8 * 8 + 8;
        // values, then the per-(batch, system) unit-diagonal flags
        const size_t vbytes = (static_cast<size_t>(s->dia_stride) * A->batches * dtype_size(A->dtype) + 255) / 256 * 256;
        const size_t bytes = vbytes + static_cast<size_t>(s->n_sys) * A->batches * sizeof(int32_t);
        CMCG_TRY(dev_alloc(&s->dia_vals, bytes));
        CMCG_CUDA(cudaMemsetAsync(s->dia_vals, 0, bytes, ctx->stream));
        s->dia_unit = reinterpret_cast<int32_t*>(static_cast<char*>(s->dia_vals) + vbytes);
        const int blocks = ctx->sm_count * 8;
#define CMCG_SCALE_DIA(MT)                                                                                              \
    k_scale_dia<MT><<<blocks, 256, 0, ctx->stream>>>(p->d_row_ptr, p->d_col, static_cast<const MT*>(A->d_vals), A->stride, \
                                                     D.d_pos, s->mix_s, p->rows, A->batches, static_cast<MT*>(s->dia_vals), \
                                                     s->dia_stride)
        if (A->dtype == CMCG_F32) CMCG_SCALE_DIA(float);
        else if (A->dtype == CMCG_BF16) CMCG_SCALE_DIA(__nv_bfloat16);
        else CMCG_SCALE_DIA(double);
#undef CMCG_SCALE_DIA
        count_launch();
        CMCG_CHECK_LAUNCH();
        const int ublocks = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(s->n_sys) * A->batches, 65535));
#define CMCG_DIA_UNIT(MT)                                                                                          \
    k_dia_unit<MT><<<ublocks, 256, 0, ctx->stream>>>(static_cast<const MT*>(s->dia_vals), s->dia_stride,          \
                                                     D.d_sys_base, D.d_sys_off, p->d_row_off, s->n_sys, A->batches, \
                                                     D.max_nd, s->dia_unit)
        if (A->dtype == CMCG_F32) CMCG_DIA_UNIT(float);
        else if (A->dtype == CMCG_BF16) CMCG_DIA_UNIT(__nv_bfloat16);
        else CMCG_DIA_UNIT(double);
#undef CMCG_DIA_UNIT
        count_launch();
        CMCG_CHECK_LAUNCH();
        s->dia_version = A->version;
        s->dia_plan_id = D.plan_id;
        s->dia_dtype = A->dtype;
    }
    *ok = true;
    return CMCG_OK;
}

// The matrix's values, unscaled, in the pattern's diagonal layout (rebuilt
// when the values or the systems change); false when the pattern has no
// diagonal plan or it is switched off.
cmcg_status ensure_dia_plain(cmcg_solver s, bool* ok) {
    *ok = false;
    cmcg_matrix A = s->A;
    cmcg_pattern p = A->pat;
    if (!s->dia_kernels || p->format != CMCG_CSR) return CMCG_OK;
    CMCG_TRY(ensure_dia(p));
    const DiaPlan& D = p->dia;
    if (!D.ok) return CMCG_OK;
    if (!(s->dia_plain && s->dia_plain_version == A->version && s->dia_plain_plan_id == D.plan_id &&
          s->dia_plain_dtype == A->dtype)) {
        cmcg_ctx ctx = p->ctx;
        dev_free(s->dia_plain);
        s->dia_plain = nullptr;
        s->dia_plain_stride = (D.n_slots + 7) / 8 * 8 + 8;
        const size_t bytes = static_cast<size_t>(s->dia_plain_stride) * A->batches * dtype_size(A->dtype);
        CMCG_TRY(dev_alloc(&s->dia_plain, bytes));
        CMCG_CUDA(cudaMemsetAsync(s->dia_plain, 0, bytes, ctx->stream));
        const int blocks = ctx->sm_count * 8;
#define CMCG_DIA_GATHER(MT)                                                                                   \
    k_dia_gather<MT><<<blocks, 256, 0, ctx->stream>>>(D.d_pos, p->nnz, static_cast<const MT*>(A->d_vals), A->stride, \
                                                      A->batches, static_cast<MT*>(s->dia_plain), s->dia_plain_stride)
        if (A->dtype == CMCG_F32) CMCG_DIA_GATHER(float);
        else if (A->dtype == CMCG_BF16) CMCG_DIA_GATHER(__nv_bfloat16);
        else CMCG_DIA_GATHER(double);
#undef CMCG_DIA_GATHER
        count_launch();
        CMCG_CHECK_LAUNCH();
        s->dia_plain_version = A->version;
        s->dia_plain_plan_id = D.plan_id;
        s->dia_plain_dtype = A->dtype;
    }
    *ok = true;
    return CMCG_OK;
}

template <typename VT, typename MT, bool RX>
cmcg_status launch_cg_fast(cmcg_solver s, SolveArgs<VT, MT>& a, int nmax) {
    cmcg_ctx ctx = s->A->pat->ctx;
    const size_t sm = static_cast<size_t>(nmax) * sizeof(VT) * (RX ? 3 : 1);
    CMCG_TRY(allow_smem(k_cg_fast<VT, MT, RX>, sm));
    const int n_inst = a.n_sys * a.ob;
    const int grid = std::max(1, std::min(n_inst, ctx->sm_count));
    CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 3 * sizeof(int32_t), ctx->stream));
    k_cg_fast<VT, MT, RX><<<grid, kSmemThreads, sm, ctx->stream>>>(a, compact_args(s->A->pat), nmax);
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

// Plain FP64 batched PCG over the diagonal layout in three CTA tiers (the
// mixed kernel's machinery): systems above kMixSmallRows rows on 1024-thread
// CTAs, then up to kMixSmallRows on 512-thread CTAs (two per SM), then up to
// kMixTinyRows on 256-thread CTAs (four per SM), larger tiers on
// higher-priority streams. *done = false when the shared memory of p with its
// halo does not fit.
template <typename MT>
cmcg_status run_plain_dia(cmcg_solver s, SolveArgs<double, MT>& a, bool* done) {
    *done = false;
    cmcg_pattern p = s->A->pat;
    cmcg_ctx ctx = p->ctx;
    const DiaPlan& D = p->dia;
    const int32_t n_inst = a.n_sys * a.ob;
    const int cta[3] = {kSmemThreads, 512, 256};
    const int tier_rows[3] = {s->max_sys_rows, std::min<int>(s->max_sys_rows, kMixSmallRows),
                              std::min<int>(s->max_sys_rows, kMixTinyRows)};
    const size_t tier_limit[3] = {kDiaSmemLimit, kMixSmallSmemLimit, kMixTinySmemLimit};
    int nmax_t[3];
    size_t sm_t[3];
    for (int t = 0; t < 3; ++t) {
        nmax_t[t] = (tier_rows[t] + cta[t] - 1) / cta[t] * cta[t];
        sm_t[t] = (static_cast<size_t>(nmax_t[t]) + 2 * static_cast<size_t>(D.margin)) * sizeof(double);
    }
    if (sm_t[0] > tier_limit[0]) return CMCG_OK;
    PlainDiaArgs<MT> m{};
    m.rows = p->rows;
    m.n_sys = s->n_sys;
    m.ob = a.ob;
    m.mb = s->A->batches;
    m.row_off = p->d_row_off;
    m.order = s->d_order;
    m.vals = static_cast<const MT*>(s->dia_plain);
    m.vstride = s->dia_plain_stride;
    m.base = D.d_sys_base;
    m.off = D.d_sys_off;
    m.margin = D.margin;
    m.dinv = a.dinv;
    m.dinv_b = a.dinv_b;
    m.b = a.b;
    m.b_b = a.b_b;
    m.x = a.x;
    m.r = a.r;
    m.q = a.q;
    m.tol = a.tol;
    m.max_iter = a.max_iter;
    m.abs_zero_test = a.abs_zero_test;
    m.st = a.st;
    int32_t lo[4] = {0, n_inst, n_inst, n_inst};
    if (s->mix_small && sm_t[1] <= tier_limit[1]) {
        lo[1] = std::min<int32_t>(n_inst, s->mix_split * a.ob);
        if (sm_t[2] <= tier_limit[2]) lo[2] = std::max(lo[1], std::min<int32_t>(n_inst, s->mix_split2 * a.ob));
    }
    int tiers[3], nt = 0;
    for (int t = 0; t < 3; ++t)
        if (lo[t + 1] > lo[t]) tiers[nt++] = t;
    CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 3 * sizeof(int32_t), ctx->stream));
    if (nt > 1) {
        CMCG_TRY(ensure_aux_stream(s));
        CMCG_CUDA(cudaEventRecord(s->ev_fork, ctx->stream));
    }
    for (int j = 0; j < nt; ++j) {
        const int t = tiers[j];
        cudaStream_t st = (j == nt - 1) ? ctx->stream : s->aux_stream[j];
        if (j < nt - 1) CMCG_CUDA(cudaStreamWaitEvent(st, s->ev_fork, 0));
        PlainDiaArgs<MT> mt = m;
        mt.item_begin = lo[t];
        mt.item_end = lo[t + 1];
        mt.next = s->counters + t;
        const int grid = std::max(1, std::min(lo[t + 1] - lo[t], ctx->sm_count * (kSmemThreads / cta[t])));
        CMCG_TRY(launch_plain_dia<MT>(mt, cta[t], nmax_t[t], sm_t[t], D.max_nd, grid, st));
        CMCG_CHECK_LAUNCH();
        count_launch();
    }
    for (int j = 0; j < nt - 1; ++j) {
        CMCG_CUDA(cudaEventRecord(s->ev_join[j], s->aux_stream[j]));
        CMCG_CUDA(cudaStreamWaitEvent(ctx->stream, s->ev_join[j], 0));
    }
    *done = true;
    return CMCG_OK;
}

template <typename VT, typename MT, int FMT>
cmcg_status run_persistent(cmcg_solver s, SolveArgs<VT, MT>& a) {
    cmcg_ctx ctx = s->A->pat->ctx;
    // FP64 vectors on stencil-shaped patterns: the diagonal-layout tiers
    if constexpr (std::is_same<VT, double>::value &&
                  (std::is_same<MT, double>::value || std::is_same<MT, float>::value)) {
        if (FMT == CMCG_CSR && !a.guess && s->fast_kernels && s->use_smem && s->max_sys_rows <= kSmemMaxRows) {
            bool dia = false;
            CMCG_TRY(ensure_dia_plain(s, &dia));
            bool done = false;
            if (dia) CMCG_TRY(run_plain_dia<MT>(s, a, &done));
            if (done) return CMCG_OK;
        }
    }
    if (FMT == CMCG_CSR && compact_ok(s)) {
        const int nmax = smem_rows(s->max_sys_rows);
        // FP32: p, r, x in shared memory (12 B/row); FP64: all three when they
        // fit (24 B/row, up to 8192 rows), else p only and r, x in global memory
        if (sizeof(VT) == 4 || nmax <= kSmemMaxRows / 2) return launch_cg_fast<VT, MT, true>(s, a, nmax);
        return launch_cg_fast<VT, MT, false>(s, a, nmax);
    }
    if constexpr (std::is_same<VT, float>::value) {
        if (s->max_sys_rows <= kSmemMaxRows && s->use_smem) {
            const int nmax = smem_rows(s->max_sys_rows);
            const size_t sm = smem_bytes(nmax);
            CMCG_TRY(allow_smem(k_cg_smem<MT, FMT>, sm));
            const int n_inst = a.n_sys * a.ob;
            const int grid = std::max(1, std::min(n_inst, ctx->sm_count));
            CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 3 * sizeof(int32_t), ctx->stream));
            k_cg_smem<MT, FMT><<<grid, kSmemThreads, sm, ctx->stream>>>(a, nmax);
            count_launch();
            CMCG_CHECK_LAUNCH();
            return CMCG_OK;
        }
    }
    int occ = 0;
    CMCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_persistent_cg<VT, MT, FMT>, kPersistThreads, 0));
    const int n_inst = a.n_sys * a.ob;
    const int grid = std::max(1, std::min(n_inst, ctx->sm_count * std::max(occ, 1)));
    CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 3 * sizeof(int32_t), ctx->stream));
    k_persistent_cg<VT, MT, FMT><<<grid, kPersistThreads, 0, ctx->stream>>>(a);
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

// Whether the grid path's product forms p_k itself (one launch less per
// iteration) or reads it from a separate p-update kernel. Forming it re-reads
// r, M^-1 and p_{k-1} at every gathered offset, which costs nothing while
// those vectors of the whole batch (vec_bytes) stay in L2, and triples their
// DRAM traffic when they do not: measured on the B200, 2D Poisson 1024^2 26.0
// against 27.2 us per iteration formed, 10000^2 1436 against 1199 us. The
// split is half the L2.
bool fuse_p_update(cmcg_solver s, double vec_bytes) {
    if (s->fuse_p >= 0) return s->fuse_p != 0;
    int l2 = 0;
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, s->A->pat->ctx->device) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return vec_bytes <= 0.5 * l2;
}

template <typename VT, typename MT, int FMT>
cmcg_status run_grid(cmcg_solver s, SolveArgs<VT, MT>& a) {
    cmcg_ctx ctx = s->A->pat->ctx;
    cudaStream_t st = ctx->stream;
    // one partial per (batch, segment); the grid is the plan's CTA count
    const int64_t items = static_cast<int64_t>(a.n_seg) * a.ob;
    const int grid = s->grid_ctas;
    const size_t need = 2 * sizeof(VT) * static_cast<size_t>(items) + 64;
    if (s->part_ws_bytes < need) {
        CMCG_TRY(ensure_buffer(&s->part_ws, &s->part_ws_bytes, need));
        if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
        if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
        s->gkey.clear();
    }
    a.part1 = static_cast<VT*>(s->part_ws);
    a.part2 = a.part1 + items;
    int64_t cap = 0;
    if (s->max_iter >= 0) cap = s->max_iter;
    else cap = 2 * static_cast<int64_t>(s->max_sys_rows);
    a.loop_cap = static_cast<int32_t>(std::min<int64_t>(cap + 2, INT32_MAX - 1));

    // stencil-shaped CSR patterns: the product reads the diagonal layout
    int nd = 0;
    a.dia = DiaArgs<MT>{};
    if (FMT == CMCG_CSR) {
        bool dia = false;
        CMCG_TRY(ensure_dia_plain(s, &dia));
        if (dia) {
            const DiaPlan& D = s->A->pat->dia;
            nd = D.max_nd;
            a.dia = DiaArgs<MT>{static_cast<const MT*>(s->dia_plain), s->dia_plain_stride, D.d_sys_base, D.d_sys_off,
                                nullptr, s->A->batches};
        }
    }

    const bool fused = fuse_p_update(s, 3.0 * sizeof(VT) * static_cast<double>(a.rows) * a.ob);
    if (!fused) a.p2 = a.p;   // (one p buffer: the kernels read p_k as stored)
    CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 3 * sizeof(int32_t), st));
    k_grid_init<VT, MT, FMT><<<grid, kTile, 0, st>>>(a);
    k_grid_init2<VT, MT, FMT><<<grid, kTile, 0, st>>>(a);
    count_launch(2);
    CMCG_CHECK_LAUNCH();

    // one iteration's kernels on stream t: p update + product + p.q (or the
    // product alone and a separate p update), then the x / r update
    const auto iteration = [&](cudaStream_t t) {
        const auto product = [&](auto fuse) {
            constexpr bool F = decltype(fuse)::value;
            if constexpr (FMT == CMCG_CSR) {
                if (nd == 5) k_grid_spmv_pq<VT, MT, FMT, 5, F><<<grid, kTile, 0, t>>>(a);
                else if (nd == 7) k_grid_spmv_pq<VT, MT, FMT, 7, F><<<grid, kTile, 0, t>>>(a);
                else k_grid_spmv_pq<VT, MT, FMT, 0, F><<<grid, kTile, 0, t>>>(a);
            } else {
                k_grid_spmv_pq<VT, MT, FMT, 0, F><<<grid, kTile, 0, t>>>(a);
            }
        };
        if (fused) product(std::true_type{});
        else product(std::false_type{});
        k_grid_update<VT, MT, FMT><<<grid, kTile, 0, t>>>(a);
        if (!fused) k_grid_pupdate<VT, MT, FMT><<<grid, kTile, 0, t>>>(a);
    };
    const int per_iter = fused ? 2 : 3;
    if (!s->graph_loop) {
        return host_loop(st, a.active, a.loop_cap, per_iter + 1, [&] {
            iteration(st);
            k_loop_step<<<1, 1, 0, st>>>(a.loops);
        });
    }

    // graph with a WHILE node over the iteration kernels; rebuilt when any
    // kernel argument changes
    std::vector<char> key(sizeof(a) + sizeof(int) * 2);
    {
        SolveArgs<VT, MT> k = a;
        k.cond = 0;
        std::memcpy(key.data(), &k, sizeof(k));
        const int ids[2] = {DT<VT>::id, FMT};
        std::memcpy(key.data() + sizeof(k), ids, sizeof(ids));
    }
    if (!s->gexec || key != s->gkey) {
        if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
        if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
        cudaGraph_t g;
        CMCG_CUDA(cudaGraphCreate(&g, 0));
        s->graph = g;
        cudaGraphConditionalHandle h;
        CMCG_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CMCG_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        a.cond = h;
        if (!ctx->capture_stream) CMCG_CUDA(cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking));
        cudaStream_t cs = ctx->capture_stream;
        CMCG_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        iteration(cs);
        k_grid_cond<<<1, 1, 0, cs>>>(a.active, a.loops, a.loop_cap, h);
        cudaGraph_t captured = nullptr;
        cudaError_t ce = cudaStreamEndCapture(cs, &captured);
        if (ce != cudaSuccess) return cuda_fail(ce, "capture of the CG iteration", __FILE__, __LINE__);
        CMCG_CUDA(cudaGraphInstantiate(&s->gexec, g, 0));
        s->gkey = key;
    }
    CMCG_CUDA(cudaGraphLaunch(s->gexec, st));
    // kernels inside the graph: per_iter + 1 per executed iteration (counted as
    // launched by the graph, not by the host)
    count_launch(1);
    return CMCG_OK;
}

// One thread-block cluster per instance (cg_cluster.cu), when the largest
// system has more than kClusterMinRows rows yet its vectors fit the shared
// memory of at most kClusterMaxCtas CTAs, and all instances' clusters can be
// resident at once. *done = false leaves the solve to the cooperative launch
// or the graph loop.
template <typename VT, typename MT, int FMT>
cmcg_status run_cluster(cmcg_solver s, SolveArgs<VT, MT>& a, bool* done) {
    *done = false;
    cmcg_ctx ctx = s->A->pat->ctx;
    const int n_inst = a.n_sys * a.ob;
    if (!s->cluster || s->max_sys_rows <= kClusterMinRows) return CMCG_OK;
    int optin = 0;
    CMCG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    int ctas = 0;
    // (2 KB of the CTA's shared memory hold the reduction scratch)
    const int lg = cluster_rows_log2(s->max_sys_rows, sizeof(VT), static_cast<size_t>(std::max(0, optin - 2048)), &ctas);
    if (lg == 0 || ctas < 2) return CMCG_OK;
    // stencil-shaped CSR patterns: the product reads the diagonal layout
    SolveArgs<VT, MT> c = a;
    int nd = 0;
    c.dia = DiaArgs<MT>{};
    if (FMT == CMCG_CSR) {
        bool dia = false;
        CMCG_TRY(ensure_dia_plain(s, &dia));
        if (dia) {
            const DiaPlan& D = s->A->pat->dia;
            nd = D.max_nd;
            c.dia = DiaArgs<MT>{static_cast<const MT*>(s->dia_plain), s->dia_plain_stride, D.d_sys_base, D.d_sys_off,
                                nullptr, s->A->batches};
        }
    }
    if (nd != 5 && nd != 7) nd = 0;
    bool launched = false;
    CMCG_TRY((cluster_cg_launch<VT, MT, FMT>(c, n_inst, ctas, lg, nd, n_inst, ctx->stream, &launched)));
    if (!launched) {
        if (log_on(1))
            log_msg(1, "cluster solve not launched: %d clusters of %d CTAs cannot be resident at once", n_inst, ctas);
        return CMCG_OK;
    }
    if (log_on(2))
        log_msg(2, "cluster solve: %d clusters of %d CTAs x %d rows, %s layout", n_inst, ctas, 1 << lg,
                nd ? "diagonal" : "sliced");
    count_launch();
    CMCG_CHECK_LAUNCH();
    *done = true;
    return CMCG_OK;
}

// One cooperative launch for the whole grid-path solve, when the instances are
// few (the closing sums run in one CTA per barrier) and the segment plan's
// CTAs can all be resident. *done = false leaves the solve to the graph path.
template <typename VT, typename MT, int FMT>
cmcg_status run_coop(cmcg_solver s, SolveArgs<VT, MT>& a, VT* p_alt, bool* done) {
    *done = false;
    cmcg_ctx ctx = s->A->pat->ctx;
    const int n_inst = a.n_sys * a.ob;
    if (!s->coop || n_inst > kCoopMaxInst || s->coop_ctas < 1 || s->coop_max_segs > kCoopMaxSegs) return CMCG_OK;
    // systems large enough to hide the graph's per-kernel launches run faster
    // on the graph kernels (more threads per SM in flight)
    if (s->max_sys_rows > kCoopMaxRows && s->coop < 2) return CMCG_OK;
    int coop_attr = 0, occ = 0;
    CMCG_CUDA(cudaDeviceGetAttribute(&coop_attr, cudaDevAttrCooperativeLaunch, ctx->device));
    CMCG_TRY((coop_cg_occupancy<VT, MT, FMT>(&occ)));
    if (!coop_attr || occ * ctx->sm_count < s->coop_ctas) {
        if (log_on(1))
            log_msg(1, "cooperative solve not launched: %d CTAs per SM resident, %d CTAs needed", occ, s->coop_ctas);
        return CMCG_OK;
    }
    // the cooperative launch has its own segment plan (one CTA per SM)
    SolveArgs<VT, MT> c = a;
    c.n_seg = s->coop_n_seg;
    c.seg_t0 = s->d_cseg_t0;
    c.seg_t1 = s->d_cseg_t1;
    c.seg_sys = s->d_cseg_sys;
    c.cta_seg0 = s->d_ccta_seg0;
    c.sys_seg0 = s->d_csys_seg0;
    const int64_t items = static_cast<int64_t>(c.n_seg) * c.ob;
    CMCG_TRY(ensure_buffer(&s->part_ws, &s->part_ws_bytes, 2 * sizeof(VT) * static_cast<size_t>(items) + 64));
    c.part1 = static_cast<VT*>(s->part_ws);
    c.part2 = c.part1 + items;
    const int64_t cap = s->max_iter >= 0 ? s->max_iter : 2 * static_cast<int64_t>(s->max_sys_rows);
    c.loop_cap = static_cast<int32_t>(std::min<int64_t>(cap + 2, INT32_MAX - 1));
    // counters: next, active, loops, -, grid barrier (count, generation)
    CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 8 * sizeof(int32_t), ctx->stream));
    // every instance starts as running (-1), so that a launch that leaves
    // early (a grid barrier whose wait ran out) is finalised as not converged
    // instead of keeping a previous solve's status; its norms read as zero
    CMCG_CUDA(cudaMemsetAsync(s->st.status, 0xFF, sizeof(int32_t) * static_cast<size_t>(n_inst), ctx->stream));
    CMCG_CUDA(cudaMemsetAsync(s->st.rr, 0, sizeof(double) * static_cast<size_t>(n_inst), ctx->stream));
    CMCG_CUDA(cudaMemsetAsync(s->st.bb, 0, sizeof(double) * static_cast<size_t>(n_inst), ctx->stream));
    // counters[4..7]: the grid barrier's two 64-bit words
    CMCG_TRY((coop_cg_launch<VT, MT, FMT>(c, s->counters + 4, ctx->d_err, n_inst, p_alt, s->coop_ctas, ctx->stream)));
    count_launch();
    *done = true;
    return CMCG_OK;
}

cmcg_status ensure_vec_ws(cmcg_solver s, size_t bytes) {
    if (s->vec_ws_bytes >= bytes && s->vec_ws) return CMCG_OK;
    CMCG_TRY(ensure_buffer(&s->vec_ws, &s->vec_ws_bytes, bytes));
    if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
    if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
    s->gkey.clear();
    return CMCG_OK;
}

template <typename VT, typename MT, int FMT>
cmcg_status solve_t(cmcg_solver s, const VT* b, int32_t b_b, const VT* guess, VT* x, int32_t ob) {
    cmcg_pattern p = s->A->pat;
    cmcg_ctx ctx = p->ctx;
    const int32_t n_inst = ob * s->n_sys;
    CMCG_TRY(ensure_state(s, n_inst));
    const void* dinv = nullptr;
    CMCG_TRY(get_dinv(s, DT<VT>::id, &dinv));
    CMCG_TRY(ensure_sell_values(s->A));
    const bool smem_ok = (FMT == CMCG_CSR && compact_ok(s)) || (sizeof(VT) == 4 && s->use_smem);
    const int32_t path = choose_path(s, n_inst, smem_ok, /*cluster_ok=*/true);
    if (log_on(2))
        log_msg(2, "solve: %d instances of up to %d rows, %s vectors, %s path", n_inst, s->max_sys_rows,
                sizeof(VT) == 8 ? "FP64" : "FP32", path == CMCG_PATH_GRID ? "grid" : "persistent");
    const size_t vbytes = sizeof(VT) * static_cast<size_t>(p->rows) * ob;
    SolveArgs<VT, MT> a = base_args<VT, MT>(s, ob);
    a.dinv = static_cast<const VT*>(dinv);
    a.dinv_b = s->A->batches;
    if (path == CMCG_PATH_PERSISTENT) {
        CMCG_TRY(ensure_vec_ws(s, 3 * vbytes + 256));
        VT* w = static_cast<VT*>(s->vec_ws);
        a.b = b; a.b_b = b_b; a.guess = guess; a.g_b = ob; a.x = x;
        a.r = w; a.p = w + p->rows * static_cast<size_t>(ob); a.q = a.p + p->rows * static_cast<size_t>(ob);
        CMCG_TRY((run_persistent<VT, MT, FMT>(s, a)));
    } else {
        // the graph iterates on internal copies of x so that its arguments do not
        // depend on the caller's buffers
        CMCG_TRY(ensure_vec_ws(s, 5 * vbytes + 256));
        VT* w = static_cast<VT*>(s->vec_ws);
        const size_t nv = p->rows * static_cast<size_t>(ob);
        a.r = w; a.p = w + nv; a.q = w + 2 * nv; a.x = w + 3 * nv;
        a.p2 = w + 4 * nv;   // (the graph loop's second p buffer, the cooperative launch's p_alt)
        a.b = b; a.b_b = b_b; a.guess = guess; a.g_b = ob;
        bool done = false;
        CMCG_TRY((run_cluster<VT, MT, FMT>(s, a, &done)));
        if (!done) CMCG_TRY((run_coop<VT, MT, FMT>(s, a, w + 4 * nv, &done)));
        if (!done) CMCG_TRY((run_grid<VT, MT, FMT>(s, a)));
        const int fb = (n_inst + 255) / 256;
        k_finalize<<<fb, 256, 0, ctx->stream>>>(s->st, n_inst);
        count_launch();
        CMCG_CHECK_LAUNCH();
        CMCG_CUDA(cudaMemcpyAsync(x, a.x, vbytes, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    s->last_inst = n_inst;
    s->last_refined = false;
    return CMCG_OK;
}

template <typename VT>
cmcg_status solve_vt(cmcg_solver s, const VT* b, int32_t b_b, const VT* g, VT* x, int32_t ob) {
    const int fmt = s->A->pat->format;
    switch (s->A->dtype) {
        case CMCG_F32:
            return fmt == CMCG_CSR ? solve_t<VT, float, CMCG_CSR>(s, b, b_b, g, x, ob) : solve_t<VT, float, CMCG_ELLPACK>(s, b, b_b, g, x, ob);
        case CMCG_F64:
            return fmt == CMCG_CSR ? solve_t<VT, double, CMCG_CSR>(s, b, b_b, g, x, ob) : solve_t<VT, double, CMCG_ELLPACK>(s, b, b_b, g, x, ob);
        case CMCG_BF16:
            return fmt == CMCG_CSR ? solve_t<VT, __nv_bfloat16, CMCG_CSR>(s, b, b_b, g, x, ob)
                                   : solve_t<VT, __nv_bfloat16, CMCG_ELLPACK>(s, b, b_b, g, x, ob);
    }
    return fail(CMCG_ERR_INVALID_ARGUMENT, "unsupported matrix dtype");
}

// ---- refined solve ----------------------------------------------------------------

template <typename MI, typename MO, int FMT>
cmcg_status refined_persistent(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_b, double* x, int32_t ob,
                               double outer_tol, int32_t max_outer) {
    cmcg_pattern p = s->A->pat;
    cmcg_ctx ctx = p->ctx;
    const int32_t n_inst = ob * s->n_sys;
    CMCG_TRY(ensure_state(s, n_inst));
    const void* dinv = nullptr;
    CMCG_TRY(get_dinv(s, CMCG_F32, &dinv));
    const size_t nv = static_cast<size_t>(p->rows) * ob;
    CMCG_TRY(ensure_buffer(&s->ref_ws, &s->ref_ws_bytes, 5 * nv * sizeof(float) + 256));
    CMCG_TRY(ensure_sell_values(s->A));
    if (Ao != s->A) CMCG_TRY(ensure_sell_values(Ao));
    float* w = static_cast<float*>(s->ref_ws);
    RefineArgs<MI, MO> a{};
    a.inner = mat_args<MI>(s->A);
    a.outer = mat_args<MO>(Ao);
    a.rows = p->rows;
    a.n_sys = s->n_sys;
    a.ob = ob;
    a.row_off = p->d_row_off;
    a.order = s->d_order;
    a.next = s->counters;
    a.dinv = static_cast<const float*>(dinv);
    a.dinv_b = s->A->batches;
    a.b = b;
    a.b_b = b_b;
    a.x = x;
    a.r32 = w; a.d32 = w + nv; a.r = w + 2 * nv; a.p = w + 3 * nv; a.q = w + 4 * nv;
    a.inner_tol = s->tol;
    a.outer_tol = outer_tol;
    a.max_inner = s->max_iter;
    a.max_outer = max_outer;
    a.st = s->st;
    CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 3 * sizeof(int32_t), ctx->stream));
    if (s->refine_method == CMCG_REFINE_RELIABLE && FMT == CMCG_CSR && compact_ok(s)) {
        CMCG_TRY(ensure_mix(s));
        MixArgs<MI, MO> m{};
        m.rows = p->rows;
        m.n_sys = s->n_sys;
        m.ob = ob;
        m.mb = s->A->batches;
        m.row_off = p->d_row_off;
        m.order = s->d_order;
        m.next = s->counters;
        m.c = compact_args(p);
        m.vin = static_cast<const MI*>(s->mix_vals);
        m.vin_stride = s->mix_stride;
        m.vout = static_cast<const MO*>(Ao->d_sell_vals);
        m.vout_stride = Ao->sell_stride;
        m.s = s->mix_s;
        m.b = b;
        m.b_b = b_b;
        m.x = x;
        m.outer_tol = outer_tol;
        m.max_inner = s->max_iter;
        m.max_updates = max_outer;
        m.delta = refine_delta_for(s);
        m.st = s->st;
        const int nmax = smem_rows(s->max_sys_rows);
        const size_t sm = smem_bytes(nmax);
        bool dia = false;
        if (s->dia_kernels) CMCG_TRY(ensure_dia_vals(s, &dia));
        // the zero halo of p must fit next to the vectors in shared memory
        // (vectors of whole 1024-row blocks in the diagonal layout)
        const int nmax_dia = (s->max_sys_rows + kDiaBlockRows - 1) / kDiaBlockRows * kDiaBlockRows;
        const size_t sm_dia = dia ? smem_bytes(nmax_dia) + 2 * sizeof(float) * static_cast<size_t>(p->dia.margin) : 0;
        const bool use_dia = dia && sm_dia <= kDiaSmemLimit;
        const size_t halo = use_dia ? 2 * sizeof(float) * static_cast<size_t>(p->dia.margin) : 0;
        int nd = 0;
        if (use_dia) {
            m.vdia = static_cast<const MI*>(s->dia_vals);
            m.vdia_stride = s->dia_stride;
            m.dia_base = p->dia.d_sys_base;
            m.dia_off = p->dia.d_sys_off;
            m.margin = p->dia.margin;
            m.dia_unit = s->dia_unit;
            nd = p->dia.max_nd;
        }
        // Three tiers by position in the size order: systems above
        // kMixSmallRows rows on 1024-thread CTAs (one per SM), then systems of
        // at most kMixSmallRows rows on 512-thread CTAs (two per SM), then
        // systems of at most kMixTinyRows rows on 256-thread CTAs (four per
        // SM), so that small systems share an SM's latencies. Larger tiers
        // launch on higher-priority streams and take the SMs first; the next
        // tier's CTAs fill the SMs they leave.
        const int cta[3] = {kSmemThreads, 512, 256};
        const int tier_rows[3] = {s->max_sys_rows, std::min<int>(s->max_sys_rows, kMixSmallRows),
                                  std::min<int>(s->max_sys_rows, kMixTinyRows)};
        const size_t tier_limit[3] = {use_dia ? kDiaSmemLimit : sm, kMixSmallSmemLimit, kMixTinySmemLimit};
        int nmax_t[3];
        size_t sm_t[3];
        for (int t = 0; t < 3; ++t) {
            nmax_t[t] = use_dia ? (tier_rows[t] + kDiaBlockRows - 1) / kDiaBlockRows * kDiaBlockRows
                                : smem_rows(tier_rows[t]);
            sm_t[t] = smem_bytes(nmax_t[t]) + halo;
        }
        // item ranges [lo[t], lo[t + 1])
        int32_t lo[4] = {0, n_inst, n_inst, n_inst};
        if (s->mix_small && sm_t[1] <= tier_limit[1]) {
            lo[1] = std::min<int32_t>(n_inst, s->mix_split * ob);
            if (sm_t[2] <= tier_limit[2]) lo[2] = std::max(lo[1], std::min<int32_t>(n_inst, s->mix_split2 * ob));
        }
        int tiers[3], nt = 0;
        for (int t = 0; t < 3; ++t)
            if (lo[t + 1] > lo[t]) tiers[nt++] = t;
        if (nt > 1) {
            CMCG_TRY(ensure_aux_stream(s));
            CMCG_CUDA(cudaEventRecord(s->ev_fork, ctx->stream));
        }
        if (log_on(2))
            log_msg(2, "refined solve: %d instances on %d CTA tier(s) [%d, %d, %d instances], %s layout", n_inst, nt,
                    lo[1] - lo[0], lo[2] - lo[1], lo[3] - lo[2], nd ? "diagonal" : "sliced");
        for (int j = 0; j < nt; ++j) {
            const int t = tiers[j];
            // the last (smallest) tier runs on the caller's stream
            cudaStream_t st = (j == nt - 1) ? ctx->stream : s->aux_stream[j];
            if (j < nt - 1) CMCG_CUDA(cudaStreamWaitEvent(st, s->ev_fork, 0));
            MixArgs<MI, MO> mt = m;
            mt.item_begin = lo[t];
            mt.item_end = lo[t + 1];
            mt.next = s->counters + t;
            const int grid = std::max(1, std::min(lo[t + 1] - lo[t], ctx->sm_count * (kSmemThreads / cta[t])));
            CMCG_TRY((launch_mixed_fast<MI, MO>(mt, cta[t], nmax_t[t], sm_t[t], nd, grid, st)));
            CMCG_CHECK_LAUNCH();
            count_launch();
        }
        for (int j = 0; j < nt - 1; ++j) {
            CMCG_CUDA(cudaEventRecord(s->ev_join[j], s->aux_stream[j]));
            CMCG_CUDA(cudaStreamWaitEvent(ctx->stream, s->ev_join[j], 0));
        }
        s->last_inst = n_inst;
        s->last_refined = true;
        return CMCG_OK;
    }
    if (s->refine_method == CMCG_REFINE_RELIABLE && s->max_sys_rows <= kSmemMaxRows && s->use_smem) {
        const int nmax = smem_rows(s->max_sys_rows);
        const size_t sm = smem_bytes(nmax);
        CMCG_TRY(allow_smem(k_reliable_smem<MI, MO, FMT>, sm));
        const int grid = std::max(1, std::min(n_inst, ctx->sm_count));
        k_reliable_smem<MI, MO, FMT><<<grid, kSmemThreads, sm, ctx->stream>>>(a, nmax, refine_delta_for(s));
        count_launch();
        CMCG_CHECK_LAUNCH();
        s->last_inst = n_inst;
        s->last_refined = true;
        return CMCG_OK;
    }
    int occ = 0;
    CMCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_persistent_refined<MI, MO, FMT>, kPersistThreads, 0));
    const int grid = std::max(1, std::min(n_inst, ctx->sm_count * std::max(occ, 1)));
    k_persistent_refined<MI, MO, FMT><<<grid, kPersistThreads, 0, ctx->stream>>>(a);
    count_launch();
    CMCG_CHECK_LAUNCH();
    s->last_inst = n_inst;
    s->last_refined = true;
    return CMCG_OK;
}

// FP64 residual r = b - A x (values of Ao) into r32 (rounded) and per-system
// |r|^2 / |b|^2, for the host-driven refinement of the grid path.
__global__ void k_axpy_f32_to_f64(double* __restrict__ x, const float* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[i] += static_cast<double>(d[i]);
}
__global__ void k_sub_round(const double* __restrict__ b, int32_t b_b, const double* __restrict__ ax, float* __restrict__ r32,
                            double* __restrict__ r64, int32_t rows, int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double bi = b[b_b == 1 ? (i % rows) : i];
        const double ri = bi - ax[i];
        r64[i] = ri;
        r32[i] = static_cast<float>(ri);
    }
}

cmcg_status refined_grid(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_b, double* x, int32_t ob,
                         double outer_tol, int32_t max_outer) {
    // Host-driven outer loop for large systems: one sync per refinement step.
    // Supports a single system per batch (the grid path's use case).
    cmcg_pattern p = s->A->pat;
    cmcg_ctx ctx = p->ctx;
    cudaStream_t st = ctx->stream;
    const size_t nv = static_cast<size_t>(p->rows) * ob;
    const int32_t n_inst = ob * s->n_sys;
    // buffers: r64, ax (FP64) + r32, d32 (FP32) + norms
    void* buf = nullptr;
    CMCG_TRY(dev_alloc(&buf, nv * (8 + 8 + 4 + 4) + 2 * 8 * static_cast<size_t>(ob) + 512));
    double* r64 = static_cast<double*>(buf);
    double* ax = r64 + nv;
    float* r32 = reinterpret_cast<float*>(ax + nv);
    float* d32 = r32 + nv;
    double* nrm = reinterpret_cast<double*>(d32 + nv + 64);
    auto cleanup = [&](cmcg_status code) { cudaStreamSynchronize(st); dev_free(buf); return code; };
    cmcg_status rc;
    const int blocks = ctx->sm_count * 8;
    std::vector<double> hb(ob), hr(ob);
    std::vector<int32_t> outer(n_inst, 0), it_tot(n_inst, 0), status(n_inst, ST_RUNNING);
    if (cudaMemsetAsync(x, 0, nv * 8, st) != cudaSuccess) return cleanup(fail(CMCG_ERR_CUDA, "memset x"));
    // |b|^2 per batch (b broadcast when b_b == 1)
    if ((rc = dot_dispatch(ctx, CMCG_F64, p->rows, b, b_b, b, b_b, nrm, b_b)) != CMCG_OK) return cleanup(rc);
    if (cudaMemcpyAsync(hb.data(), nrm, 8 * b_b, cudaMemcpyDeviceToHost, st) != cudaSuccess) return cleanup(fail(CMCG_ERR_CUDA, "D2H"));
    if (cudaStreamSynchronize(st) != cudaSuccess) return cleanup(fail(CMCG_ERR_CUDA, "sync"));
    for (int32_t i = b_b; i < ob; ++i) hb[i] = hb[0];
    {
        // x == 0: r = b
        const int32_t bb = b_b;
        for (int32_t i = 0; i < ob; ++i) {
            const double* src = b + (bb == 1 ? 0 : static_cast<size_t>(i) * p->rows);
            if (cudaMemcpyAsync(r64 + static_cast<size_t>(i) * p->rows, src, 8 * p->rows, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                return cleanup(fail(CMCG_ERR_CUDA, "copy b"));
        }
        if ((rc = convert(ctx, CMCG_F64, r64, CMCG_F32, r32, static_cast<int64_t>(nv))) != CMCG_OK) return cleanup(rc);
    }
    for (int32_t i = 0; i < ob; ++i) hr[i] = hb[i];
    for (int32_t step = 0;; ++step) {
        bool all_done = true;
        for (int32_t i = 0; i < ob; ++i) {
            if (status[i] != ST_RUNNING) continue;
            if (hb[i] == 0.0) status[i] = CMCG_SOLVE_ZERO_RHS;
            else if (!std::isfinite(hr[i])) status[i] = CMCG_SOLVE_NON_FINITE;
            else if (hr[i] < outer_tol * outer_tol * hb[i]) status[i] = CMCG_SOLVE_CONVERGED;
            else if (step >= max_outer) status[i] = CMCG_SOLVE_MAX_ITER;
            else all_done = false;
        }
        if (all_done) break;
        // inner solve A d = r32 (FP32) on the grid path
        const int32_t saved = s->path;
        s->path = CMCG_PATH_GRID;
        s->inner_solve = true;   // the inner rhs shrinks with the residual: no absolute early-out
        rc = solve_vt<float>(s, r32, ob, nullptr, d32, ob);
        s->inner_solve = false;
        s->path = saved;
        if (rc != CMCG_OK) return cleanup(rc);
        std::vector<int32_t> it(n_inst);
        if (cudaMemcpyAsync(it.data(), s->st.it, 4 * n_inst, cudaMemcpyDeviceToHost, st) != cudaSuccess) return cleanup(fail(CMCG_ERR_CUDA, "D2H"));
        k_axpy_f32_to_f64<<<blocks, 256, 0, st>>>(x, d32, static_cast<int64_t>(nv));
        count_launch();
        if ((rc = spmv_dispatch(Ao, CMCG_F64, x, ob, ax, CMCG_ASSIGN)) != CMCG_OK) return cleanup(rc);
        k_sub_round<<<blocks, 256, 0, st>>>(b, b_b, ax, r32, r64, p->rows, static_cast<int64_t>(nv));
        count_launch();
        if ((rc = dot_dispatch(ctx, CMCG_F64, p->rows, r64, ob, r64, ob, nrm, ob)) != CMCG_OK) return cleanup(rc);
        if (cudaMemcpyAsync(hr.data(), nrm, 8 * ob, cudaMemcpyDeviceToHost, st) != cudaSuccess) return cleanup(fail(CMCG_ERR_CUDA, "D2H"));
        if (cudaStreamSynchronize(st) != cudaSuccess) return cleanup(fail(CMCG_ERR_CUDA, "refinement step"));
        for (int32_t i = 0; i < ob; ++i)
            if (status[i] == ST_RUNNING) { outer[i]++; it_tot[i] += it[i]; }
    }
    // publish stats in the instance state
    std::vector<double> err(n_inst), rrv(n_inst), bbv(n_inst);
    for (int32_t i = 0; i < n_inst; ++i) {
        err[i] = status[i] == CMCG_SOLVE_ZERO_RHS ? 0.0 : std::sqrt(hr[i] / hb[i]);
        rrv[i] = hr[i];
        bbv[i] = hb[i];
    }
    if (cudaMemcpyAsync(s->st.err, err.data(), 8 * n_inst, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->st.rr, rrv.data(), 8 * n_inst, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->st.bb, bbv.data(), 8 * n_inst, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->st.it, it_tot.data(), 4 * n_inst, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->st.outer, outer.data(), 4 * n_inst, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->st.status, status.data(), 4 * n_inst, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return cleanup(fail(CMCG_ERR_CUDA, "stats upload"));
    s->last_inst = n_inst;
    s->last_refined = true;
    return cleanup(CMCG_OK);
}

// Reliable-update mixed solve on the grid path (CSR patterns): the iteration is
// one WHILE-node graph (product, update, fold, FP64 residual, p update, loop
// condition); b and x go through internal copies so the graph's arguments do
// not depend on the caller's buffers.
template <typename MI, typename MO>
cmcg_status refined_grid_mixed(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_b, double* x, int32_t ob,
                               double outer_tol, int32_t max_outer) {
    cmcg_pattern p = s->A->pat;
    cmcg_ctx ctx = p->ctx;
    cudaStream_t st = ctx->stream;
    const int32_t n_inst = ob * s->n_sys;
    CMCG_TRY(ensure_state(s, n_inst));
    CMCG_TRY(ensure_sell_values(s->A));
    if (Ao != s->A) CMCG_TRY(ensure_sell_values(Ao));
    CMCG_TRY(ensure_mix(s));
    const size_t nv = static_cast<size_t>(p->rows) * ob, nb = static_cast<size_t>(p->rows) * b_b;
    const size_t need = (nv + nb) * sizeof(double) + 5 * nv * sizeof(float) + 512;
    CMCG_TRY(ensure_buffer(&s->ref_ws, &s->ref_ws_bytes, need));
    double* x64 = static_cast<double*>(s->ref_ws);
    double* b64 = x64 + nv;
    float* f = reinterpret_cast<float*>(b64 + nb);
    const int64_t items = static_cast<int64_t>(s->n_seg) * ob;
    CMCG_TRY(ensure_buffer(&s->part_ws, &s->part_ws_bytes, items * (2 * sizeof(double) + 2 * sizeof(float)) + 256));
    double* p1 = static_cast<double*>(s->part_ws);
    GMixArgs<MI, MO> m{};
    m.g = base_args<float, MI>(s, ob);
    m.g.m.sell_vals = static_cast<const MI*>(s->mix_vals);
    m.g.m.sell_vstride = s->mix_stride;
    m.g.b_b = b_b;
    m.g.r = f; m.g.p = f + nv; m.g.q = f + 2 * nv; m.g.p2 = f + 4 * nv;   // (f + 3 nv: xh)
    m.g.part1 = reinterpret_cast<float*>(p1 + 2 * items);
    m.g.part2 = m.g.part1 + items;
    m.g.abs_zero_test = 0;
    int64_t cap = s->max_iter >= 0 ? s->max_iter : 2 * static_cast<int64_t>(s->max_sys_rows);
    m.g.loop_cap = static_cast<int32_t>(std::min<int64_t>(cap + 2, INT32_MAX - 1));
    m.mo = mat_args<MO>(Ao);
    m.s = s->mix_s;
    m.b64 = b64;
    m.x64 = x64;
    m.xh = f + 3 * nv;
    m.p1 = p1;
    m.p2 = p1 + items;
    m.outer_tol = outer_tol;
    m.max_updates = max_outer;
    m.delta = refine_delta_for(s);
    const int grid = s->grid_ctas;
    // stencil-shaped patterns: the inner product reads the scaled values in the
    // diagonal layout
    int nd = 0;
    if (s->dia_kernels) {
        bool dia = false;
        CMCG_TRY(ensure_dia_vals(s, &dia));
        if (dia) {
            const DiaPlan& D = p->dia;
            nd = D.max_nd;
            m.g.dia = DiaArgs<MI>{static_cast<const MI*>(s->dia_vals), s->dia_stride, D.d_sys_base, D.d_sys_off,
                                  s->dia_unit, s->A->batches};
        }
    }

    // the product forms p_k when r and p of the batch stay in L2 (fuse_p_update)
    const bool fused = fuse_p_update(s, 2.0 * sizeof(float) * static_cast<double>(nv));
    if (!fused) m.g.p2 = m.g.p;   // (one p buffer: the kernels read p_k as stored)
    CMCG_CUDA(cudaMemcpyAsync(b64, b, nb * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CMCG_CUDA(cudaMemsetAsync(s->counters, 0, 3 * sizeof(int32_t), st));
    k_gmix_init<MI, MO><<<grid, kTile, 0, st>>>(m);
    count_launch();
    CMCG_CHECK_LAUNCH();
    // one iteration's kernels on stream t
    const auto iteration = [&](cudaStream_t t) {
        const auto product = [&](auto fuse) {
            constexpr bool F = decltype(fuse)::value;
            if (nd == 5) k_gmix_spmv<MI, MO, 5, F><<<grid, kTile, 0, t>>>(m);
            else if (nd == 7) k_gmix_spmv<MI, MO, 7, F><<<grid, kTile, 0, t>>>(m);
            else k_gmix_spmv<MI, MO, 0, F><<<grid, kTile, 0, t>>>(m);
        };
        if (fused) product(std::true_type{});
        else product(std::false_type{});
        k_gmix_update<MI, MO><<<grid, kTile, 0, t>>>(m);
        k_gmix_fold<MI, MO, false><<<grid, kTile, 0, t>>>(m);
        k_gmix_residual<MI, MO, false><<<grid, kTile, 0, t>>>(m);
        if (!fused) k_gmix_pupdate<MI, MO><<<grid, kTile, 0, t>>>(m);
    };
    if (!s->graph_loop) {
        CMCG_TRY(host_loop(st, m.g.active, m.g.loop_cap, fused ? 5 : 6, [&] {
            iteration(st);
            k_loop_step<<<1, 1, 0, st>>>(m.g.loops);
        }));
    } else {
        std::vector<char> key(sizeof(m) + sizeof(int) * 2);
        {
            GMixArgs<MI, MO> k = m;
            k.g.cond = 0;
            std::memcpy(key.data(), &k, sizeof(k));
            const int ids[2] = {DT<MI>::id, DT<MO>::id};
            std::memcpy(key.data() + sizeof(k), ids, sizeof(ids));
        }
        if (!s->gexec_mix || key != s->gkey_mix) {
            if (s->gexec_mix) { cudaGraphExecDestroy(s->gexec_mix); s->gexec_mix = nullptr; }
            if (s->graph_mix) { cudaGraphDestroy(s->graph_mix); s->graph_mix = nullptr; }
            cudaGraph_t g;
            CMCG_CUDA(cudaGraphCreate(&g, 0));
            s->graph_mix = g;
            cudaGraphConditionalHandle h;
            CMCG_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            CMCG_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            m.g.cond = h;
            if (!ctx->capture_stream) CMCG_CUDA(cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking));
            cudaStream_t cs = ctx->capture_stream;
            CMCG_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            iteration(cs);
            k_grid_cond<<<1, 1, 0, cs>>>(m.g.active, m.g.loops, m.g.loop_cap, h);
            cudaGraph_t captured = nullptr;
            cudaError_t ce = cudaStreamEndCapture(cs, &captured);
            if (ce != cudaSuccess) return cuda_fail(ce, "capture of the mixed CG iteration", __FILE__, __LINE__);
            CMCG_CUDA(cudaGraphInstantiate(&s->gexec_mix, g, 0));
            s->gkey_mix = key;
        }
        CMCG_CUDA(cudaGraphLaunch(s->gexec_mix, st));
    }
    k_gmix_fold<MI, MO, true><<<grid, kTile, 0, st>>>(m);
    k_gmix_residual<MI, MO, true><<<grid, kTile, 0, st>>>(m);
    k_finalize<<<(n_inst + 255) / 256, 256, 0, st>>>(s->st, n_inst);
    count_launch(4);
    CMCG_CHECK_LAUNCH();
    CMCG_CUDA(cudaMemcpyAsync(x, x64, nv * sizeof(double), cudaMemcpyDeviceToDevice, st));
    s->last_inst = n_inst;
    s->last_refined = true;
    return CMCG_OK;
}

template <typename MI, int FMT>
cmcg_status refined_mi(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_b, double* x, int32_t ob, double ot,
                       int32_t mo) {
    if (Ao->dtype == CMCG_F32) return refined_persistent<MI, float, FMT>(s, Ao, b, b_b, x, ob, ot, mo);
    if (Ao->dtype == CMCG_F64) return refined_persistent<MI, double, FMT>(s, Ao, b, b_b, x, ob, ot, mo);
    return fail(CMCG_ERR_INVALID_ARGUMENT, "refined solve: the outer matrix must be F32 or F64");
}

}  // namespace

extern "C" {

cmcg_status cmcg_cg_create(cmcg_matrix A, int32_t precond, cmcg_solver* out) {
    CMCG_REQUIRE(A && out, "cmcg_cg_create: NULL argument");
    *out = nullptr;
    CMCG_REQUIRE(A->pat->rows == A->pat->cols, "cmcg_cg_create: matrix must be square");
    CMCG_REQUIRE(precond == CMCG_PRECOND_IDENTITY || precond == CMCG_PRECOND_JACOBI, "cmcg_cg_create: bad preconditioner");
    CMCG_CUDA(cudaSetDevice(A->pat->ctx->device));
    auto* s = new cmcg_solver_s();
    s->A = A;
    A->refs++;
    s->precond = precond;
    // default tolerance: epsilon of the scalar type (IterativeSolverBase.h:131)
    s->tol = (A->dtype == CMCG_F64) ? 2.220446049250313e-16 : 1.1920928955078125e-07;
    if (const char* e = std::getenv("CUMAT_CG_FAST")) s->fast_kernels = std::atoi(e) != 0;
    if (const char* e = std::getenv("CUMAT_CG_DIA")) s->dia_kernels = std::atoi(e) != 0;
    if (const char* e = std::getenv("CUMAT_CG_SMALL")) s->mix_small = std::atoi(e) != 0;
    if (const char* e = std::getenv("CUMAT_CG_COOP")) s->coop = std::max(0, std::min(2, std::atoi(e)));
    if (const char* e = std::getenv("CUMAT_CG_CLUSTER")) s->cluster = std::atoi(e) != 0;
    if (const char* e = std::getenv("CUMAT_CG_FUSE")) s->fuse_p = std::atoi(e) != 0;
    if (const char* e = std::getenv("CUMAT_CG_GRAPH")) s->graph_loop = std::atoi(e) != 0;
    if (const char* e = std::getenv("CUMAT_CG_BF16_FALLBACK")) s->bf16_fallback = std::atoi(e) != 0;
    cmcg_status st = build_plan(s);
    if (st == CMCG_OK) st = dev_alloc(reinterpret_cast<void**>(&s->counters), 64);
    if (st == CMCG_OK && cudaMemsetAsync(s->counters, 0, 64, A->pat->ctx->stream) != cudaSuccess) st = fail(CMCG_ERR_CUDA, "memset");
    if (st != CMCG_OK) { cmcg_cg_destroy(s); return st; }
    // Jacobi is extracted at construction like the reference's DiagonalPreconditioner(A)
    if (precond == CMCG_PRECOND_JACOBI) {
        const void* d;
        st = get_dinv(s, A->dtype == CMCG_F64 ? CMCG_F64 : CMCG_F32, &d);
        if (st != CMCG_OK) { cmcg_cg_destroy(s); return st; }
    }
    *out = s;
    return CMCG_OK;
}

cmcg_status cmcg_cg_destroy(cmcg_solver s) {
    if (!s) return CMCG_OK;
    cudaSetDevice(s->A->pat->ctx->device);
    cudaStreamSynchronize(s->A->pat->ctx->stream);
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->graph) cudaGraphDestroy(s->graph);
    for (cudaStream_t st : s->aux_stream)
        if (st) cudaStreamDestroy(st);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    for (cudaEvent_t e : s->ev_join)
        if (e) cudaEventDestroy(e);
    if (s->gexec_mix) cudaGraphExecDestroy(s->gexec_mix);
    if (s->graph_mix) cudaGraphDestroy(s->graph_mix);
    for (void* p : {static_cast<void*>(s->d_order), static_cast<void*>(s->d_tile_row0), static_cast<void*>(s->d_seg_t0),
                    static_cast<void*>(s->d_seg_t1), static_cast<void*>(s->d_seg_sys), static_cast<void*>(s->d_cta_seg0),
                    static_cast<void*>(s->d_sys_seg0), static_cast<void*>(s->d_cseg_t0), static_cast<void*>(s->d_cseg_t1),
                    static_cast<void*>(s->d_cseg_sys), static_cast<void*>(s->d_ccta_seg0),
                    static_cast<void*>(s->d_csys_seg0), s->dinv[0], s->dinv[1], s->vec_ws, s->ref_ws, s->part_ws,
                    s->st_ws, static_cast<void*>(s->counters), s->mix_vals, static_cast<void*>(s->mix_s),
                    s->dia_vals, s->dia_plain})
        dev_free(p);
    if (s->host_io) cudaFreeHost(s->host_io);
    dev_free(s->fb_x);
    dev_free(s->fb_list);
    if (s->fb) cmcg_cg_destroy(s->fb);
    if (s->fb_mat) cmcg_matrix_destroy(s->fb_mat);
    cmcg_matrix A = s->A;
    delete s;
    matrix_release(A);
    return CMCG_OK;
}

cmcg_status cmcg_cg_set_tolerance(cmcg_solver s, double tol) {
    CMCG_REQUIRE(s, "cmcg_cg_set_tolerance: NULL solver");
    CMCG_REQUIRE(tol >= 0.0 && std::isfinite(tol), "cmcg_cg_set_tolerance: tolerance must be finite and >= 0");
    s->tol = tol;
    return CMCG_OK;
}

cmcg_status cmcg_cg_set_max_iterations(cmcg_solver s, int64_t max_iter) {
    CMCG_REQUIRE(s, "cmcg_cg_set_max_iterations: NULL solver");
    CMCG_REQUIRE(max_iter < INT32_MAX, "cmcg_cg_set_max_iterations: too large");
    s->max_iter = max_iter < 0 ? -1 : max_iter;
    return CMCG_OK;
}

cmcg_status cmcg_cg_get_settings(cmcg_solver s, double* tol, int64_t* max_iter) {
    CMCG_REQUIRE(s, "cmcg_cg_get_settings: NULL solver");
    if (tol) *tol = s->tol;
    if (max_iter) *max_iter = s->max_iter < 0 ? 2 * static_cast<int64_t>(s->max_sys_rows) : s->max_iter;
    return CMCG_OK;
}

cmcg_status cmcg_cg_set_path(cmcg_solver s, int32_t path) {
    CMCG_REQUIRE(s, "cmcg_cg_set_path: NULL solver");
    CMCG_REQUIRE(path == CMCG_PATH_AUTO || path == CMCG_PATH_PERSISTENT || path == CMCG_PATH_GRID ||
                     path == CMCG_PATH_PERSISTENT_GLOBAL,
                 "cmcg_cg_set_path: bad path");
    s->path = path == CMCG_PATH_PERSISTENT_GLOBAL ? CMCG_PATH_PERSISTENT : path;
    s->use_smem = path != CMCG_PATH_PERSISTENT_GLOBAL;
    return CMCG_OK;
}

cmcg_status cmcg_cg_set_refinement(cmcg_solver s, int32_t method, double delta) {
    CMCG_REQUIRE(s, "cmcg_cg_set_refinement: NULL solver");
    CMCG_REQUIRE(method == CMCG_REFINE_RELIABLE || method == CMCG_REFINE_RESTART, "cmcg_cg_set_refinement: bad method");
    CMCG_REQUIRE(delta >= 0.0 && delta < 1.0, "cmcg_cg_set_refinement: delta must be 0 (automatic) or in (0, 1)");
    s->refine_method = method;
    s->refine_delta = delta;
    return CMCG_OK;
}

cmcg_status cmcg_cg_solve(cmcg_solver s, int32_t vdt, const void* b, int32_t b_batches, const void* guess, void* x) {
    NvtxRange nvtx_("cmcg_cg_solve");
    CMCG_REQUIRE(s && b && x, "cmcg_cg_solve: NULL argument");
    CMCG_REQUIRE(b_batches >= 1, "cmcg_cg_solve: b_batches must be >= 1");
    CMCG_REQUIRE(s->A->batches == 1 || b_batches == 1 || b_batches == s->A->batches,
                 "cmcg_cg_solve: batch counts of matrix and rhs must match or be 1");
    CMCG_CUDA(cudaSetDevice(s->A->pat->ctx->device));
    CMCG_TRY(refresh_plan(s));
    const int32_t ob = std::max(s->A->batches, b_batches);
    CMCG_REQUIRE(static_cast<int64_t>(ob) * s->n_sys <= INT32_MAX / 2, "cmcg_cg_solve: too many systems");
    if (vdt == CMCG_F32)
        return solve_vt<float>(s, static_cast<const float*>(b), b_batches, static_cast<const float*>(guess), static_cast<float*>(x), ob);
    if (vdt == CMCG_F64)
        return solve_vt<double>(s, static_cast<const double*>(b), b_batches, static_cast<const double*>(guess), static_cast<double*>(x), ob);
    return fail(CMCG_ERR_INVALID_ARGUMENT, "cmcg_cg_solve: vector dtype must be F32 or F64");
}

cmcg_status cmcg_cg_solve_host(cmcg_solver s, int32_t vdt, const void* b_host, int32_t b_batches, const void* guess_host,
                               void* x_host) {
    NvtxRange nvtx_("cmcg_cg_solve_host");
    CMCG_REQUIRE(s && b_host && x_host, "cmcg_cg_solve_host: NULL argument");
    CMCG_REQUIRE(vdt == CMCG_F32 || vdt == CMCG_F64, "cmcg_cg_solve_host: vector dtype must be F32 or F64");
    CMCG_REQUIRE(b_batches >= 1, "cmcg_cg_solve_host: b_batches must be >= 1");
    cmcg_ctx ctx = s->A->pat->ctx;
    CMCG_CUDA(cudaSetDevice(ctx->device));
    const int32_t ob = std::max(s->A->batches, b_batches);
    const size_t es = dtype_size(vdt);
    const size_t nb = es * s->A->pat->rows * static_cast<size_t>(b_batches);
    const size_t nx = es * s->A->pat->rows * static_cast<size_t>(ob);
    // device staging: b | guess | x
    void* dbuf = nullptr;
    CMCG_TRY(dev_alloc(&dbuf, nb + 2 * nx + 512));
    char* db = static_cast<char*>(dbuf);
    char* dg = db + ((nb + 255) / 256) * 256;
    char* dx = dg + ((nx + 255) / 256) * 256;
    cudaStream_t st = ctx->stream;
    cmcg_status rc = CMCG_OK;
    if (cudaMemcpyAsync(db, b_host, nb, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = fail(CMCG_ERR_CUDA, "upload b");
    if (rc == CMCG_OK && guess_host && cudaMemcpyAsync(dg, guess_host, nx, cudaMemcpyHostToDevice, st) != cudaSuccess)
        rc = fail(CMCG_ERR_CUDA, "upload guess");
    if (rc == CMCG_OK) rc = cmcg_cg_solve(s, vdt, db, b_batches, guess_host ? dg : nullptr, dx);
    if (rc == CMCG_OK && cudaMemcpyAsync(x_host, dx, nx, cudaMemcpyDeviceToHost, st) != cudaSuccess) rc = fail(CMCG_ERR_CUDA, "download x");
    if (cudaStreamSynchronize(st) != cudaSuccess && rc == CMCG_OK) rc = fail(CMCG_ERR_CUDA, "solve failed");
    dev_free(dbuf);
    return rc;
}

static cmcg_status fetch_stats(cmcg_solver s, std::vector<int32_t>* it, std::vector<double>* err, std::vector<int32_t>* st,
                               std::vector<int32_t>* outer) {
    CMCG_REQUIRE(s->last_inst > 0, "no solve has been run");
    cudaStream_t stream = s->A->pat->ctx->stream;
    CMCG_CUDA(cudaStreamSynchronize(stream));
    const size_t n = s->last_inst;
    if (it) { it->resize(n); CMCG_CUDA(cudaMemcpy(it->data(), s->st.it, 4 * n, cudaMemcpyDeviceToHost)); }
    if (err) { err->resize(n); CMCG_CUDA(cudaMemcpy(err->data(), s->st.err, 8 * n, cudaMemcpyDeviceToHost)); }
    if (st) { st->resize(n); CMCG_CUDA(cudaMemcpy(st->data(), s->st.status, 4 * n, cudaMemcpyDeviceToHost)); }
    if (outer) { outer->resize(n); CMCG_CUDA(cudaMemcpy(outer->data(), s->st.outer, 4 * n, cudaMemcpyDeviceToHost)); }
    return CMCG_OK;
}

cmcg_status cmcg_cg_iterations(cmcg_solver s, int64_t* iterations) {
    CMCG_REQUIRE(s && iterations, "cmcg_cg_iterations: NULL argument");
    std::vector<int32_t> it;
    CMCG_TRY(fetch_stats(s, &it, nullptr, nullptr, nullptr));
    *iterations = it.empty() ? 0 : *std::max_element(it.begin(), it.end());
    return CMCG_OK;
}

cmcg_status cmcg_cg_error(cmcg_solver s, double* error) {
    CMCG_REQUIRE(s && error, "cmcg_cg_error: NULL argument");
    std::vector<double> e;
    CMCG_TRY(fetch_stats(s, nullptr, &e, nullptr, nullptr));
    double m = 0.0;
    for (double v : e) m = (std::isnan(v) || std::isnan(m)) ? NAN : std::max(m, v);
    *error = m;
    return CMCG_OK;
}

cmcg_status cmcg_cg_system_stats(cmcg_solver s, int32_t* iters, double* err, int32_t* status, int32_t* outer) {
    CMCG_REQUIRE(s, "cmcg_cg_system_stats: NULL solver");
    std::vector<int32_t> it, st, ou;
    std::vector<double> e;
    CMCG_TRY(fetch_stats(s, iters ? &it : nullptr, err ? &e : nullptr, status ? &st : nullptr, outer ? &ou : nullptr));
    if (iters) std::copy(it.begin(), it.end(), iters);
    if (err) std::copy(e.begin(), e.end(), err);
    if (status) std::copy(st.begin(), st.end(), status);
    if (outer) std::copy(ou.begin(), ou.end(), outer);
    return CMCG_OK;
}

}  // extern "C"

namespace {

cmcg_status solve_refined_impl(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_batches, double* x,
                               double outer_tol, int32_t max_outer);

// Takes the FP32-value re-solve of the listed instances: their rows of x and
// their statistics (one CTA per instance).
__global__ void k_take_fallback(const int32_t* __restrict__ list, int32_t n_list, InstState dst, InstState src,
                                const int32_t* __restrict__ row_off, int32_t n_sys, int32_t rows, double* __restrict__ x,
                                const double* __restrict__ xf) {
    for (int j = blockIdx.x; j < n_list; j += gridDim.x) {
        const int inst = list[j];
        const int b = inst / n_sys, sys = inst - b * n_sys;
        const int64_t o = static_cast<int64_t>(b) * rows;
        for (int i = row_off[sys] + threadIdx.x; i < row_off[sys + 1]; i += blockDim.x) x[o + i] = xf[o + i];
        if (threadIdx.x == 0) {
            dst.it[inst] = src.it[inst];
            dst.status[inst] = src.status[inst];
            dst.outer[inst] = src.outer[inst];
            dst.err[inst] = src.err[inst];
            dst.rr[inst] = src.rr[inst];
            dst.bb[inst] = src.bb[inst];
        }
    }
}

// BF16 inner values round the Jacobi-scaled matrix by up to 2^-9 relative;
// where that times the condition number approaches 1 the reliable updates
// stop contracting and the system ends unconverged. Such systems are solved
// again with the FP32 values of the outer matrix (converted once when the
// outer matrix is FP64) and their results replace the BF16 ones; the
// instances are reported by cmcg_cg_fallbacks.
cmcg_status bf16_fallback(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_batches, double* x, double outer_tol,
                          int32_t max_outer) {
    cmcg_ctx ctx = s->A->pat->ctx;
    const int32_t n = s->last_inst;
    s->fallback.assign(n, 0);
    std::vector<int32_t> st(n);
    CMCG_CUDA(cudaStreamSynchronize(ctx->stream));
    CMCG_CUDA(cudaMemcpy(st.data(), s->st.status, 4 * static_cast<size_t>(n), cudaMemcpyDeviceToHost));
    std::vector<int32_t> list;
    for (int32_t i = 0; i < n; ++i)
        if (st[i] != CMCG_SOLVE_CONVERGED && st[i] != CMCG_SOLVE_ZERO_RHS) list.push_back(i);
    if (list.empty()) return CMCG_OK;
    cmcg_matrix Af = Ao;
    if (Ao->dtype != CMCG_F32) {
        if (!s->fb_mat || s->fb_mat->version != Ao->version) {
            if (!s->fb_mat) CMCG_TRY(cmcg_matrix_create(Ao->pat, CMCG_F32, Ao->batches, &s->fb_mat));
            // FP64 values rounded to FP32 on the device (same layout and stride)
            CMCG_TRY(convert(ctx, Ao->dtype, Ao->d_vals, CMCG_F32, s->fb_mat->d_vals, Ao->stride * Ao->batches));
            s->fb_mat->version = Ao->version;   // tracks the source's values
        }
        Af = s->fb_mat;
    }
    if (!s->fb || s->fb->A != Af) {
        if (s->fb) cmcg_cg_destroy(s->fb);
        s->fb = nullptr;
        CMCG_TRY(cmcg_cg_create(Af, s->precond, &s->fb));
    }
    cmcg_solver f = s->fb;
    f->tol = s->tol;
    f->max_iter = s->max_iter;
    f->path = s->path;
    f->refine_method = s->refine_method;
    f->refine_delta = 0.0;   // the FP32 default
    const size_t nv = static_cast<size_t>(s->A->pat->rows) * std::max(s->A->batches, b_batches);
    CMCG_TRY(ensure_buffer(reinterpret_cast<void**>(&s->fb_x), &s->fb_x_bytes, nv * sizeof(double)));
    CMCG_TRY(solve_refined_impl(f, Ao, b, b_batches, s->fb_x, outer_tol, max_outer));
    CMCG_TRY(ensure_buffer(reinterpret_cast<void**>(&s->fb_list), &s->fb_list_bytes, list.size() * sizeof(int32_t)));
    CMCG_CUDA(cudaMemcpyAsync(s->fb_list, list.data(), list.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    const int grid = static_cast<int>(std::min<size_t>(list.size(), 65535));
    k_take_fallback<<<grid, 256, 0, ctx->stream>>>(s->fb_list, static_cast<int32_t>(list.size()), s->st, f->st,
                                                   s->A->pat->d_row_off, s->n_sys, s->A->pat->rows, x, s->fb_x);
    count_launch();
    CMCG_CHECK_LAUNCH();
    // the list upload must finish before the host vector goes away
    CMCG_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int32_t i : list) s->fallback[i] = 1;
    log_msg(1, "refined solve: %zu of %d systems did not converge with BF16 values and were solved with FP32 values",
            list.size(), n);
    return CMCG_OK;
}

}  // namespace

extern "C" {

cmcg_status cmcg_cg_solve_refined(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_batches, double* x,
                                  double outer_tol, int32_t max_outer) {
    NvtxRange nvtx_("cmcg_cg_solve_refined");
    CMCG_REQUIRE(s && b && x, "cmcg_cg_solve_refined: NULL argument");
    if (!Ao) Ao = s->A;
    s->fallback.clear();
    CMCG_TRY(solve_refined_impl(s, Ao, b, b_batches, x, outer_tol, max_outer));
    if (s->A->dtype == CMCG_BF16 && s->bf16_fallback) CMCG_TRY(bf16_fallback(s, Ao, b, b_batches, x, outer_tol, max_outer));
    return CMCG_OK;
}

cmcg_status cmcg_cg_fallbacks(cmcg_solver s, int32_t* flags, int64_t* count) {
    CMCG_REQUIRE(s, "cmcg_cg_fallbacks: NULL solver");
    CMCG_REQUIRE(s->last_inst > 0, "cmcg_cg_fallbacks: no solve has been run");
    int64_t c = 0;
    for (int32_t i = 0; i < s->last_inst; ++i) {
        const int32_t v = (s->last_refined && i < static_cast<int32_t>(s->fallback.size())) ? s->fallback[i] : 0;
        if (flags) flags[i] = v;
        c += v;
    }
    if (count) *count = c;
    return CMCG_OK;
}

}  // extern "C"

namespace {

cmcg_status solve_refined_impl(cmcg_solver s, cmcg_matrix Ao, const double* b, int32_t b_batches, double* x,
                               double outer_tol, int32_t max_outer) {
    CMCG_REQUIRE(s && b && x, "cmcg_cg_solve_refined: NULL argument");
    if (!Ao) Ao = s->A;
    CMCG_REQUIRE(Ao->pat == s->A->pat, "cmcg_cg_solve_refined: outer matrix must share the solver's pattern");
    CMCG_REQUIRE(Ao->batches == s->A->batches, "cmcg_cg_solve_refined: outer matrix batch count differs");
    CMCG_REQUIRE(Ao->dtype == CMCG_F32 || Ao->dtype == CMCG_F64, "cmcg_cg_solve_refined: outer values must be F32 or F64");
    CMCG_REQUIRE(s->A->dtype == CMCG_F32 || s->A->dtype == CMCG_BF16, "cmcg_cg_solve_refined: inner values must be F32 or BF16");
    CMCG_REQUIRE(outer_tol > 0.0 && max_outer >= 1, "cmcg_cg_solve_refined: need outer_tol > 0 and max_outer >= 1");
    CMCG_REQUIRE(b_batches >= 1 && (s->A->batches == 1 || b_batches == 1 || b_batches == s->A->batches),
                 "cmcg_cg_solve_refined: batch counts must match or be 1");
    CMCG_CUDA(cudaSetDevice(s->A->pat->ctx->device));
    CMCG_TRY(refresh_plan(s));
    const int32_t ob = std::max(s->A->batches, b_batches);
    const int fmt = s->A->pat->format;
    int32_t path = choose_path(s, ob * s->n_sys, s->use_smem && s->refine_method == CMCG_REFINE_RELIABLE);
    // the grid path's reliable-update solver needs the sliced layout (CSR)
    const bool grid_mixed = fmt == CMCG_CSR && s->refine_method == CMCG_REFINE_RELIABLE;
    // packed systems run persistent (one CTA per system, vectors in shared
    // memory where they fit) unless they are too large for shared memory and
    // the grid solver handles them
    if (s->n_sys > 1 && s->path == CMCG_PATH_AUTO && (!grid_mixed || s->max_sys_rows <= kSmemMaxRows))
        path = CMCG_PATH_PERSISTENT;
    if (path == CMCG_PATH_GRID) {
        if (grid_mixed) {
            if (s->A->dtype == CMCG_F32)
                return Ao->dtype == CMCG_F64 ? refined_grid_mixed<float, double>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer)
                                             : refined_grid_mixed<float, float>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer);
            return Ao->dtype == CMCG_F64
                       ? refined_grid_mixed<__nv_bfloat16, double>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer)
                       : refined_grid_mixed<__nv_bfloat16, float>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer);
        }
        CMCG_REQUIRE(s->n_sys == 1, "cmcg_cg_solve_refined: the grid path's restart refinement takes one system per batch");
        return refined_grid(s, Ao, b, b_batches, x, ob, outer_tol, max_outer);
    }
    if (s->A->dtype == CMCG_F32)
        return fmt == CMCG_CSR ? refined_mi<float, CMCG_CSR>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer)
                               : refined_mi<float, CMCG_ELLPACK>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer);
    return fmt == CMCG_CSR ? refined_mi<__nv_bfloat16, CMCG_CSR>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer)
                           : refined_mi<__nv_bfloat16, CMCG_ELLPACK>(s, Ao, b, b_batches, x, ob, outer_tol, max_outer);
}

}  // namespace

extern "C" {

cmcg_status cmcg_cg_adjoint(cmcg_solver s, cmcg_matrix Ao, const double* x, const double* gx, int32_t batches, double* gb,
                            double* gA, double outer_tol, int32_t max_outer) {
    NvtxRange nvtx_("cmcg_cg_adjoint");
    CMCG_REQUIRE(s && x && gx && gb, "cmcg_cg_adjoint: NULL argument");
    // A symmetric: A^T lambda = gx is A lambda = gx, solved by the same fused CG
    CMCG_TRY(cmcg_cg_solve_refined(s, Ao, gx, batches, gb, outer_tol, max_outer));
    if (gA) {
        // dL/dA_ij = -lambda_i x_j on the pattern (one sampled outer product)
        const int32_t ob = std::max(s->A->batches, batches);
        CMCG_TRY(sddmm_dispatch(s->A, CMCG_F64, -1.0, gb, ob, x, ob, gA, ob));
    }
    return CMCG_OK;
}

}  // extern "C"
