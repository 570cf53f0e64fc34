// Grid path, cooperative: the whole PCG loop of a few large systems in one
// launch over all SMs (one 1024-thread CTA per SM), with two grid barriers per
// iteration instead of kernel boundaries.
//
// Iteration k (reference loop cuMat/src/ConjugateGradient.h:180-203):
//   phase 1: p_k = z + beta p_{k-1} on this CTA's rows (written to the other
//            of two p buffers), q = A p_k with the gathered p_k(j) formed on
//            the fly from z(j) = M^-1 r(j) and p_{k-1}(j), partial p_k.q
//   barrier: alpha = r.z / p.q (last CTA to arrive)
//   phase 2: x += alpha p_k, r -= alpha q, partials |r|^2 and r.z
//   barrier: convergence, beta (last CTA to arrive)
// Forming p_k inside the product removes the separate p update pass and its
// barrier; the owner and every gatherer evaluate p_k(j) with the same
// expression, so they agree bit for bit. When a CTA's rows lie in one system
// and all their column indices in a window [c0, c1) that fits the CTA's
// shared memory (stencils: the rows plus a halo as wide as the largest
// offset), phase 1 first forms p_k over the whole window with coalesced
// loads into shared memory and the product gathers from there: three
// coalesced vector reads per window entry instead of three L2 gathers per
// matrix entry, with the same expression and therefore the same values. The last CTA to reach a barrier adds
// the phase's per-segment partials of every instance in a fixed order and
// writes the scalars (alpha, beta, statuses, running count) before releasing
// the others, so every CTA sees the same values and leaves the loop in the
// same iteration. Vectors and scalars written by other CTAs are read through
// L2 (ld.global.cg); the matrix and the inverse diagonal through the read-only
// path.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "cg_grid.cuh"
#include "grid_sync.cuh"

namespace cmcg {
namespace {

template <typename VT>
struct WindowX {     // gathers from the shared-memory window [c0, c0 + width)
    const VT* w;
    int c0, width;
    // every stored entry's column lies in the window; a padding slot of the
    // sliced layout (value 0) may name a column outside it and reads an
    // entry of the window instead
    __device__ __forceinline__ VT operator()(int c) const { return w[min(max(c - c0, 0), width - 1)]; }
};

// entries of p_k the window of one CTA may hold (dynamic shared memory)
constexpr int kCoopWindowBytes = 192 * 1024;

template <typename VT>
struct CoherentX {   // gathers of a vector that other CTAs of the launch write
    const VT* __restrict__ x;
    __device__ __forceinline__ VT operator()(int c) const { return __ldcg(x + c); }
};

// p_k(j) = z(j) + beta p_{k-1}(j), z = M^-1 r; one expression for owner and gatherers
template <typename VT>
__device__ __forceinline__ VT p_next(VT dinv, VT r, VT pprev, VT beta) {
    return fma(beta, pprev, dinv * r);
}

template <typename VT>
struct PNextX {      // gathers of p_k formed from r, M^-1 and p_{k-1}
    const VT* __restrict__ r;
    const VT* __restrict__ dinv;   // null: identity
    const VT* __restrict__ pprev;
    VT beta;
    __device__ __forceinline__ VT operator()(int c) const {
        const VT d = dinv ? __ldg(dinv + c) : VT(1);
        return p_next(d, __ldcg(r + c), __ldcg(pprev + c), beta);
    }
};

template <typename VT>
struct CoopArgs {
    GridSync* sync;
    int32_t* err;
    int32_t n_inst;
    VT* p_alt;   // second p buffer, [batch][rows]
    BarrierLimits lim;
    int32_t window;   // stage p_k over each CTA's column window (else form it inside the gathers)
};

// Totals of NV partial arrays over the segments of instance `inst` (whole CTA,
// fixed order; every thread receives them).
template <typename VT, typename MT, int NV>
__device__ __forceinline__ void coop_inst_sum(const SolveArgs<VT, MT>& a, VT* const (&part)[NV], int inst, VT (&tot)[NV],
                                              VT* red) {
    const int b = inst / a.n_sys, s = inst - b * a.n_sys;
    const int64_t base = static_cast<int64_t>(b) * a.n_seg + a.sys_seg0[s];
    const int count = a.sys_seg0[s + 1] - a.sys_seg0[s];
#pragma unroll
    for (int j = 0; j < NV; ++j) tot[j] = VT(0);
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
#pragma unroll
        for (int j = 0; j < NV; ++j) tot[j] += __ldcg(part[j] + base + i);
    }
    block_sum<VT, NV>(tot, red);
}

template <typename VT>
__device__ __forceinline__ VT ld_cg_scalar(const double* p) { return static_cast<VT>(__ldcg(p)); }

// This CTA's segments (batch-independent part), cached in shared memory for
// the whole launch.
struct SegCache {
    int s, seg, sr0, r0, r1, sys_seg0;
};

template <typename VT, typename MT, int FMT>
__global__ void __launch_bounds__(kCoopThreads, 1) k_coop_cg(SolveArgs<VT, MT> a, CoopArgs<VT> c) {
    extern __shared__ __align__(16) unsigned char coop_smem[];
    VT* const win = reinterpret_cast<VT*>(coop_smem);
    __shared__ VT red[2 * (kCoopThreads / 32)];
    __shared__ SegCache segs[kCoopMaxSegs];
    __shared__ int nseg_s;
    __shared__ int win_lo, win_hi, win_sys;
    VT* const parts2[2] = {a.part1, a.part2};
    VT* const parts1[1] = {a.part1};
    const VT tol = static_cast<VT>(a.tol);
    unsigned long long epoch = 0;   // barriers passed (the same count in every CTA)

    if (threadIdx.x == 0) nseg_s = min(a.cta_seg0[blockIdx.x + 1] - a.cta_seg0[blockIdx.x], kCoopMaxSegs);
    __syncthreads();
    const int nseg = nseg_s;
    if (threadIdx.x < nseg) {
        const int seg = a.cta_seg0[blockIdx.x] + threadIdx.x;
        const SegInfo g = seg_info(a, 0, seg);
        segs[threadIdx.x] = SegCache{g.s, seg, g.sr0, g.r0, g.r1, a.sys_seg0[g.s]};
    }
    __syncthreads();
    // the column window of this CTA's rows (CSR patterns whose CTA rows lie in
    // one system); win_sys < 0: gather from global memory
    if (threadIdx.x == 0) {
        // the window holds the CTA's own rows (whose p_k the product emits)
        // and every column its rows reference
        win_lo = nseg > 0 ? segs[0].r0 : 0;
        win_hi = nseg > 0 ? segs[nseg - 1].r1 - 1 : -1;
        win_sys = (FMT == CMCG_CSR && nseg > 0 && nseg == a.cta_seg0[blockIdx.x + 1] - a.cta_seg0[blockIdx.x])
                      ? segs[0].s : -1;
        for (int k = 1; k < nseg; ++k)
            if (segs[k].s != win_sys) win_sys = -1;
    }
    __syncthreads();
    if (FMT == CMCG_CSR && win_sys >= 0) {
        int lo = INT32_MAX, hi = -1;
        for (int k = 0; k < nseg; ++k)
            for (int e = __ldg(a.m.rp + segs[k].r0) + threadIdx.x; e < __ldg(a.m.rp + segs[k].r1); e += kCoopThreads) {
                const int cidx = __ldg(a.m.ci + e);
                lo = min(lo, cidx);
                hi = max(hi, cidx);
            }
        atomicMin(&win_lo, lo);
        atomicMax(&win_hi, hi);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int sr0 = a.row_off[win_sys], send = a.row_off[win_sys + 1];
            const bool fits = win_hi >= win_lo && win_lo >= sr0 && win_hi < send &&
                              static_cast<int64_t>(win_hi - win_lo + 1) * static_cast<int64_t>(sizeof(VT)) <= kCoopWindowBytes;
            if (!fits) win_sys = -1;
        }
        __syncthreads();
    }
    const bool use_win = c.window && win_sys >= 0;
    const int wlo = win_lo, whi = win_hi + 1;

// loop over this CTA's (batch, segment) pairs: b_, g (SegCache), inst, pidx, vo
#define CMCG_COOP_SEGMENTS                                                        \
    for (int b_ = 0; b_ < a.ob; ++b_)                                             \
        for (int k_ = 0; k_ < nseg; ++k_)                                         \
            if (const SegCache g = segs[k_]; true)                                \
                if (const int inst = b_ * a.n_sys + g.s, pidx = b_ * a.n_seg + g.seg; true) \
                    if (const int64_t vo = static_cast<int64_t>(b_) * a.rows; true)

    // init A: x = guess or 0, r = b - A x; partials |b|^2, |r|^2
    CMCG_COOP_SEGMENTS {
        const VT* bv = a.b + (a.b_b == 1 ? 0 : vo);
        VT* x = a.x + vo;
        VT* r = a.r + vo;
        VT acc[2] = {VT(0), VT(0)};
        const VT* gv = a.guess ? a.guess + (a.g_b == 1 ? 0 : vo) : nullptr;
        if (gv) {
            const auto A = inst_matrix<MT, FMT>(a.m, b_);
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
            for (int i = g.r0 + threadIdx.x; i < g.r1; i += kCoopThreads) {
                const VT bi = bv[i];
                r[i] = bi;
                x[i] = VT(0);
                acc[0] += bi * bi;
                acc[1] += bi * bi;
            }
        }
        block_sum<VT, 2>(acc, red);
        if (threadIdx.x == 0) { a.part1[pidx] = acc[0]; a.part2[pidx] = acc[1]; }
    }
    if (!grid_barrier(c.sync, c.err, c.lim, epoch, [&] {
            for (int inst = 0; inst < c.n_inst; ++inst) {
                VT tot[2];
                coop_inst_sum<VT, MT, 2>(a, parts2, inst, tot, red);
                if (threadIdx.x == 0) {
                    const VT bb = tot[0], rr = tot[1];
                    a.st.bb[inst] = bb;
                    a.st.rr[inst] = rr;
                    a.st.it[inst] = 0;
                    a.st.outer[inst] = 0;
                    a.st.beta[inst] = 0.0;
                    int32_t status = ST_RUNNING;
                    if ((a.abs_zero_test && bb < tol * tol) || bb == VT(0)) status = CMCG_SOLVE_ZERO_RHS;
                    else if (!finite_(bb) || !finite_(rr)) status = CMCG_SOLVE_NON_FINITE;
                    else if (rr < tol * tol * bb) status = CMCG_SOLVE_CONVERGED;
                    a.st.status[inst] = status;
                }
            }
        }))
        return;

    // init B: zero x of zero-rhs systems; p_{-1} = 0 (with beta = 0, p_0 = z);
    // partial r.z
    CMCG_COOP_SEGMENTS {
        const int32_t st = ld_status(a.st.status + inst);
        VT acc[1] = {VT(0)};
        if (st == CMCG_SOLVE_ZERO_RHS) {
#pragma unroll 4
            for (int i = g.r0 + threadIdx.x; i < g.r1; i += kCoopThreads) a.x[vo + i] = VT(0);
        } else if (st == ST_RUNNING) {
            const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
#pragma unroll 4
            for (int i = g.r0 + threadIdx.x; i < g.r1; i += kCoopThreads) {
                const VT ri = a.r[vo + i];
                const VT zi = dinv ? dinv[i] * ri : ri;
                a.p[vo + i] = VT(0);
                acc[0] += ri * zi;
            }
        }
        block_sum<VT, 1>(acc, red);
        if (threadIdx.x == 0) a.part1[pidx] = acc[0];
    }
    if (!grid_barrier(c.sync, c.err, c.lim, epoch, [&] {
            int32_t running = 0;
            for (int inst = 0; inst < c.n_inst; ++inst) {
                VT tot[1];
                coop_inst_sum<VT, MT, 1>(a, parts1, inst, tot, red);
                if (threadIdx.x == 0 && ld_status(a.st.status + inst) == ST_RUNNING) {
                    const VT rz = tot[0];
                    a.st.rz[inst] = rz;
                    int32_t status = ST_RUNNING;
                    if (!finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
                    else if (!(rz > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
                    a.st.status[inst] = status;
                    running += status == ST_RUNNING;
                }
            }
            if (threadIdx.x == 0) *a.active = running;
        }))
        return;

    VT* pprev = a.p;
    VT* pcur = c.p_alt;
    for (int32_t loop = 0; *reinterpret_cast<volatile int32_t*>(a.active) > 0 && loop < a.loop_cap; ++loop) {
        // phase 1: p_k = z + beta p_{k-1}; q = A p_k; partial p_k.q
        if (use_win) {
            // one system: stage p_k over the window, then the product
            for (int b_ = 0; b_ < a.ob; ++b_) {
                const int inst = b_ * a.n_sys + win_sys;
                const int64_t vo = static_cast<int64_t>(b_) * a.rows;
                const VT beta = ld_cg_scalar<VT>(a.st.beta + inst);
                const bool running = ld_status(a.st.status + inst) == ST_RUNNING;
                const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
                const VT* rv = a.r + vo;
                const VT* pp = pprev + vo;
                if (running) {
                    for (int j = wlo + threadIdx.x; j < whi; j += kCoopThreads)
                        win[j - wlo] = p_next(dinv ? __ldg(dinv + j) : VT(1), __ldcg(rv + j), __ldcg(pp + j), beta);
                }
                __syncthreads();
                for (int k_ = 0; k_ < nseg; ++k_) {
                    const SegCache g = segs[k_];
                    const int pidx = b_ * a.n_seg + g.seg;
                    VT acc[1] = {VT(0)};
                    if (running) {
                        VT* pc = pcur + vo;
                        VT* q = a.q + vo;
                        const auto A = inst_matrix<MT, FMT>(a.m, b_);
                        cta_rows4_seg<VT>(A, g.s, g.sr0, g.r0 - g.sr0, g.r1 - g.r0, WindowX<VT>{win, wlo, whi - wlo},
                                          [&](int row, VT v) {
                                              const VT pk = win[row - wlo];
                                              pc[row] = pk;
                                              q[row] = v;
                                              acc[0] += pk * v;
                                          });
                    }
                    block_sum<VT, 1>(acc, red);
                    if (threadIdx.x == 0) a.part1[pidx] = acc[0];
                }
            }
        } else {
        CMCG_COOP_SEGMENTS {
            const VT beta = ld_cg_scalar<VT>(a.st.beta + inst);
            const int32_t st = ld_status(a.st.status + inst);
            VT acc[1] = {VT(0)};
            if (st == ST_RUNNING) {
                const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
                const VT* rv = a.r + vo;
                const VT* pp = pprev + vo;
                VT* pc = pcur + vo;
                VT* q = a.q + vo;
                const auto A = inst_matrix<MT, FMT>(a.m, b_);
                cta_rows4_seg<VT>(A, g.s, g.sr0, g.r0 - g.sr0, g.r1 - g.r0, PNextX<VT>{rv, dinv, pp, beta},
                                 [&](int row, VT v) {
                                     const VT pk = p_next(dinv ? __ldg(dinv + row) : VT(1), rv[row], pp[row], beta);
                                     pc[row] = pk;
                                     q[row] = v;
                                     acc[0] += pk * v;
                                 });
            }
            block_sum<VT, 1>(acc, red);
            if (threadIdx.x == 0) a.part1[pidx] = acc[0];
        }
        }
        if (!grid_barrier(c.sync, c.err, c.lim, epoch, [&] {
                int32_t running = 0;
                for (int inst = 0; inst < c.n_inst; ++inst) {
                    VT tot[1];
                    coop_inst_sum<VT, MT, 1>(a, parts1, inst, tot, red);
                    if (threadIdx.x == 0 && ld_status(a.st.status + inst) == ST_RUNNING) {
                        const VT pq = tot[0];
                        const VT alpha = ld_cg_scalar<VT>(a.st.rz + inst) / pq;
                        int32_t status = ST_RUNNING;
                        if (!finite_(pq) || !finite_(alpha)) status = CMCG_SOLVE_NON_FINITE;
                        else if (!(pq > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
                        a.st.status[inst] = status;
                        a.st.alpha[inst] = alpha;
                        running += status == ST_RUNNING;
                    }
                }
                if (threadIdx.x == 0) *a.active = running;
            }))
            return;

        // phase 2: x += alpha p_k, r -= alpha q; partials |r|^2, r.z
        CMCG_COOP_SEGMENTS {
            const VT alpha = ld_cg_scalar<VT>(a.st.alpha + inst);
            const int32_t st = ld_status(a.st.status + inst);
            VT acc[2] = {VT(0), VT(0)};
            if (st == ST_RUNNING) {
                const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
                const VT* pc = pcur + vo;
#pragma unroll 4
                for (int i = g.r0 + threadIdx.x; i < g.r1; i += kCoopThreads) {
                    a.x[vo + i] += alpha * pc[i];
                    const VT ri = a.r[vo + i] - alpha * a.q[vo + i];
                    a.r[vo + i] = ri;
                    const VT zi = dinv ? dinv[i] * ri : ri;
                    acc[0] += ri * ri;
                    acc[1] += ri * zi;
                }
            }
            block_sum<VT, 2>(acc, red);
            if (threadIdx.x == 0) { a.part1[pidx] = acc[0]; a.part2[pidx] = acc[1]; }
        }
        if (!grid_barrier(c.sync, c.err, c.lim, epoch, [&] {
                int32_t running = 0;
                for (int inst = 0; inst < c.n_inst; ++inst) {
                    VT tot[2];
                    coop_inst_sum<VT, MT, 2>(a, parts2, inst, tot, red);
                    if (threadIdx.x == 0 && ld_status(a.st.status + inst) == ST_RUNNING) {
                        const VT rr = tot[0], rzn = tot[1];
                        const VT bb = ld_cg_scalar<VT>(a.st.bb + inst);
                        a.st.rr[inst] = rr;
                        const int b = inst / a.n_sys, s = inst - b * a.n_sys;
                        const int n = a.row_off[s + 1] - a.row_off[s];
                        int32_t status = ST_RUNNING;
                        if (!finite_(rr) || !finite_(rzn)) status = CMCG_SOLVE_NON_FINITE;
                        else if (rr < tol * tol * bb) status = CMCG_SOLVE_CONVERGED;
                        else if (!(rzn > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
                        else {
                            a.st.beta[inst] = rzn / ld_cg_scalar<VT>(a.st.rz + inst);
                            a.st.rz[inst] = rzn;
                            const int32_t it = ld_status(a.st.it + inst) + 1;
                            a.st.it[inst] = it;
                            if (it >= sys_max_iter(a.max_iter, n)) status = CMCG_SOLVE_MAX_ITER;
                        }
                        a.st.status[inst] = status;
                        running += status == ST_RUNNING;
                    }
                }
                if (threadIdx.x == 0) *a.active = running;
            }))
            return;
        VT* t = pprev;
        pprev = pcur;
        pcur = t;
    }
#undef CMCG_COOP_SEGMENTS
}

}  // namespace

template <typename VT, typename MT, int FMT>
cmcg_status coop_cg_occupancy(int* ctas_per_sm) {
    CMCG_CUDA(cudaFuncSetAttribute(k_coop_cg<VT, MT, FMT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kCoopWindowBytes));
    CMCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, k_coop_cg<VT, MT, FMT>, kCoopThreads,
                                                            kCoopWindowBytes));
    return CMCG_OK;
}

template <typename VT, typename MT, int FMT>
cmcg_status coop_cg_launch(const SolveArgs<VT, MT>& a, void* sync, int32_t* err, int n_inst, VT* p_alt, int grid,
                           cudaStream_t st) {
    SolveArgs<VT, MT> args = a;
    // the barrier's wait limit; CUMAT_TEST_GRID_SPINS / CUMAT_TEST_GRID_EXTRA
    // (tests of the bounded wait) set a short limit and an arrival that never
    // comes
    BarrierLimits lim{kGridBarrierSpins, 0u};
    if (const char* e = std::getenv("CUMAT_TEST_GRID_SPINS")) lim.spins = std::max(1LL, std::atoll(e));
    if (const char* e = std::getenv("CUMAT_TEST_GRID_EXTRA")) lim.extra = static_cast<unsigned>(std::max(0, std::atoi(e)));
    // CUMAT_CG_COOP_WINDOW=0 forms p_k inside the gathers instead of staging it
    int32_t window = 1;
    if (const char* e = std::getenv("CUMAT_CG_COOP_WINDOW")) window = std::atoi(e) != 0;
    CoopArgs<VT> c{static_cast<GridSync*>(sync), err, n_inst, p_alt, lim, window};
    void* params[] = {&args, &c};
    CMCG_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_coop_cg<VT, MT, FMT>), grid, kCoopThreads,
                                          params, kCoopWindowBytes, st));
    return CMCG_OK;
}

#define CMCG_COOP_INSTANTIATE(VT, MT, FMT)                                                              \
    template cmcg_status coop_cg_occupancy<VT, MT, FMT>(int*);                                          \
    template cmcg_status coop_cg_launch<VT, MT, FMT>(const SolveArgs<VT, MT>&, void*, int32_t*, int, VT*, int, \
                                                     cudaStream_t);
#define CMCG_COOP_FORMATS(VT, MT)           \
    CMCG_COOP_INSTANTIATE(VT, MT, CMCG_CSR) \
    CMCG_COOP_INSTANTIATE(VT, MT, CMCG_ELLPACK)
CMCG_COOP_FORMATS(float, float)
CMCG_COOP_FORMATS(float, double)
CMCG_COOP_FORMATS(float, __nv_bfloat16)
CMCG_COOP_FORMATS(double, float)
CMCG_COOP_FORMATS(double, double)
CMCG_COOP_FORMATS(double, __nv_bfloat16)

}  // namespace cmcg
