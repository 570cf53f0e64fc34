// Grid-path PCG on thread-block clusters: systems too large for one CTA but
// small enough for the shared memory of one cluster (up to 16 CTAs of 1024
// threads on B200) are solved by one cluster each, without grid barriers.
//
// CTA k of a cluster owns the 2^lg rows [k 2^lg, (k + 1) 2^lg) of its system
// and keeps their p, q, r, x and inverse diagonal in its shared memory (x is
// written back at the end). The product reads the values from global memory
// (L2) in the pattern's diagonal layout for stencil patterns (no column
// indices), else in the sliced layout, and gathers p from the CTA that owns
// each column through distributed shared memory (the column's owner is a
// shift of its local row). A scalar (p.q, |r|^2, r.z) is summed per CTA, each
// CTA writes its partial into every CTA's shared memory, and after one cluster
// barrier every CTA adds the partials in rank order, so all CTAs hold the same
// scalars and take the same decisions. An iteration has three cluster
// barriers: p published, p.q summed, |r|^2 and r.z summed. The algorithm,
// early-outs, statuses and iteration count are those of the one-CTA solver
// (reference cuMat/src/ConjugateGradient.h:123-206).
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include <cooperative_groups.h>

#include "cg_cluster.cuh"
#include "cg_dev.cuh"
#include "objects.h"

namespace cmcg {
namespace {

namespace cgrp = cooperative_groups;

// p of the instance: column c (a global row of the system starting at r0)
// lives at (c - r0) mod 2^lg in CTA (c - r0) >> lg of the cluster
template <typename VT>
struct ClusterP {
    const VT* p;   // this CTA's slice (shared memory)
    int r0, lg, rank;
    __device__ __forceinline__ VT operator()(int c) const {
        const int l = c - r0;
        const int owner = l >> lg;
        const int idx = l & ((1 << lg) - 1);
        if (owner == rank) return p[idx];
        return cgrp::this_cluster().map_shared_rank(p, owner)[idx];
    }
};

// NV CTA totals summed over the cluster (see the file comment); part is this
// CTA's [NV][kClusterMaxCtas] array, written by every CTA of the cluster.
// Every thread gets the sums; one cluster barrier.
template <typename VT, int NV>
__device__ __forceinline__ void cluster_sum(VT (&v)[NV], VT* red, VT* part, int rank, int ctas) {
    block_sum<VT, NV>(v, red);
    cgrp::cluster_group cl = cgrp::this_cluster();
    if (static_cast<int>(threadIdx.x) < ctas) {
        VT* dst = cl.map_shared_rank(part, static_cast<int>(threadIdx.x));
#pragma unroll
        for (int j = 0; j < NV; ++j) dst[j * kClusterMaxCtas + rank] = v[j];
    }
    cl.sync();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        VT t = VT(0);
        for (int k = 0; k < ctas; ++k) t += part[j * kClusterMaxCtas + k];
        v[j] = t;
    }
}

// Thread-per-row product over the CTA's local rows [lo, lo + cnt) of system s
// (lo a multiple of 32): two rows per thread in flight (the 64-register budget
// of 1024-thread CTAs); f(global row, value) in increasing row order per thread.
template <typename VT, typename MT, int FMT, typename XF, typename F>
__device__ __forceinline__ void cluster_rows(const InstMatrix<MT, FMT>& A, int s, int r0, int lo, int cnt, const XF& xf,
                                             F&& f) {
    const int T = blockDim.x;
    for (int ib = threadIdx.x; ib < cnt; ib += 2 * T) {
        const int ii[2] = {lo + ib, lo + ib + T};
        const bool ok[2] = {true, ib + T < cnt};
        VT v[2];
        row_products<VT, 2>(A.rm, s, r0, ii, ok, xf, v);
        f(r0 + ii[0], v[0]);
        if (ok[1]) f(r0 + ii[1], v[1]);
    }
}

// The same over the diagonal layout (ND diagonals per system, ascending
// offsets, the row's CSR order): the values of both rows are loaded before
// the first gather; a column index is clamped into the system, where a zero
// value meets it.
template <typename VT, typename MT, int ND, typename XF, typename F>
__device__ __forceinline__ void cluster_dia_rows(const MT* __restrict__ v, const int (&off)[ND], int r0, int n, int lo,
                                                 int cnt, const XF& xf, F&& f) {
    const int T = blockDim.x;
    for (int ib = threadIdx.x; ib < cnt; ib += 2 * T) {
        const bool ok1 = ib + T < cnt;
        const int ii[2] = {lo + ib, ok1 ? lo + ib + T : lo + ib};
        MT w[2][ND];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const MT* vr = v + static_cast<int64_t>(ii[k] / kDiaBlockRows) * ND * kDiaBlockRows + ii[k] % kDiaBlockRows;
#pragma unroll
            for (int d = 0; d < ND; ++d) w[k][d] = vr[d * kDiaBlockRows];
        }
        VT acc[2] = {VT(0), VT(0)};
#pragma unroll
        for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int k = 0; k < 2; ++k)
                acc[k] = fma(mval<VT>(w[k][d]), xf(r0 + min(max(ii[k] + off[d], 0), n - 1)), acc[k]);
        f(r0 + ii[0], acc[0]);
        if (ok1) f(r0 + ii[1], acc[1]);
    }
}

struct ClusterArgs {
    int32_t ctas;   // CTAs per cluster
    int32_t lg;     // log2 of the rows per CTA
};

template <typename VT, typename MT, int FMT, int ND>
__global__ void __launch_bounds__(kClusterThreads, 1) k_cluster_cg(SolveArgs<VT, MT> a, ClusterArgs c) {
    extern __shared__ __align__(16) unsigned char cl_smem[];
    const int R = 1 << c.lg;
    VT* const p = reinterpret_cast<VT*>(cl_smem);
    VT* const q = p + R;
    VT* const r = q + R;
    VT* const x = r + R;
    VT* const dv = x + R;   // inverse diagonal (Jacobi)
    __shared__ VT red[2 * (kClusterThreads / 32)];
    // partial sums written by the cluster's CTAs: A for p.q and r.z, B for
    // |b|^2, |r|^2 and r.z (each reuse of a buffer is a barrier after its reads)
    __shared__ VT partA[2 * kClusterMaxCtas];
    __shared__ VT partB[2 * kClusterMaxCtas];
    cgrp::cluster_group cl = cgrp::this_cluster();
    const int rank = static_cast<int>(cl.block_rank());
    const int ctas = c.ctas;
    const int inst = blockIdx.x / ctas;
    const int bi = inst / a.n_sys, s = inst - bi * a.n_sys;
    const int r0 = a.row_off[s], n = a.row_off[s + 1] - r0;
    const int lo = rank << c.lg;
    const int cnt = max(0, min(R, n - lo));
    const int T = blockDim.x, tid = threadIdx.x;
    const int64_t vo = static_cast<int64_t>(bi) * a.rows;
    const auto A = inst_matrix<MT, FMT>(a.m, bi);
    int off[ND > 0 ? ND : 1];
    const MT* dvals = nullptr;
    if constexpr (ND > 0) {
#pragma unroll
        for (int j = 0; j < ND; ++j) off[j] = __ldg(a.dia.off + s * kDiaMax + j);
        dvals = a.dia.vals + (a.dia.mb == 1 ? 0 : static_cast<int64_t>(bi) * a.dia.vstride) + __ldg(a.dia.base + s);
    }
    // q_i = (A y)_i for the CTA's rows, f(global row, value)
    const auto product = [&](const auto& xf, auto&& f) {
        if constexpr (ND > 0) cluster_dia_rows<VT, MT, ND>(dvals, off, r0, n, lo, cnt, xf, f);
        else cluster_rows<VT>(A, s, r0, lo, cnt, xf, f);
    };
    const VT* bv = a.b + (a.b_b == 1 ? 0 : vo);
    const VT* g = a.guess ? a.guess + (a.g_b == 1 ? 0 : vo) : nullptr;
    const VT* dinv = a.dinv ? a.dinv + (a.dinv_b == 1 ? 0 : vo) : nullptr;
    const bool jacobi = dinv != nullptr;
    const VT tol = static_cast<VT>(a.tol);
    const int64_t maxit = sys_max_iter(a.max_iter, n);

    // r = b - A x0 (x0 = guess or 0); |b|^2, |r|^2
    VT acc[2] = {VT(0), VT(0)};
    if (g) {
        product(GlobalX<VT>{g}, [&](int row, VT v) {
            const int li = row - r0 - lo;
            const VT b_i = bv[row];
            const VT ri = b_i - v;
            r[li] = ri;
            x[li] = g[row];
            acc[0] += b_i * b_i;
            acc[1] += ri * ri;
        });
    } else {
        for (int li = tid; li < cnt; li += T) {
            const VT b_i = bv[r0 + lo + li];
            r[li] = b_i;
            x[li] = VT(0);
            acc[0] += b_i * b_i;
        }
    }
    if (jacobi)
        for (int li = tid; li < cnt; li += T) dv[li] = dinv[r0 + lo + li];
    cluster_sum<VT, 2>(acc, red, partB, rank, ctas);   // (its barriers also order the shared stores above)
    const VT bb = acc[0];
    VT rr = g ? acc[1] : bb;
    const VT thr = tol * tol * bb;
    int32_t status = ST_RUNNING;
    int32_t it = 0;
    if ((a.abs_zero_test && bb < tol * tol) || bb == VT(0)) {
        for (int li = tid; li < cnt; li += T) x[li] = VT(0);
        status = CMCG_SOLVE_ZERO_RHS;
    } else if (!finite_(rr) || !finite_(bb)) {
        status = CMCG_SOLVE_NON_FINITE;
    } else if (rr < thr) {
        status = CMCG_SOLVE_CONVERGED;
    } else {
        VT rzv[1] = {VT(0)};
        for (int li = tid; li < cnt; li += T) {
            const VT ri = r[li];
            const VT zi = jacobi ? dv[li] * ri : ri;
            p[li] = zi;
            rzv[0] += ri * zi;
        }
        cluster_sum<VT, 1>(rzv, red, partA, rank, ctas);
        VT rz = rzv[0];
        if (!finite_(rz)) status = CMCG_SOLVE_NON_FINITE;
        else if (!(rz > VT(0))) status = CMCG_SOLVE_BREAKDOWN;
        while (status == ST_RUNNING) {
            if (it >= maxit) { status = CMCG_SOLVE_MAX_ITER; break; }
            cl.sync();   // p of every CTA written
            VT pq[1] = {VT(0)};
            product(ClusterP<VT>{p, r0, c.lg, rank}, [&](int row, VT v) {
                const int li = row - r0 - lo;
                q[li] = v;
                pq[0] += p[li] * v;
            });
            cluster_sum<VT, 1>(pq, red, partA, rank, ctas);   // (also: every gather of p is done)
            const VT alpha = rz / pq[0];
            if (!finite_(pq[0]) || !finite_(alpha)) { status = CMCG_SOLVE_NON_FINITE; break; }
            if (!(pq[0] > VT(0))) { status = CMCG_SOLVE_BREAKDOWN; break; }
            VT s2[2] = {VT(0), VT(0)};
            for (int li = tid; li < cnt; li += T) {
                x[li] += alpha * p[li];
                const VT ri = r[li] - alpha * q[li];
                r[li] = ri;
                const VT zi = jacobi ? dv[li] * ri : ri;
                s2[0] += ri * ri;
                s2[1] += ri * zi;
            }
            cluster_sum<VT, 2>(s2, red, partB, rank, ctas);
            rr = s2[0];
            if (!finite_(rr) || !finite_(s2[1])) { status = CMCG_SOLVE_NON_FINITE; break; }
            if (rr < thr) { status = CMCG_SOLVE_CONVERGED; break; }
            const VT rzn = s2[1];
            if (!(rzn > VT(0))) { status = CMCG_SOLVE_BREAKDOWN; break; }
            const VT beta = rzn / rz;
            rz = rzn;
            for (int li = tid; li < cnt; li += T) {
                const VT ri = r[li];
                const VT zi = jacobi ? dv[li] * ri : ri;
                p[li] = zi + beta * p[li];
            }
            ++it;
        }
    }
    VT* xg = a.x + vo;
    for (int li = tid; li < cnt; li += T) xg[r0 + lo + li] = x[li];
    if (rank == 0 && tid == 0) {
        a.st.it[inst] = it;
        a.st.status[inst] = status;
        a.st.rr[inst] = static_cast<double>(rr);
        a.st.bb[inst] = static_cast<double>(bb);
        a.st.outer[inst] = 0;
    }
    cl.sync();   // no CTA leaves while another may still address its shared memory
}

}  // namespace

int cluster_rows_log2(int64_t max_rows, size_t elem_bytes, size_t smem_limit, int* ctas) {
    *ctas = 0;
    for (int lg = 10; lg <= 20; ++lg) {
        const int64_t R = int64_t(1) << lg;
        const int64_t c = (max_rows + R - 1) / R;
        if (c > kClusterMaxCtas) continue;
        if (kClusterVectors * static_cast<size_t>(R) * elem_bytes > smem_limit) return 0;
        *ctas = static_cast<int>(std::max<int64_t>(c, 1));
        return lg;
    }
    return 0;
}

template <typename VT, typename MT, int FMT>
cmcg_status cluster_cg_launch(const SolveArgs<VT, MT>& a, int n_inst, int ctas, int rows_log2, int nd, int min_resident,
                              cudaStream_t st, bool* launched) {
    *launched = false;
    const auto kern = nd == 5 ? k_cluster_cg<VT, MT, FMT, 5> : nd == 7 ? k_cluster_cg<VT, MT, FMT, 7>
                                                                        : k_cluster_cg<VT, MT, FMT, 0>;
    const size_t smem = kClusterVectors * sizeof(VT) * (size_t(1) << rows_log2);
    int device = 0;
    CMCG_CUDA(cudaGetDevice(&device));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(n_inst) * static_cast<unsigned>(ctas));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(ctas);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // (the shared-memory attribute belongs to the kernel, not to the shape:
    // set on every launch)
    CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    // the resident-cluster count of a (device, kernel, shape) is looked up once
    // per process (the occupancy query costs more than a small solve)
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int, size_t>, int> resident_of;
    const auto key = std::make_tuple(device, reinterpret_cast<const void*>(kern), ctas, smem);
    int resident = -1;
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto it = resident_of.find(key);
        if (it != resident_of.end()) resident = it->second;
    }
    if (resident < 0) {
        if (cudaOccupancyMaxActiveClusters(&resident, kern, &cfg) != cudaSuccess) {
            (void)cudaGetLastError();   // (a cluster shape the device cannot place: leave the solve to the others)
            resident = 0;
        }
        std::lock_guard<std::mutex> lock(mu);
        resident_of[key] = resident;
    }
    if (resident < min_resident) return CMCG_OK;
    const ClusterArgs c{ctas, rows_log2};
    CMCG_CUDA(cudaLaunchKernelEx(&cfg, kern, a, c));
    *launched = true;
    return CMCG_OK;
}

#define CMCG_CLUSTER_INSTANTIATE(VT, MT, FMT)                                                                    \
    template cmcg_status cluster_cg_launch<VT, MT, FMT>(const SolveArgs<VT, MT>&, int, int, int, int, int,   \
                                                        cudaStream_t, bool*);
#define CMCG_CLUSTER_FORMATS(VT, MT)           \
    CMCG_CLUSTER_INSTANTIATE(VT, MT, CMCG_CSR) \
    CMCG_CLUSTER_INSTANTIATE(VT, MT, CMCG_ELLPACK)
CMCG_CLUSTER_FORMATS(float, float)
CMCG_CLUSTER_FORMATS(float, double)
CMCG_CLUSTER_FORMATS(float, __nv_bfloat16)
CMCG_CLUSTER_FORMATS(double, float)
CMCG_CLUSTER_FORMATS(double, double)
CMCG_CLUSTER_FORMATS(double, __nv_bfloat16)

}  // namespace cmcg
