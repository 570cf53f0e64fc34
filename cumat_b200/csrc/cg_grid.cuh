// Argument blocks and work plan of the CG kernels, shared by the solver's
// translation units (persistent, grid-graph and cooperative kernels).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cumat_cg.h"
#include "cg_dev.cuh"
#include "common.cuh"

namespace cmcg {

constexpr int kTile = 256;          // rows per tile of the grid path (= threads per CTA)
constexpr int kGridCtasPerSm = 4;   // grid path CTAs per SM (segment plan size)
constexpr int kPersistThreads = 256;

// ---------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------

template <typename MT>
struct MatArgs {
    const int32_t* rp;
    const int32_t* ci;
    const int32_t* ell;
    int32_t width, rows_pad;
    const MT* vals;
    int64_t vstride;
    int32_t mb;
    // sliced ELLPACK copy (CSR patterns)
    const int32_t* sell_col;
    const MT* sell_vals;
    int64_t sell_vstride;
    const int64_t* slice_off;
    const int32_t* slice_w;
    const int32_t* sys_slice0;
};

template <typename MT, int FMT>
__device__ __forceinline__ InstMatrix<MT, FMT> inst_matrix(const MatArgs<MT>& m, int b) {
    InstMatrix<MT, FMT> A;
    const MT* v = m.vals + (m.mb == 1 ? 0 : static_cast<int64_t>(b) * m.vstride);
    A.csr = CsrView<MT>{m.rp, m.ci, v};
    A.ell = EllView<MT>{m.ell, v, m.width, m.rows_pad};
    if (FMT == CMCG_CSR)
        A.rm = RowMat<MT>{m.sell_col, m.sell_vals + (m.mb == 1 ? 0 : static_cast<int64_t>(b) * m.sell_vstride),
                          m.slice_off, m.slice_w, m.sys_slice0, 0, 0};
    else
        A.rm = RowMat<MT>{m.ell, v, nullptr, nullptr, nullptr, m.rows_pad, m.width};
    return A;
}

// Diagonal-layout copy of a stencil-shaped CSR pattern's values (see DiaPlan):
// system s stores diagonal d (offset off[s * 8 + d], ascending) of its local
// row i at vals[b * vstride + base[s] + 1024 ((i / 1024) nd + d) + i % 1024];
// absent entries hold zeros. vals == nullptr: not used.
template <typename MT>
struct DiaArgs {
    const MT* vals;
    int64_t vstride;
    const int64_t* base;
    const int32_t* off;
    const int32_t* unit;   // [mb][n_sys]: middle diagonal is offset 0 with all values 1 (null: none)
    int32_t mb;
};

// Per-instance state (instance = batch * n_sys + system).
struct InstState {
    double* bb;      // |b|^2
    double* rr;      // |r|^2 (latest)
    double* rz;      // r.z
    double* alpha;
    double* beta;
    int32_t* it;     // iterations (reference semantics)
    int32_t* status;
    int32_t* outer;  // refinement steps
    double* err;     // sqrt(rr / bb) written by the finaliser
    unsigned* tk1;
    unsigned* tk2;
    double* rmax;    // mixed solver: scaled |r|^2 at the last residual replacement
    double* goal;    //   scaled |r|^2 that would meet the FP64 target
    int32_t* flag;   //   1: replace the residual in this iteration
    int32_t* rep_it; //   iteration of the last replacement
    int32_t* cyc0;   //   length of the first replacement cycle
    int32_t* stall;  //   consecutive replacements whose true residual did not drop
};

// Progress guard of the reliable updates. Inner values too coarse for the
// system's conditioning (BF16 at a condition number of ~1e6) make the inner
// recursion stagnate or diverge, and its residual may then never drop far
// enough to trigger a replacement. A replacement is therefore also forced
// after kStallFirst iterations in the first cycle (see below), and later after 4 times the
// first cycle's length plus kStallPad, kept within [kStallMin, kStallFirst]. A
// replacement whose true residual norm fell by less than 10 % is a stall;
// kStallMax stalls in a row stop the system with CMCG_SOLVE_BREAKDOWN. (A
// healthy FP32 cycle at condition 1e8 still cuts the residual by more than
// half in kStallFirst iterations.)
// With a coarse replacement threshold (delta >= 0.05, the BF16 default, whose
// cycles are short) the first cycle is forced after kStallMin iterations.
constexpr int kStallFirst = 4096;
constexpr int kStallMin = 1024;
constexpr int kStallPad = 256;
constexpr int kStallMax = 3;
constexpr double kStallRatio = 0.81;   // |r|^2 ratio of a 10 % norm drop
__host__ __device__ __forceinline__ int stall_len(int replacements, int cyc0, float delta) {
    const int l = 4 * cyc0 + kStallPad;
    if (replacements == 0) return delta >= 0.05f ? kStallMin : kStallFirst;
    return l < kStallMin ? kStallMin : (l > kStallFirst ? kStallFirst : l);
}

template <typename VT, typename MT>
struct SolveArgs {
    MatArgs<MT> m;
    DiaArgs<MT> dia;
    int32_t rows, n_sys, ob;
    const int32_t* row_off;
    const int32_t* order;          // persistent: systems, largest first
    int32_t* next;                 // persistent: work counter
    // grid path tiles
    int32_t n_tiles;
    const int32_t* tile_row0;
    int32_t n_seg;
    const int32_t* seg_t0;       // segment = tiles [seg_t0, seg_t1) of one CTA in one system
    const int32_t* seg_t1;
    const int32_t* seg_sys;
    const int32_t* cta_seg0;     // segments of CTA c: [cta_seg0[c], cta_seg0[c+1])
    const int32_t* sys_seg0;     // segments of system s: [sys_seg0[s], sys_seg0[s+1])
    VT* part1;
    VT* part2;
    int32_t* active;
    int32_t* loops;
    int32_t loop_cap;
    cudaGraphConditionalHandle cond;
    // vectors, [batch][rows]
    const VT* dinv;
    int32_t dinv_b;
    const VT* b;
    int32_t b_b;
    const VT* guess;
    int32_t g_b;
    VT* x;
    VT* r;
    VT* p;
    VT* p2;        // graph loop: p_k is in p for even k, in p2 for odd k
    VT* q;
    double tol;
    int64_t max_iter;              // < 0: 2 * rows of the system
    int32_t abs_zero_test;         // reference early-out |b|^2 < tol^2 (0 for refinement inner solves)
    InstState st;
};

__device__ __forceinline__ int64_t sys_max_iter(int64_t mi, int n) { return mi < 0 ? 2 * static_cast<int64_t>(n) : mi; }

// ---------------------------------------------------------------------------
// Grid path work plan and reductions
// ---------------------------------------------------------------------------

__device__ __forceinline__ int32_t ld_status(const int32_t* s) { return *reinterpret_cast<const volatile int32_t*>(s); }

// Publishes this tile's NV partial sums and, if it is the last tile of its
// system instance, returns true with the instance totals (fixed order) in tot.
template <typename VT, int NV>
__device__ bool tile_ticket(const VT (&v)[NV], VT* const (&part)[NV], int64_t pbase, int t_begin, int t_count,
                            int64_t pidx, unsigned* tk, int inst, VT (&tot)[NV], VT* red, bool* last_s) {
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) part[j][pidx] = v[j];
        __threadfence();
        const unsigned t = atomicAdd(tk + inst, 1u);
        *last_s = (t == static_cast<unsigned>(t_count - 1));
    }
    __syncthreads();
    const bool last = *last_s;
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int j = 0; j < NV; ++j) tot[j] = VT(0);
    for (int i = threadIdx.x; i < t_count; i += blockDim.x) {
#pragma unroll
        for (int j = 0; j < NV; ++j) tot[j] += __ldcg(part[j] + pbase + t_begin + i);
    }
    block_sum<VT, NV>(tot, red);
    if (threadIdx.x == 0) tk[inst] = 0u;
    return true;
}

// The grid path's work plan: the tiles are split into gridDim.x contiguous
// ranges, one per CTA; a "segment" is the part of one CTA's range that lies in
// one system. Each CTA keeps its running sums in registers over a segment's
// tiles and publishes one partial per segment; the last segment of a system
// instance to finish (ticket) adds that system's partials in segment order.
// A system's segments have consecutive ids, so the closing sum reads at most
// gridDim.x values.
struct SegInfo {
    int s, inst, t0, t1, sr0, send, r0, r1, pidx, pbase, count;   // rows [r0, r1) of the segment
};

template <typename VT, typename MT>
__device__ __forceinline__ SegInfo seg_info(const SolveArgs<VT, MT>& a, int b, int seg) {
    SegInfo g;
    g.s = a.seg_sys[seg];
    g.inst = b * a.n_sys + g.s;
    g.t0 = a.seg_t0[seg];
    g.t1 = a.seg_t1[seg];
    g.sr0 = a.row_off[g.s];
    g.send = a.row_off[g.s + 1];
    // the tiles of a system are consecutive kTile-row blocks from its first row
    g.r0 = a.tile_row0[g.t0];
    g.r1 = min(g.r0 + (g.t1 - g.t0) * kTile, g.send);
    g.pidx = b * a.n_seg + seg;
    g.pbase = b * a.n_seg + a.sys_seg0[g.s];
    g.count = a.sys_seg0[g.s + 1] - a.sys_seg0[g.s];
    return g;
}

// Four consecutive vector elements moved with 16-byte accesses (float4, or
// two double2).
template <typename VT> struct V4;
template <> struct V4<float> {
    float v[4];
    __device__ __forceinline__ void load(const float* p) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
    __device__ __forceinline__ void store(float* p) const { *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]); }
};
template <> struct V4<double> {
    double v[4];
    __device__ __forceinline__ void load(const double* p) {
        const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    __device__ __forceinline__ void store(double* p) const {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
};

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Row loop of a segment [r0, r1) for the vector passes: when every pointer in
// `ptrs` is 16-byte aligned at r0, thread t takes the 4-row chunks
// r0 + 4 (t + k T) through body4(i), the rest (or everything) goes row by row
// through body1(i).
template <int NP, typename F4, typename F1>
__device__ __forceinline__ void seg_rows_vec(int r0, int r1, const void* const (&ptrs)[NP], F4&& body4, F1&& body1) {
    bool vec = true;
#pragma unroll
    for (int j = 0; j < NP; ++j) vec = vec && (ptrs[j] == nullptr || aligned16(ptrs[j]));
    int tail = r0;
    if (vec) {
        const int n4 = (r1 - r0) >> 2;
#pragma unroll 2
        for (int c = threadIdx.x; c < n4; c += blockDim.x) body4(r0 + 4 * c);
        tail = r0 + 4 * n4;
    }
    for (int i = tail + threadIdx.x; i < r1; i += blockDim.x) body1(i);
}

#define CMCG_FOR_SEGMENTS(a)                                                     \
    for (int b_ = 0; b_ < (a).ob; ++b_)                                          \
        for (int seg_ = (a).cta_seg0[blockIdx.x]; seg_ < (a).cta_seg0[blockIdx.x + 1]; ++seg_)

// ---------------------------------------------------------------------------
// Cooperative grid solve (cg_coop.cu): the whole PCG loop of at most
// kCoopMaxInst instances in one launch of one kCoopThreads-thread CTA per SM
// ---------------------------------------------------------------------------

constexpr int kCoopMaxInst = 16;
constexpr int kCoopThreads = 1024;
constexpr int kCoopMaxSegs = 32;   // segments one CTA may own (cached in shared memory)
constexpr int kCoopMaxRows = 1 << 15;   // largest system for which the cooperative launch is chosen (larger: graph loop faster)

template <typename VT, typename MT, int FMT>
cmcg_status coop_cg_occupancy(int* ctas_per_sm);
// sync: a zeroed grid barrier (two 64-bit words) in device memory; err: device
// error word; p_alt: a second p buffer of the vectors' size
template <typename VT, typename MT, int FMT>
cmcg_status coop_cg_launch(const SolveArgs<VT, MT>& a, void* sync, int32_t* err, int n_inst, VT* p_alt, int grid,
                           cudaStream_t st);

}  // namespace cmcg
