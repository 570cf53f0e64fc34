// Stand-alone sparse products and batched reductions behind the C ABI.
//
//  cmcg_spmv          replaces ProductAssignment<... SparseMatrix<CSR|ELLPACK> ...>
//                     (cuMat/src/SparseProductEvaluation.h:95-139, :232-276) and their
//                     thread-per-row kernels (:43-88, :194-226)
//  cmcg_dot,
//  cmcg_squared_norm  replace dot / squaredNorm (cuMat/src/ReductionOpsPlugin.inl:279-315),
//                     which run CUB DeviceReduce / segmented reductions with a
//                     temporary allocation per call (ReductionOps.h:563-598)
//  cmcg_sddmm         replaces the sparse outer product on a pattern
//                     (SparseProductEvaluation.h:16-37 + SparseEvaluation.h:15-34)
//
// Design: CSR is thread per row with the row's index and value loads issued
// before its gathers (bulk-staged tiles and warp row blocks are variants);
// ELLPACK is four rows per thread with 16-byte loads of the column-major slabs.
// The first product of a pattern picks among the variants that add in the same
// order by timing them (launch_spmv). Reductions are warp shuffles, one
// partial per CTA and a single deterministic combine by the last CTA of each
// batch (ticket counter, no spinning).

#include <sys/stat.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "objects.h"
#include "spmv_dev.cuh"
#include "tma.cuh"

namespace cmcg {
namespace {

constexpr int kSpmvThreads = 256;

// Stand-alone product kernels: 0 = row-unrolled CSR / four-rows-per-thread
// ELLPACK, 1 = warp row-block CSR / thread-per-row ELLPACK, 2 = bulk-staged
// CSR / four-rows-per-thread ELLPACK, 3 .. 6 = CSR with 4 .. 32 lanes per row,
// 7 = CSR with four rows per thread and 16-byte chunks, 8 = CSR with
// warp-staged entries. CUMAT_SPMV_VARIANT forces one (a comparison knob, read
// at each product); unset, each pattern picks by timing on its first product
// (see launch_spmv).
int spmv_variant() {
    const char* e = std::getenv("CUMAT_SPMV_VARIANT");
    return e ? std::atoi(e) : -1;
}

template <int MODE, typename VT>
__device__ __forceinline__ void assign_out(VT* y, VT v) {
    if (MODE == CMCG_ASSIGN) *y = v;
    else if (MODE == CMCG_ADD) *y += v;
    else *y -= v;
}

template <typename MT, typename VT, int MODE>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_csr(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                           const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                           const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                           VT* __restrict__ y, int32_t rows, int32_t ob) {
    __shared__ WarpStage<VT> stage[kSpmvThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nblk = (rows + 31) >> 5;
    const int64_t items = static_cast<int64_t>(nblk) * ob;
    const int64_t wstride = static_cast<int64_t>(gridDim.x) * (kSpmvThreads / 32);
    for (int64_t it = static_cast<int64_t>(blockIdx.x) * (kSpmvThreads / 32) + warp; it < items; it += wstride) {
        const int b = static_cast<int>(it / nblk);
        const int r0 = static_cast<int>(it - static_cast<int64_t>(b) * nblk) * 32;
        const int nr = min(32, rows - r0);
        CsrView<MT> A{rp, ci, vals + (mb == 1 ? 0 : b * vstride)};
        GlobalX<VT> xf{x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols)};
        const VT v = warp_csr_rows<VT>(A, r0, nr, xf, stage[warp]);
        if (lane < nr) assign_out<MODE>(y + static_cast<int64_t>(b) * rows + r0 + lane, v);
    }
}

template <typename MT, typename VT, int MODE>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_ell(const int32_t* __restrict__ idx, int32_t width, int32_t rows_pad,
                                                           const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                           const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                           VT* __restrict__ y, int32_t rows, int32_t ob) {
    const int64_t items = static_cast<int64_t>(rows) * ob;
    for (int64_t it = static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * kSpmvThreads) {
        const int b = static_cast<int>(it / rows);
        const int r = static_cast<int>(it - static_cast<int64_t>(b) * rows);
        EllView<MT> A{idx, vals + (mb == 1 ? 0 : b * vstride), width, rows_pad};
        GlobalX<VT> xf{x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols)};
        assign_out<MODE>(y + it, ell_row<VT>(A, r, xf));
    }
}

// ---- CSR, thread per row, unrolled ------------------------------------------------
//
// The reference's thread-per-row loop (SparseProductEvaluation.h:55-87) with
// the loads taken out of the dependency chain: a thread loads up to
// kCsrUnroll column indices and values of its row (predicated on the row end)
// before the first gather, so each thread keeps 2 * kCsrUnroll independent
// loads and then kCsrUnroll gathers in flight (variant 0). Variant 9 works on
// R = 2 rows per thread at once (items it and it + stride of the flattened
// (batch, row) index), with twice the loads in flight per thread at half the
// resident threads, (batch, row) advanced by a step computed once per thread,
// and a grid sized so that every grid-stride pass is equally full. The
// scattered 4-byte loads of neighbouring rows fall into the same cache lines,
// which L1 merges. Each row is summed in entry order with fused multiply-adds,
// like the reference, so both give the same bits.

constexpr int kCsrUnroll = 8;

template <typename MT, typename VT, int MODE>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_csr_rows(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                                const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                                const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                                VT* __restrict__ y, int32_t rows, int32_t ob) {
    const int64_t items = static_cast<int64_t>(rows) * ob;
    for (int64_t it = static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * kSpmvThreads) {
        const int b = static_cast<int>(it / rows);
        const int r = static_cast<int>(it - static_cast<int64_t>(b) * rows);
        const MT* v = vals + (mb == 1 ? 0 : b * vstride);
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        const int e = __ldg(rp + r + 1);
        VT acc = VT(0);
        for (int k = __ldg(rp + r); k < e; k += kCsrUnroll) {
            int c[kCsrUnroll];
            MT w[kCsrUnroll];
#pragma unroll
            for (int u = 0; u < kCsrUnroll; ++u) {
                const bool in = k + u < e;
                c[u] = in ? __ldg(ci + k + u) : -1;
                w[u] = in ? v[k + u] : MT{};
            }
#pragma unroll
            for (int u = 0; u < kCsrUnroll; ++u)
                if (c[u] >= 0) acc = fma(mval<VT>(w[u]), __ldg(xv + c[u]), acc);
        }
        assign_out<MODE>(y + it, acc);
    }
}

template <typename MT, typename VT, int MODE, int R>
__global__ void __launch_bounds__(kSpmvThreads, 4) k_spmv_csr_rows2(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                                const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                                const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                                VT* __restrict__ y, int32_t rows, int32_t ob) {
    const int64_t items = static_cast<int64_t>(rows) * ob;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kSpmvThreads;
    int64_t it = static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x;
    if (it >= items) return;
    const int64_t db = stride / rows, dr = stride - db * rows;
    int64_t b0 = it / rows, r0 = it - b0 * rows;
    const auto advance = [&](int64_t& b, int64_t& r) {
        r += dr;
        b += db;
        if (r >= rows) {
            r -= rows;
            ++b;
        }
    };
    for (; it < items; it += R * stride) {
        // the thread's rows of this pass: items it + j * stride
        int64_t bb[R], rr[R];
        bool has[R];
        int k[R], e[R];
        VT acc[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            if (j == 0) {
                bb[0] = b0;
                rr[0] = r0;
            } else {
                bb[j] = bb[j - 1];
                rr[j] = rr[j - 1];
                advance(bb[j], rr[j]);
            }
            has[j] = it + j * stride < items;
            k[j] = has[j] ? __ldg(rp + rr[j]) : 0;
            e[j] = has[j] ? __ldg(rp + rr[j] + 1) : 0;
            acc[j] = VT(0);
        }
        bool more = true;
        while (more) {
            int c[R][kCsrUnroll];
            MT w[R][kCsrUnroll];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const MT* v = vals + (mb == 1 ? 0 : bb[j] * vstride);
#pragma unroll
                for (int u = 0; u < kCsrUnroll; ++u) {
                    const bool in = k[j] + u < e[j];
                    c[j][u] = in ? __ldg(ci + k[j] + u) : -1;
                    w[j][u] = in ? v[k[j] + u] : MT{};
                }
            }
            more = false;
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const VT* xv = x + (xb == 1 ? 0 : bb[j] * cols);
#pragma unroll
                for (int u = 0; u < kCsrUnroll; ++u)
                    if (c[j][u] >= 0) acc[j] = fma(mval<VT>(w[j][u]), __ldg(xv + c[j][u]), acc[j]);
                k[j] += kCsrUnroll;
                more = more || k[j] < e[j];
            }
        }
#pragma unroll
        for (int j = 0; j < R; ++j)
            if (has[j]) assign_out<MODE>(y + it + j * stride, acc[j]);
        b0 = bb[R - 1];
        r0 = rr[R - 1];
        advance(b0, r0);
    }
}

// ---- CSR, V lanes per row (long or skewed rows) ----------------------------------
//
// V lanes (4, 8, 16 or 32) share a row: its entries are read in 4-entry chunks
// aligned to 16 bytes (one int4 of column indices and one 16-byte load of
// values per lane and chunk, 8-byte for BF16; the index and value arrays are
// padded so the last chunk stays in bounds, and entries of a chunk outside the
// row are masked), lane l of the group taking chunks l, l + V, ...; the group's
// partial sums are combined with __shfl_xor_sync. Used for rows much longer
// than a stencil's, where thread per row serialises a long row on one thread.

template <typename MT, typename VT, int MODE, int V>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_csr_vec(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                               const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                               const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                               VT* __restrict__ y, int32_t rows, int32_t ob) {
    static_assert(V >= 4 && V <= 32 && (V & (V - 1)) == 0, "V lanes per row: 4, 8, 16 or 32");
    constexpr int GPW = 32 / V;   // rows per warp and step
    const int lane = threadIdx.x & 31, sub = lane & (V - 1);
    const int64_t items = static_cast<int64_t>(rows) * ob;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * kSpmvThreads) >> 5;
    // the loop bound is the warp's (uniform), so every lane reaches the shuffles
    for (int64_t w = warp; w * GPW < items; w += nwarps) {
        const int64_t it = w * GPW + lane / V;
        VT acc = VT(0);
        if (it < items) {
            const int b = static_cast<int>(it / rows);
            const int r = static_cast<int>(it - static_cast<int64_t>(b) * rows);
            const MT* v = vals + (mb == 1 ? 0 : b * vstride);
            const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
            const int a = __ldg(rp + r), e = __ldg(rp + r + 1);
#pragma unroll 2
            for (int k = (a & ~3) + 4 * sub; k < e; k += 4 * V) {
                const int4 c = __ldg(reinterpret_cast<const int4*>(ci + k));
                Vals4<MT> w4;
                w4.load(v + k);
                if (k >= a && k < e) acc += mval<VT>(w4.v[0]) * __ldg(xv + c.x);
                if (k + 1 >= a && k + 1 < e) acc += mval<VT>(w4.v[1]) * __ldg(xv + c.y);
                if (k + 2 >= a && k + 2 < e) acc += mval<VT>(w4.v[2]) * __ldg(xv + c.z);
                if (k + 3 >= a && k + 3 < e) acc += mval<VT>(w4.v[3]) * __ldg(xv + c.w);
            }
        }
#pragma unroll
        for (int o = V / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
        if (sub == 0 && it < items) assign_out<MODE>(y + it, acc);
    }
}

// ---- CSR, four consecutive rows per thread, 16-byte chunks ------------------------
//
// The four rows r .. r + 3 of a thread (r a multiple of 4) own one contiguous
// entry range [rp[r], rp[r + 4]); the thread reads it in 4-entry chunks
// aligned to 16 bytes (one int4 of column indices and one 16-byte load of
// values, 8-byte for BF16; the padded index and value arrays keep the last
// chunk in bounds), so neighbouring threads read neighbouring chunks and a
// warp's loads are whole lines, as in the ELLPACK kernel. Each entry is added
// to its row's sum in entry order, the same sums as thread per row.

template <typename MT, typename VT, int MODE>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_csr4(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                            const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                            const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                            VT* __restrict__ y, int32_t rows, int32_t ob) {
    const int64_t quads = (static_cast<int64_t>(rows) + 3) / 4;
    const int64_t items = quads * ob;
    for (int64_t it = static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * kSpmvThreads) {
        const int b = static_cast<int>(it / quads);
        const int r = static_cast<int>(it - static_cast<int64_t>(b) * quads) * 4;
        const MT* v = vals + (mb == 1 ? 0 : b * vstride);
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        // row pointers of the four rows (padded with copies of nnz past the end)
        const int4 bp = __ldg(reinterpret_cast<const int4*>(rp + r));
        const int b4 = __ldg(rp + r + 4);
        VT a0 = VT(0), a1 = VT(0), a2 = VT(0), a3 = VT(0);
#pragma unroll 2
        for (int k = bp.x & ~3; k < b4; k += 4) {
            const int4 c = __ldg(reinterpret_cast<const int4*>(ci + k));
            Vals4<MT> w;
            w.load(v + k);
            const int cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int kk = k + u;
                if (kk < bp.x || kk >= b4) continue;
                const VT t = mval<VT>(w.v[u]);
                if (kk < bp.y) a0 += t * __ldg(xv + cc[u]);
                else if (kk < bp.z) a1 += t * __ldg(xv + cc[u]);
                else if (kk < bp.w) a2 += t * __ldg(xv + cc[u]);
                else a3 += t * __ldg(xv + cc[u]);
            }
        }
        VT* yv = y + static_cast<int64_t>(b) * rows + r;
        if (r < rows) assign_out<MODE>(yv, a0);
        if (r + 1 < rows) assign_out<MODE>(yv + 1, a1);
        if (r + 2 < rows) assign_out<MODE>(yv + 2, a2);
        if (r + 3 < rows) assign_out<MODE>(yv + 3, a3);
    }
}

// ---- CSR, warp-staged entries ----------------------------------------------------
//
// A warp takes 32 consecutive rows, whose entries form one contiguous range. It
// reads the range in rounds of kCsrStage entries with coalesced loads (lane l
// takes entries l, l + 32, ...), converting each value to the vector type and
// gathering its x into shared memory; lane l then adds up the staged entries
// of row l in entry order with fused multiply-adds, which is the
// thread-per-row kernel's sum bit for bit. Rows longer than a round carry
// their sum into the next one.

constexpr int kCsrStage = 256;   // entries per warp and round

template <typename MT, typename VT, int MODE>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_csr_warp(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                                const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                                const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                                VT* __restrict__ y, int32_t rows, int32_t ob) {
    __shared__ VT sw[kSpmvThreads / 32][kCsrStage];
    __shared__ VT sx[kSpmvThreads / 32][kCsrStage];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t groups = (static_cast<int64_t>(rows) + 31) / 32;
    const int64_t items = groups * ob;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * kSpmvThreads) >> 5;
    // the loop bound is the warp's (uniform), so every lane reaches the
    // shuffles and __syncwarp
    for (int64_t w = (static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x) >> 5; w < items; w += nwarps) {
        const int b = static_cast<int>(w / groups);
        const int r0 = static_cast<int>(w - static_cast<int64_t>(b) * groups) * 32;
        const int r = r0 + lane;
        const MT* v = vals + (mb == 1 ? 0 : b * vstride);
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        const int a = r < rows ? __ldg(rp + r) : 0;
        const int e = r < rows ? __ldg(rp + r + 1) : 0;
        const int g0 = __shfl_sync(FULL, a, 0);
        const int g1 = __shfl_sync(FULL, e, min(32, rows - r0) - 1);
        VT acc = VT(0);
        for (int cs = g0; cs < g1; cs += kCsrStage) {
            const int ce = min(cs + kCsrStage, g1);
            for (int k = cs + lane; k < ce; k += 32) {
                sw[wib][k - cs] = mval<VT>(v[k]);
                sx[wib][k - cs] = __ldg(xv + __ldg(ci + k));
            }
            __syncwarp();
            const int lo = max(a, cs), hi = min(e, ce);
            for (int k = lo; k < hi; ++k) acc = fma(sw[wib][k - cs], sx[wib][k - cs], acc);
            __syncwarp();
        }
        if (r < rows) assign_out<MODE>(y + static_cast<int64_t>(b) * rows + r, acc);
    }
}

// ---- bulk-staged CSR product ----------------------------------------------------
//
// Persistent CTAs walk precomputed row tiles (<= kTileRows rows, <= kTileNnz
// entries). For each tile one thread issues three cp.async.bulk copies (the
// tile's row pointers, column indices and values, 16-byte aligned ranges) into a
// shared-memory stage, completing on that stage's mbarrier; two stages are in
// flight per CTA. Threads then take rows (thread per row), read their entries
// from shared memory, gather x through the read-only path and write y. A tile
// that is one row longer than kTileNnz is summed by the whole CTA from global
// memory. (A variant the autotuner may pick: with two stages the copies often
// stall behind the gathers, and the row-unrolled kernel above wins.)

constexpr int kTileRows = 512;
constexpr int kTileNnz = 2048;
constexpr int kTmaThreads = 256;

template <typename MT>
struct TileSmem {
    static constexpr int kEpv = 16 / static_cast<int>(sizeof(MT));   // values per 16 bytes
    static constexpr int kRp = kTileRows + 8;
    static constexpr int kCol = kTileNnz + 8;
    static constexpr int kVal = kTileNnz + 2 * kEpv;
    static constexpr size_t kStageBytes = ((kRp + kCol) * 4 + kVal * sizeof(MT) + 15) / 16 * 16;
};

template <typename MT, typename VT, int MODE>
__global__ void __launch_bounds__(kTmaThreads) k_spmv_csr_tma(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                             const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                             const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                             VT* __restrict__ y, int32_t rows, int32_t ob,
                                                             const int32_t* __restrict__ tiles, int32_t ntiles,
                                                             int32_t* err, uint32_t wait_limit, int32_t test_no_copy) {
    using L = TileSmem<MT>;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ VT red[kTmaThreads / 32];
    const int tid = threadIdx.x;
    const int64_t items = static_cast<int64_t>(ntiles) * ob;
    const int64_t G = gridDim.x;

    auto stage_ptr = [&](int s) { return smem + s * L::kStageBytes; };
    // issue the copies of item `it` into stage s (thread 0 only)
    auto issue = [&](int64_t it, int s) {
        const int b = static_cast<int>(it / ntiles);
        const int t = static_cast<int>(it - static_cast<int64_t>(b) * ntiles);
        const int r0 = __ldg(tiles + t), r1 = __ldg(tiles + t + 1);
        const int k0 = __ldg(rp + r0), k1 = __ldg(rp + r1);
        unsigned char* st = stage_ptr(s);
        const int ra = r0 & ~3, rb = (r1 + 1 + 3) & ~3;
        uint32_t bytes = static_cast<uint32_t>(rb - ra) * 4u;
        const bool stage_entries = (k1 - k0) <= kTileNnz && k1 > k0;
        int ca = 0, cb = 0, va = 0, vb = 0;
        if (stage_entries) {
            ca = k0 & ~3; cb = (k1 + 3) & ~3;
            va = k0 & ~(L::kEpv - 1); vb = (k1 + L::kEpv - 1) & ~(L::kEpv - 1);
            bytes += static_cast<uint32_t>(cb - ca) * 4u + static_cast<uint32_t>(vb - va) * static_cast<uint32_t>(sizeof(MT));
        }
        mbar_arrive_expect_tx(&bar[s], bytes);
        // (test of the bounded wait: the stage is armed but nothing is copied,
        // so the wait runs out with no copy in flight)
        if (test_no_copy) return;
        bulk_g2s(st, rp + ra, static_cast<uint32_t>(rb - ra) * 4u, &bar[s]);
        if (stage_entries) {
            const MT* vb_ = vals + (mb == 1 ? 0 : b * vstride);
            bulk_g2s(st + L::kRp * 4, ci + ca, static_cast<uint32_t>(cb - ca) * 4u, &bar[s]);
            bulk_g2s(st + (L::kRp + L::kCol) * 4, vb_ + va, static_cast<uint32_t>(vb - va) * sizeof(MT), &bar[s]);
        }
    };

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        if (blockIdx.x < items) issue(blockIdx.x, 0);
        if (blockIdx.x + G < items) issue(blockIdx.x + G, 1);
    }
    int j = 0;
    for (int64_t it = blockIdx.x; it < items; it += G, ++j) {
        const int s = j & 1;
        // uniform over the CTA: the compute below has barriers
        const bool ok = __syncthreads_and(mbar_wait(&bar[s], (j >> 1) & 1, err, wait_limit)) != 0;
        if (!ok) {
            // the wait ran out (recorded in *err): wait once more, bounded, for
            // this stage's copies and for the other stage's, which may still be
            // in flight, then leave without issuing anything
            if (tid == 0) {
                mbar_wait(&bar[s], (j >> 1) & 1, nullptr, wait_limit);
                if (it + G < items) mbar_wait(&bar[s ^ 1], ((j + 1) >> 1) & 1, nullptr, wait_limit);
            }
            __syncthreads();
            return;
        }
        const int b = static_cast<int>(it / ntiles);
        const int t = static_cast<int>(it - static_cast<int64_t>(b) * ntiles);
        const int r0 = __ldg(tiles + t), r1 = __ldg(tiles + t + 1);
        const unsigned char* st = stage_ptr(s);
        const int32_t* srp = reinterpret_cast<const int32_t*>(st);
        const int32_t* sci = reinterpret_cast<const int32_t*>(st + L::kRp * 4);
        const MT* sva = reinterpret_cast<const MT*>(st + (L::kRp + L::kCol) * 4);
        const int ra = r0 & ~3;
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        VT* yv = y + static_cast<int64_t>(b) * rows;
        {
            const int k0 = srp[r0 - ra], k1 = srp[r1 - ra];
            if (k1 - k0 <= kTileNnz) {
                const int ca = k0 & ~3, va = k0 & ~(L::kEpv - 1);
                for (int r = r0 + tid; r < r1; r += kTmaThreads) {
                    const int a = srp[r - ra], e = srp[r - ra + 1];
                    VT acc = VT(0);
                    for (int k = a; k < e; ++k) acc += mval<VT>(sva[k - va]) * __ldg(xv + sci[k - ca]);
                    assign_out<MODE>(yv + r, acc);
                }
            } else {
                // one long row: the CTA sums it from global memory
                const MT* vb_ = vals + (mb == 1 ? 0 : b * vstride);
                VT acc[1] = {VT(0)};
                for (int k = k0 + tid; k < k1; k += kTmaThreads) acc[0] += mval<VT>(vb_[k]) * __ldg(xv + __ldg(ci + k));
                block_sum<VT, 1>(acc, red);
                if (tid == 0) assign_out<MODE>(yv + r0, acc[0]);
            }
        }
        __syncthreads();   // stage s fully consumed
        if (tid == 0 && it + 2 * G < items) {
            fence_proxy_async();
            issue(it + 2 * G, s);
        }
    }
}

// ---- ELLPACK, four rows per thread ---------------------------------------------------
//
// Column-major slabs with rows padded to a multiple of 4: each thread loads one
// 16-byte vector of column indices and the matching values per slot for four
// consecutive rows (coalesced across the warp), skips padding (index < 0) and
// gathers x through the read-only path.

template <typename MT> struct Vec4Load;
template <> struct Vec4Load<float> {
    __device__ __forceinline__ static void load(const float* p, float (&v)[4]) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
};
template <> struct Vec4Load<double> {
    __device__ __forceinline__ static void load(const double* p, double (&v)[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 c = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = c.x; v[3] = c.y;
    }
};
template <> struct Vec4Load<__nv_bfloat16> {
    __device__ __forceinline__ static void load(const __nv_bfloat16* p, __nv_bfloat16 (&v)[4]) {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
        const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&t.x);
        const __nv_bfloat162 c = *reinterpret_cast<const __nv_bfloat162*>(&t.y);
        v[0] = a.x; v[1] = a.y; v[2] = c.x; v[3] = c.y;
    }
};

// one slot of four rows: padding (index < 0) contributes nothing
template <typename MT, typename VT>
__device__ __forceinline__ void ell4_slot(const int4 c, const MT (&w)[4], const VT* __restrict__ xv, VT (&acc)[4]) {
    if (c.x >= 0) acc[0] += mval<VT>(w[0]) * __ldg(xv + c.x);
    if (c.y >= 0) acc[1] += mval<VT>(w[1]) * __ldg(xv + c.y);
    if (c.z >= 0) acc[2] += mval<VT>(w[2]) * __ldg(xv + c.z);
    if (c.w >= 0) acc[3] += mval<VT>(w[3]) * __ldg(xv + c.w);
}

// W > 0: the width is a compile-time constant and every slot's index and value
// vectors are loaded before the first gather (2 W independent 16-byte loads in
// flight per thread); W == 0: any width, slot by slot
template <typename MT, typename VT, int MODE, int W>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_ell4(const int32_t* __restrict__ idx, int32_t width, int32_t rows_pad,
                                                            const MT* __restrict__ vals, int64_t vstride, int32_t mb,
                                                            const VT* __restrict__ x, int32_t cols, int32_t xb,
                                                            VT* __restrict__ y, int32_t rows, int32_t ob) {
    const int quads = rows_pad >> 2;
    const int64_t items = static_cast<int64_t>(quads) * ob;
    for (int64_t it = static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * kSpmvThreads) {
        const int b = static_cast<int>(it / quads);
        const int r = static_cast<int>(it - static_cast<int64_t>(b) * quads) * 4;
        const MT* v = vals + (mb == 1 ? 0 : b * vstride);
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        VT acc[4] = {VT(0), VT(0), VT(0), VT(0)};
        if constexpr (W > 0) {
            int4 c[W];
            MT w[W][4];
#pragma unroll
            for (int j = 0; j < W; ++j) {
                const int64_t o = r + static_cast<int64_t>(j) * rows_pad;
                c[j] = __ldg(reinterpret_cast<const int4*>(idx + o));
                Vec4Load<MT>::load(v + o, w[j]);
            }
#pragma unroll
            for (int j = 0; j < W; ++j) ell4_slot<MT, VT>(c[j], w[j], xv, acc);
        } else {
            for (int j = 0; j < width; ++j) {
                const int64_t o = r + static_cast<int64_t>(j) * rows_pad;
                const int4 c = __ldg(reinterpret_cast<const int4*>(idx + o));
                MT w[4];
                Vec4Load<MT>::load(v + o, w);
                ell4_slot<MT, VT>(c, w, xv, acc);
            }
        }
        VT* yv = y + static_cast<int64_t>(b) * rows + r;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (r + q < rows) assign_out<MODE>(yv + q, acc[q]);
    }
}

cmcg_status ensure_spmv_tiles(cmcg_pattern p) {
    if (p->d_spmv_tiles) return CMCG_OK;
    std::vector<int32_t> t;
    const auto& rp = p->h_row_ptr;
    int32_t r = 0;
    while (r < p->rows) {
        t.push_back(r);
        const int32_t start = r;
        ++r;  // a tile holds at least one row (a long row alone)
        if (rp[r] - rp[start] > kTileNnz) continue;
        while (r < p->rows && r - start < kTileRows && rp[r + 1] - rp[start] <= kTileNnz) ++r;
    }
    t.push_back(p->rows);
    CMCG_TRY(dev_alloc(reinterpret_cast<void**>(&p->d_spmv_tiles), t.size() * sizeof(int32_t)));
    CMCG_CUDA(cudaMemcpy(p->d_spmv_tiles, t.data(), t.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    p->n_spmv_tiles = static_cast<int32_t>(t.size() - 1);
    return CMCG_OK;
}

template <typename MT, typename VT, int MODE>
cmcg_status launch_csr_tma(cmcg_matrix A, const VT* xv, int32_t xb, VT* yv, int32_t ob) {
    cmcg_pattern p = A->pat;
    cmcg_ctx ctx = p->ctx;
    CMCG_TRY(ensure_spmv_tiles(p));
    const size_t sm = 2 * TileSmem<MT>::kStageBytes;
    auto kern = k_spmv_csr_tma<MT, VT, MODE>;
    static thread_local bool attr_set[3][2][3] = {};
    bool& done = attr_set[DT<MT>::id][DT<VT>::id][MODE];
    if (!done) {
        CMCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
        done = true;
    }
    int occ = 0;
    CMCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kTmaThreads, sm));
    const int64_t items = static_cast<int64_t>(p->n_spmv_tiles) * ob;
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, static_cast<int64_t>(ctx->sm_count) * std::max(occ, 1))));
    // wait limit of the stage barriers; CUMAT_TEST_WAIT_LIMIT and
    // CUMAT_TEST_NO_COPY (tests of the bounded wait) set a short limit and
    // stages that are armed but never filled
    uint32_t limit = kWaitLimit;
    int32_t no_copy = 0;
    if (const char* e = std::getenv("CUMAT_TEST_WAIT_LIMIT")) limit = static_cast<uint32_t>(std::max(1, std::atoi(e)));
    if (const char* e = std::getenv("CUMAT_TEST_NO_COPY")) no_copy = std::atoi(e) != 0;
    kern<<<grid, kTmaThreads, sm, ctx->stream>>>(p->d_row_ptr, p->d_col, static_cast<const MT*>(A->d_vals), A->stride,
                                                A->batches, xv, p->cols, xb, yv, p->rows, ob, p->d_spmv_tiles,
                                                p->n_spmv_tiles, ctx->d_err, limit, no_copy);
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

// ELLPACK widths 1..8 get the width-specialised kernel; the grid is at most one
// wave of resident CTAs (grid-stride loop over the row quads)
template <typename K>
int resident_grid(K kern, int needed, int sm_count) {
    // resident CTAs per SM, queried once per kernel (a host call per product
    // would show in small products)
    static std::mutex mu;
    static std::map<const void*, int> occ_of;
    int occ = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = occ_of.find(reinterpret_cast<const void*>(kern));
        if (it != occ_of.end()) occ = it->second;
    }
    if (occ == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kSpmvThreads, 0) != cudaSuccess || occ < 1) occ = 1;
        std::lock_guard<std::mutex> lk(mu);
        occ_of[reinterpret_cast<const void*>(kern)] = occ;
    }
    return std::max(1, std::min(needed, sm_count * occ));
}

// CTAs for `units` CTA-passes of grid-stride work: all of them when they fit
// at once, else as few passes as the resident grid needs with every pass
// equally full (no last pass that leaves most of the GPU idle)
template <typename K>
int balanced_grid(K kern, int64_t units, int sm_count) {
    const int cap = resident_grid(kern, INT32_MAX, sm_count);
    if (units <= cap) return static_cast<int>(std::max<int64_t>(1, units));
    const int64_t passes = (units + cap - 1) / cap;
    return static_cast<int>((units + passes - 1) / passes);
}

template <typename MT, typename VT, int MODE>
void launch_ell4(cmcg_matrix A, int blocks, const MT* vals, const VT* xv, int32_t xb, VT* yv, int32_t ob) {
    cmcg_pattern p = A->pat;
    cudaStream_t st = p->ctx->stream;
    const int sms = p->ctx->sm_count;
#define CMCG_ELL4_W(W)                                                                                            \
    k_spmv_ell4<MT, VT, MODE, W><<<resident_grid(k_spmv_ell4<MT, VT, MODE, W>, blocks, sms), kSpmvThreads, 0, st>>>( \
        p->d_ell, p->width, p->rows_pad, vals, A->stride, A->batches, xv, p->cols, xb, yv, p->rows, ob)
    switch (p->width) {
        case 1: CMCG_ELL4_W(1); break;
        case 2: CMCG_ELL4_W(2); break;
        case 3: CMCG_ELL4_W(3); break;
        case 4: CMCG_ELL4_W(4); break;
        case 5: CMCG_ELL4_W(5); break;
        case 6: CMCG_ELL4_W(6); break;
        case 7: CMCG_ELL4_W(7); break;
        case 8: CMCG_ELL4_W(8); break;
        default: CMCG_ELL4_W(0);
    }
#undef CMCG_ELL4_W
}

template <typename MT, typename VT>
cmcg_status launch_spmv_variant(cmcg_matrix A, const void* x, int32_t xb, void* y, int32_t mode, int variant) {
    cmcg_pattern p = A->pat;
    cmcg_ctx ctx = p->ctx;
    const int32_t ob = std::max(A->batches, xb);
    const MT* vals = static_cast<const MT*>(A->d_vals);
    const VT* xv = static_cast<const VT*>(x);
    VT* yv = static_cast<VT*>(y);
    const int max_blocks = ctx->sm_count * 8;
    if (p->format == CMCG_CSR && variant == 2) {
        if (mode == CMCG_ASSIGN) return launch_csr_tma<MT, VT, CMCG_ASSIGN>(A, xv, xb, yv, ob);
        if (mode == CMCG_ADD) return launch_csr_tma<MT, VT, CMCG_ADD>(A, xv, xb, yv, ob);
        return launch_csr_tma<MT, VT, CMCG_SUB>(A, xv, xb, yv, ob);
    }
    if (p->format == CMCG_CSR && variant >= 3 && variant <= 6) {
        const int V = 4 << (variant - 3);
        const int64_t threads = static_cast<int64_t>(p->rows) * ob * V;
        const int needed = static_cast<int>(std::min<int64_t>((threads + kSpmvThreads - 1) / kSpmvThreads, max_blocks));
#define CMCG_LAUNCH_CSR_VEC(M, VV)                                                                                   \
    k_spmv_csr_vec<MT, VT, M, VV><<<resident_grid(k_spmv_csr_vec<MT, VT, M, VV>, needed, ctx->sm_count), kSpmvThreads, \
                                    0, ctx->stream>>>(p->d_row_ptr, p->d_col, vals, A->stride, A->batches, xv, p->cols,  \
                                                      xb, yv, p->rows, ob)
#define CMCG_LAUNCH_CSR_VEC_V(M)              \
    switch (V) {                              \
        case 4: CMCG_LAUNCH_CSR_VEC(M, 4); break;   \
        case 8: CMCG_LAUNCH_CSR_VEC(M, 8); break;   \
        case 16: CMCG_LAUNCH_CSR_VEC(M, 16); break; \
        default: CMCG_LAUNCH_CSR_VEC(M, 32);        \
    }
        if (mode == CMCG_ASSIGN) { CMCG_LAUNCH_CSR_VEC_V(CMCG_ASSIGN) }
        else if (mode == CMCG_ADD) { CMCG_LAUNCH_CSR_VEC_V(CMCG_ADD) }
        else { CMCG_LAUNCH_CSR_VEC_V(CMCG_SUB) }
#undef CMCG_LAUNCH_CSR_VEC_V
#undef CMCG_LAUNCH_CSR_VEC
        count_launch();
        CMCG_CHECK_LAUNCH();
        return CMCG_OK;
    }
    if (p->format == CMCG_CSR && variant == 7) {
        const int64_t threads = (static_cast<int64_t>(p->rows) + 3) / 4 * ob;
        const int needed = static_cast<int>(std::min<int64_t>((threads + kSpmvThreads - 1) / kSpmvThreads, max_blocks));
#define CMCG_LAUNCH_CSR4(M)                                                                                    \
    k_spmv_csr4<MT, VT, M><<<resident_grid(k_spmv_csr4<MT, VT, M>, needed, ctx->sm_count), kSpmvThreads, 0,      \
                             ctx->stream>>>(p->d_row_ptr, p->d_col, vals, A->stride, A->batches, xv, p->cols, xb, yv, \
                                            p->rows, ob)
        if (mode == CMCG_ASSIGN) CMCG_LAUNCH_CSR4(CMCG_ASSIGN);
        else if (mode == CMCG_ADD) CMCG_LAUNCH_CSR4(CMCG_ADD);
        else CMCG_LAUNCH_CSR4(CMCG_SUB);
#undef CMCG_LAUNCH_CSR4
        count_launch();
        CMCG_CHECK_LAUNCH();
        return CMCG_OK;
    }
    if (p->format == CMCG_CSR && variant == 8) {
        const int64_t warps = (static_cast<int64_t>(p->rows) + 31) / 32 * ob;
        const int needed = static_cast<int>(std::min<int64_t>((warps + kSpmvThreads / 32 - 1) / (kSpmvThreads / 32), max_blocks));
#define CMCG_LAUNCH_CSR_WARP(M)                                                                                       \
    k_spmv_csr_warp<MT, VT, M><<<resident_grid(k_spmv_csr_warp<MT, VT, M>, needed, ctx->sm_count), kSpmvThreads, 0,     \
                                 ctx->stream>>>(p->d_row_ptr, p->d_col, vals, A->stride, A->batches, xv, p->cols, xb, yv, \
                                                p->rows, ob)
        if (mode == CMCG_ASSIGN) CMCG_LAUNCH_CSR_WARP(CMCG_ASSIGN);
        else if (mode == CMCG_ADD) CMCG_LAUNCH_CSR_WARP(CMCG_ADD);
        else CMCG_LAUNCH_CSR_WARP(CMCG_SUB);
#undef CMCG_LAUNCH_CSR_WARP
        count_launch();
        CMCG_CHECK_LAUNCH();
        return CMCG_OK;
    }
    if (p->format == CMCG_CSR && (variant == 0 || variant == 9)) {
        const int64_t items = static_cast<int64_t>(p->rows) * ob;
        const int rpt = variant == 9 ? 2 : 1;   // rows in flight per thread
        const int64_t units = (items + static_cast<int64_t>(kSpmvThreads) * rpt - 1) / (static_cast<int64_t>(kSpmvThreads) * rpt);
#define CMCG_LAUNCH_CSR_ROW1(M)                                                                                  \
    k_spmv_csr_rows<MT, VT, M><<<resident_grid(k_spmv_csr_rows<MT, VT, M>, needed, ctx->sm_count), kSpmvThreads, 0, \
                                 ctx->stream>>>(p->d_row_ptr, p->d_col, vals, A->stride, A->batches, xv, p->cols, xb, \
                                                yv, p->rows, ob)
#define CMCG_LAUNCH_CSR_ROWS(M, R)                                                                                     \
    k_spmv_csr_rows2<MT, VT, M, R><<<balanced_grid(k_spmv_csr_rows2<MT, VT, M, R>, units, ctx->sm_count), kSpmvThreads, \
                                     0, ctx->stream>>>(p->d_row_ptr, p->d_col, vals, A->stride, A->batches, xv, p->cols, \
                                                      xb, yv, p->rows, ob)
        if (variant == 0) {
            const int needed = static_cast<int>(std::min<int64_t>((items + kSpmvThreads - 1) / kSpmvThreads, max_blocks));
            if (mode == CMCG_ASSIGN) CMCG_LAUNCH_CSR_ROW1(CMCG_ASSIGN);
            else if (mode == CMCG_ADD) CMCG_LAUNCH_CSR_ROW1(CMCG_ADD);
            else CMCG_LAUNCH_CSR_ROW1(CMCG_SUB);
        } else {
            if (mode == CMCG_ASSIGN) CMCG_LAUNCH_CSR_ROWS(CMCG_ASSIGN, 2);
            else if (mode == CMCG_ADD) CMCG_LAUNCH_CSR_ROWS(CMCG_ADD, 2);
            else CMCG_LAUNCH_CSR_ROWS(CMCG_SUB, 2);
        }
#undef CMCG_LAUNCH_CSR_ROW1
#undef CMCG_LAUNCH_CSR_ROWS
        count_launch();
        CMCG_CHECK_LAUNCH();
        return CMCG_OK;
    }
    if (p->format == CMCG_ELLPACK && variant != 1) {
        const int64_t threads = static_cast<int64_t>(p->rows_pad / 4) * ob;
        const int blocks = static_cast<int>(std::min<int64_t>((threads + kSpmvThreads - 1) / kSpmvThreads, max_blocks));
        if (mode == CMCG_ASSIGN) launch_ell4<MT, VT, CMCG_ASSIGN>(A, blocks, vals, xv, xb, yv, ob);
        else if (mode == CMCG_ADD) launch_ell4<MT, VT, CMCG_ADD>(A, blocks, vals, xv, xb, yv, ob);
        else launch_ell4<MT, VT, CMCG_SUB>(A, blocks, vals, xv, xb, yv, ob);
        count_launch();
        CMCG_CHECK_LAUNCH();
        return CMCG_OK;
    }
    if (p->format == CMCG_CSR) {
        const int64_t warps = static_cast<int64_t>((p->rows + 31) / 32) * ob;
        const int blocks = static_cast<int>(std::min<int64_t>((warps + 7) / 8, max_blocks));
#define CMCG_LAUNCH_CSR(M)                                                                                       \
    k_spmv_csr<MT, VT, M><<<blocks, kSpmvThreads, 0, ctx->stream>>>(p->d_row_ptr, p->d_col, vals, A->stride,     \
                                                                    A->batches, xv, p->cols, xb, yv, p->rows, ob)
        if (mode == CMCG_ASSIGN) CMCG_LAUNCH_CSR(CMCG_ASSIGN);
        else if (mode == CMCG_ADD) CMCG_LAUNCH_CSR(CMCG_ADD);
        else CMCG_LAUNCH_CSR(CMCG_SUB);
#undef CMCG_LAUNCH_CSR
    } else {
        const int64_t threads = static_cast<int64_t>(p->rows) * ob;
        const int blocks = static_cast<int>(std::min<int64_t>((threads + kSpmvThreads - 1) / kSpmvThreads, max_blocks));
#define CMCG_LAUNCH_ELL(M)                                                                                      \
    k_spmv_ell<MT, VT, M><<<blocks, kSpmvThreads, 0, ctx->stream>>>(p->d_ell, p->width, p->rows_pad, vals,       \
                                                                    A->stride, A->batches, xv, p->cols, xb, yv,  \
                                                                    p->rows, ob)
        if (mode == CMCG_ASSIGN) CMCG_LAUNCH_ELL(CMCG_ASSIGN);
        else if (mode == CMCG_ADD) CMCG_LAUNCH_ELL(CMCG_ADD);
        else CMCG_LAUNCH_ELL(CMCG_SUB);
#undef CMCG_LAUNCH_ELL
    }
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

// ---- batched dot / squared norm -------------------------------------------------

constexpr int kRedThreads = 256;

// grid (gx, ob): CTA (bx, b) sums a grid-stride slice of batch b; the last CTA
// of batch b (ticket) adds the gx partials in index order and resets the ticket.
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_dot(int64_t n, const VT* __restrict__ x, int32_t xb,
                                                     const VT* __restrict__ y, int32_t yb, VT* __restrict__ out,
                                                     VT* __restrict__ partial, unsigned* __restrict__ ticket) {
    __shared__ VT red[kRedThreads / 32];
    __shared__ bool last;
    const int b = blockIdx.y;
    const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * n);
    const VT* yv = y + (yb == 1 ? 0 : static_cast<int64_t>(b) * n);
    // four grid strides per pass: eight independent loads in flight per thread,
    // summed into four accumulators that are added in a fixed order
    VT acc[1] = {VT(0)};
    VT a4[4] = {VT(0), VT(0), VT(0), VT(0)};
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kRedThreads;
    int64_t i = static_cast<int64_t>(blockIdx.x) * kRedThreads + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {
        VT xs[4], ys[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            xs[j] = __ldg(xv + i + j * stride);
            ys[j] = __ldg(yv + i + j * stride);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) a4[j] += xs[j] * ys[j];
    }
#pragma unroll
    for (int j = 0; j < 3; ++j)
        if (i + j * stride < n) a4[j] += __ldg(xv + i + j * stride) * __ldg(yv + i + j * stride);
    acc[0] = (a4[0] + a4[1]) + (a4[2] + a4[3]);
    block_sum<VT, 1>(acc, red);
    if (threadIdx.x == 0) {
        partial[static_cast<int64_t>(b) * gridDim.x + blockIdx.x] = acc[0];
        __threadfence();
        const unsigned t = atomicAdd(ticket + b, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    VT s[1] = {VT(0)};
    const volatile VT* pv = partial + static_cast<int64_t>(b) * gridDim.x;
    for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += kRedThreads) s[0] += pv[i];
    block_sum<VT, 1>(s, red);
    if (threadIdx.x == 0) {
        out[b] = s[0];
        ticket[b] = 0;
    }
}

// CTAs per batch of the dot product: one per 4 x 256 x 4 entries (four
// passes of four loads per thread), at most 8 per SM over all batches (a full
// SM of 256-thread CTAs), at most `cap`
int dot_grid(cmcg_ctx ctx, int64_t n, int32_t ob, int cap) {
    const int64_t want = std::max<int64_t>(1, (n + kRedThreads * 16 - 1) / (kRedThreads * 16));
    const int most = std::max(1, std::min(cap, (ctx->sm_count * 8) / std::max(1, ob) + 1));
    return static_cast<int>(std::min<int64_t>(want, most));
}

template <typename VT>
cmcg_status launch_dot(cmcg_ctx ctx, int64_t n, const void* x, int32_t xb, const void* y, int32_t yb, void* out,
                       int32_t ob) {
    const int gx = dot_grid(ctx, n, ob, INT32_MAX);
    CMCG_TRY(ensure_buffer(&ctx->red_partial, &ctx->red_partial_bytes, static_cast<size_t>(gx) * ob * sizeof(VT)));
    if (ctx->red_ticket_count < static_cast<size_t>(ob)) {
        dev_free(ctx->red_ticket);
        ctx->red_ticket = nullptr;
        ctx->red_ticket_count = 0;
        CMCG_TRY(dev_alloc(reinterpret_cast<void**>(&ctx->red_ticket), ob * sizeof(unsigned)));
        CMCG_CUDA(cudaMemsetAsync(ctx->red_ticket, 0, ob * sizeof(unsigned), ctx->stream));
        ctx->red_ticket_count = ob;
    }
    dim3 grid(gx, ob);
    k_dot<VT><<<grid, kRedThreads, 0, ctx->stream>>>(n, static_cast<const VT*>(x), xb, static_cast<const VT*>(y), yb,
                                                     static_cast<VT*>(out), static_cast<VT*>(ctx->red_partial),
                                                     ctx->red_ticket);
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

// ---- sampled outer product on the pattern -----------------------------------------

// Sampled outer product on a CSR pattern, out_k = alpha * u[row(k)] * v[col(k)]
// for every stored entry k: thread per row, two rows per thread in flight (r
// and r + stride), with kCsrUnroll column indices of each loaded before the
// first gather and reused for all value batches; each product is
// (alpha * u) * v, the reference's order.
template <typename VT>
__global__ void __launch_bounds__(kSpmvThreads) k_sddmm_csr(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                            int32_t rows, int32_t cols, int64_t vstride, VT alpha,
                                                            const VT* __restrict__ u, int32_t ub,
                                                            const VT* __restrict__ v, int32_t vb,
                                                            VT* __restrict__ out, int32_t ob) {
    // two rows per thread in flight: r and r + stride
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kSpmvThreads;
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * kSpmvThreads + threadIdx.x; r < rows; r += 2 * stride) {
        const int64_t rr[2] = {r, r + stride};
        const bool has1 = r + stride < rows;
        int k[2], e[2];
        k[0] = __ldg(rp + r);
        e[0] = __ldg(rp + r + 1);
        k[1] = has1 ? __ldg(rp + rr[1]) : 0;
        e[1] = has1 ? __ldg(rp + rr[1] + 1) : 0;
        while (k[0] < e[0] || k[1] < e[1]) {
            int c[2][kCsrUnroll];
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int q = 0; q < kCsrUnroll; ++q) c[j][q] = k[j] + q < e[j] ? __ldg(ci + k[j] + q) : -1;
            for (int b = 0; b < ob; ++b) {
                const VT* uu = u + (ub == 1 ? 0 : static_cast<int64_t>(b) * rows);
                const VT* vv = v + (vb == 1 ? 0 : static_cast<int64_t>(b) * cols);
                VT g[2][kCsrUnroll];
#pragma unroll
                for (int j = 0; j < 2; ++j)
#pragma unroll
                    for (int q = 0; q < kCsrUnroll; ++q) g[j][q] = c[j][q] >= 0 ? __ldg(vv + c[j][q]) : VT(0);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if (k[j] >= e[j]) continue;
                    const VT au = alpha * __ldg(uu + rr[j]);
                    VT* o = out + static_cast<int64_t>(b) * vstride + k[j];
#pragma unroll
                    for (int q = 0; q < kCsrUnroll; ++q)
                        if (c[j][q] >= 0) o[q] = au * g[j][q];
                }
            }
            k[0] += kCsrUnroll;
            k[1] += kCsrUnroll;
        }
    }
}

template <typename VT>
__global__ void k_sddmm_ell(const int32_t* __restrict__ idx, int32_t width, int32_t rows_pad, int32_t rows, int32_t cols,
                            int64_t vstride, VT alpha, const VT* __restrict__ u, int32_t ub, const VT* __restrict__ v,
                            int32_t vb, VT* __restrict__ out, int32_t ob) {
    const int64_t per = static_cast<int64_t>(rows) * width;
    const int64_t items = per * ob;
    for (int64_t it = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(it / per);
        const int64_t rem = it - b * per;
        const int j = static_cast<int>(rem / rows);
        const int r = static_cast<int>(rem - static_cast<int64_t>(j) * rows);
        const int c = __ldg(idx + r + static_cast<int64_t>(j) * rows_pad);
        const VT* ub_ = u + (ub == 1 ? 0 : static_cast<int64_t>(b) * rows);
        const VT* vb_ = v + (vb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        // output in the caller's dense [batch][slot][row] layout
        out[it] = (c >= 0) ? alpha * ub_[r] * vb_[c] : VT(0);
    }
}

template <typename VT>
cmcg_status launch_sddmm(cmcg_matrix M, double alpha, const void* u, int32_t ub, const void* v, int32_t vb, void* out,
                         int32_t ob) {
    cmcg_pattern p = M->pat;
    cmcg_ctx ctx = p->ctx;
    if (p->format == CMCG_CSR) {
        // two rows per thread; 64 registers leave 4 CTAs per SM
        const int64_t need = (static_cast<int64_t>(p->rows) + 2 * kSpmvThreads - 1) / (2 * kSpmvThreads);
        const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, ctx->sm_count * 4)));
        k_sddmm_csr<VT><<<blocks, kSpmvThreads, 0, ctx->stream>>>(p->d_row_ptr, p->d_col, p->rows, p->cols, p->nnz,
                                                         static_cast<VT>(alpha), static_cast<const VT*>(u), ub,
                                                         static_cast<const VT*>(v), vb, static_cast<VT*>(out), ob);
    } else {
        const int64_t n = p->nnz * ob;
        const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, ctx->sm_count * 8));
        k_sddmm_ell<VT><<<blocks, 256, 0, ctx->stream>>>(p->d_ell, p->width, p->rows_pad, p->rows, p->cols, p->nnz,
                                                         static_cast<VT>(alpha), static_cast<const VT*>(u), ub,
                                                         static_cast<const VT*>(v), vb, static_cast<VT*>(out), ob);
    }
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

}  // namespace

// Row-length rule of the CSR product (deterministic, from the pattern): when
// the longest row has at least 256 entries and 32 times the mean, thread per
// row would leave a few threads summing long rows alone, and a warp per row
// (V = 32) takes over. Otherwise the product stays thread per row, which adds
// every row in entry order exactly as the solvers' products do (so that, for
// instance, b = A x0 followed by a solve from x0 finds a zero residual). The
// V = 4 .. 16 kernels are there for callers that force them. Returns the
// variant (3 + log2(V / 4)) or -1.
int csr_vec_variant(cmcg_pattern p) {
    const auto& rp = p->h_row_ptr;
    int64_t mx = 0;
    for (int32_t r = 0; r < p->rows; ++r) mx = std::max<int64_t>(mx, rp[r + 1] - rp[r]);
    const double mean = static_cast<double>(p->nnz) / std::max(1, p->rows);
    return (mx >= 256 && static_cast<double>(mx) >= 32.0 * mean) ? 6 : -1;
}

// Persistent cache of the timed choices: one line "key variant" per tuned
// case, key = GPU name | format | value type | vector type | rows | nnz |
// width, in $CUMAT_TUNE_CACHE (default ~/.cache/cumat_b200/spmv_tune.txt;
// empty: no file). A process reuses the choice a previous one timed on the
// same GPU model and pattern shape instead of timing again.
std::mutex g_tune_mu;

std::string tune_path() {
    if (const char* e = std::getenv("CUMAT_TUNE_CACHE")) return e;
    const char* h = std::getenv("HOME");
    return h ? std::string(h) + "/.cache/cumat_b200/spmv_tune.txt" : std::string();
}

std::string tune_key(cmcg_pattern p, int mt, int vt) {
    cudaDeviceProp prop{};
    std::string gpu = cudaGetDeviceProperties(&prop, p->ctx->device) == cudaSuccess ? prop.name : "unknown";
    for (char& c : gpu)
        if (c == ' ' || c == '|') c = '_';
    return gpu + "|" + (p->format == CMCG_CSR ? "csr" : "ell") + "|" + std::to_string(mt) + "|" + std::to_string(vt) +
           "|" + std::to_string(p->rows) + "|" + std::to_string(p->nnz) + "|" + std::to_string(p->width);
}

int tune_lookup(const std::string& key) {
    const std::string path = tune_path();
    if (path.empty()) return -1;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return -1;
    char line[512];
    int found = -1;
    while (std::fgets(line, sizeof(line), f)) {
        const char* sp = std::strrchr(line, ' ');
        if (!sp) continue;
        if (std::string(line, sp - line) == key) found = std::atoi(sp + 1);   // the last entry wins
    }
    std::fclose(f);
    return found;
}

void tune_store(const std::string& key, int variant) {
    const std::string path = tune_path();
    if (path.empty()) return;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    // create the parent directories (a failure shows as the open failing)
    for (size_t i = path.find('/', 1); i != std::string::npos; i = path.find('/', i + 1))
        ::mkdir(path.substr(0, i).c_str(), 0755);
    if (FILE* f = std::fopen(path.c_str(), "a")) {
        std::fprintf(f, "%s %d\n", key.c_str(), variant);
        std::fclose(f);
    }
}

// Internal entry used by the solver (device pointers, no validation).
// Autotuner of the stand-alone product: CSR patterns with long or skewed rows
// take the V-lanes-per-row kernel by the row-length rule above. Otherwise,
// among the kernels that add every
// row's products in the same order (CSR: row-unrolled, bulk-staged; ELLPACK:
// four rows per thread, thread per row), so that the choice never changes a
// result, it times each candidate on the caller's operands (one warm-up and
// three timed launches, CUDA events on the context stream) the first time a
// pattern is multiplied with a given value / vector type, and keeps the
// fastest in the pattern. Tuning needs an assigning product (the candidates
// write y) and a stream that is not being captured; otherwise the default
// kernel runs untuned.
template <typename MT, typename VT>
cmcg_status launch_spmv(cmcg_matrix A, const void* x, int32_t xb, void* y, int32_t mode) {
    const int forced = spmv_variant();
    if (forced >= 0) return launch_spmv_variant<MT, VT>(A, x, xb, y, mode, forced);
    cmcg_pattern p = A->pat;
    int8_t& choice = p->spmv_choice[DT<MT>::id][DT<VT>::id];
    if (choice >= 0) return launch_spmv_variant<MT, VT>(A, x, xb, y, mode, choice);
    if (p->format == CMCG_CSR) {
        const int vec = csr_vec_variant(p);
        if (vec >= 0) {
            log_msg(1, "product: skewed rows (%d rows, %lld entries), %d lanes per row", p->rows,
                    static_cast<long long>(p->nnz), 4 << (vec - 3));
            choice = static_cast<int8_t>(vec);
            return launch_spmv_variant<MT, VT>(A, x, xb, y, mode, vec);
        }
    }
    const std::string key = tune_key(p, DT<MT>::id, DT<VT>::id);
    const int cached = tune_lookup(key);
    if (cached == 0 || cached == 1 || cached == 2 || ((cached == 7 || cached == 8 || cached == 9) && p->format == CMCG_CSR)) {
        choice = static_cast<int8_t>(cached);
        return launch_spmv_variant<MT, VT>(A, x, xb, y, mode, cached);
    }
    cudaStream_t st = p->ctx->stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (mode != CMCG_ASSIGN || cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
        return launch_spmv_variant<MT, VT>(A, x, xb, y, mode, 0);
    // CSR: thread per row (one or two rows in flight), warp-staged entries,
    // four rows per thread with 16-byte chunks, bulk-staged tiles (the last
    // candidate's output stays in y); ELLPACK: four rows per thread, thread
    // per row
    int cands[5] = {0, 9, 8, 7, 2};
    int nc = 5;
    if (p->format != CMCG_CSR) {
        cands[1] = 1;
        nc = 2;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CMCG_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(CMCG_ERR_CUDA, "spmv autotune: event creation failed");
    }
    float best = 0.0f;
    int pick = cands[0];
    cmcg_status rc = CMCG_OK;
    for (int j = 0; j < nc; ++j) {
        const int c = cands[j];
        if ((rc = launch_spmv_variant<MT, VT>(A, x, xb, y, mode, c)) != CMCG_OK) break;
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3 && rc == CMCG_OK; ++r) rc = launch_spmv_variant<MT, VT>(A, x, xb, y, mode, c);
        cudaEventRecord(e1, st);
        float ms = 0.0f;
        if (rc != CMCG_OK || cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            if (rc == CMCG_OK) rc = fail(CMCG_ERR_CUDA, "spmv autotune: timing failed");
            break;
        }
        if (c == cands[0] || ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != CMCG_OK) return rc;
    choice = static_cast<int8_t>(pick);
    tune_store(key, pick);
    log_msg(1, "product %s: variant %d timed fastest (%.3f ms for 3 calls)", key.c_str(), pick, best);
    // the last candidate's output is in y; rerun the pick if it was another one
    return pick == cands[nc - 1] ? CMCG_OK : launch_spmv_variant<MT, VT>(A, x, xb, y, mode, pick);
}

cmcg_status spmv_dispatch(cmcg_matrix A, int32_t vec_dtype, const void* x, int32_t xb, void* y, int32_t mode) {
    if (vec_dtype == CMCG_F32) {
        switch (A->dtype) {
            case CMCG_F32: return launch_spmv<float, float>(A, x, xb, y, mode);
            case CMCG_BF16: return launch_spmv<__nv_bfloat16, float>(A, x, xb, y, mode);
            case CMCG_F64: return launch_spmv<double, float>(A, x, xb, y, mode);
        }
    } else if (vec_dtype == CMCG_F64) {
        switch (A->dtype) {
            case CMCG_F32: return launch_spmv<float, double>(A, x, xb, y, mode);
            case CMCG_BF16: return launch_spmv<__nv_bfloat16, double>(A, x, xb, y, mode);
            case CMCG_F64: return launch_spmv<double, double>(A, x, xb, y, mode);
        }
    }
    return fail(CMCG_ERR_INVALID_ARGUMENT, "cmcg_spmv: vector dtype must be F32 or F64");
}

cmcg_status dot_dispatch(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t xb, const void* y, int32_t yb,
                         void* out, int32_t ob) {
    if (dtype == CMCG_F32) return launch_dot<float>(ctx, n, x, xb, y, yb, out, ob);
    if (dtype == CMCG_F64) return launch_dot<double>(ctx, n, x, xb, y, yb, out, ob);
    return fail(CMCG_ERR_INVALID_ARGUMENT, "dot: dtype must be F32 or F64");
}

cmcg_status sddmm_dispatch(cmcg_matrix M, int32_t dt, double alpha, const void* u, int32_t ub, const void* v,
                           int32_t vb, void* out, int32_t ob) {
    if (dt != CMCG_F32 && dt != CMCG_F64) return fail(CMCG_ERR_INVALID_ARGUMENT, "sddmm: dtype must be F32 or F64");
    cmcg_pattern p = M->pat;
    // CSC / BSR patterns: the product in CSR order, then scattered into the
    // caller's value order
    void* tmp = nullptr;
    void* dst = out;
    if (p->d_val_perm) {
        CMCG_TRY(dev_alloc(&tmp, std::max<size_t>(static_cast<size_t>(p->nnz) * ob * dtype_size(dt), 16)));
        dst = tmp;
    }
    cmcg_status st = dt == CMCG_F32 ? launch_sddmm<float>(M, alpha, u, ub, v, vb, dst, ob)
                                    : launch_sddmm<double>(M, alpha, u, ub, v, vb, dst, ob);
    if (tmp) {
        if (st == CMCG_OK) st = permute_values(p, dt, tmp, p->nnz, out, p->nnz, ob, false);
        cudaStreamSynchronize(p->ctx->stream);
        dev_free(tmp);
    }
    return st;
}

}  // namespace cmcg

using namespace cmcg;

extern "C" {

cmcg_status cmcg_spmv(cmcg_matrix A, int32_t vec_dtype, const void* x, int32_t x_batches, void* y, int32_t mode) {
    NvtxRange nvtx_("cmcg_spmv");
    CMCG_REQUIRE(A && x && y, "cmcg_spmv: NULL argument");
    CMCG_REQUIRE(x_batches >= 1, "cmcg_spmv: x_batches must be >= 1");
    CMCG_REQUIRE(A->batches == 1 || x_batches == 1 || A->batches == x_batches,
                 "cmcg_spmv: batch counts of matrix and vector must match or be 1");
    CMCG_REQUIRE(mode == CMCG_ASSIGN || mode == CMCG_ADD || mode == CMCG_SUB, "cmcg_spmv: bad assignment mode");
    CMCG_CUDA(cudaSetDevice(A->pat->ctx->device));
    return spmv_dispatch(A, vec_dtype, x, x_batches, y, mode);
}

cmcg_status cmcg_dot(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t xb, const void* y, int32_t yb,
                     void* out) {
    NvtxRange nvtx_("cmcg_dot");
    CMCG_REQUIRE(ctx && x && y && out, "cmcg_dot: NULL argument");
    CMCG_REQUIRE(n >= 0 && xb >= 1 && yb >= 1, "cmcg_dot: bad size");
    CMCG_REQUIRE(xb == 1 || yb == 1 || xb == yb, "cmcg_dot: batch counts must match or be 1");
    CMCG_REQUIRE(std::max(xb, yb) <= 65535, "cmcg_dot: at most 65535 batches");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    return dot_dispatch(ctx, dtype, n, x, xb, y, yb, out, std::max(xb, yb));
}

cmcg_status cmcg_squared_norm(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t batches, void* out) {
    NvtxRange nvtx_("cmcg_squared_norm");
    return cmcg_dot(ctx, dtype, n, x, batches, x, batches, out);
}

}  // extern "C"

// ---- batched dot product without any allocation ----------------------------------
//
// cmcg_dot keeps its per-CTA partial sums and per-batch tickets in a context
// buffer that it allocates with cudaMalloc the first time (and grows). Some
// callers cannot let a library allocate: a host that has handed all device
// memory to its own pool or framework allocator (a cudaMalloc from the library
// would fail or fragment that memory), or a loop with a latency budget in which
// cudaMalloc / cudaFree and the synchronisation they can imply are not allowed.
// For them cmcg_dot_noalloc runs the same kernel with its scratch in the
// fixed-size device array below, which exists once per GPU that loads this
// library and stays allocated until the process exits.

namespace {

constexpr int kNoAllocMaxBatches = 1024;     // largest batch count accepted
constexpr int kNoAllocMaxPartials = 4096;    // partial sums (all batches together)

// [partials: kNoAllocMaxPartials doubles (room for floats too)][tickets: one
// unsigned per batch]. In host code this name is only a stand-in: its device
// address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_dot_scratch[kNoAllocMaxPartials * sizeof(double) +
                                                             kNoAllocMaxBatches * sizeof(unsigned)];

std::mutex g_dot_scratch_mu;
void* g_dot_scratch_addr[1024] = {};   // device address per device ordinal

// Address of the scratch array on `device`, looked up once per device with that
// device current (the caller has made it current).
cmcg_status dot_scratch_address(int device, void** out) {
    CMCG_REQUIRE(device >= 0 && device < 1024, "cmcg_dot_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_dot_scratch_mu);
    if (!g_dot_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_dot_scratch)", __FILE__, __LINE__);
        g_dot_scratch_addr[device] = p;
    }
    *out = g_dot_scratch_addr[device];
    return CMCG_OK;
}

template <typename VT>
cmcg_status launch_dot_noalloc(cmcg_ctx ctx, int64_t n, const void* x, int32_t xb, const void* y, int32_t yb,
                               void* out, int32_t ob) {
    void* base = nullptr;
    CMCG_TRY(dot_scratch_address(ctx->device, &base));
    VT* partial = static_cast<VT*>(base);
    unsigned* ticket = reinterpret_cast<unsigned*>(static_cast<unsigned char*>(base) + kNoAllocMaxPartials * sizeof(double));
    const int gx = dot_grid(ctx, n, ob, std::max(1, kNoAllocMaxPartials / ob));
    // the tickets must start at zero; every call clears them (no allocation)
    CMCG_CUDA(cudaMemsetAsync(ticket, 0, ob * sizeof(unsigned), ctx->stream));
    dim3 grid(gx, ob);
    k_dot<VT><<<grid, kRedThreads, 0, ctx->stream>>>(n, static_cast<const VT*>(x), xb, static_cast<const VT*>(y), yb,
                                                     static_cast<VT*>(out), partial, ticket);
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

}  // namespace

extern "C" {

cmcg_status cmcg_dot_noalloc(cmcg_ctx ctx, int32_t dtype, int64_t n, const void* x, int32_t xb, const void* y,
                             int32_t yb, void* out) {
    NvtxRange nvtx_("cmcg_dot_noalloc");
    CMCG_REQUIRE(ctx && x && y && out, "cmcg_dot_noalloc: NULL argument");
    CMCG_REQUIRE(n >= 0 && xb >= 1 && yb >= 1, "cmcg_dot_noalloc: bad size");
    CMCG_REQUIRE(xb == 1 || yb == 1 || xb == yb, "cmcg_dot_noalloc: batch counts must match or be 1");
    const int32_t ob = std::max(xb, yb);
    if (ob > kNoAllocMaxBatches)
        return fail(CMCG_ERR_INVALID_ARGUMENT, "cmcg_dot_noalloc: " + std::to_string(ob) +
                                                   " batches requested, the fixed scratch holds at most " +
                                                   std::to_string(kNoAllocMaxBatches) + " (use cmcg_dot)");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    if (dtype == CMCG_F32) return launch_dot_noalloc<float>(ctx, n, x, xb, y, yb, out, ob);
    if (dtype == CMCG_F64) return launch_dot_noalloc<double>(ctx, n, x, xb, y, yb, out, ob);
    return fail(CMCG_ERR_INVALID_ARGUMENT, "cmcg_dot_noalloc: dtype must be F32 or F64");
}

cmcg_status cmcg_sddmm(cmcg_matrix M, int32_t vec_dtype, double alpha, const void* u, int32_t ub, const void* v,
                       int32_t vb, void* out, int32_t ob) {
    NvtxRange nvtx_("cmcg_sddmm");
    CMCG_REQUIRE(M && u && v && out, "cmcg_sddmm: NULL argument");
    CMCG_REQUIRE(ub >= 1 && vb >= 1 && ob >= 1, "cmcg_sddmm: batch counts must be >= 1");
    CMCG_REQUIRE((ub == 1 || ub == ob) && (vb == 1 || vb == ob), "cmcg_sddmm: batch counts must match or be 1");
    CMCG_CUDA(cudaSetDevice(M->pat->ctx->device));
    return sddmm_dispatch(M, vec_dtype, alpha, u, ub, v, vb, out, ob);
}

}  // extern "C"
