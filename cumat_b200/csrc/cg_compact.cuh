// Device helpers of the persistent kernels over the compact sliced layout
// (CSR patterns whose systems have at most 65536 rows), shared by the plain
// and the mixed-precision kernels, and the launch interface of the mixed one.
#pragma once

#include "cg_dev.cuh"
#include "cg_grid.cuh"
#include "cg_smem.cuh"
#include "common.cuh"

namespace cmcg {

// Next work item of a persistent CTA (one atomic per CTA, broadcast through
// shared memory).
__device__ __forceinline__ int fetch_item(int32_t* next, int* slot) {
    if (threadIdx.x == 0) *slot = atomicAdd(next, 1);
    __syncthreads();
    const int item = *slot;
    __syncthreads();
    return item;
}

// Compact sliced layout: 16-bit system-local column indices, the slice offsets
// / widths a warp visits cached in shared memory once per system (no dependent
// global loads per row), 32-bit offsets.

struct SliceEnt {
    int32_t off;
    int32_t w;
};

// tab[w][k]: slice w + 32 k of the system (local rows 32 (w + 32 k) ...), the
// slice holding the rows tid + k * 1024 of warp w.
// (T threads per CTA: warp w's rows in slot k are those of slice w + (T / 32) k)
template <int T = kSmemThreads>
__device__ __forceinline__ void load_slice_table(SliceEnt (*tab)[kSmemNK], const int32_t* __restrict__ off32,
                                                 const int32_t* __restrict__ sw, int sl0, int nsl) {
    for (int t = threadIdx.x; t < (T / 32) * kSmemNK; t += blockDim.x) {
        const int w = t / kSmemNK, k = t - (t / kSmemNK) * kSmemNK, sl = w + (T / 32) * k;
        tab[w][k] = sl < nsl ? SliceEnt{__ldg(off32 + sl0 + sl), __ldg(sw + sl0 + sl)} : SliceEnt{0, 0};
    }
}

template <typename T>
struct LocalX {
    const T* p;
    __device__ __forceinline__ T operator()(int c) const { return p[c]; }
};

// W entries of a row, fully unrolled: every load is the row's base pointer
// plus an immediate offset; all loads issue before the first product; the
// products are summed in entry order.
template <int W, typename VT, typename MT, typename XF>
__device__ __forceinline__ VT row_w(const uint16_t* __restrict__ c, const MT* __restrict__ v, const XF& xf) {
    int ci[W];
    MT vi[W];
#pragma unroll
    for (int j = 0; j < W; ++j) {
        ci[j] = __ldg(c + 32 * j);
        vi[j] = v[32 * j];
    }
    VT acc = VT(0);
#pragma unroll
    for (int j = 0; j < W; ++j) acc += mval<VT>(vi[j]) * xf(ci[j]);
    return acc;
}

// Entries of the lane's row in one compact slice, summed in entry order.
template <typename VT, typename MT, typename XF>
__device__ __forceinline__ VT fast_row(const uint16_t* __restrict__ col, const MT* __restrict__ val, SliceEnt e, int lane,
                                       const XF& xf) {
    const uint16_t* c = col + e.off + lane;
    const MT* v = val + e.off + lane;
    switch (e.w) {   // warp-uniform: one slice per warp
        case 0: return VT(0);
        case 1: return row_w<1, VT>(c, v, xf);
        case 2: return row_w<2, VT>(c, v, xf);
        case 3: return row_w<3, VT>(c, v, xf);
        case 4: return row_w<4, VT>(c, v, xf);
        case 5: return row_w<5, VT>(c, v, xf);
        case 6: return row_w<6, VT>(c, v, xf);
        case 7: return row_w<7, VT>(c, v, xf);
        case 8: return row_w<8, VT>(c, v, xf);
        default: break;
    }
    VT acc = VT(0);
    int j = 0;
    for (; j + 4 <= e.w; j += 4) {
        const int c0 = __ldg(c + 32 * j), c1 = __ldg(c + 32 * (j + 1)), c2 = __ldg(c + 32 * (j + 2)),
                  c3 = __ldg(c + 32 * (j + 3));
        const MT v0 = v[32 * j], v1 = v[32 * (j + 1)], v2 = v[32 * (j + 2)], v3 = v[32 * (j + 3)];
        acc += mval<VT>(v0) * xf(c0);
        acc += mval<VT>(v1) * xf(c1);
        acc += mval<VT>(v2) * xf(c2);
        acc += mval<VT>(v3) * xf(c3);
    }
    for (; j < e.w; ++j) acc += mval<VT>(v[32 * j]) * xf(__ldg(c + 32 * j));
    return acc;
}

// Two rows of equal width W (the lane's rows in two slices): the 4 W index
// and value loads of both rows issue before the first product, so the two
// rows cost one memory latency instead of two; each row sums in entry order.
template <int W, typename VT, typename MT, typename XF>
__device__ __forceinline__ void row_w2(const uint16_t* __restrict__ c0, const MT* __restrict__ v0,
                                       const uint16_t* __restrict__ c1, const MT* __restrict__ v1, const XF& xf, VT& q0,
                                       VT& q1) {
    int ci0[W], ci1[W];
    MT vi0[W], vi1[W];
#pragma unroll
    for (int j = 0; j < W; ++j) {
        ci0[j] = __ldg(c0 + 32 * j);
        vi0[j] = v0[32 * j];
        ci1[j] = __ldg(c1 + 32 * j);
        vi1[j] = v1[32 * j];
    }
    VT a0 = VT(0), a1 = VT(0);
#pragma unroll
    for (int j = 0; j < W; ++j) {
        a0 += mval<VT>(vi0[j]) * xf(ci0[j]);
        a1 += mval<VT>(vi1[j]) * xf(ci1[j]);
    }
    q0 = a0;
    q1 = a1;
}

// fast_row for the lane's rows in two slices (e1.w == 0: no second row).
template <typename VT, typename MT, typename XF>
__device__ __forceinline__ void fast_rows2(const uint16_t* __restrict__ col, const MT* __restrict__ val, SliceEnt e0,
                                           SliceEnt e1, int lane, const XF& xf, VT& q0, VT& q1) {
    if (e0.w == e1.w) {   // warp-uniform
        const uint16_t* c0 = col + e0.off + lane;
        const MT* v0 = val + e0.off + lane;
        const uint16_t* c1 = col + e1.off + lane;
        const MT* v1 = val + e1.off + lane;
        switch (e0.w) {
            case 0: q0 = q1 = VT(0); return;
            case 3: row_w2<3>(c0, v0, c1, v1, xf, q0, q1); return;
            case 4: row_w2<4>(c0, v0, c1, v1, xf, q0, q1); return;
            case 5: row_w2<5>(c0, v0, c1, v1, xf, q0, q1); return;
            default: break;
        }
        // wider rows only with 4-byte values (register budget of 1024-thread CTAs)
        if constexpr (sizeof(MT) <= 4) {
            if (e0.w == 6) { row_w2<6>(c0, v0, c1, v1, xf, q0, q1); return; }
            if (e0.w == 7) { row_w2<7>(c0, v0, c1, v1, xf, q0, q1); return; }
        }
    }
    q0 = fast_row<VT>(col, val, e0, lane, xf);
    q1 = fast_row<VT>(col, val, e1, lane, xf);
}

struct CompactArgs {
    const uint16_t* col16;
    const int32_t* off32;
    const int32_t* sw;
    const int32_t* sys_slice0;
};

template <typename MI, typename MO>
struct MixArgs {
    int32_t rows, n_sys, ob, mb;
    const int32_t* row_off;
    const int32_t* order;
    int32_t* next;                 // work counter of this launch
    int32_t item_begin, item_end;  // its work items: (position in order) * ob + batch
    CompactArgs c;
    const MI* vin;          // Jacobi-scaled inner values, sliced layout
    int64_t vin_stride;
    const MO* vout;         // unscaled outer values, sliced layout
    int64_t vout_stride;
    const double* s;        // scale 1/sqrt(a_ii) (or 1), [mb][rows]
    const double* b;
    int32_t b_b;
    double* x;
    double outer_tol;
    int64_t max_inner;
    int32_t max_updates;
    float delta;
    InstState st;
    // diagonal layout of the scaled inner values (kernels built with ND > 0)
    const MI* vdia;         // [mb][vdia_stride]
    int64_t vdia_stride;
    const int64_t* dia_base;   // n_sys
    const int32_t* dia_off;    // n_sys * kDiaMax
    int32_t margin;            // largest |offset|: zero halo around p in shared memory
    const int32_t* dia_unit;   // [mb][n_sys]: 1 = middle diagonal is offset 0 with all values 1
};

// Systems of at most this many rows may run on 512-thread CTAs, two per SM,
// or on 256-thread CTAs, four per SM.
constexpr int kMixSmallRows = kSmemNK * 512;
constexpr int kMixTinyRows = kSmemNK * 256;

// Launches k_mixed_fast (cg_mixed.cu) with `threads` (1024, 512 or 256) threads per
// CTA and `smem` bytes of dynamic shared memory: nd = 0 sliced layout, nd = 5
// or 7 diagonal layout.
template <typename MI, typename MO>
cmcg_status launch_mixed_fast(const MixArgs<MI, MO>& m, int threads, int nmax, size_t smem, int nd, int grid,
                              cudaStream_t stream);

}  // namespace cmcg
