// Storage formats beside CSR and ELLPACK, the transposed product, and dense
// <-> sparse evaluation on a pattern.
//
//  cmcg_pattern_create_csc   replaces SparsityPattern<CSC> (cuMat/src/SparseMatrixBase.h:29-87)
//  cmcg_pattern_create_bsr   replaces a CSR pattern of block scalars (a row-major float3x3 with
//                            float3 vectors, tests/TestBlockedConjugateGradient.cu:10-237)
//  cmcg_spmv_transposed      y = A^T x (the reference leaves transposed operands as a TODO,
//                            SparseProductEvaluation.h:94)
//  cmcg_matrix_to_dense,
//  cmcg_matrix_from_dense    sparse -> dense and dense -> sparse on the pattern (the coefficient-wise
//                            evaluation of SparseEvaluation.h:15-34, tests TestSparseMatrix.cu:10-384)
//
// Design: a CSC or BSR pattern is turned, on the host and once, into the
// equivalent CSR pattern that every kernel of the library already takes (a
// BSR block row becomes `block` scalar rows whose entries follow the row's
// blocks in order), plus a map from each CSR entry to the caller's value
// index. Matrices keep their values in CSR order; uploads gather through the
// map and downloads scatter back, so products, the CG kernels (persistent,
// grid, mixed precision, adjoint) and reductions need no format of their own.
// The transposed product walks the pattern's transpose (built once per
// pattern, counting sort by column) thread per column, over a copy of the
// values in the transpose's entry order (gathered once per value upload, so
// the product streams them like a CSR product): no atomics, a fixed
// summation order.

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "objects.h"

namespace cmcg {
namespace {

template <typename T>
__global__ void k_permute(const T* __restrict__ src, int64_t sstride, T* __restrict__ dst, int64_t dstride,
                          const int32_t* __restrict__ perm, int64_t nnz, int32_t batches, int32_t gather) {
    const int64_t items = nnz * batches;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < items;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = i / nnz, k = i - b * nnz;
        if (gather) dst[b * dstride + k] = src[b * sstride + perm[k]];
        else dst[b * dstride + perm[k]] = src[b * sstride + k];
    }
}

template <int MODE, typename VT>
__device__ __forceinline__ void put(VT* y, VT v) {
    if (MODE == CMCG_ASSIGN) *y = v;
    else if (MODE == CMCG_ADD) *y += v;
    else *y -= v;
}

// y[b][c] (mode)= sum over the entries (r, c) of A of a_rc x[b][r]: thread per
// column c of A over the transpose's entries (row index trow[k], value tv[k]
// in the transpose's order), entries in ascending row order; kTUnroll entries
// of the column are loaded before the first gather
constexpr int kTUnroll = 8;

template <typename MT, typename VT, int MODE>
__global__ void __launch_bounds__(256) k_spmv_t(const int32_t* __restrict__ trp, const int32_t* __restrict__ trow,
                                                const MT* __restrict__ tvals, int64_t tstride, int32_t mb,
                                                const VT* __restrict__ x, int32_t rows, int32_t xb, VT* __restrict__ y,
                                                int32_t cols, int32_t ob) {
    const int64_t items = static_cast<int64_t>(cols) * ob;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(it / cols);
        const int c = static_cast<int>(it - static_cast<int64_t>(b) * cols);
        const MT* tv = tvals + (mb == 1 ? 0 : b * tstride);
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * rows);
        VT acc = VT(0);
        const int e = __ldg(trp + c + 1);
        for (int k = __ldg(trp + c); k < e; k += kTUnroll) {
            int r[kTUnroll];
            MT w[kTUnroll];
#pragma unroll
            for (int u = 0; u < kTUnroll; ++u) {
                const bool in = k + u < e;
                r[u] = in ? __ldg(trow + k + u) : -1;
                w[u] = in ? tv[k + u] : MT{};
            }
#pragma unroll
            for (int u = 0; u < kTUnroll; ++u)
                if (r[u] >= 0) acc = fma(mval<VT>(w[u]), __ldg(xv + r[u]), acc);
        }
        put<MODE>(y + it, acc);
    }
}

// dense index of (r, c) in batch b
__device__ __forceinline__ int64_t dense_at(int64_t b, int r, int c, int rows, int cols, int row_major) {
    return row_major ? (b * rows + r) * static_cast<int64_t>(cols) + c : (b * cols + c) * static_cast<int64_t>(rows) + r;
}

// thread per (batch, row): TO = true writes the stored values into the dense
// matrix, false reads the dense values at the stored entries
template <typename T, bool TO>
__global__ void k_dense_csr(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, T* vals, int64_t vstride,
                            int32_t mb, T* dense, int32_t rows, int32_t cols, int32_t row_major) {
    const int64_t items = static_cast<int64_t>(rows) * mb;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = it / rows;
        const int r = static_cast<int>(it - b * rows);
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            const int64_t d = dense_at(b, r, ci[k], rows, cols, row_major);
            if (TO) dense[d] = vals[b * vstride + k];
            else vals[b * vstride + k] = dense[d];
        }
    }
}

template <typename T, bool TO>
__global__ void k_dense_ell(const int32_t* __restrict__ idx, int32_t width, int32_t rows_pad, T* vals, int64_t vstride,
                            int32_t mb, T* dense, int32_t rows, int32_t cols, int32_t row_major) {
    const int64_t items = static_cast<int64_t>(rows) * mb;
    for (int64_t it = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = it / rows;
        const int r = static_cast<int>(it - b * rows);
        for (int j = 0; j < width; ++j) {
            const int64_t o = static_cast<int64_t>(j) * rows_pad + r;
            const int c = idx[o];
            if (c < 0) continue;
            const int64_t d = dense_at(b, r, c, rows, cols, row_major);
            if (TO) dense[d] = vals[b * vstride + o];
            else vals[b * vstride + o] = dense[d];
        }
    }
}

int grid_for(cmcg_ctx ctx, int64_t items) {
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((items + 255) / 256, ctx->sm_count * 16)));
}

// Marks a CSR pattern just created from the caller's CSC / BSR arrays and
// uploads the value map.
cmcg_status attach_declared(cmcg_pattern p, int32_t declared, const std::vector<int32_t>& perm,
                            std::vector<int32_t>&& ptr, std::vector<int32_t>&& idx, int64_t decl_nnz) {
    p->declared = declared;
    p->decl_nnz = decl_nnz;
    p->h_decl_ptr = std::move(ptr);
    p->h_decl_idx = std::move(idx);
    CMCG_TRY(dev_alloc(reinterpret_cast<void**>(&p->d_val_perm), std::max<size_t>(perm.size(), 1) * sizeof(int32_t)));
    if (!perm.empty())
        CMCG_CUDA(cudaMemcpy(p->d_val_perm, perm.data(), perm.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    return CMCG_OK;
}

// the pattern's transpose (counting sort of the entries by column; within a
// column ascending rows, since rows are visited in order)
cmcg_status ensure_transpose(cmcg_pattern p) {
    if (p->d_t_row_ptr) return CMCG_OK;
    const auto& rp = p->h_row_ptr;
    const auto& ci = p->h_col;
    std::vector<int32_t> trp(static_cast<size_t>(p->cols) + 1, 0), trow(static_cast<size_t>(p->nnz)),
        tperm(static_cast<size_t>(p->nnz));
    for (int64_t k = 0; k < p->nnz; ++k) trp[ci[k] + 1]++;
    for (int32_t c = 0; c < p->cols; ++c) trp[c + 1] += trp[c];
    std::vector<int32_t> next(trp.begin(), trp.end() - 1);
    for (int32_t r = 0; r < p->rows; ++r)
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) {
            const int32_t pos = next[ci[k]]++;
            trow[pos] = r;
            tperm[pos] = k;
        }
    int32_t *a = nullptr, *b = nullptr, *c = nullptr;
    cmcg_status st = dev_alloc(reinterpret_cast<void**>(&a), trp.size() * sizeof(int32_t));
    if (st == CMCG_OK) st = dev_alloc(reinterpret_cast<void**>(&b), std::max<size_t>(trow.size(), 1) * sizeof(int32_t));
    if (st == CMCG_OK) st = dev_alloc(reinterpret_cast<void**>(&c), std::max<size_t>(tperm.size(), 1) * sizeof(int32_t));
    if (st == CMCG_OK &&
        (cudaMemcpy(a, trp.data(), trp.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
         (p->nnz && cudaMemcpy(b, trow.data(), trow.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) ||
         (p->nnz && cudaMemcpy(c, tperm.data(), tperm.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)))
        st = fail(CMCG_ERR_CUDA, "transposed pattern: upload failed");
    if (st != CMCG_OK) {
        dev_free(a);
        dev_free(b);
        dev_free(c);
        return st;
    }
    p->d_t_row_ptr = a;
    p->d_t_col = b;
    p->d_t_perm = c;
    return CMCG_OK;
}

// A's values in the transpose's entry order (gathered through d_t_perm once
// per value upload)
cmcg_status ensure_t_values(cmcg_matrix A) {
    if (A->d_t_vals && A->t_version == A->version) return CMCG_OK;
    cmcg_pattern p = A->pat;
    cmcg_ctx ctx = p->ctx;
    const int64_t stride = csr_padded_nnz(p->nnz);
    if (!A->d_t_vals) {
        CMCG_TRY(dev_alloc(&A->d_t_vals, static_cast<size_t>(stride) * A->batches * dtype_size(A->dtype)));
        A->t_stride = stride;
    }
    if (p->nnz > 0) {
        const int grid = grid_for(ctx, p->nnz * A->batches);
        switch (dtype_size(A->dtype)) {
            case 2:
                k_permute<uint16_t><<<grid, 256, 0, ctx->stream>>>(static_cast<const uint16_t*>(A->d_vals), A->stride,
                                                                   static_cast<uint16_t*>(A->d_t_vals), stride,
                                                                   p->d_t_perm, p->nnz, A->batches, 1);
                break;
            case 4:
                k_permute<uint32_t><<<grid, 256, 0, ctx->stream>>>(static_cast<const uint32_t*>(A->d_vals), A->stride,
                                                                   static_cast<uint32_t*>(A->d_t_vals), stride,
                                                                   p->d_t_perm, p->nnz, A->batches, 1);
                break;
            default:
                k_permute<uint64_t><<<grid, 256, 0, ctx->stream>>>(static_cast<const uint64_t*>(A->d_vals), A->stride,
                                                                   static_cast<uint64_t*>(A->d_t_vals), stride,
                                                                   p->d_t_perm, p->nnz, A->batches, 1);
        }
        count_launch();
        CMCG_CHECK_LAUNCH();
    }
    A->t_version = A->version;
    return CMCG_OK;
}

template <typename MT, typename VT>
cmcg_status launch_spmv_t(cmcg_matrix A, const void* x, int32_t xb, void* y, int32_t mode) {
    cmcg_pattern p = A->pat;
    cmcg_ctx ctx = p->ctx;
    CMCG_TRY(ensure_t_values(A));
    const int32_t ob = std::max(A->batches, xb);
    const int grid = grid_for(ctx, static_cast<int64_t>(p->cols) * ob);
#define CMCG_SPMV_T(M)                                                                                              \
    k_spmv_t<MT, VT, M><<<grid, 256, 0, ctx->stream>>>(p->d_t_row_ptr, p->d_t_col, static_cast<const MT*>(A->d_t_vals), \
                                                       A->t_stride, A->batches, static_cast<const VT*>(x), p->rows, xb, \
                                                       static_cast<VT*>(y), p->cols, ob)
    if (mode == CMCG_ASSIGN) CMCG_SPMV_T(CMCG_ASSIGN);
    else if (mode == CMCG_ADD) CMCG_SPMV_T(CMCG_ADD);
    else CMCG_SPMV_T(CMCG_SUB);
#undef CMCG_SPMV_T
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

template <typename T>
cmcg_status dense_t(cmcg_matrix A, void* dense, int32_t row_major, bool to) {
    cmcg_pattern p = A->pat;
    cmcg_ctx ctx = p->ctx;
    T* v = static_cast<T*>(A->d_vals);
    T* d = static_cast<T*>(dense);
    const int grid = grid_for(ctx, static_cast<int64_t>(p->rows) * A->batches);
    if (to) {
        CMCG_CUDA(cudaMemsetAsync(dense, 0, static_cast<size_t>(p->rows) * p->cols * A->batches * sizeof(T), ctx->stream));
        if (p->format == CMCG_CSR)
            k_dense_csr<T, true><<<grid, 256, 0, ctx->stream>>>(p->d_row_ptr, p->d_col, v, A->stride, A->batches, d,
                                                                p->rows, p->cols, row_major);
        else
            k_dense_ell<T, true><<<grid, 256, 0, ctx->stream>>>(p->d_ell, p->width, p->rows_pad, v, A->stride,
                                                                A->batches, d, p->rows, p->cols, row_major);
    } else {
        if (p->format == CMCG_CSR)
            k_dense_csr<T, false><<<grid, 256, 0, ctx->stream>>>(p->d_row_ptr, p->d_col, v, A->stride, A->batches, d,
                                                                 p->rows, p->cols, row_major);
        else
            k_dense_ell<T, false><<<grid, 256, 0, ctx->stream>>>(p->d_ell, p->width, p->rows_pad, v, A->stride,
                                                                 A->batches, d, p->rows, p->cols, row_major);
        A->version++;
    }
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

cmcg_status dense_dispatch(cmcg_matrix A, void* dense, int32_t row_major, bool to) {
    switch (A->dtype) {
        case CMCG_F32: return dense_t<float>(A, dense, row_major, to);
        case CMCG_F64: return dense_t<double>(A, dense, row_major, to);
        default: return dense_t<__nv_bfloat16>(A, dense, row_major, to);
    }
}

}  // namespace

cmcg_status permute_values(cmcg_pattern p, int32_t dtype, const void* src, int64_t src_stride, void* dst,
                           int64_t dst_stride, int32_t batches, bool to_internal) {
    cmcg_ctx ctx = p->ctx;
    const int64_t n = p->nnz;
    if (n == 0) return CMCG_OK;
    const int grid = grid_for(ctx, n * batches);
    const int g = to_internal ? 1 : 0;
    switch (dtype_size(dtype)) {
        case 2:
            k_permute<uint16_t><<<grid, 256, 0, ctx->stream>>>(static_cast<const uint16_t*>(src), src_stride,
                                                               static_cast<uint16_t*>(dst), dst_stride, p->d_val_perm, n,
                                                               batches, g);
            break;
        case 4:
            k_permute<uint32_t><<<grid, 256, 0, ctx->stream>>>(static_cast<const uint32_t*>(src), src_stride,
                                                               static_cast<uint32_t*>(dst), dst_stride, p->d_val_perm, n,
                                                               batches, g);
            break;
        default:
            k_permute<uint64_t><<<grid, 256, 0, ctx->stream>>>(static_cast<const uint64_t*>(src), src_stride,
                                                               static_cast<uint64_t*>(dst), dst_stride, p->d_val_perm, n,
                                                               batches, g);
    }
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

void free_declared(cmcg_pattern p) {
    dev_free(p->d_val_perm);
    dev_free(p->d_t_row_ptr);
    dev_free(p->d_t_col);
    dev_free(p->d_t_perm);
    p->d_val_perm = p->d_t_row_ptr = p->d_t_col = p->d_t_perm = nullptr;
}

}  // namespace cmcg

using namespace cmcg;

extern "C" {

cmcg_status cmcg_pattern_create_csc(cmcg_ctx ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* col_ptr,
                                    const int32_t* row_idx, int32_t is_device, cmcg_pattern* out) {
    CMCG_REQUIRE(ctx && out, "cmcg_pattern_create_csc: NULL context or output");
    *out = nullptr;
    CMCG_REQUIRE(rows > 0 && cols > 0, "cmcg_pattern_create_csc: rows and cols must be positive");
    CMCG_REQUIRE(nnz >= 0 && nnz <= INT32_MAX, "cmcg_pattern_create_csc: nnz must be in [0, 2^31)");
    CMCG_REQUIRE(col_ptr != nullptr && (nnz == 0 || row_idx != nullptr), "cmcg_pattern_create_csc: NULL index array");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    std::vector<int32_t> cp(static_cast<size_t>(cols) + 1), ri(static_cast<size_t>(nnz));
    const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    CMCG_CUDA(cudaMemcpy(cp.data(), col_ptr, cp.size() * sizeof(int32_t), kind));
    if (nnz) CMCG_CUDA(cudaMemcpy(ri.data(), row_idx, ri.size() * sizeof(int32_t), kind));
    CMCG_REQUIRE(cp[0] == 0 && cp[cols] == nnz, "CSC col_ptr must start at 0 and end at nnz");
    for (int32_t c = 0; c < cols; ++c)
        if (cp[c + 1] < cp[c]) return fail(CMCG_ERR_INVALID_ARGUMENT, "CSC col_ptr must be non-decreasing (column " + std::to_string(c) + ")");
    for (int64_t k = 0; k < nnz; ++k)
        if (ri[k] < 0 || ri[k] >= rows)
            return fail(CMCG_ERR_INVALID_ARGUMENT, "CSC row index out of range at entry " + std::to_string(k));
    // the equivalent CSR pattern: entries of a row in ascending column order
    std::vector<int32_t> rp(static_cast<size_t>(rows) + 1, 0), col(static_cast<size_t>(nnz)), perm(static_cast<size_t>(nnz));
    for (int64_t k = 0; k < nnz; ++k) rp[ri[k] + 1]++;
    for (int32_t r = 0; r < rows; ++r) rp[r + 1] += rp[r];
    std::vector<int32_t> next(rp.begin(), rp.end() - 1);
    for (int32_t c = 0; c < cols; ++c)
        for (int32_t k = cp[c]; k < cp[c + 1]; ++k) {
            const int32_t pos = next[ri[k]]++;
            col[pos] = c;
            perm[pos] = k;
        }
    cmcg_pattern p = nullptr;
    CMCG_TRY(cmcg_pattern_create_csr(ctx, rows, cols, nnz, rp.data(), col.data(), 0, &p));
    cmcg_status st = attach_declared(p, CMCG_CSC, perm, std::move(cp), std::move(ri), nnz);
    if (st != CMCG_OK) {
        cmcg_pattern_destroy(p);
        return st;
    }
    *out = p;
    return CMCG_OK;
}

cmcg_status cmcg_pattern_create_bsr(cmcg_ctx ctx, int32_t block_rows, int32_t block_cols, int32_t block_size,
                                    int64_t nnz_blocks, const int32_t* row_ptr, const int32_t* col_idx,
                                    int32_t is_device, cmcg_pattern* out) {
    CMCG_REQUIRE(ctx && out, "cmcg_pattern_create_bsr: NULL context or output");
    *out = nullptr;
    CMCG_REQUIRE(block_rows > 0 && block_cols > 0, "cmcg_pattern_create_bsr: block rows and columns must be positive");
    CMCG_REQUIRE(block_size >= 2 && block_size <= 8, "cmcg_pattern_create_bsr: block size must be 2 .. 8");
    const int64_t B = block_size;
    CMCG_REQUIRE(static_cast<int64_t>(block_rows) * B <= INT32_MAX && static_cast<int64_t>(block_cols) * B <= INT32_MAX,
                 "cmcg_pattern_create_bsr: too many rows");
    CMCG_REQUIRE(nnz_blocks >= 0 && nnz_blocks * B * B <= INT32_MAX, "cmcg_pattern_create_bsr: too many entries");
    CMCG_REQUIRE(row_ptr != nullptr && (nnz_blocks == 0 || col_idx != nullptr), "cmcg_pattern_create_bsr: NULL index array");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    std::vector<int32_t> brp(static_cast<size_t>(block_rows) + 1), bci(static_cast<size_t>(nnz_blocks));
    const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    CMCG_CUDA(cudaMemcpy(brp.data(), row_ptr, brp.size() * sizeof(int32_t), kind));
    if (nnz_blocks) CMCG_CUDA(cudaMemcpy(bci.data(), col_idx, bci.size() * sizeof(int32_t), kind));
    CMCG_REQUIRE(brp[0] == 0 && brp[block_rows] == nnz_blocks, "BSR row_ptr must start at 0 and end at nnz_blocks");
    for (int32_t r = 0; r < block_rows; ++r)
        if (brp[r + 1] < brp[r]) return fail(CMCG_ERR_INVALID_ARGUMENT, "BSR row_ptr must be non-decreasing (block row " + std::to_string(r) + ")");
    for (int64_t k = 0; k < nnz_blocks; ++k)
        if (bci[k] < 0 || bci[k] >= block_cols)
            return fail(CMCG_ERR_INVALID_ARGUMENT, "BSR block column out of range at block " + std::to_string(k));
    // block row I -> scalar rows I B + i; each holds, block by block in order,
    // the B entries (i, j) of the row's blocks: columns J B + j, caller's value
    // k B^2 + i B + j
    const int32_t rows = static_cast<int32_t>(block_rows * B), cols = static_cast<int32_t>(block_cols * B);
    const int64_t nnz = nnz_blocks * B * B;
    std::vector<int32_t> rp(static_cast<size_t>(rows) + 1), col(static_cast<size_t>(nnz)), perm(static_cast<size_t>(nnz));
    int64_t pos = 0;
    rp[0] = 0;
    for (int32_t I = 0; I < block_rows; ++I)
        for (int64_t i = 0; i < B; ++i) {
            for (int32_t k = brp[I]; k < brp[I + 1]; ++k)
                for (int64_t j = 0; j < B; ++j) {
                    col[pos] = static_cast<int32_t>(bci[k] * B + j);
                    perm[pos] = static_cast<int32_t>(k * B * B + i * B + j);
                    ++pos;
                }
            rp[I * B + i + 1] = static_cast<int32_t>(pos);
        }
    cmcg_pattern p = nullptr;
    CMCG_TRY(cmcg_pattern_create_csr(ctx, rows, cols, nnz, rp.data(), col.data(), 0, &p));
    p->block = block_size;
    p->decl_rows = block_rows;
    p->decl_cols = block_cols;
    cmcg_status st = attach_declared(p, CMCG_BSR, perm, std::move(brp), std::move(bci), nnz_blocks);
    if (st != CMCG_OK) {
        cmcg_pattern_destroy(p);
        return st;
    }
    *out = p;
    return CMCG_OK;
}

cmcg_status cmcg_spmv_transposed(cmcg_matrix A, int32_t vec_dtype, const void* x, int32_t x_batches, void* y,
                                 int32_t mode) {
    NvtxRange nvtx_("cmcg_spmv_transposed");
    CMCG_REQUIRE(A && x && y, "cmcg_spmv_transposed: NULL argument");
    CMCG_REQUIRE(A->pat->format == CMCG_CSR, "cmcg_spmv_transposed: CSR, CSC or BSR patterns only");
    CMCG_REQUIRE(x_batches >= 1 && (A->batches == 1 || x_batches == 1 || x_batches == A->batches),
                 "cmcg_spmv_transposed: batch counts must match or be 1");
    CMCG_REQUIRE(mode == CMCG_ASSIGN || mode == CMCG_ADD || mode == CMCG_SUB, "cmcg_spmv_transposed: bad mode");
    CMCG_CUDA(cudaSetDevice(A->pat->ctx->device));
    CMCG_TRY(ensure_transpose(A->pat));
    if (vec_dtype == CMCG_F32) {
        switch (A->dtype) {
            case CMCG_F32: return launch_spmv_t<float, float>(A, x, x_batches, y, mode);
            case CMCG_F64: return launch_spmv_t<double, float>(A, x, x_batches, y, mode);
            default: return launch_spmv_t<__nv_bfloat16, float>(A, x, x_batches, y, mode);
        }
    }
    if (vec_dtype == CMCG_F64) {
        switch (A->dtype) {
            case CMCG_F32: return launch_spmv_t<float, double>(A, x, x_batches, y, mode);
            case CMCG_F64: return launch_spmv_t<double, double>(A, x, x_batches, y, mode);
            default: return launch_spmv_t<__nv_bfloat16, double>(A, x, x_batches, y, mode);
        }
    }
    return fail(CMCG_ERR_INVALID_ARGUMENT, "cmcg_spmv_transposed: vector dtype must be F32 or F64");
}

cmcg_status cmcg_matrix_to_dense(cmcg_matrix A, void* dense, int32_t row_major) {
    CMCG_REQUIRE(A && dense, "cmcg_matrix_to_dense: NULL argument");
    CMCG_CUDA(cudaSetDevice(A->pat->ctx->device));
    return dense_dispatch(A, dense, row_major, true);
}

cmcg_status cmcg_matrix_from_dense(cmcg_matrix A, const void* dense, int32_t row_major) {
    CMCG_REQUIRE(A && dense, "cmcg_matrix_from_dense: NULL argument");
    CMCG_CUDA(cudaSetDevice(A->pat->ctx->device));
    return dense_dispatch(A, const_cast<void*>(dense), row_major, false);
}

}  // extern "C"
