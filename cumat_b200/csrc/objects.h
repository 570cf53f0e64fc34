// Library-owned objects behind the C ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/cumat_cg.h"

struct cmcg_ctx_s {
    int32_t device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 148;
    // scratch for the batched dot / squared-norm combine (grown on demand)
    void* red_partial = nullptr;
    size_t red_partial_bytes = 0;
    unsigned* red_ticket = nullptr;
    size_t red_ticket_count = 0;
};

// Sparsity pattern. CSR: row_ptr (rows+1) + col_idx (nnz), the reference's JA /
// IA (cuMat/src/SparseMatrixBase.h:89-147). ELLPACK: column-major indices with
// rows padded to a multiple of 4 ([width][rows_pad], -1 padding), the
// reference's `indices` matrix (SparseMatrixBase.h:149-206) with the padding
// rows added for 16-byte vector loads.
struct cmcg_pattern_s {
    cmcg_ctx ctx = nullptr;
    int32_t format = CMCG_CSR;
    int32_t rows = 0, cols = 0;
    int64_t nnz = 0;         // CSR: stored entries; ELL: rows * width
    int32_t width = 0;       // ELL entries per row
    int32_t rows_pad = 0;    // ELL: rows rounded up to 4
    int32_t* d_row_ptr = nullptr;
    int32_t* d_col = nullptr;
    int32_t* d_ell = nullptr;
    std::vector<int32_t> h_row_ptr;   // CSR host copy (planning)
    std::vector<int32_t> h_col;       // host copy of col_idx / ell indices (planning, validation)
    // independent systems (diagonal blocks); default one system of all rows
    std::vector<int64_t> row_off;
    int32_t* d_row_off = nullptr;     // int32 copy, n_sys + 1
    int refs = 1;
};

struct cmcg_matrix_s {
    cmcg_pattern pat = nullptr;
    int32_t dtype = CMCG_F32;
    int32_t batches = 1;
    int64_t stride = 0;      // elements between batches (CSR: nnz padded to 4; ELL: width * rows_pad)
    void* d_vals = nullptr;
};

namespace cmcg {
// shared helpers implemented in runtime.cu
cmcg_status dev_alloc(void** p, size_t bytes);
void dev_free(void* p);
cmcg_status ensure_buffer(void** p, size_t* cur, size_t need);
void pattern_release(cmcg_pattern p);
int64_t csr_padded_nnz(int64_t nnz);
// converts n elements between element types on the context stream
cmcg_status convert(cmcg_ctx ctx, int src_dt, const void* src, int dst_dt, void* dst, int64_t n);
}  // namespace cmcg
