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
    // private stream used only to capture CUDA graphs (capture is not allowed on
    // the legacy default stream); the captured graphs are launched on `stream`
    cudaStream_t capture_stream = nullptr;
    int sm_count = 148;
    // scratch for the batched dot / squared-norm combine (grown on demand)
    void* red_partial = nullptr;
    size_t red_partial_bytes = 0;
    unsigned* red_ticket = nullptr;
    size_t red_ticket_count = 0;
    // device error word (bounded waits that ran out set bits; read and cleared by
    // cmcg_ctx_device_errors)
    int32_t* d_err = nullptr;
    // handle + every pattern created on it; freed when the last one is released
    int refs = 1;
};

// Sliced ELLPACK copy of a CSR pattern used by the CG kernels: every system's
// rows are cut into slices of 32 consecutive rows; a slice of width w (its
// longest row) stores entry j of its row l at slice_off[slice] + j * 32 + l, so
// a warp reading one entry of 32 rows makes one coalesced 128-byte access.
// Padding slots carry the row's own column and value 0.
struct SellPlan {
    int64_t n_slots = 0;
    int32_t n_slices = 0;
    int32_t* d_col = nullptr;         // n_slots, global column index
    int32_t* d_perm = nullptr;        // n_slots, CSR entry of the slot or -1 (padding)
    int64_t* d_slice_off = nullptr;   // n_slices + 1
    int32_t* d_slice_w = nullptr;     // n_slices
    int32_t* d_sys_slice0 = nullptr;  // n_sys + 1, first slice of each system
    int32_t* d_slice_row0 = nullptr;  // n_slices, first global row of each slice
    // compact form for the fast kernels (present when every system has at most
    // 65536 rows and n_slots < 2^31): 16-bit column indices local to the
    // system, 32-bit slice offsets
    uint16_t* d_col16 = nullptr;
    int32_t* d_slice_off32 = nullptr;
    int64_t plan_id = 0;              // changes when the systems change
};

// Diagonal (DIA) copy of a CSR pattern whose systems each have at most
// kDiaMax distinct column offsets col - row (stencils on structured grids,
// banded matrices), in blocks of kDiaBlockRows rows: system s stores diagonal
// d (offset sys_off[s][d], sorted ascending, padded with offset 0) of its
// local row i = kDiaBlockRows k + j at slot
// sys_base[s] + kDiaBlockRows (k nd + d) + j (nd = max_nd); entries missing
// from a row, and the rows of the last block past the system's end, hold
// value 0. Feeds the mixed-precision persistent kernel, whose thread j then
// reads every value of its rows from one pointer with immediate offsets and
// needs no column indices.
constexpr int kDiaMax = 8;
constexpr int kDiaBlockRows = 1024;
struct DiaPlan {
    bool built = false;
    bool ok = false;            // every system has at most kDiaMax offsets
    int32_t max_nd = 0;         // diagonals stored per system (5 or 7)
    int32_t margin = 0;         // largest |offset|
    int64_t n_slots = 0;
    int32_t* d_pos = nullptr;       // per CSR entry: its slot
    int64_t* d_sys_base = nullptr;  // n_sys
    int32_t* d_sys_off = nullptr;   // n_sys * kDiaMax
    int64_t plan_id = 0;            // changes when the systems change
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
    // row tiles of the bulk-staged CSR product (built on first use): tile t
    // covers rows [tile_row0[t], tile_row0[t+1]), at most kTileRows rows and,
    // unless it is a single long row, at most kTileNnz entries
    int32_t n_spmv_tiles = 0;
    int32_t* d_spmv_tiles = nullptr;
    // sliced ELLPACK copy for the CG kernels (CSR only, built on first use)
    SellPlan sell;
    // diagonal copy for the mixed-precision kernel (CSR only, built on first use)
    DiaPlan dia;
    // stand-alone product kernel picked by timing on first use, per
    // [value dtype][vector dtype] (-1: not tuned yet)
    int8_t spmv_choice[3][2] = {{-1, -1}, {-1, -1}, {-1, -1}};
    int64_t systems_version = 0;      // incremented by cmcg_pattern_set_systems
    // The caller's storage when it is not CSR or ELLPACK: CMCG_CSC (the
    // reference's SparsityPattern<CSC>: column pointers + row indices, values in
    // column order) or CMCG_BSR (block CSR, block x block values per stored
    // block, row-major). The kernels see the equivalent CSR pattern (format ==
    // CMCG_CSR; a BSR block row expands to `block` scalar rows) and matrices
    // keep their values in its order: CSR entry k is the caller's value
    // d_val_perm[k] (null for plain CSR / ELLPACK).
    int32_t declared = -1;            // CMCG_CSC, CMCG_BSR, or -1 (as format)
    int32_t* d_val_perm = nullptr;
    int32_t block = 1;                // BSR block size
    int64_t decl_nnz = 0;             // the caller's stored entries (CSC) or blocks (BSR)
    int32_t decl_rows = 0, decl_cols = 0;   // BSR: block rows / block columns
    std::vector<int32_t> h_decl_ptr, h_decl_idx;   // the caller's index arrays (for download)
    // transpose of the CSR pattern (built by the first transposed product):
    // row r of A^T holds entries d_t_col[k] of A's column r, k in
    // [d_t_row_ptr[r], d_t_row_ptr[r + 1]), whose values are A's entries d_t_perm[k]
    int32_t* d_t_row_ptr = nullptr;
    int32_t* d_t_col = nullptr;
    int32_t* d_t_perm = nullptr;
    int refs = 1;
};

struct cmcg_matrix_s {
    cmcg_pattern pat = nullptr;
    int32_t dtype = CMCG_F32;
    int32_t batches = 1;
    int64_t stride = 0;      // elements between batches (CSR: nnz padded to 4; ELL: width * rows_pad)
    void* d_vals = nullptr;
    int64_t version = 0;              // incremented by every value upload
    // values in the pattern's sliced ELLPACK layout ([batch][n_slots_pad]),
    // regathered when `version` or the plan changes
    void* d_sell_vals = nullptr;
    int64_t sell_stride = 0;
    int64_t sell_version = -1;
    int64_t sell_plan_id = -1;
    // values in the entry order of the pattern's transpose ([batch][t_stride]),
    // regathered when `version` changes (the transposed product)
    void* d_t_vals = nullptr;
    int64_t t_stride = 0;
    int64_t t_version = -1;
    // handle + every solver created on it; freed when the last one is released
    int refs = 1;
};

namespace cmcg {
// shared helpers implemented in runtime.cu
cmcg_status dev_alloc(void** p, size_t bytes);
void dev_free(void* p);
cmcg_status ensure_buffer(void** p, size_t* cur, size_t need);
void pattern_release(cmcg_pattern p);
void matrix_release(cmcg_matrix m);
void ctx_release(cmcg_ctx c);
int64_t csr_padded_nnz(int64_t nnz);
// converts n elements between element types on the context stream
cmcg_status convert(cmcg_ctx ctx, int src_dt, const void* src, int dst_dt, void* dst, int64_t n);
// builds the pattern's sliced ELLPACK plan (CSR) and the matrix's values in it
cmcg_status ensure_sell(cmcg_pattern p);
cmcg_status ensure_sell_values(cmcg_matrix m);
void free_sell(SellPlan& s);
// builds the pattern's diagonal plan (CSR; dia.ok tells whether it applies)
cmcg_status ensure_dia(cmcg_pattern p);
void free_dia(DiaPlan& d);
// values between the caller's order and the internal CSR order of a pattern
// with d_val_perm (sparse_ops.cu): to_internal gathers dst[b][k] =
// src[b][perm[k]], otherwise dst[b][perm[k]] = src[b][k]; dtype of both
cmcg_status permute_values(cmcg_pattern p, int32_t dtype, const void* src, int64_t src_stride, void* dst,
                           int64_t dst_stride, int32_t batches, bool to_internal);
void free_declared(cmcg_pattern p);
}  // namespace cmcg
