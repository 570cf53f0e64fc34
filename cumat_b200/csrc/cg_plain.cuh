// Arguments and launcher of the plain FP64 diagonal-layout persistent CG
// kernel (cg_plain.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cg_grid.cuh"

namespace cmcg {

template <typename MT>
struct PlainDiaArgs {
    int32_t rows, n_sys, ob, mb;
    const int32_t* row_off;
    const int32_t* order;          // systems, largest first
    int32_t* next;                 // work counter of this launch
    int32_t item_begin, item_end;  // its work items: (position in order) * ob + batch
    const MT* vals;                // unscaled values in the diagonal layout, [mb][vstride]
    int64_t vstride;
    const int64_t* base;           // n_sys
    const int32_t* off;            // n_sys * kDiaMax
    int32_t margin;                // largest |offset|: zero halo around p in shared memory
    const double* dinv;            // Jacobi inverse diagonal (null: identity)
    int32_t dinv_b;
    const double* b;
    int32_t b_b;
    double* x;                     // [batch][rows]
    double* r;                     // work vectors, [batch][rows]
    double* q;
    double tol;
    int64_t max_iter;              // < 0: 2 * rows of the system
    int32_t abs_zero_test;
    InstState st;
};

// Launches k_plain_dia with `threads` (1024, 512 or 256) threads per CTA and
// `smem` bytes of dynamic shared memory (p of nmax rows plus its two halos);
// nd = 5 or 7 diagonals.
template <typename MT>
cmcg_status launch_plain_dia(const PlainDiaArgs<MT>& a, int threads, int nmax, size_t smem, int nd, int grid,
                             cudaStream_t stream);

}  // namespace cmcg
