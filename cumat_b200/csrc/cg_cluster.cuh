// Cluster solve of the grid path (cg_cluster.cu): one thread-block cluster per
// system instance, the instance's p, q and r in the cluster's shared memory.
#pragma once

#include "cg_grid.cuh"

namespace cmcg {

constexpr int kClusterThreads = 1024;
constexpr int kClusterMaxCtas = 16;   // non-portable cluster size (B200 allows 16)
constexpr int kClusterVectors = 5;    // p, q, r, x and 1/diag of a CTA's rows in shared memory

// Rows per CTA for systems of up to max_rows rows: the smallest power of two R
// >= 1024 with ceil(max_rows / R) <= kClusterMaxCtas; *ctas = that quotient.
// Returns 0 when the kClusterVectors vectors of R rows do not fit in
// smem_limit bytes.
int cluster_rows_log2(int64_t max_rows, size_t elem_bytes, size_t smem_limit, int* ctas);

// Launches the cluster solve of n_inst instances (cluster i solves instance i;
// nd = 5 or 7: the values in a.dia's diagonal layout, else the sliced layout)
// when the device can hold at least min_resident clusters at once; *launched
// = false leaves the solve to the other grid-path loops.
template <typename VT, typename MT, int FMT>
cmcg_status cluster_cg_launch(const SolveArgs<VT, MT>& a, int n_inst, int ctas, int rows_log2, int nd, int min_resident,
                              cudaStream_t st, bool* launched);

}  // namespace cmcg
