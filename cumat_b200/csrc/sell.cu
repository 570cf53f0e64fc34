// Sliced ELLPACK (32-row slices) copy of CSR patterns for the CG kernels.
//
// The reference streams CSR thread-per-row with strided scalar loads
// (cuMat/src/SparseProductEvaluation.h:55-87). The CG kernels here keep the
// thread-per-row shape (one row per lane, rows of a warp consecutive) but read a
// column-major slice layout, so every load of a warp is one 128-byte access and
// the inner loop is four instructions per entry. The layout is built once per
// pattern on the host (slices never cross a system boundary) and the values are
// gathered into it on the device whenever the matrix values change.

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "objects.h"

namespace cmcg {

void free_sell(SellPlan& s) {
    dev_free(s.d_col);
    dev_free(s.d_perm);
    dev_free(s.d_slice_off);
    dev_free(s.d_slice_w);
    dev_free(s.d_sys_slice0);
    dev_free(s.d_col16);
    dev_free(s.d_slice_off32);
    dev_free(s.d_slice_row0);
    const int64_t id = s.plan_id;
    s = SellPlan();
    s.plan_id = id;
}

cmcg_status ensure_sell(cmcg_pattern p) {
    if (p->format != CMCG_CSR) return CMCG_OK;
    SellPlan& S = p->sell;
    if (S.d_col) return CMCG_OK;
    const auto& rp = p->h_row_ptr;
    const auto& ci = p->h_col;
    const auto& ro = p->row_off;
    const int64_t n_sys = static_cast<int64_t>(ro.size()) - 1;
    std::vector<int64_t> off;
    std::vector<int32_t> width, sys0(n_sys + 1);
    int64_t slots = 0;
    for (int64_t s = 0; s < n_sys; ++s) {
        sys0[s] = static_cast<int32_t>(width.size());
        for (int64_t r = ro[s]; r < ro[s + 1]; r += 32) {
            const int64_t e = std::min<int64_t>(r + 32, ro[s + 1]);
            int32_t w = 0;
            for (int64_t q = r; q < e; ++q) w = std::max(w, rp[q + 1] - rp[q]);
            off.push_back(slots);
            width.push_back(w);
            slots += static_cast<int64_t>(w) * 32;
        }
    }
    sys0[n_sys] = static_cast<int32_t>(width.size());
    off.push_back(slots);
    if (width.size() > static_cast<size_t>(INT32_MAX))
        return fail(CMCG_ERR_NOT_SUPPORTED, "sliced ELLPACK: too many slices");
    std::vector<int32_t> col(static_cast<size_t>(slots)), perm(static_cast<size_t>(slots));
    int64_t max_rows = 0;
    for (int64_t s = 0; s < n_sys; ++s) max_rows = std::max(max_rows, ro[s + 1] - ro[s]);
    const bool compact = max_rows <= 65536 && slots < INT32_MAX;
    std::vector<uint16_t> col16(compact ? static_cast<size_t>(slots) : 0);
    std::vector<int32_t> off32(compact ? off.size() : 0), row0(width.size());
    size_t sl = 0;
    for (int64_t s = 0; s < n_sys; ++s) {
        for (int64_t r = ro[s]; r < ro[s + 1]; r += 32, ++sl) {
            row0[sl] = static_cast<int32_t>(r);
            const int64_t e = std::min<int64_t>(r + 32, ro[s + 1]);
            const int32_t w = width[sl];
            for (int64_t q = r; q < r + 32; ++q) {
                const int64_t lane = q - r;
                const int32_t a = q < e ? rp[q] : 0, len = q < e ? rp[q + 1] - rp[q] : 0;
                // padding points at a valid column of the system (the row itself,
                // or the system's first row for lanes past its end) with value 0
                const int32_t pad_col = static_cast<int32_t>(q < e ? q : ro[s]);
                for (int32_t j = 0; j < w; ++j) {
                    const int64_t o = off[sl] + static_cast<int64_t>(j) * 32 + lane;
                    if (j < len) { col[o] = ci[a + j]; perm[o] = a + j; }
                    else { col[o] = pad_col; perm[o] = -1; }
                    if (compact) col16[o] = static_cast<uint16_t>(col[o] - ro[s]);
                }
            }
        }
    }
    S.n_slots = slots;
    S.n_slices = static_cast<int32_t>(width.size());
    auto up = [](void** d, const void* h, size_t bytes) -> cmcg_status {
        CMCG_TRY(dev_alloc(d, std::max<size_t>(bytes, 16)));
        if (bytes) CMCG_CUDA(cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
        return CMCG_OK;
    };
    cmcg_status st;
    if ((st = up(reinterpret_cast<void**>(&S.d_col), col.data(), col.size() * 4)) != CMCG_OK ||
        (st = up(reinterpret_cast<void**>(&S.d_perm), perm.data(), perm.size() * 4)) != CMCG_OK ||
        (st = up(reinterpret_cast<void**>(&S.d_slice_off), off.data(), off.size() * 8)) != CMCG_OK ||
        (st = up(reinterpret_cast<void**>(&S.d_slice_w), width.data(), width.size() * 4)) != CMCG_OK ||
        (st = up(reinterpret_cast<void**>(&S.d_sys_slice0), sys0.data(), sys0.size() * 4)) != CMCG_OK ||
        (st = up(reinterpret_cast<void**>(&S.d_slice_row0), row0.data(), row0.size() * 4)) != CMCG_OK) {
        free_sell(S);
        return st;
    }
    if (compact) {
        for (size_t i = 0; i < off.size(); ++i) off32[i] = static_cast<int32_t>(off[i]);
        if ((st = up(reinterpret_cast<void**>(&S.d_col16), col16.data(), col16.size() * 2)) != CMCG_OK ||
            (st = up(reinterpret_cast<void**>(&S.d_slice_off32), off32.data(), off32.size() * 4)) != CMCG_OK) {
            free_sell(S);
            return st;
        }
    }
    return CMCG_OK;
}

void free_dia(DiaPlan& d) {
    dev_free(d.d_pos);
    dev_free(d.d_sys_base);
    dev_free(d.d_sys_off);
    const int64_t id = d.plan_id;
    d = DiaPlan();
    d.plan_id = id;
}

cmcg_status ensure_dia(cmcg_pattern p) {
    DiaPlan& D = p->dia;
    if (p->format != CMCG_CSR || D.built) return CMCG_OK;
    D.built = true;   // a failed or inapplicable plan is not retried until the systems change
    const auto& rp = p->h_row_ptr;
    const auto& ci = p->h_col;
    const auto& ro = p->row_off;
    const int64_t n_sys = static_cast<int64_t>(ro.size()) - 1;
    std::vector<int32_t> off(static_cast<size_t>(n_sys) * kDiaMax, 0);
    std::vector<int64_t> base(n_sys);
    std::vector<int32_t> nd(n_sys);
    int64_t slots = 0;
    int32_t max_nd = 0, margin = 0;
    for (int64_t s = 0; s < n_sys; ++s) {
        std::vector<int32_t> o;
        for (int64_t r = ro[s]; r < ro[s + 1]; ++r) {
            for (int32_t k = rp[r]; k < rp[r + 1]; ++k) {
                const int32_t d = static_cast<int32_t>(ci[k] - r);
                if (std::find(o.begin(), o.end(), d) == o.end()) {
                    if (static_cast<int>(o.size()) == kDiaMax) return CMCG_OK;   // not diagonal-shaped: D.ok stays false
                    o.push_back(d);
                }
            }
        }
        std::sort(o.begin(), o.end());
        for (size_t j = 0; j < o.size(); ++j) {
            off[static_cast<size_t>(s) * kDiaMax + j] = o[j];
            margin = std::max(margin, std::abs(o[j]));
        }
        nd[s] = static_cast<int32_t>(o.size());
        max_nd = std::max(max_nd, nd[s]);
    }
    // every system stores the same number of diagonals (5 or 7, the widths the
    // kernel is built for); unused ones hold zeros
    const int32_t nd_alloc = max_nd <= 5 ? 5 : max_nd <= 7 ? 7 : 0;
    if (nd_alloc == 0) return CMCG_OK;
    constexpr int64_t B = kDiaBlockRows;
    for (int64_t s = 0; s < n_sys; ++s) {
        base[s] = slots;
        slots += static_cast<int64_t>(nd_alloc) * ((ro[s + 1] - ro[s] + B - 1) / B) * B;
    }
    if (slots >= INT32_MAX) return CMCG_OK;
    std::vector<int32_t> pos(static_cast<size_t>(p->nnz));
    for (int64_t s = 0; s < n_sys; ++s) {
        const int32_t* o = off.data() + s * kDiaMax;
        for (int64_t r = ro[s]; r < ro[s + 1]; ++r) {
            const int64_t i = r - ro[s];
            for (int32_t k = rp[r]; k < rp[r + 1]; ++k) {
                const int32_t d = static_cast<int32_t>(std::find(o, o + nd[s], static_cast<int32_t>(ci[k] - r)) - o);
                pos[k] = static_cast<int32_t>(base[s] + B * ((i / B) * nd_alloc + d) + i % B);
            }
        }
    }
    auto up = [](void** dptr, const void* h, size_t bytes) -> cmcg_status {
        CMCG_TRY(dev_alloc(dptr, std::max<size_t>(bytes, 16)));
        if (bytes) CMCG_CUDA(cudaMemcpy(*dptr, h, bytes, cudaMemcpyHostToDevice));
        return CMCG_OK;
    };
    cmcg_status st;
    if ((st = up(reinterpret_cast<void**>(&D.d_pos), pos.data(), pos.size() * 4)) != CMCG_OK ||
        (st = up(reinterpret_cast<void**>(&D.d_sys_base), base.data(), base.size() * 8)) != CMCG_OK ||
        (st = up(reinterpret_cast<void**>(&D.d_sys_off), off.data(), off.size() * 4)) != CMCG_OK) {
        free_dia(D);
        D.built = true;
        return st;
    }
    D.n_slots = slots;
    D.max_nd = nd_alloc;
    D.margin = margin;
    D.ok = true;
    return CMCG_OK;
}

namespace {

template <typename MT>
__global__ void k_sell_gather(const int32_t* __restrict__ perm, int64_t n_slots, const MT* __restrict__ vals,
                              int64_t vstride, MT* __restrict__ out, int64_t ostride, int32_t batches) {
    const int64_t total = n_slots * batches;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = i / n_slots, k = i - b * n_slots;
        const int32_t e = perm[k];
        out[b * ostride + k] = e >= 0 ? vals[b * vstride + e] : MT{};
    }
}

}  // namespace

cmcg_status ensure_sell_values(cmcg_matrix m) {
    cmcg_pattern p = m->pat;
    if (p->format != CMCG_CSR) return CMCG_OK;
    CMCG_TRY(ensure_sell(p));
    const SellPlan& S = p->sell;
    if (m->d_sell_vals && m->sell_version == m->version && m->sell_plan_id == S.plan_id) return CMCG_OK;
    const size_t es = dtype_size(m->dtype);
    const int64_t stride = (S.n_slots + 7) / 8 * 8 + 8;
    if (!m->d_sell_vals || m->sell_stride != stride || m->sell_plan_id != S.plan_id) {
        dev_free(m->d_sell_vals);
        m->d_sell_vals = nullptr;
        CMCG_TRY(dev_alloc(&m->d_sell_vals, static_cast<size_t>(stride) * m->batches * es));
        m->sell_stride = stride;
    }
    cmcg_ctx ctx = p->ctx;
    const int64_t total = S.n_slots * m->batches;
    const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, static_cast<int64_t>(ctx->sm_count) * 16));
    if (total > 0) {
        switch (m->dtype) {
            case CMCG_F32:
                k_sell_gather<float><<<blocks, 256, 0, ctx->stream>>>(S.d_perm, S.n_slots, static_cast<const float*>(m->d_vals),
                                                                      m->stride, static_cast<float*>(m->d_sell_vals), stride, m->batches);
                break;
            case CMCG_F64:
                k_sell_gather<double><<<blocks, 256, 0, ctx->stream>>>(S.d_perm, S.n_slots, static_cast<const double*>(m->d_vals),
                                                                       m->stride, static_cast<double*>(m->d_sell_vals), stride, m->batches);
                break;
            default:
                k_sell_gather<__nv_bfloat16><<<blocks, 256, 0, ctx->stream>>>(
                    S.d_perm, S.n_slots, static_cast<const __nv_bfloat16*>(m->d_vals), m->stride,
                    static_cast<__nv_bfloat16*>(m->d_sell_vals), stride, m->batches);
        }
        count_launch();
        CMCG_CHECK_LAUNCH();
    }
    m->sell_version = m->version;
    m->sell_plan_id = S.plan_id;
    return CMCG_OK;
}

}  // namespace cmcg
