// CPU ORACLE — test infrastructure only.
//
// A plain, single-threaded restatement of the reference's algorithms for the
// batched sparse CG path, used to check the CUDA library. Only the tests, the
// smoke check and the benchmark's CPU-baseline leg may load this file's
// library, and only as the checker: the product never calls it and has no CPU
// fallback.
//
// What each function restates (paths relative to the reference repository):
//   orc_spmv_csr_*   cuMat/src/SparseProductEvaluation.h:43-88   (CSRMVKernel_StaticBatches)
//   orc_spmv_ell_*   cuMat/src/SparseProductEvaluation.h:194-226 (ELLPACKMVKernel_StaticBatches)
//   orc_dot_*, orc_sqnorm_*   cuMat/src/ReductionOpsPlugin.inl:279-315 (dot = cwiseDot().sum,
//                    squaredNorm = cwiseAbs2().sum, per batch)
//   orc_inv_diag_*   cuMat/src/ConjugateGradient.h:228-230 with UnaryOps.h:177
//                    (cwiseInverseCheck: 1/a_ii, or 1 where a_ii == 0) and the
//                    diagonal lookup of SparseMatrixBase.h:258-271 (0 when absent)
//   orc_cg_*         cuMat/src/ConjugateGradient.h:123-206 (_solve_with_guess_impl),
//                    defaults from IterativeSolverBase.h:83-86 / :131
//   orc_sddmm_*      the sparse outer product on a pattern,
//                    SparseProductEvaluation.h:16-37 + SparseEvaluation.h:15-34
//   orc_refined_*    FP64 iterative refinement around an FP32 inner CG (no
//                    reference counterpart; classical mixed-precision iterative
//                    refinement: r = b - A x in FP64, solve A d = r at low
//                    precision, x += d, repeat)
//
// Summation order: reductions use pairwise summation in the vector's scalar
// type, standing in for the reference's CUB tree reductions (whose order is not
// specified), so FP32 results agree with a GPU tree sum to rounding, not bitwise.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace {

template <typename T>
T pairwise_sum(const T* a, int64_t n) {
    if (n <= 32) {
        T s = T(0);
        for (int64_t i = 0; i < n; ++i) s += a[i];
        return s;
    }
    const int64_t h = n / 2;
    return pairwise_sum(a, h) + pairwise_sum(a + h, n - h);
}

template <typename T>
T dot(const T* x, const T* y, int64_t n, std::vector<T>& tmp) {
    tmp.resize(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) tmp[i] = x[i] * y[i];
    return pairwise_sum(tmp.data(), n);
}

// y[b] = A[b] * x[b] with broadcasting of a single-batch matrix or vector.
// Rows without entries produce 0.
template <typename MT, typename VT>
void spmv_csr(int32_t rows, const int32_t* rp, const int32_t* ci, const MT* val, int64_t nnz,
              int32_t mb, const VT* x, int32_t cols, int32_t xb, VT* y, int32_t ob) {
    for (int32_t b = 0; b < ob; ++b) {
        const MT* v = val + (mb == 1 ? 0 : static_cast<int64_t>(b) * nnz);
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        VT* yv = y + static_cast<int64_t>(b) * rows;
        for (int32_t r = 0; r < rows; ++r) {
            VT acc = VT(0);
            for (int32_t k = rp[r]; k < rp[r + 1]; ++k) acc += static_cast<VT>(v[k]) * xv[ci[k]];
            yv[r] = acc;
        }
    }
}

template <typename MT, typename VT>
void spmv_ell(int32_t rows, int32_t width, const int32_t* idx, const MT* val, int32_t mb,
              const VT* x, int32_t cols, int32_t xb, VT* y, int32_t ob) {
    const int64_t slab = static_cast<int64_t>(rows) * width;
    for (int32_t b = 0; b < ob; ++b) {
        const MT* v = val + (mb == 1 ? 0 : static_cast<int64_t>(b) * slab);
        const VT* xv = x + (xb == 1 ? 0 : static_cast<int64_t>(b) * cols);
        VT* yv = y + static_cast<int64_t>(b) * rows;
        for (int32_t r = 0; r < rows; ++r) {
            VT acc = VT(0);
            for (int32_t j = 0; j < width; ++j) {
                const int64_t o = r + static_cast<int64_t>(j) * rows;
                const int32_t c = idx[o];
                if (c < 0) continue;
                acc += static_cast<VT>(v[o]) * xv[c];
            }
            yv[r] = acc;
        }
    }
}

template <typename T>
void inv_diag(int32_t rows, const int32_t* rp, const int32_t* ci, const T* val, int64_t row_base, T* out) {
    for (int32_t r = 0; r < rows; ++r) {
        T d = T(0);
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k)
            if (ci[k] == r + row_base) { d = val[k]; break; }
        out[r] = (d != T(0)) ? T(1) / d : T(1);
    }
}

// One CSR system: rows [r0, r0+n) of a (possibly block-diagonal) CSR matrix
// whose columns for these rows lie in [r0, r0+n).
template <typename T>
struct System {
    int64_t n;
    int64_t r0;
    const int32_t* rp;   // rp[0..n], absolute offsets into ci / val
    const int32_t* ci;   // absolute column indices
    const T* val;
    void apply(const T* x_local, T* y_local) const {
        for (int64_t r = 0; r < n; ++r) {
            T acc = T(0);
            for (int32_t k = rp[r]; k < rp[r + 1]; ++k) acc += val[k] * x_local[ci[k] - r0];
            y_local[r] = acc;
        }
    }
};

// The reference's PCG loop for a lock-stepped batch of `nb` systems sharing
// the iteration counter (ConjugateGradient.h:123-206). With nb == 1 it is the
// per-system solve used for packed batches. Returns the iteration count and
// writes per-system squared-residual ratios to ratio[] (error = sqrt(max)).
template <typename T>
int64_t cg_lockstep(const std::vector<System<T>>& sys, const T* const* rhs, const T* const* guess,
                    T* const* x, T tol, int64_t max_iter, int precond, double* ratio, int32_t* early,
                    bool abs_zero_test = true) {
    const size_t nb = sys.size();
    std::vector<T> tmpd;
    std::vector<std::vector<T>> r(nb), p(nb), z(nb), q(nb), dinv(nb);
    std::vector<T> rhsN2(nb), thr(nb), resN2(nb), absNew(nb);
    for (size_t s = 0; s < nb; ++s) {
        const int64_t n = sys[s].n;
        r[s].resize(n); p[s].resize(n); z[s].resize(n); q[s].resize(n); dinv[s].assign(n, T(1));
        for (int64_t i = 0; i < n; ++i) x[s][i] = guess ? guess[s][i] : T(0);
        if (precond == 1) {
            // inverse diagonal with absolute column indices
            for (int64_t i = 0; i < n; ++i) {
                T d = T(0);
                for (int32_t k = sys[s].rp[i]; k < sys[s].rp[i + 1]; ++k)
                    if (sys[s].ci[k] == sys[s].r0 + i) { d = sys[s].val[k]; break; }
                dinv[s][i] = (d != T(0)) ? T(1) / d : T(1);
            }
        }
    }
    // r = b - A x
    for (size_t s = 0; s < nb; ++s) {
        sys[s].apply(x[s], q[s].data());
        for (int64_t i = 0; i < sys[s].n; ++i) r[s][i] = rhs[s][i] - q[s][i];
        rhsN2[s] = dot(rhs[s], rhs[s], sys[s].n, tmpd);
    }
    bool all = true;
    // the reference's absolute early-out (ConjugateGradient.h:152-159); the
    // refinement's inner solves only stop early on an exactly zero rhs, since
    // their right-hand sides shrink with the outer residual
    for (size_t s = 0; s < nb; ++s) all = all && (abs_zero_test ? rhsN2[s] < tol * tol : rhsN2[s] == T(0));
    if (all) {
        for (size_t s = 0; s < nb; ++s) {
            for (int64_t i = 0; i < sys[s].n; ++i) x[s][i] = T(0);
            ratio[s] = 0.0;
        }
        if (early) *early = 1;
        return 0;
    }
    for (size_t s = 0; s < nb; ++s) {
        thr[s] = tol * tol * rhsN2[s];
        resN2[s] = dot(r[s].data(), r[s].data(), sys[s].n, tmpd);
    }
    all = true;
    for (size_t s = 0; s < nb; ++s) all = all && (resN2[s] < thr[s]);
    if (all) {
        for (size_t s = 0; s < nb; ++s) ratio[s] = static_cast<double>(resN2[s] / rhsN2[s]);
        if (early) *early = 2;
        return 0;
    }
    for (size_t s = 0; s < nb; ++s) {
        for (int64_t i = 0; i < sys[s].n; ++i) p[s][i] = dinv[s][i] * r[s][i];
        absNew[s] = dot(r[s].data(), p[s].data(), sys[s].n, tmpd);
    }
    int64_t it = 0;
    while (it < max_iter) {
        for (size_t s = 0; s < nb; ++s) {
            const int64_t n = sys[s].n;
            sys[s].apply(p[s].data(), q[s].data());
            const T alpha = absNew[s] / dot(p[s].data(), q[s].data(), n, tmpd);
            for (int64_t i = 0; i < n; ++i) x[s][i] += alpha * p[s][i];
            for (int64_t i = 0; i < n; ++i) r[s][i] -= alpha * q[s][i];
            resN2[s] = dot(r[s].data(), r[s].data(), n, tmpd);
        }
        all = true;
        for (size_t s = 0; s < nb; ++s) all = all && (resN2[s] < thr[s]);
        if (all) break;
        for (size_t s = 0; s < nb; ++s) {
            const int64_t n = sys[s].n;
            for (int64_t i = 0; i < n; ++i) z[s][i] = dinv[s][i] * r[s][i];
            const T absOld = absNew[s];
            absNew[s] = dot(r[s].data(), z[s].data(), n, tmpd);
            const T beta = absNew[s] / absOld;
            for (int64_t i = 0; i < n; ++i) p[s][i] = z[s][i] + beta * p[s][i];
        }
        ++it;
    }
    for (size_t s = 0; s < nb; ++s) ratio[s] = static_cast<double>(resN2[s] / rhsN2[s]);
    if (early) *early = 0;
    return it;
}

template <typename T>
int cg_csr(int32_t n, const int32_t* rp, const int32_t* ci, const T* val, int64_t nnz, int32_t mb,
           const T* rhs, int32_t batches, const T* guess, T* x, double tol, int64_t max_iter, int precond,
           int lockstep, int64_t* iters, double* err) {
    if (max_iter < 0) max_iter = 2 * static_cast<int64_t>(n);
    std::vector<System<T>> all(batches);
    for (int32_t b = 0; b < batches; ++b)
        all[b] = System<T>{n, 0, rp, ci, val + (mb == 1 ? 0 : static_cast<int64_t>(b) * nnz)};
    std::vector<const T*> R(batches), G(batches);
    std::vector<T*> X(batches);
    for (int32_t b = 0; b < batches; ++b) {
        R[b] = rhs + static_cast<int64_t>(b) * n;
        G[b] = guess ? guess + static_cast<int64_t>(b) * n : nullptr;
        X[b] = x + static_cast<int64_t>(b) * n;
    }
    std::vector<double> ratio(batches);
    const T t = static_cast<T>(tol);
    if (lockstep) {
        const int64_t it = cg_lockstep<T>(all, R.data(), guess ? G.data() : nullptr, X.data(), t, max_iter,
                                          precond, ratio.data(), nullptr);
        double m = 0.0;
        for (double v : ratio) m = std::max(m, v);
        for (int32_t b = 0; b < batches; ++b) { iters[b] = it; err[b] = std::sqrt(m); }
    } else {
        for (int32_t b = 0; b < batches; ++b) {
            std::vector<System<T>> one{all[b]};
            const T* Rb = R[b];
            const T* Gb = G[b];
            T* Xb = X[b];
            double rt = 0.0;
            iters[b] = cg_lockstep<T>(one, &Rb, guess ? &Gb : nullptr, &Xb, t, max_iter, precond, &rt, nullptr);
            err[b] = std::sqrt(rt);
        }
    }
    return 0;
}

// Independent systems packed block-diagonally (row_off[n_sys+1]).
template <typename T>
int cg_packed(int64_t n_sys, const int64_t* row_off, const int32_t* rp, const int32_t* ci, const T* val,
              const T* rhs, const T* guess, T* x, double tol, int64_t max_iter, int precond,
              int64_t* iters, double* err) {
    for (int64_t s = 0; s < n_sys; ++s) {
        const int64_t r0 = row_off[s], n = row_off[s + 1] - row_off[s];
        std::vector<System<T>> one{System<T>{n, r0, rp + r0, ci, val}};
        const T* Rb = rhs + r0;
        const T* Gb = guess ? guess + r0 : nullptr;
        T* Xb = x + r0;
        const int64_t mi = max_iter < 0 ? 2 * n : max_iter;
        double rt = 0.0;
        iters[s] = cg_lockstep<T>(one, &Rb, guess ? &Gb : nullptr, &Xb, static_cast<T>(tol), mi, precond, &rt, nullptr);
        err[s] = std::sqrt(rt);
    }
    return 0;
}

inline float bf16_round(float f) {
    // round-to-nearest-even to the top 16 bits of the IEEE binary32 pattern
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) {  // inf / nan: truncate, keep nan quiet
        u &= 0xffff0000u;
        if ((u & 0x007f0000u) == 0 && std::isnan(f)) u |= 0x00400000u;
    } else {
        const uint32_t lsb = (u >> 16) & 1u;
        u += 0x7fffu + lsb;
        u &= 0xffff0000u;
    }
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

}  // namespace

extern "C" {

int orc_spmv_csr_f32(int32_t rows, const int32_t* rp, const int32_t* ci, const float* val, int64_t nnz,
                     int32_t mb, const float* x, int32_t cols, int32_t xb, float* y, int32_t ob) {
    spmv_csr<float, float>(rows, rp, ci, val, nnz, mb, x, cols, xb, y, ob);
    return 0;
}
int orc_spmv_csr_f64(int32_t rows, const int32_t* rp, const int32_t* ci, const double* val, int64_t nnz,
                     int32_t mb, const double* x, int32_t cols, int32_t xb, double* y, int32_t ob) {
    spmv_csr<double, double>(rows, rp, ci, val, nnz, mb, x, cols, xb, y, ob);
    return 0;
}
// FP32 matrix values upcast into an FP64 product (the refinement residual).
int orc_spmv_csr_f32f64(int32_t rows, const int32_t* rp, const int32_t* ci, const float* val, int64_t nnz,
                        int32_t mb, const double* x, int32_t cols, int32_t xb, double* y, int32_t ob) {
    spmv_csr<float, double>(rows, rp, ci, val, nnz, mb, x, cols, xb, y, ob);
    return 0;
}
int orc_spmv_ell_f32(int32_t rows, int32_t width, const int32_t* idx, const float* val, int32_t mb,
                     const float* x, int32_t cols, int32_t xb, float* y, int32_t ob) {
    spmv_ell<float, float>(rows, width, idx, val, mb, x, cols, xb, y, ob);
    return 0;
}
int orc_spmv_ell_f64(int32_t rows, int32_t width, const int32_t* idx, const double* val, int32_t mb,
                     const double* x, int32_t cols, int32_t xb, double* y, int32_t ob) {
    spmv_ell<double, double>(rows, width, idx, val, mb, x, cols, xb, y, ob);
    return 0;
}

// out[b] = sum_i x[b][i] * y[b][i]; xb / yb == 1 broadcasts.
int orc_dot_f32(int64_t n, int32_t ob, const float* x, int32_t xb, const float* y, int32_t yb, float* out) {
    std::vector<float> t;
    for (int32_t b = 0; b < ob; ++b) {
        const float* xv = x + (xb == 1 ? 0 : b * n);
        const float* yv = y + (yb == 1 ? 0 : b * n);
        out[b] = dot(xv, yv, n, t);
    }
    return 0;
}
int orc_dot_f64(int64_t n, int32_t ob, const double* x, int32_t xb, const double* y, int32_t yb, double* out) {
    std::vector<double> t;
    for (int32_t b = 0; b < ob; ++b) {
        const double* xv = x + (xb == 1 ? 0 : b * n);
        const double* yv = y + (yb == 1 ? 0 : b * n);
        out[b] = dot(xv, yv, n, t);
    }
    return 0;
}
int orc_sqnorm_f32(int64_t n, int32_t ob, const float* x, float* out) { return orc_dot_f32(n, ob, x, ob, x, ob, out); }
int orc_sqnorm_f64(int64_t n, int32_t ob, const double* x, double* out) { return orc_dot_f64(n, ob, x, ob, x, ob, out); }

int orc_inv_diag_f32(int32_t rows, const int32_t* rp, const int32_t* ci, const float* val, float* out) {
    inv_diag<float>(rows, rp, ci, val, 0, out);
    return 0;
}
int orc_inv_diag_f64(int32_t rows, const int32_t* rp, const int32_t* ci, const double* val, double* out) {
    inv_diag<double>(rows, rp, ci, val, 0, out);
    return 0;
}

// Reference CG on a shared-pattern batch. lockstep = 1 follows the reference
// exactly (all batches iterate until all converged, one iteration count);
// lockstep = 0 solves every batch on its own (per-system convergence).
// max_iter < 0 selects the reference default 2 * n. iters / err: per batch.
int orc_cg_csr_f32(int32_t n, const int32_t* rp, const int32_t* ci, const float* val, int64_t nnz, int32_t mb,
                   const float* rhs, int32_t batches, const float* guess, float* x, double tol, int64_t max_iter,
                   int precond, int lockstep, int64_t* iters, double* err) {
    return cg_csr<float>(n, rp, ci, val, nnz, mb, rhs, batches, guess, x, tol, max_iter, precond, lockstep, iters, err);
}
int orc_cg_csr_f64(int32_t n, const int32_t* rp, const int32_t* ci, const double* val, int64_t nnz, int32_t mb,
                   const double* rhs, int32_t batches, const double* guess, double* x, double tol, int64_t max_iter,
                   int precond, int lockstep, int64_t* iters, double* err) {
    return cg_csr<double>(n, rp, ci, val, nnz, mb, rhs, batches, guess, x, tol, max_iter, precond, lockstep, iters, err);
}

int orc_cg_packed_f32(int64_t n_sys, const int64_t* row_off, const int32_t* rp, const int32_t* ci, const float* val,
                      const float* rhs, const float* guess, float* x, double tol, int64_t max_iter, int precond,
                      int64_t* iters, double* err) {
    return cg_packed<float>(n_sys, row_off, rp, ci, val, rhs, guess, x, tol, max_iter, precond, iters, err);
}
int orc_cg_packed_f64(int64_t n_sys, const int64_t* row_off, const int32_t* rp, const int32_t* ci, const double* val,
                      const double* rhs, const double* guess, double* x, double tol, int64_t max_iter, int precond,
                      int64_t* iters, double* err) {
    return cg_packed<double>(n_sys, row_off, rp, ci, val, rhs, guess, x, tol, max_iter, precond, iters, err);
}

// Mixed-precision solve of packed systems: FP64 residual r = b - A x with the
// FP32 values upcast; inner FP32 Jacobi/identity CG on A d = r to inner_tol
// (relative to |r|), with the matrix values optionally rounded to BF16 for the
// inner solve; x += d in FP64; stop when |r|^2 < outer_tol^2 |b|^2.
// outer[s] = refinement steps, inner[s] = total inner iterations, err[s] =
// final |b - A x| / |b| in FP64.
int orc_refined_packed(int64_t n_sys, const int64_t* row_off, const int32_t* rp, const int32_t* ci, const float* val,
                       const double* rhs, double* x, double inner_tol, double outer_tol, int64_t max_inner,
                       int32_t max_outer, int precond, int bf16_inner, int32_t* outer, int64_t* inner, double* err) {
    std::vector<double> t64;
    for (int64_t s = 0; s < n_sys; ++s) {
        const int64_t r0 = row_off[s], n = row_off[s + 1] - row_off[s];
        const int32_t* srp = rp + r0;
        const int32_t nz0 = srp[0], nz1 = srp[n];
        std::vector<float> v32(val + nz0, val + nz1);
        if (bf16_inner)
            for (auto& v : v32) v = bf16_round(v);
        // inner system views its own (possibly rounded) copy of the values
        std::vector<int32_t> lrp(n + 1);
        for (int64_t i = 0; i <= n; ++i) lrp[i] = srp[i] - nz0;
        System<float> inner_sys{n, r0, lrp.data(), ci + nz0, v32.data()};
        const double* b = rhs + r0;
        double* xs = x + r0;
        for (int64_t i = 0; i < n; ++i) xs[i] = 0.0;
        const double bb = dot(b, b, n, t64);
        std::vector<double> r(n), ax(n);
        std::vector<float> r32(n), d32(n);
        int32_t o = 0;
        int64_t tot = 0;
        double rr = bb;
        for (int64_t i = 0; i < n; ++i) r[i] = b[i];
        const int64_t mi = max_inner < 0 ? 2 * n : max_inner;
        while (true) {
            if (!(rr >= outer_tol * outer_tol * bb) || o >= max_outer) break;
            for (int64_t i = 0; i < n; ++i) r32[i] = static_cast<float>(r[i]);
            std::vector<System<float>> one{inner_sys};
            const float* R = r32.data();
            float* D = d32.data();
            double rt = 0.0;
            tot += cg_lockstep<float>(one, &R, nullptr, &D, static_cast<float>(inner_tol), mi, precond, &rt, nullptr,
                                      /*abs_zero_test=*/false);
            for (int64_t i = 0; i < n; ++i) xs[i] += static_cast<double>(d32[i]);
            // r = b - A x with the exact FP32 values in FP64 arithmetic
            for (int64_t i = 0; i < n; ++i) {
                double acc = 0.0;
                for (int32_t k = srp[i]; k < srp[i + 1]; ++k) acc += static_cast<double>(val[k]) * xs[ci[k] - r0];
                ax[i] = acc;
            }
            for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
            rr = dot(r.data(), r.data(), n, t64);
            ++o;
        }
        outer[s] = o;
        inner[s] = tot;
        err[s] = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    }
    return 0;
}

// Mixed precision with reliable updates, per system (no reference counterpart;
// residual replacement after van der Vorst & Ye 2000, reliable updates after
// Clark et al. 2010): FP32 Jacobi/identity PCG whose increments are folded
// into the FP64 solution and whose recursive residual is replaced by the FP64
// residual b - A x (FP32 values upcast) whenever |r|^2 < delta^2 |r_last|^2 or
// |r|^2 < tol^2 |b|^2; the direction p is kept. Stops when the FP64 residual
// satisfies |r| < tol |b|. iters[s] = FP32 iterations, updates[s] =
// replacements, err[s] = final FP64 relative residual.
int orc_reliable_packed(int64_t n_sys, const int64_t* row_off, const int32_t* rp, const int32_t* ci, const float* val,
                        const double* rhs, double* x, double tol, double delta, int64_t max_iter, int32_t max_updates,
                        int precond, int bf16_inner, int64_t* iters, int32_t* updates, double* err) {
    std::vector<float> t32;
    std::vector<double> t64;
    for (int64_t s = 0; s < n_sys; ++s) {
        const int64_t r0 = row_off[s], n = row_off[s + 1] - row_off[s];
        const int32_t* srp = rp + r0;
        std::vector<float> vin(val + srp[0], val + srp[n]);
        if (bf16_inner)
            for (auto& v : vin) v = bf16_round(v);
        const int32_t k0 = srp[0];
        auto apply32 = [&](const float* xin, float* y) {
            for (int64_t i = 0; i < n; ++i) {
                float acc = 0.0f;
                for (int32_t k = srp[i]; k < srp[i + 1]; ++k) acc += vin[k - k0] * xin[ci[k] - r0];
                y[i] = acc;
            }
        };
        const double* b = rhs + r0;
        double* xs = x + r0;
        std::vector<float> d(n, 1.0f), r(n), p(n), q(n), xk(n, 0.0f);
        if (precond == 1)
            for (int64_t i = 0; i < n; ++i) {
                float dv = 0.0f;
                for (int32_t k = srp[i]; k < srp[i + 1]; ++k)
                    if (ci[k] == r0 + i) { dv = val[k]; break; }
                d[i] = dv != 0.0f ? 1.0f / dv : 1.0f;
            }
        for (int64_t i = 0; i < n; ++i) {
            xs[i] = 0.0;
            r[i] = static_cast<float>(b[i]);
            p[i] = d[i] * r[i];
        }
        const double bb = dot(b, b, n, t64);
        std::vector<float> z(n);
        for (int64_t i = 0; i < n; ++i) z[i] = r[i] * (d[i] * r[i]);
        float rz = pairwise_sum(z.data(), n);
        const double thr = tol * tol * bb;
        double rr64 = bb, rmax2 = bb;
        int64_t it = 0;
        int32_t up = 0;
        const int64_t mi = max_iter < 0 ? 2 * n : max_iter;
        bool done = (bb == 0.0) || (rr64 < thr);
        while (!done && it < mi && up < max_updates) {
            apply32(p.data(), q.data());
            const float pq = dot(p.data(), q.data(), n, t32);
            const float alpha = rz / pq;
            if (!(pq > 0.0f) || !std::isfinite(alpha)) break;
            for (int64_t i = 0; i < n; ++i) {
                xk[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            const float rr = dot(r.data(), r.data(), n, t32);
            for (int64_t i = 0; i < n; ++i) z[i] = r[i] * (d[i] * r[i]);
            float rzn = pairwise_sum(z.data(), n);
            ++it;
            if (rr < static_cast<float>(delta * delta) * static_cast<float>(rmax2) || rr < static_cast<float>(thr)) {
                for (int64_t i = 0; i < n; ++i) { xs[i] += static_cast<double>(xk[i]); xk[i] = 0.0f; }
                std::vector<double> r64(n);
                for (int64_t i = 0; i < n; ++i) {
                    double acc = 0.0;
                    for (int32_t k = srp[i]; k < srp[i + 1]; ++k) acc += static_cast<double>(val[k]) * xs[ci[k] - r0];
                    r64[i] = b[i] - acc;
                    r[i] = static_cast<float>(r64[i]);
                }
                rr64 = dot(r64.data(), r64.data(), n, t64);
                rmax2 = rr64;
                ++up;
                for (int64_t i = 0; i < n; ++i) z[i] = r[i] * (d[i] * r[i]);
                rzn = pairwise_sum(z.data(), n);
                if (rr64 < thr) { done = true; break; }
            }
            if (!(rzn > 0.0f)) break;
            const float beta = rzn / rz;
            rz = rzn;
            for (int64_t i = 0; i < n; ++i) p[i] = d[i] * r[i] + beta * p[i];
        }
        bool pending = false;
        for (int64_t i = 0; i < n; ++i)
            if (xk[i] != 0.0f) { xs[i] += static_cast<double>(xk[i]); pending = true; }
        if (pending) {
            std::vector<double> r64(n);
            for (int64_t i = 0; i < n; ++i) {
                double acc = 0.0;
                for (int32_t k = srp[i]; k < srp[i + 1]; ++k) acc += static_cast<double>(val[k]) * xs[ci[k] - r0];
                r64[i] = b[i] - acc;
            }
            rr64 = dot(r64.data(), r64.data(), n, t64);
        }
        iters[s] = it;
        updates[s] = up;
        err[s] = bb > 0 ? std::sqrt(rr64 / bb) : 0.0;
    }
    return 0;
}

// The same reliable-update method in the Jacobi-scaled form used by the CUDA
// fast path: the inner FP32 CG (no preconditioner) runs on S A S with
// S = diag(1/sqrt(a_ii)) (1 where a_ii <= 0 or precond == 0), scaled values
// rounded to FP32 (or BF16); x += S xh at every fold; the inner residual is
// S (b - A x); replacement when |r^|^2 < delta^2 |r^_last|^2 or
// |r^|^2 < (tol^2 |b|^2 / |r_last|^2) |r^_last|^2.
int orc_reliable_scaled_packed(int64_t n_sys, const int64_t* row_off, const int32_t* rp, const int32_t* ci,
                               const float* val, const double* rhs, double* x, double tol, double delta,
                               int64_t max_iter, int32_t max_updates, int precond, int bf16_inner, int64_t* iters,
                               int32_t* updates, double* err) {
    std::vector<float> t32;
    std::vector<double> t64;
    for (int64_t s = 0; s < n_sys; ++s) {
        const int64_t r0 = row_off[s], n = row_off[s + 1] - row_off[s];
        const int32_t* srp = rp + r0;
        const int32_t k0 = srp[0];
        std::vector<double> sc(n, 1.0);
        if (precond == 1)
            for (int64_t i = 0; i < n; ++i)
                for (int32_t k = srp[i]; k < srp[i + 1]; ++k)
                    if (ci[k] == r0 + i) { if (val[k] > 0.0f) sc[i] = 1.0 / std::sqrt(static_cast<double>(val[k])); break; }
        std::vector<float> vin(srp[n] - k0);
        for (int64_t i = 0; i < n; ++i)
            for (int32_t k = srp[i]; k < srp[i + 1]; ++k) {
                const float v = static_cast<float>(static_cast<double>(bf16_inner ? bf16_round(val[k]) : val[k]) * sc[i] *
                                                   sc[ci[k] - r0]);
                vin[k - k0] = bf16_inner ? bf16_round(v) : v;
            }
        const double* b = rhs + r0;
        double* xs = x + r0;
        std::vector<float> r(n), p(n), q(n), xh(n, 0.0f), sq(n);
        for (int64_t i = 0; i < n; ++i) {
            xs[i] = 0.0;
            r[i] = static_cast<float>(sc[i] * b[i]);
            p[i] = r[i];
        }
        const double bb = dot(b, b, n, t64);
        float rz = dot(r.data(), r.data(), n, t32);
        const double thr = tol * tol * bb;
        double rr64 = bb;
        float rmax = rz;
        int64_t it = 0;
        int32_t up = 0;
        const int64_t mi = max_iter < 0 ? 2 * n : max_iter;
        bool folded = true;
        auto residual = [&](std::vector<double>& r64) {
            for (int64_t i = 0; i < n; ++i) {
                double acc = 0.0;
                for (int32_t k = srp[i]; k < srp[i + 1]; ++k) acc += static_cast<double>(val[k]) * xs[ci[k] - r0];
                r64[i] = b[i] - acc;
            }
        };
        bool done = (bb == 0.0) || (rr64 < thr);
        while (!done && it < mi && up < max_updates) {
            for (int64_t i = 0; i < n; ++i) {
                float acc = 0.0f;
                for (int32_t k = srp[i]; k < srp[i + 1]; ++k) acc += vin[k - k0] * p[ci[k] - r0];
                q[i] = acc;
            }
            const float pq = dot(p.data(), q.data(), n, t32);
            const float alpha = rz / pq;
            if (!(pq > 0.0f) || !std::isfinite(alpha)) break;
            for (int64_t i = 0; i < n; ++i) {
                xh[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            float rzn = dot(r.data(), r.data(), n, t32);
            ++it;
            folded = false;
            if (rzn < static_cast<float>(delta * delta) * rmax || rzn < static_cast<float>(thr / rr64) * rmax) {
                for (int64_t i = 0; i < n; ++i) { xs[i] += sc[i] * static_cast<double>(xh[i]); xh[i] = 0.0f; }
                std::vector<double> r64(n), rh2(n);
                residual(r64);
                for (int64_t i = 0; i < n; ++i) {
                    r[i] = static_cast<float>(sc[i] * r64[i]);
                    rh2[i] = static_cast<double>(r[i]) * static_cast<double>(r[i]);
                }
                rr64 = dot(r64.data(), r64.data(), n, t64);
                rzn = static_cast<float>(pairwise_sum(rh2.data(), n));
                rmax = rzn;
                ++up;
                folded = true;
                if (rr64 < thr) { done = true; break; }
            }
            if (!(rzn > 0.0f)) break;
            const float beta = rzn / rz;
            rz = rzn;
            for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
        }
        if (!folded) {
            for (int64_t i = 0; i < n; ++i) xs[i] += sc[i] * static_cast<double>(xh[i]);
            std::vector<double> r64(n);
            residual(r64);
            rr64 = dot(r64.data(), r64.data(), n, t64);
        }
        iters[s] = it;
        updates[s] = up;
        err[s] = bb > 0 ? std::sqrt(rr64 / bb) : 0.0;
    }
    return 0;
}

// out[k] = alpha * u[row(k)] * v[col(k)] at the pattern's entries.
int orc_sddmm_csr_f64(int32_t rows, const int32_t* rp, const int32_t* ci, double alpha, const double* u,
                      const double* v, double* out) {
    for (int32_t r = 0; r < rows; ++r)
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) out[k] = alpha * u[r] * v[ci[k]];
    return 0;
}
int orc_sddmm_csr_f32(int32_t rows, const int32_t* rp, const int32_t* ci, float alpha, const float* u,
                      const float* v, float* out) {
    for (int32_t r = 0; r < rows; ++r)
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) out[k] = alpha * u[r] * v[ci[k]];
    return 0;
}

float orc_bf16_round(float f) { return bf16_round(f); }

}  // extern "C"
