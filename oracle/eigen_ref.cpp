// CPU ORACLE (reference build) — test infrastructure only.
//
// A thin C-ABI driver around the reference's bundled Eigen 3.3.90
// (third-party/Eigen in the reference repository), which is the CPU path the
// reference benchmarks its GPU solver against
// (benchmarks/conjugate_gradient/Implementation_Eigen.cpp:59-61,
// benchmarks/csrmv/Implementation_Eigen.cpp). The Eigen headers are compiled
// from where they lie in the reference checkout by oracle/Makefile into
// oracle/_ref/libeigen_ref.so; nothing of Eigen is copied into this repository.
//
// Used as (1) a second, independent check of the oracle restatement (iteration
// counts, SpMV results), (2) the FP64 truth for solution errors
// (SimplicialLLT / dense PartialPivLU), and (3) the timed CPU baseline: Eigen's
// ConjugateGradient<SparseMatrix<double, RowMajor>, Lower|Upper, Diagonal|Identity>
// over a batch of independent systems, OpenMP-parallel across systems.

#include <Eigen/Dense>
#include <Eigen/IterativeLinearSolvers>
#include <Eigen/Sparse>
#include <Eigen/SparseCholesky>

#include <chrono>
#include <cstdint>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename T>
using SpR = Eigen::SparseMatrix<T, Eigen::RowMajor, int>;

template <typename T>
SpR<T> make_csr(int64_t rows, int64_t cols, const int32_t* rp, const int32_t* ci, const float* val,
                int64_t col_base = 0) {
    std::vector<Eigen::Triplet<T>> trip;
    const int64_t nz = rp[rows] - rp[0];
    trip.reserve(static_cast<size_t>(nz));
    for (int64_t r = 0; r < rows; ++r)
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k)
            trip.emplace_back(static_cast<int>(r), static_cast<int>(ci[k] - col_base), static_cast<T>(val[k]));
    SpR<T> m(rows, cols);
    m.setFromTriplets(trip.begin(), trip.end());
    m.makeCompressed();
    return m;
}

template <typename T, typename Pre>
void cg_one(const SpR<T>& A, const T* b, T* x, double tol, int64_t maxit, int64_t* iters, double* err) {
    using Vec = Eigen::Matrix<T, Eigen::Dynamic, 1>;
    Eigen::ConjugateGradient<SpR<T>, Eigen::Lower | Eigen::Upper, Pre> cg;
    cg.setTolerance(static_cast<T>(tol));
    if (maxit >= 0) cg.setMaxIterations(maxit);
    cg.compute(A);
    Eigen::Map<const Vec> bv(b, A.rows());
    Eigen::Map<Vec> xv(x, A.rows());
    xv = cg.solve(bv);
    *iters = cg.iterations();
    *err = static_cast<double>(cg.error());
}

struct Packed {
    std::vector<SpR<double>> sys;
    std::vector<int64_t> row_off;
};

}  // namespace

extern "C" {

int eref_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Eigen CG on one CSR system (FP32 matrix + vectors). precond: 0 identity, 1 Jacobi.
int eref_cg_csr_f32(int32_t n, const int32_t* rp, const int32_t* ci, const float* val, const float* b, float* x,
                    double tol, int64_t maxit, int precond, int64_t* iters, double* err) {
    SpR<float> A = make_csr<float>(n, n, rp, ci, val);
    if (precond == 1) cg_one<float, Eigen::DiagonalPreconditioner<float>>(A, b, x, tol, maxit, iters, err);
    else cg_one<float, Eigen::IdentityPreconditioner>(A, b, x, tol, maxit, iters, err);
    return 0;
}

// Same with the FP32 values upcast to FP64 and FP64 vectors.
int eref_cg_csr_f64(int32_t n, const int32_t* rp, const int32_t* ci, const float* val, const double* b, double* x,
                    double tol, int64_t maxit, int precond, int64_t* iters, double* err) {
    SpR<double> A = make_csr<double>(n, n, rp, ci, val);
    if (precond == 1) cg_one<double, Eigen::DiagonalPreconditioner<double>>(A, b, x, tol, maxit, iters, err);
    else cg_one<double, Eigen::IdentityPreconditioner>(A, b, x, tol, maxit, iters, err);
    return 0;
}

// y = A x with Eigen's row-major sparse * dense product (OpenMP inside Eigen
// when built with it). reps repetitions; returns seconds for all of them.
double eref_spmv_csr_f32(int32_t rows, int32_t cols, const int32_t* rp, const int32_t* ci, const float* val,
                         const float* x, float* y, int32_t reps, int32_t nthreads) {
    SpR<float> A = make_csr<float>(rows, cols, rp, ci, val);
    if (nthreads > 0) Eigen::setNbThreads(nthreads);
    Eigen::Map<const Eigen::VectorXf> xv(x, cols);
    Eigen::Map<Eigen::VectorXf> yv(y, rows);
    const auto t0 = std::chrono::steady_clock::now();
    for (int32_t i = 0; i < reps; ++i) yv.noalias() = A * xv;
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// FP64 direct solve (SimplicialLLT, AMD ordering) of one SPD CSR system with
// FP32 values upcast. Returns 0 on success.
int eref_llt_solve(int32_t n, const int32_t* rp, const int32_t* ci, const float* val, const double* b, double* x,
                   int64_t col_base) {
    SpR<double> Ar = make_csr<double>(n, n, rp, ci, val, col_base);
    Eigen::SparseMatrix<double> A = Ar;  // column-major copy for the factorisation
    Eigen::SimplicialLLT<Eigen::SparseMatrix<double>> llt(A);
    if (llt.info() != Eigen::Success) return 1;
    Eigen::Map<const Eigen::VectorXd> bv(b, n);
    Eigen::Map<Eigen::VectorXd> xv(x, n);
    xv = llt.solve(bv);
    return llt.info() == Eigen::Success ? 0 : 2;
}

// FP64 dense LU solve, A row-major n x n.
int eref_dense_solve(int32_t n, const double* a_rowmajor, const double* b, double* x) {
    Eigen::Map<const Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor>> A(a_rowmajor, n, n);
    Eigen::Map<const Eigen::VectorXd> bv(b, n);
    Eigen::Map<Eigen::VectorXd> xv(x, n);
    xv = A.partialPivLu().solve(bv);
    return 0;
}

// ---- packed batch of independent systems (the CPU baseline) ----------------

void* eref_packed_create(int64_t n_sys, const int64_t* row_off, const int32_t* rp, const int32_t* ci,
                         const float* val) {
    auto* P = new Packed();
    P->row_off.assign(row_off, row_off + n_sys + 1);
    P->sys.resize(static_cast<size_t>(n_sys));
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t s = 0; s < n_sys; ++s) {
        const int64_t r0 = row_off[s], n = row_off[s + 1] - row_off[s];
        P->sys[s] = make_csr<double>(n, n, rp + r0, ci, val, r0);
    }
    return P;
}

void eref_packed_destroy(void* h) { delete static_cast<Packed*>(h); }

// Solves systems [s0, s1) with Eigen's FP64 ConjugateGradient (compute + solve
// per system) on nthreads OpenMP threads; b / x are the packed FP64 vectors.
// Returns the wall-clock seconds of the parallel region.
double eref_packed_cg_f64(void* h, int64_t s0, int64_t s1, const double* b, double* x, double tol, int64_t maxit,
                          int precond, int32_t nthreads, int64_t* iters, double* err) {
    auto* P = static_cast<Packed*>(h);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Eigen::setNbThreads(1);
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t s = s0; s < s1; ++s) {
        const int64_t r0 = P->row_off[s];
        int64_t it = 0;
        double e = 0.0;
        if (precond == 1)
            cg_one<double, Eigen::DiagonalPreconditioner<double>>(P->sys[s], b + r0, x + r0, tol, maxit, &it, &e);
        else
            cg_one<double, Eigen::IdentityPreconditioner>(P->sys[s], b + r0, x + r0, tol, maxit, &it, &e);
        iters[s - s0] = it;
        err[s - s0] = e;
    }
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
