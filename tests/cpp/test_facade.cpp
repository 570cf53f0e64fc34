// The reference's own test cases for the batched sparse CG path, written
// against the C++ facade (include/cuMat/*) and run on the GPU:
//   tests/TestSparseMultOp.cu:70-519   CSR / ELLPACK products, batched matrix / vector
//   tests/TestReductionOps4.cu:39-87   dot {49, 32}, squaredNorm {46, 130}, norm
//   tests/TestConjugateGradient.cu     early outs, dense solves, batched dense solve
//   tests/TestSparseMatrix.cu:53-101   CSC pattern, sparse -> dense
//   tests/TestBlockedConjugateGradient.cu:244-275   blocked (3x3) Poisson CG
// plus a sparse 2D Poisson CG against the bundled Eigen's iteration count and
// an FP64-refined solve. Prints one line per case; the exit status is the
// number of failed cases.
#include <cuMat/Core>
#include <cuMat/IterativeLinearSolvers>
#include <cuMat/Sparse>

#include <cmath>
#include <cstdio>
#include <functional>
#include <random>
#include <string>
#include <vector>

using namespace cuMat;

namespace {

int g_failed = 0;
std::string g_msg;

#define REQUIRE(cond)                                                                    \
    do {                                                                                 \
        if (!(cond)) {                                                                   \
            g_msg = std::string(#cond) + " (line " + std::to_string(__LINE__) + ")";    \
            throw std::runtime_error("requirement failed");                              \
        }                                                                                \
    } while (0)

void run(const char* name, const std::function<void()>& f) {
    g_msg.clear();
    try {
        f();
        std::printf("PASS %s\n", name);
    } catch (const std::exception& e) {
        ++g_failed;
        std::printf("FAIL %s: %s %s\n", name, e.what(), g_msg.c_str());
    }
    std::fflush(stdout);
}

template <typename M>
std::vector<double> host(const M& m) {
    auto h = m.toHost();
    return std::vector<double>(h.begin(), h.end());
}

bool close_rel(const std::vector<double>& a, const std::vector<double>& b, double tol) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (std::abs(a[i] - b[i]) > tol * std::max(1.0, std::abs(b[i]))) return false;
    return true;
}

// {1,4,0,0,0},{0,2,3,0,0},{5,0,0,7,8},{0,0,9,0,6} (TestSparseMultOp.cu:73-88)
SparsityPattern<CSR> kat_csr() {
    SparsityPattern<CSR> p;
    p.rows = 4;
    p.cols = 5;
    p.nnz = 9;
    p.IA = SparsityPattern<CSR>::IndexVector::fromHost({0, 1, 1, 2, 0, 3, 4, 2, 4}, 9);
    p.JA = SparsityPattern<CSR>::IndexVector::fromHost({0, 2, 4, 7, 9}, 5);
    return p;
}
const std::vector<float> kKatVals = {1, 4, 2, 3, 5, 7, 8, 9, 6};
const std::vector<float> kKatRhs = {2, 5, 3, -4, 1};
const std::vector<double> kKatOut = {22, 19, -10, 33};

SparsityPattern<ELLPACK> kat_ell() {
    SparsityPattern<ELLPACK> p;
    p.rows = 4;
    p.cols = 5;
    p.nnzPerRow = 3;
    // column-major 4 x 3: rows {0,1,-1} {1,2,-1} {0,3,4} {2,4,-1}
    p.indices = SparsityPattern<ELLPACK>::IndexMatrix::fromHost({0, 1, 0, 2, 1, 2, 3, 4, -1, -1, 4, -1}, 4, 3);
    return p;
}
// padding values are unspecified in the reference (666 there)
const std::vector<float> kKatEllVals = {1, 2, 5, 9, 4, 3, 7, 6, 666, 666, 8, 666};

std::vector<double> scaled(const std::vector<double>& v, double s) {
    std::vector<double> o(v);
    for (auto& x : o) x *= s;
    return o;
}

// symmetric, diagonally dominant dense matrix: (R + R^T) / 2 + n I with R
// uniform in [0, 1) (the reference adds n I to R; CG needs the symmetric part)
template <typename T>
std::vector<T> spd_dense(int n, std::mt19937& rng) {
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::vector<double> r(static_cast<size_t>(n * n));
    for (auto& v : r) v = u(rng);
    std::vector<T> a(static_cast<size_t>(n * n));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            a[static_cast<size_t>(i + n * j)] = static_cast<T>(0.5 * (r[i + n * j] + r[j + n * i]) + (i == j ? n : 0));
    return a;
}

template <typename T>
std::vector<T> uniform(size_t n, std::mt19937& rng, double lo = 0.0, double hi = 1.0) {
    std::uniform_real_distribution<double> u(lo, hi);
    std::vector<T> v(n);
    for (auto& x : v) x = static_cast<T>(u(rng));
    return v;
}

}  // namespace

int main() {
    run("CSR Matrix-Vector Product", [] {
        SparseMatrix<float, 1, CSR> A(kat_csr());
        A.getData().copyFromHost(kKatVals.data());
        VectorXf b = VectorXf::fromHost(kKatRhs, 5);
        VectorXf x = A * b;
        REQUIRE(close_rel(host(x), kKatOut, 1e-6));
    });
    run("CSR BMatrix-Vector Product", [] {
        SparseMatrix<float, 3, CSR> A(kat_csr());
        std::vector<float> v;
        for (float s : {1.f, 2.f, 3.f})
            for (float e : kKatVals) v.push_back(e * s);
        A.getData().copyFromHost(v.data());
        BVectorXf x = A * VectorXf::fromHost(kKatRhs, 5);
        std::vector<double> want;
        for (double s : {1.0, 2.0, 3.0})
            for (double e : scaled(kKatOut, s)) want.push_back(e);
        REQUIRE(x.batches() == 3 && close_rel(host(x), want, 1e-6));
    });
    run("CSR BMatrix-BVector Product", [] {
        SparseMatrix<float, 3, CSR> A(kat_csr());
        std::vector<float> v, bb;
        for (float s : {1.f, 2.f, -1.f})
            for (float e : kKatVals) v.push_back(e * s);
        for (float s : {1.f, 2.f, 3.f})
            for (float e : kKatRhs) bb.push_back(e * s);
        A.getData().copyFromHost(v.data());
        BVectorXf x = A * BVectorXf::fromHost(bb, 5, 1, 3);
        std::vector<double> want;
        for (double s : {1.0, 4.0, -3.0})
            for (double e : scaled(kKatOut, s)) want.push_back(e);
        REQUIRE(close_rel(host(x), want, 1e-6));
    });
    run("CSR product assignment modes", [] {
        SparseMatrix<double, 1, CSR> A(kat_csr());
        std::vector<double> v(kKatVals.begin(), kKatVals.end());
        A.getData().copyFromHost(v.data());
        VectorXd b = VectorXd::fromHost(std::vector<double>(kKatRhs.begin(), kKatRhs.end()), 5);
        VectorXd y = VectorXd::fromHost({1, 1, 1, 1}, 4);
        A.product(b, y, AssignmentMode::ADD);
        REQUIRE(close_rel(host(y), {23, 20, -9, 34}, 1e-12));
        A.product(b, y, AssignmentMode::SUB);
        REQUIRE(close_rel(host(y), {1, 1, 1, 1}, 1e-12));
    });
    run("ELLPACK Matrix-Vector Product", [] {
        SparseMatrix<float, 1, ELLPACK> A(kat_ell());
        A.getData().copyFromHost(kKatEllVals.data());
        VectorXf x = A * VectorXf::fromHost(kKatRhs, 5);
        REQUIRE(close_rel(host(x), kKatOut, 1e-6));
    });
    run("ELLPACK BMatrix-Vector Product", [] {
        SparseMatrix<float, 3, ELLPACK> A(kat_ell());
        std::vector<float> v;
        for (float s : {1.f, 2.f, 3.f})
            for (float e : kKatEllVals) v.push_back(e * s);
        A.getData().copyFromHost(v.data());
        BVectorXf x = A * VectorXf::fromHost(kKatRhs, 5);
        std::vector<double> want;
        for (double s : {1.0, 2.0, 3.0})
            for (double e : scaled(kKatOut, s)) want.push_back(e);
        REQUIRE(close_rel(host(x), want, 1e-6));
    });
    run("pattern validation throws invalid_argument", [] {
        SparsityPattern<CSR> p = kat_csr();
        p.nnz = 8;
        bool thrown = false;
        try {
            p.assertValid();
        } catch (const std::invalid_argument&) {
            thrown = true;
        }
        REQUIRE(thrown);
        SparsityPattern<CSR> q = kat_csr();
        q.IA = SparsityPattern<CSR>::IndexVector::fromHost({0, 1, 1, 2, 0, 3, 7, 2, 4}, 9);   // column 7 >= cols
        thrown = false;
        try {
            SparseMatrix<float, 1, CSR> A(q);
        } catch (const std::invalid_argument&) {
            thrown = true;
        }
        REQUIRE(thrown);
    });
    run("dot", [] {
        // TestReductionOps4.cu:39-62 (float instead of int storage)
        const float d1[2][1][3] = {{{1, 2, 6}}, {{2, 1, 3}}};
        const float d2[1][1][3] = {{{5, -2, 8}}};
        auto m1 = BRowVectorXfR::fromArray(d1);
        auto m2 = RowVectorXfR::fromArray(d2);
        REQUIRE(close_rel(host(m1.dot(m2)), {49, 32}, 0));
        REQUIRE(close_rel(host(m2.dot(m1)), {49, 32}, 0));
    });
    run("norm", [] {
        // TestReductionOps4.cu:64-87
        const double d[2][1][4] = {{{5, 2, 4, 1}}, {{11, 0, 0, -3}}};
        auto m = BMatrixXdR::fromArray(d);
        REQUIRE(close_rel(host(m.squaredNorm()), {46, 130}, 0));
        REQUIRE(close_rel(host(m.norm()), {6.782329983125268139, 11.401754250991379791}, 1e-15));
    });
    run("linear combination", [] {
        // the reference's linear-combination benchmark expression with 3 terms
        std::mt19937 rng(11);
        const int n = 1001;   // not a multiple of 4: the element-wise path
        std::vector<VectorXf> vs;
        std::vector<std::vector<float>> hv;
        for (int t = 0; t < 3; ++t) {
            hv.push_back(uniform<float>(n, rng));
            vs.push_back(VectorXf::fromHost(hv.back(), n));
        }
        const std::vector<double> f = {0.5, -2.0, 3.25};
        VectorXf out = linearCombination(vs, f);
        std::vector<double> want(n);
        for (int i = 0; i < n; ++i) want[i] = 0.5 * hv[0][i] - 2.0 * hv[1][i] + 3.25 * hv[2][i];
        REQUIRE(close_rel(host(out), want, 1e-6));
    });
    for (int size : {5, 10, 50, 100}) {
        const std::string n = "Conjugate Gradient - Early Out Rhs, size " + std::to_string(size);
        run(n.c_str(), [size] {
            std::mt19937 rng(size);
            MatrixXf A = MatrixXf::fromHost(spd_dense<float>(size, rng), size, size);
            VectorXf b = VectorXf::Zero(size);
            ConjugateGradient<MatrixXf> cg(A);
            VectorXf x = cg.solve(b);
            REQUIRE(cg.iterations() == 0);
            REQUIRE(cg.error() == 0);
            REQUIRE(host(x.squaredNorm())[0] == 0);
        });
    }
    for (int size : {5, 10, 50, 100}) {
        const std::string n = "Conjugate Gradient - Early Out X, size " + std::to_string(size);
        // double storage: b = A * xt and the solver's first residual then agree
        // to the last bit, so the exact guess passes the epsilon test
        run(n.c_str(), [size] {
            std::mt19937 rng(100 + size);
            MatrixXd A = MatrixXd::fromHost(spd_dense<double>(size, rng), size, size);
            VectorXd xt = VectorXd::fromHost(uniform<double>(size, rng), size);
            VectorXd b = A * xt;
            ConjugateGradient<MatrixXd> cg(A);
            VectorXd x = cg.solveWithGuess(b, xt);
            REQUIRE(cg.iterations() == 0);
            REQUIRE(cg.error() <= 1e-10);
            REQUIRE(close_rel(host(x), host(xt), 0));
        });
    }
    for (int size : {5, 10, 50, 100}) {
        const std::string n = "Conjugate Gradient - Solve Dense, size " + std::to_string(size);
        run(n.c_str(), [size] {
            std::mt19937 rng(200 + size);
            MatrixXd A = MatrixXd::fromHost(spd_dense<double>(size, rng), size, size);
            VectorXd xt = VectorXd::fromHost(uniform<double>(size, rng), size);
            VectorXd b = A * xt;
            ConjugateGradient<MatrixXd> cg(A);
            cg.setMaxIterations(10 * size);
            VectorXd x = cg.solve(b);
            REQUIRE(cg.iterations() > 0);
            REQUIRE(cg.error() > 0);
            REQUIRE(cg.iterations() < cg.maxIterations());
            REQUIRE(cg.error() <= cg.tolerance());
            REQUIRE(close_rel(host(x), host(xt), 1e-4));
        });
    }
    run("Conjugate Gradient - Solve Dense Batched", [] {
        const int size = 10, batches = 3;
        std::mt19937 rng(7);
        MatrixXd A = MatrixXd::fromHost(spd_dense<double>(size, rng), size, size);
        typedef Matrix<double, Dynamic, 1, batches, ColumnMajor> Vec;
        Vec xt = Vec::fromHost(uniform<double>(size * batches, rng), size, 1, batches);
        Vec b = A * xt;
        ConjugateGradient<MatrixXd> cg(A);
        cg.setMaxIterations(10 * size);
        Vec x = cg.solve(b);
        REQUIRE(cg.iterations() > 0);
        REQUIRE(cg.error() > 0);
        REQUIRE(cg.iterations() < cg.maxIterations());
        REQUIRE(cg.error() <= cg.tolerance());
        REQUIRE(close_rel(host(x), host(xt), 1e-4));
    });
    run("Sparse CG, 2D Poisson 64x64 unpreconditioned vs bundled Eigen", [] {
        // 5-point Poisson, IDX(x, y) = y + x * g, b uniform[-1, 1] from mt19937(0)
        const int g = 64, n = g * g;
        std::vector<int> rp(1, 0), ci;
        std::vector<float> v;
        for (int x = 0; x < g; ++x)
            for (int y = 0; y < g; ++y) {
                const int i = y + x * g;
                auto add = [&](int j, float a) { ci.push_back(j); v.push_back(a); };
                if (x > 0) add(i - g, -1);
                if (y > 0) add(i - 1, -1);
                add(i, 4);
                if (y < g - 1) add(i + 1, -1);
                if (x < g - 1) add(i + g, -1);
                rp.push_back(static_cast<int>(ci.size()));
            }
        SparsityPattern<CSR> p;
        p.rows = p.cols = n;
        p.nnz = static_cast<Index>(ci.size());
        p.JA = SparsityPattern<CSR>::IndexVector::fromHost(rp, n + 1);
        p.IA = SparsityPattern<CSR>::IndexVector::fromHost(ci, p.nnz);
        SparseMatrix<float, 1, CSR> A(p);
        A.getData().copyFromHost(v.data());
        std::mt19937 rng(0);
        std::uniform_real_distribution<float> u(-1.0f, 1.0f);
        std::vector<float> hb(n);
        for (auto& e : hb) e = u(rng);
        VectorXf b = VectorXf::fromHost(hb, n);
        ConjugateGradient<SparseMatrix<float, 1, CSR>, IdentityPreconditioner> cg(A);
        cg.setTolerance(1e-6).setMaxIterations(1000);
        VectorXf x = cg.solve(b);
        // the bundled Eigen ConjugateGradient takes 164 iterations on this system
        REQUIRE(std::abs(static_cast<long>(cg.iterations()) - 164) <= 2);
        REQUIRE(cg.error() < 1e-6);
        // FP64 refinement of the same float system to 1e-10
        SparseMatrix<float, 1, CSR> A2 = A;
        ConjugateGradient<SparseMatrix<float, 1, CSR>> cg2(A2);
        VectorXd b64 = VectorXd::fromHost(std::vector<double>(hb.begin(), hb.end()), n);
        VectorXd x64 = cg2.solveRefined(b64, 1e-10);
        REQUIRE(cg2.error() < 1e-10);
        auto st = cg2.systemStats(1);
        REQUIRE(st.status[0] == CMCG_SOLVE_CONVERGED);
    });
    run("CSC sparse matrix to dense", [] {
        // TestSparseMatrix.cu:53-101: 4 x 5, column pointers JA, row indices IA
        SparsityPattern<CSC> p;
        p.rows = 4;
        p.cols = 5;
        p.nnz = 9;
        p.IA = SparsityPattern<CSC>::IndexVector::fromHost(std::vector<int>{0, 2, 0, 1, 1, 3, 2, 2, 3}, 9);
        p.JA = SparsityPattern<CSC>::IndexVector::fromHost(std::vector<int>{0, 2, 4, 6, 7, 9}, 6);
        p.assertValid();
        SparseMatrix<float, 2, CSC> A(p);
        std::vector<float> v{1, 5, 4, 2, 3, 9, 7, 8, 6, -1, -5, -4, -2, -3, -9, -7, -8, -6};
        A.getData().copyFromHost(v.data());
        auto d = host(A.toDense());
        const double want[4][5] = {{1, 4, 0, 0, 0}, {0, 2, 3, 0, 0}, {5, 0, 0, 7, 8}, {0, 0, 9, 0, 6}};
        for (int b = 0; b < 2; ++b)
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 5; ++c) REQUIRE(d[static_cast<size_t>(b * 20 + r * 5 + c)] == (b ? -1 : 1) * want[r][c]);
        // the transposed product of the CSC matrix: A^T (1, 1, 1, 1) = column sums
        VectorXf ones = VectorXf::fromHost(std::vector<float>{1, 1, 1, 1}, 4);
        SparseMatrix<float, 1, CSC> A1(p);
        A1.getData().copyFromHost(v.data());
        REQUIRE(close_rel(host(A1.transposedProduct(ones)), {6, 6, 12, 7, 14}, 1e-6));
    });
    run("Blocked CG", [] {
        // TestBlockedConjugateGradient.cu:244-275: 3 x 3 blocks of 3 x 3
        // (row-major), b = (0.1, 0, 0 | 0, 0, 0 | 0, 0, -0.1), tol 1e-5, 30 iterations
        SparsityPattern<CSR> blocks;
        blocks.rows = blocks.cols = 3;
        blocks.nnz = 7;
        blocks.JA = SparsityPattern<CSR>::IndexVector::fromHost(std::vector<int>{0, 2, 5, 7}, 4);
        blocks.IA = SparsityPattern<CSR>::IndexVector::fromHost(std::vector<int>{0, 1, 0, 1, 2, 1, 2}, 7);
        const std::vector<float> D{2, -1, 0, -1, 2, -1, 0, -1, 2}, U{0, 0, 0, 0, 0, 0, -1, 0, 0},
            L{0, 0, -1, 0, 0, 0, 0, 0, 0}, E{2, -1, 0, -1, 2, -1, 0, -1, 1};
        std::vector<float> vals;
        for (const auto* blk : {&D, &U, &L, &D, &U, &L, &E}) vals.insert(vals.end(), blk->begin(), blk->end());
        BlockSparseMatrix<float, 3> mat(blocks);
        mat.getData().copyFromHost(vals.data());
        VectorXf b = VectorXf::fromHost(std::vector<float>{0.1f, 0, 0, 0, 0, 0, 0, 0, -0.1f}, 9);
        ConjugateGradient<BlockSparseMatrix<float, 3>> cg(mat);
        cg.setMaxIterations(30);
        cg.setTolerance(1e-5);
        VectorXf x = cg.solve(b);
        REQUIRE(cg.error() < cg.tolerance());
        REQUIRE(cg.iterations() < cg.maxIterations());
        REQUIRE(cg.iterations() > 0);
        // A x reproduces b
        REQUIRE(close_rel(host(mat * x), {0.1, 0, 0, 0, 0, 0, 0, 0, -0.1}, 1e-4));
    });
    std::printf("%d failed\n", g_failed);
    return g_failed;
}
