// C++ facade over the C ABI (cumat_cg.h): the names a cuMat program uses on
// the batched sparse CG path, with the reference's argument meaning and error
// behaviour, computed by the sm_100a kernels of libcumat_cg.so.
//
// Reference interfaces mirrored (paths relative to the reference repository):
//   Matrix (dense device storage, column-major [batch][col][row])  cuMat/src/Matrix.h
//   SparsityPattern<CSR | ELLPACK>                                  cuMat/src/SparseMatrixBase.h:89-206
//   SparseMatrix<Scalar, Batches, SparseFlags>, A * x               cuMat/src/SparseMatrix.h:48-414,
//                                                                   cuMat/src/SparseProductEvaluation.h:95-276
//   dot / squaredNorm / norm (batched, 1x1xB result)                cuMat/src/ReductionOpsPlugin.inl:279-334
//   ConjugateGradient<MatrixType, Preconditioner>                   cuMat/src/ConjugateGradient.h:96-265
//   IterativeSolverBase (tolerance, maxIterations, iterations,
//   error)                                                          cuMat/src/IterativeSolverBase.h:10-135
//   Context::current() (one stream per host thread)                 cuMat/src/Context.h:132-214
//   cuda_error / std::invalid_argument                              cuMat/src/Errors.h:17-30, Macros.h:158-165
//
// What is not mirrored: the expression-template machinery (lazy cwise
// expressions, blocks, slices, sparseView). Products and reductions here
// evaluate immediately into new device storage. Dense matrices given to
// ConjugateGradient or multiplied with a vector are carried as a CSR matrix
// holding every entry (the reference runs the same CG arithmetic on dense
// storage).
//
// Link: -I include -L cumat_b200/lib -lcumat_cg (the library brings its own
// static CUDA runtime; this header needs none).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../cumat_cg.h"

namespace cuMat {

typedef std::ptrdiff_t Index;
constexpr int Dynamic = -1;

// storage order flags (cuMat/src/Constants.h:18-28)
enum Flags { ColumnMajor = 0x00, RowMajor = 0x01 };
// sparse formats (cuMat/src/Constants.h:168-183)
enum SparseFlags { CSC = 1, CSR = 2, ELLPACK = 3 };
// how a product is written to its target (cuMat/src/Constants.h)
enum class AssignmentMode { ASSIGN, ADD, SUB };

// CUDA failure (cuMat/src/Errors.h:17-30)
class cuda_error : public std::exception {
    std::string message_;

public:
    explicit cuda_error(std::string m) : message_(std::move(m)) {}
    const char* what() const noexcept override { return message_.c_str(); }
};

namespace b200 {

// Turns a C-ABI status into the reference's exception types.
inline void check(cmcg_status s) {
    if (s == CMCG_OK) return;
    std::string msg = cmcg_last_error_string();
    if (s == CMCG_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    if (s == CMCG_ERR_NOT_SUPPORTED) throw std::runtime_error(msg);
    throw cuda_error(msg);
}

template <typename T>
struct DType;
template <>
struct DType<float> {
    static constexpr int32_t id = CMCG_F32;
};
template <>
struct DType<double> {
    static constexpr int32_t id = CMCG_F64;
};
template <>
struct DType<int> {
    static constexpr int32_t id = -1;   // index storage only, no arithmetic
};

// Library context kept alive by every object created on it.
struct CtxHolder {
    cmcg_ctx ctx = nullptr;
    explicit CtxHolder(int device) { check(cmcg_ctx_create(device, nullptr, &ctx)); }
    ~CtxHolder() {
        if (ctx) cmcg_ctx_destroy(ctx);
    }
    CtxHolder(const CtxHolder&) = delete;
    CtxHolder& operator=(const CtxHolder&) = delete;
};

}  // namespace b200

// One context (device + private stream) per host thread, like the reference's
// thread-local Context. The device is Context::device() at the thread's first
// use (0 unless set).
class Context {
    std::shared_ptr<b200::CtxHolder> h_;
    explicit Context(int device) : h_(std::make_shared<b200::CtxHolder>(device)) {}

public:
    static int& device() {
        static int d = 0;
        return d;
    }
    static Context& current() {
        thread_local Context c(device());
        return c;
    }
    cmcg_ctx handle() const { return h_->ctx; }
    const std::shared_ptr<b200::CtxHolder>& holder() const { return h_; }
    void* stream() const {
        void* s = nullptr;
        b200::check(cmcg_ctx_stream(h_->ctx, &s));
        return s;
    }
    void synchronize() const { b200::check(cmcg_ctx_synchronize(h_->ctx)); }
};

namespace b200 {

// Reference-counted device buffer (reference DevicePointer, cuMat/src/DevicePointer.h:12-30).
class DeviceBuffer {
    std::shared_ptr<CtxHolder> ctx_;
    void* p_ = nullptr;
    size_t bytes_ = 0;

public:
    DeviceBuffer(size_t bytes) : ctx_(Context::current().holder()), bytes_(bytes) {
        check(cmcg_device_alloc(ctx_->ctx, static_cast<int64_t>(bytes), &p_));
    }
    ~DeviceBuffer() {
        if (p_) cmcg_device_free(ctx_->ctx, p_);
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    void* get() const { return p_; }
    size_t bytes() const { return bytes_; }
    cmcg_ctx ctx() const { return ctx_->ctx; }
};

}  // namespace b200

// Dense device matrix with a batch dimension. Element (r, c, b) lives at
// r + rows * (c + cols * b) (ColumnMajor) or c + cols * (r + rows * b)
// (RowMajor). Copies are shallow (shared storage), as in the reference.
template <typename _Scalar, int _Rows, int _Columns, int _Batches, int _Flags>
class Matrix {
public:
    typedef _Scalar Scalar;
    enum { Rows = _Rows, Columns = _Columns, Batches = _Batches, Flags = _Flags };

private:
    Index rows_ = 0, cols_ = 0, batches_ = 0;
    std::shared_ptr<b200::DeviceBuffer> buf_;

    void allocate() {
        if (rows_ < 0 || cols_ < 0 || batches_ < 0) throw std::invalid_argument("Matrix: negative size");
        if ((Rows > 0 && rows_ != Rows) || (Columns > 0 && cols_ != Columns) || (Batches > 0 && batches_ != Batches))
            throw std::invalid_argument("Matrix: size does not match the compile-time size");
        buf_ = std::make_shared<b200::DeviceBuffer>(static_cast<size_t>(size()) * sizeof(Scalar));
    }

public:
    Matrix() : rows_(Rows > 0 ? Rows : 0), cols_(Columns > 0 ? Columns : 0), batches_(Batches > 0 ? Batches : 0) {
        if (rows_ * cols_ * batches_ > 0) allocate();
    }
    // vectors: rows only; matrices: rows and columns (batch count 1 unless fixed)
    explicit Matrix(Index rows) : rows_(rows), cols_(Columns > 0 ? Columns : 1), batches_(Batches > 0 ? Batches : 1) {
        allocate();
    }
    Matrix(Index rows, Index cols) : rows_(rows), cols_(cols), batches_(Batches > 0 ? Batches : 1) { allocate(); }
    Matrix(Index rows, Index cols, Index batches) : rows_(rows), cols_(cols), batches_(batches) { allocate(); }
    // shares the storage of a matrix type with other compile-time sizes (the
    // run-time sizes must fit this type), e.g. VectorXf x = A * b
    template <int R2, int C2, int B2, int F2>
    Matrix(const Matrix<Scalar, R2, C2, B2, F2>& o) : rows_(o.rows_), cols_(o.cols_), batches_(o.batches_), buf_(o.buf_) {
        if ((Rows > 0 && rows_ != Rows) || (Columns > 0 && cols_ != Columns) || (Batches > 0 && batches_ != Batches))
            throw std::invalid_argument("Matrix: size does not match the compile-time size");
        if (F2 != Flags && rows_ > 1 && cols_ > 1) throw std::invalid_argument("Matrix: storage orders differ");
    }
    template <typename, int, int, int, int>
    friend class Matrix;

    Index rows() const { return rows_; }
    Index cols() const { return cols_; }
    Index batches() const { return batches_; }
    Index size() const { return rows_ * cols_ * batches_; }
    Scalar* data() { return buf_ ? static_cast<Scalar*>(buf_->get()) : nullptr; }
    const Scalar* data() const { return buf_ ? static_cast<const Scalar*>(buf_->get()) : nullptr; }
    cmcg_ctx context() const { return buf_ ? buf_->ctx() : Context::current().handle(); }
    bool isExclusiveUse() const { return buf_.use_count() <= 1; }

    // storage order: the raw element array as stored on the device
    void copyFromHost(const Scalar* h) {
        b200::check(cmcg_memcpy(context(), data(), h, size() * static_cast<int64_t>(sizeof(Scalar)), CMCG_HOST_TO_DEVICE));
    }
    void copyToHost(Scalar* h) const {
        b200::check(cmcg_memcpy(context(), h, data(), size() * static_cast<int64_t>(sizeof(Scalar)), CMCG_DEVICE_TO_HOST));
    }
    std::vector<Scalar> toHost() const {
        std::vector<Scalar> v(static_cast<size_t>(size()));
        if (size()) copyToHost(v.data());
        return v;
    }
    // element (r, c, b) of a host copy
    Index index(Index r, Index c, Index b) const {
        return (Flags & RowMajor) ? c + cols_ * (r + rows_ * b) : r + rows_ * (c + cols_ * b);
    }

    static Matrix fromHost(const std::vector<Scalar>& v, Index rows, Index cols = 1, Index batches = 1) {
        Matrix m(rows, cols, batches);
        if (static_cast<Index>(v.size()) != m.size()) throw std::invalid_argument("Matrix::fromHost: size mismatch");
        if (m.size()) m.copyFromHost(v.data());
        return m;
    }
    // a[batch][row][col] like the reference's fromArray
    template <int D, int R, int C>
    static Matrix fromArray(const Scalar (&a)[D][R][C]) {
        Matrix m(R, C, D);
        std::vector<Scalar> h(static_cast<size_t>(m.size()));
        for (int b = 0; b < D; ++b)
            for (int r = 0; r < R; ++r)
                for (int c = 0; c < C; ++c) h[static_cast<size_t>(m.index(r, c, b))] = a[b][r][c];
        m.copyFromHost(h.data());
        return m;
    }

    Matrix deepClone() const {
        Matrix m(rows_, cols_, batches_);
        b200::check(cmcg_memcpy(context(), m.data(), data(), size() * static_cast<int64_t>(sizeof(Scalar)),
                                CMCG_DEVICE_TO_DEVICE));
        return m;
    }
    void setZero() { b200::check(cmcg_memset_zero(context(), data(), size() * static_cast<int64_t>(sizeof(Scalar)))); }
    static Matrix Zero(Index rows, Index cols = 1, Index batches = 1) {
        Matrix m(rows, cols, batches);
        m.setZero();
        return m;
    }
    static Matrix Identity(Index n, Index batches = 1) {
        Matrix m(n, n, batches);
        std::vector<Scalar> h(static_cast<size_t>(m.size()), Scalar(0));
        for (Index b = 0; b < batches; ++b)
            for (Index i = 0; i < n; ++i) h[static_cast<size_t>(m.index(i, i, b))] = Scalar(1);
        m.copyFromHost(h.data());
        return m;
    }

    // batched reductions over rows and columns: one value per batch, on the
    // device, as a 1 x 1 x B matrix (a one-batch operand broadcasts)
    template <int R2, int C2, int B2, int F2>
    Matrix<Scalar, 1, 1, Dynamic, ColumnMajor> dot(const Matrix<Scalar, R2, C2, B2, F2>& o) const {
        static_assert(b200::DType<Scalar>::id >= 0, "dot: float or double storage");
        if (rows_ * cols_ != o.rows() * o.cols()) throw std::invalid_argument("dot: size mismatch");
        if (batches_ != o.batches() && batches_ != 1 && o.batches() != 1)
            throw std::invalid_argument("dot: batch counts must match or be 1");
        const Index ob = batches_ > o.batches() ? batches_ : o.batches();
        Matrix<Scalar, 1, 1, Dynamic, ColumnMajor> out(1, 1, ob);
        b200::check(cmcg_dot(context(), b200::DType<Scalar>::id, rows_ * cols_, data(), static_cast<int32_t>(batches_),
                             o.data(), static_cast<int32_t>(o.batches()), out.data()));
        return out;
    }
    Matrix<Scalar, 1, 1, Dynamic, ColumnMajor> squaredNorm() const {
        static_assert(b200::DType<Scalar>::id >= 0, "squaredNorm: float or double storage");
        Matrix<Scalar, 1, 1, Dynamic, ColumnMajor> out(1, 1, batches_);
        b200::check(cmcg_squared_norm(context(), b200::DType<Scalar>::id, rows_ * cols_, data(),
                                      static_cast<int32_t>(batches_), out.data()));
        return out;
    }
    // norm: square root of squaredNorm per batch (the B scalars are read back)
    Matrix<Scalar, 1, 1, Dynamic, ColumnMajor> norm() const {
        auto sq = squaredNorm();
        std::vector<Scalar> h = sq.toHost();
        for (auto& v : h) v = std::sqrt(v);
        return Matrix<Scalar, 1, 1, Dynamic, ColumnMajor>::fromHost(h, 1, 1, batches_);
    }
};

// sum_t factors[t] * vectors[t] in one fused pass (up to 16 terms): the value
// of the reference's cwise expression `v0 * f0 + v1 * f1 + ...`
// (benchmarks/linear_combination/Implementation_cuMat.cu:52-66). Vectors with
// one batch broadcast against batched ones.
template <typename S, int R, int C, int B, int F>
Matrix<S, R, C, B, F> linearCombination(const std::vector<Matrix<S, R, C, B, F>>& vectors, const std::vector<double>& factors) {
    static_assert(b200::DType<S>::id >= 0, "linearCombination: float or double storage");
    if (vectors.empty() || vectors.size() != factors.size() || vectors.size() > 16)
        throw std::invalid_argument("linearCombination: 1 to 16 (vector, factor) pairs");
    Index ob = 1;
    std::vector<const void*> ptrs;
    std::vector<int32_t> vb;
    for (const auto& v : vectors) {
        if (v.rows() * v.cols() != vectors[0].rows() * vectors[0].cols())
            throw std::invalid_argument("linearCombination: size mismatch");
        ob = v.batches() > ob ? v.batches() : ob;
        ptrs.push_back(v.data());
        vb.push_back(static_cast<int32_t>(v.batches()));
    }
    Matrix<S, R, C, B, F> out(vectors[0].rows(), vectors[0].cols(), ob);
    b200::check(cmcg_lincomb(out.context(), b200::DType<S>::id, vectors[0].rows() * vectors[0].cols(),
                             static_cast<int32_t>(vectors.size()), factors.data(), ptrs.data(), vb.data(), out.data(),
                             static_cast<int32_t>(ob), CMCG_ASSIGN));
    return out;
}

// typedefs of the reference (cuMat/src/Matrix.h:1396-1440), the ones this path uses
#define CUMAT_B200_TYPEDEFS(T, s)                                         \
    typedef Matrix<T, 1, 1, 1, ColumnMajor> Scalar##s;                    \
    typedef Matrix<T, 1, 1, Dynamic, ColumnMajor> BScalar##s;             \
    typedef Matrix<T, Dynamic, 1, 1, ColumnMajor> VectorX##s;             \
    typedef Matrix<T, Dynamic, 1, Dynamic, ColumnMajor> BVectorX##s;      \
    typedef Matrix<T, 1, Dynamic, 1, RowMajor> RowVectorX##s##R;          \
    typedef Matrix<T, 1, Dynamic, Dynamic, RowMajor> BRowVectorX##s##R;   \
    typedef Matrix<T, Dynamic, Dynamic, 1, ColumnMajor> MatrixX##s;       \
    typedef Matrix<T, Dynamic, Dynamic, Dynamic, ColumnMajor> BMatrixX##s; \
    typedef Matrix<T, Dynamic, Dynamic, Dynamic, RowMajor> BMatrixX##s##R;
CUMAT_B200_TYPEDEFS(int, i)
CUMAT_B200_TYPEDEFS(float, f)
CUMAT_B200_TYPEDEFS(double, d)
#undef CUMAT_B200_TYPEDEFS

// ---- sparsity patterns (cuMat/src/SparseMatrixBase.h:89-206) ------------------

template <int _SparseFlags>
struct SparsityPattern;

template <>
struct SparsityPattern<CSR> {
    typedef int StorageIndex;
    typedef Matrix<StorageIndex, Dynamic, 1, 1, ColumnMajor> IndexVector;
    template <typename S, int B>
    using DataMatrix = Matrix<S, Dynamic, 1, B, ColumnMajor>;

    Index nnz = 0;
    Index rows = 0;
    Index cols = 0;
    IndexVector IA;   // column index of every entry, size nnz
    IndexVector JA;   // row pointers, size rows + 1

    // sizes only, like the reference; the index contents are checked when a
    // matrix is created on the pattern
    void assertValid() const {
        if (!(JA.size() == rows + 1 && rows > 0 && cols > 0 && IA.size() == nnz))
            throw std::invalid_argument("SparsityPattern<CSR>: inconsistent sizes");
    }
    Index getNNZ() const { return nnz; }
    template <typename S, int B>
    DataMatrix<S, B> allocateDataMatrix(Index batches) const {
        return DataMatrix<S, B>(nnz, 1, batches);
    }
};

// reference SparsityPattern<CSC> (SparseMatrixBase.h:29-87): JA = column
// pointers (cols + 1), IA = row index of every entry; values in column order
template <>
struct SparsityPattern<CSC> {
    typedef int StorageIndex;
    typedef Matrix<StorageIndex, Dynamic, 1, 1, ColumnMajor> IndexVector;
    template <typename S, int B>
    using DataMatrix = Matrix<S, Dynamic, 1, B, ColumnMajor>;

    Index nnz = 0;
    Index rows = 0;
    Index cols = 0;
    IndexVector IA;   // row index of every entry, size nnz
    IndexVector JA;   // column pointers, size cols + 1

    void assertValid() const {
        if (!(JA.size() == cols + 1 && rows > 0 && cols > 0 && IA.size() == nnz))
            throw std::invalid_argument("SparsityPattern<CSC>: inconsistent sizes");
    }
    Index getNNZ() const { return nnz; }
    template <typename S, int B>
    DataMatrix<S, B> allocateDataMatrix(Index batches) const {
        return DataMatrix<S, B>(nnz, 1, batches);
    }
};

template <>
struct SparsityPattern<ELLPACK> {
    typedef int StorageIndex;
    typedef Matrix<StorageIndex, Dynamic, Dynamic, 1, ColumnMajor> IndexMatrix;
    template <typename S, int B>
    using DataMatrix = Matrix<S, Dynamic, Dynamic, B, ColumnMajor>;

    Index rows = 0;
    Index cols = 0;
    Index nnzPerRow = 0;
    IndexMatrix indices;   // rows x nnzPerRow, column-major, -1 = no entry

    void assertValid() const {
        if (!(indices.rows() == rows && indices.cols() == nnzPerRow && rows > 0 && cols > 0 && nnzPerRow > 0 &&
              nnzPerRow <= cols))
            throw std::invalid_argument("SparsityPattern<ELLPACK>: inconsistent sizes");
    }
    Index getNNZ() const { return rows * nnzPerRow; }
    template <typename S, int B>
    DataMatrix<S, B> allocateDataMatrix(Index batches) const {
        return DataMatrix<S, B>(rows, nnzPerRow, batches);
    }
};

namespace b200 {

struct PatternHandle {
    cmcg_pattern p = nullptr;
    std::shared_ptr<CtxHolder> ctx;
    ~PatternHandle() {
        if (p) cmcg_pattern_destroy(p);
    }
};
struct MatrixHandle {
    cmcg_matrix m = nullptr;
    std::shared_ptr<PatternHandle> pat;
    ~MatrixHandle() {
        if (m) cmcg_matrix_destroy(m);
    }
};

inline std::shared_ptr<PatternHandle> make_pattern(const SparsityPattern<CSR>& sp) {
    sp.assertValid();
    auto h = std::make_shared<PatternHandle>();
    h->ctx = Context::current().holder();
    check(cmcg_pattern_create_csr(h->ctx->ctx, static_cast<int32_t>(sp.rows), static_cast<int32_t>(sp.cols), sp.nnz,
                                  sp.JA.data(), sp.IA.data(), 1, &h->p));
    return h;
}
inline std::shared_ptr<PatternHandle> make_pattern(const SparsityPattern<CSC>& sp) {
    sp.assertValid();
    auto h = std::make_shared<PatternHandle>();
    h->ctx = Context::current().holder();
    check(cmcg_pattern_create_csc(h->ctx->ctx, static_cast<int32_t>(sp.rows), static_cast<int32_t>(sp.cols), sp.nnz,
                                  sp.JA.data(), sp.IA.data(), 1, &h->p));
    return h;
}
inline std::shared_ptr<PatternHandle> make_pattern(const SparsityPattern<ELLPACK>& sp) {
    sp.assertValid();
    auto h = std::make_shared<PatternHandle>();
    h->ctx = Context::current().holder();
    check(cmcg_pattern_create_ell(h->ctx->ctx, static_cast<int32_t>(sp.rows), static_cast<int32_t>(sp.cols),
                                  static_cast<int32_t>(sp.nnzPerRow), sp.indices.data(), 1, &h->p));
    return h;
}

}  // namespace b200

// ---- sparse matrix (cuMat/src/SparseMatrix.h:48-414) ---------------------------

// Values live in getData() (reference layout: [batch][nnz] for CSR,
// [batch][slot][row] for ELLPACK). They are handed to the library before the
// next product or solve after any non-const getData() call; copies of a
// SparseMatrix share pattern and values.
template <typename _Scalar, int _Batches, int _SparseFlags>
class SparseMatrix {
public:
    typedef _Scalar Scalar;
    enum { Batches = _Batches, SFlags = _SparseFlags };
    typedef SparsityPattern<_SparseFlags> SparsityPatternType;
    typedef typename SparsityPatternType::template DataMatrix<_Scalar, _Batches> DataMatrix;
    static_assert(_SparseFlags == CSR || _SparseFlags == CSC || _SparseFlags == ELLPACK,
                  "SparseMatrix: CSR, CSC or ELLPACK storage");
    static_assert(b200::DType<_Scalar>::id >= 0, "SparseMatrix: float or double values");

private:
    struct State {
        SparsityPatternType pattern;
        DataMatrix data;
        std::shared_ptr<b200::MatrixHandle> handle;
        bool dirty = true;
    };
    std::shared_ptr<State> s_;

public:
    SparseMatrix() = default;
    explicit SparseMatrix(const SparsityPatternType& pattern, Index batches = (_Batches > 0 ? _Batches : 1))
        : s_(std::make_shared<State>()) {
        s_->pattern = pattern;
        s_->data = pattern.template allocateDataMatrix<_Scalar, _Batches>(batches);
        s_->data.setZero();
        auto h = std::make_shared<b200::MatrixHandle>();
        h->pat = b200::make_pattern(pattern);
        b200::check(cmcg_matrix_create(h->pat->p, b200::DType<_Scalar>::id, static_cast<int32_t>(batches), &h->m));
        s_->handle = h;
    }

    const SparsityPatternType& getSparsityPattern() const { return s_->pattern; }
    DataMatrix& getData() {
        s_->dirty = true;
        return s_->data;
    }
    const DataMatrix& getData() const { return s_->data; }
    Index rows() const { return s_->pattern.rows; }
    Index cols() const { return s_->pattern.cols; }
    Index batches() const { return s_->data.batches(); }
    Index nnz() const { return s_->pattern.getNNZ(); }
    bool isInitialized() const { return static_cast<bool>(s_); }

    // library handle with the current values (uploads them when they may have changed)
    cmcg_matrix handle() const {
        if (!s_) throw std::runtime_error("SparseMatrix: not initialized");
        if (s_->dirty) {
            b200::check(cmcg_matrix_set_values(s_->handle->m, b200::DType<_Scalar>::id, s_->data.data(), 1));
            s_->dirty = false;
        }
        return s_->handle->m;
    }

    // out (mode)= A * x; x and out are [batch][n] device vectors
    template <typename V1, typename V2>
    void product(const V1& x, V2& out, AssignmentMode mode = AssignmentMode::ASSIGN) const {
        static_assert(std::is_same<typename V1::Scalar, typename V2::Scalar>::value, "product: vector types differ");
        if (x.rows() * x.cols() != cols()) throw std::invalid_argument("SparseMatrix * x: size mismatch");
        const Index ob = batches() > x.batches() ? batches() : x.batches();
        if (out.rows() * out.cols() != rows() || out.batches() != ob)
            throw std::invalid_argument("SparseMatrix * x: output size mismatch");
        const int32_t m = mode == AssignmentMode::ASSIGN ? CMCG_ASSIGN : mode == AssignmentMode::ADD ? CMCG_ADD : CMCG_SUB;
        b200::check(cmcg_spmv(handle(), b200::DType<typename V1::Scalar>::id, x.data(), static_cast<int32_t>(x.batches()),
                              out.data(), m));
    }
    // y = A * x, evaluated immediately into a new vector
    template <typename S, int R, int C, int B, int F>
    Matrix<S, Dynamic, 1, Dynamic, ColumnMajor> operator*(const Matrix<S, R, C, B, F>& x) const {
        const Index ob = batches() > x.batches() ? batches() : x.batches();
        Matrix<S, Dynamic, 1, Dynamic, ColumnMajor> y(rows(), 1, ob);
        product(x, y);
        return y;
    }
    // y = A^T * x, evaluated immediately (CSR / CSC storage)
    template <typename S, int R, int C, int B, int F>
    Matrix<S, Dynamic, 1, Dynamic, ColumnMajor> transposedProduct(const Matrix<S, R, C, B, F>& x) const {
        if (x.rows() * x.cols() != rows()) throw std::invalid_argument("SparseMatrix^T * x: size mismatch");
        const Index ob = batches() > x.batches() ? batches() : x.batches();
        Matrix<S, Dynamic, 1, Dynamic, ColumnMajor> y(cols(), 1, ob);
        b200::check(cmcg_spmv_transposed(handle(), b200::DType<S>::id, x.data(), static_cast<int32_t>(x.batches()),
                                         y.data(), CMCG_ASSIGN));
        return y;
    }
    // dense copy [batch][rows][cols] (row-major), zeros off the pattern: the
    // reference's assignment of a sparse matrix to a dense one
    Matrix<_Scalar, Dynamic, Dynamic, Dynamic, RowMajor> toDense() const {
        Matrix<_Scalar, Dynamic, Dynamic, Dynamic, RowMajor> d(rows(), cols(), batches());
        b200::check(cmcg_matrix_to_dense(handle(), d.data(), 1));
        return d;
    }
};

// Block CSR matrix of BlockSize x BlockSize blocks of Scalar (no reference
// class: the reference puts a user-defined block scalar type, e.g. a
// row-major float3x3 with float3 vectors, into SparseMatrix<Block, 1, CSR>,
// tests/TestBlockedConjugateGradient.cu:10-237). The pattern's JA / IA index
// blocks; values are BlockSize^2 per block, row-major, block after block;
// vectors hold BlockSize entries per block row, so rows() counts scalars.
// Works with ConjugateGradient like any SparseMatrix.
template <typename _Scalar, int BlockSize, int _Batches = 1>
class BlockSparseMatrix {
public:
    typedef _Scalar Scalar;
    enum { Batches = _Batches, Block = BlockSize };
    typedef Matrix<_Scalar, Dynamic, 1, _Batches, ColumnMajor> DataMatrix;

private:
    struct State {
        SparsityPattern<CSR> blocks;
        DataMatrix data;
        std::shared_ptr<b200::MatrixHandle> handle;
        bool dirty = true;
    };
    std::shared_ptr<State> s_;

public:
    BlockSparseMatrix() = default;
    explicit BlockSparseMatrix(const SparsityPattern<CSR>& blocks, Index batches = (_Batches > 0 ? _Batches : 1))
        : s_(std::make_shared<State>()) {
        blocks.assertValid();
        s_->blocks = blocks;
        s_->data = DataMatrix(blocks.nnz * BlockSize * BlockSize, 1, batches);
        s_->data.setZero();
        auto h = std::make_shared<b200::MatrixHandle>();
        h->pat = std::make_shared<b200::PatternHandle>();
        h->pat->ctx = Context::current().holder();
        b200::check(cmcg_pattern_create_bsr(h->pat->ctx->ctx, static_cast<int32_t>(blocks.rows),
                                            static_cast<int32_t>(blocks.cols), BlockSize, blocks.nnz, blocks.JA.data(),
                                            blocks.IA.data(), 1, &h->pat->p));
        b200::check(cmcg_matrix_create(h->pat->p, b200::DType<_Scalar>::id, static_cast<int32_t>(batches), &h->m));
        s_->handle = h;
    }
    DataMatrix& getData() {
        s_->dirty = true;
        return s_->data;
    }
    Index rows() const { return s_->blocks.rows * BlockSize; }
    Index cols() const { return s_->blocks.cols * BlockSize; }
    Index batches() const { return s_->data.batches(); }
    cmcg_matrix handle() const {
        if (s_->dirty) {
            b200::check(cmcg_matrix_set_values(s_->handle->m, b200::DType<_Scalar>::id, s_->data.data(), 1));
            s_->dirty = false;
        }
        return s_->handle->m;
    }
    template <typename S, int R, int C, int B, int F>
    Matrix<S, Dynamic, 1, Dynamic, ColumnMajor> operator*(const Matrix<S, R, C, B, F>& x) const {
        if (x.rows() * x.cols() != cols()) throw std::invalid_argument("BlockSparseMatrix * x: size mismatch");
        const Index ob = batches() > x.batches() ? batches() : x.batches();
        Matrix<S, Dynamic, 1, Dynamic, ColumnMajor> y(rows(), 1, ob);
        b200::check(cmcg_spmv(handle(), b200::DType<S>::id, x.data(), static_cast<int32_t>(x.batches()), y.data(),
                              CMCG_ASSIGN));
        return y;
    }
};

namespace b200 {

// Dense matrix -> CSR matrix with every entry stored (batch 0 of the values;
// all batches when the dense matrix is batched).
template <typename S, int R, int C, int B, int F>
SparseMatrix<S, Dynamic, CSR> dense_as_csr(const Matrix<S, R, C, B, F>& A) {
    const Index n = A.rows(), m = A.cols(), nb = A.batches();
    std::vector<S> h = A.toHost();
    std::vector<int> rp(static_cast<size_t>(n + 1)), ci(static_cast<size_t>(n * m));
    std::vector<S> v(static_cast<size_t>(n * m * nb));
    for (Index r = 0; r <= n; ++r) rp[static_cast<size_t>(r)] = static_cast<int>(r * m);
    for (Index r = 0; r < n; ++r)
        for (Index c = 0; c < m; ++c) ci[static_cast<size_t>(r * m + c)] = static_cast<int>(c);
    for (Index b = 0; b < nb; ++b)
        for (Index r = 0; r < n; ++r)
            for (Index c = 0; c < m; ++c)
                v[static_cast<size_t>(b * n * m + r * m + c)] = h[static_cast<size_t>(A.index(r, c, b))];
    SparsityPattern<CSR> sp;
    sp.rows = n;
    sp.cols = m;
    sp.nnz = n * m;
    sp.JA = SparsityPattern<CSR>::IndexVector::fromHost(rp, n + 1);
    sp.IA = SparsityPattern<CSR>::IndexVector::fromHost(ci, n * m);
    SparseMatrix<S, Dynamic, CSR> out(sp, nb);
    out.getData().copyFromHost(v.data());
    return out;
}

template <typename M>
struct SolverMatrix {   // sparse matrices are used as they are
    typedef M type;
    static const M& get(const M& A) { return A; }
};
template <typename S, int R, int C, int B, int F>
struct SolverMatrix<Matrix<S, R, C, B, F>> {
    typedef SparseMatrix<S, Dynamic, CSR> type;
    static type get(const Matrix<S, R, C, B, F>& A) { return dense_as_csr(A); }
};

}  // namespace b200

// dense matrix times vector through the same product kernel
template <typename S, int R, int C, int B, int F, int R2, int C2, int B2, int F2>
Matrix<S, Dynamic, 1, Dynamic, ColumnMajor> operator*(const Matrix<S, R, C, B, F>& A, const Matrix<S, R2, C2, B2, F2>& x) {
    return b200::dense_as_csr(A) * x;
}

// ---- preconditioners (cuMat/src/ConjugateGradient.h:218-265) -------------------

template <typename _MatrixType>
class DiagonalPreconditioner {
public:
    static constexpr int32_t id = CMCG_PRECOND_JACOBI;
};
class IdentityPreconditioner {
public:
    static constexpr int32_t id = CMCG_PRECOND_IDENTITY;
};

// ---- conjugate gradient (cuMat/src/ConjugateGradient.h:96-206) -----------------

// Per-system result of the last solve (no reference counterpart).
struct SystemStats {
    std::vector<int32_t> iterations, status, outer;
    std::vector<double> error;
};

template <typename _MatrixType, typename _Preconditioner = DiagonalPreconditioner<_MatrixType>>
class ConjugateGradient {
public:
    typedef _MatrixType MatrixType;
    typedef typename MatrixType::Scalar Scalar;
    typedef double RealScalar;
    typedef typename b200::SolverMatrix<MatrixType>::type SMatrix;

private:
    struct SolverHandle {
        cmcg_solver s = nullptr;
        ~SolverHandle() {
            if (s) cmcg_cg_destroy(s);
        }
    };
    SMatrix A_;
    std::shared_ptr<SolverHandle> h_;
    RealScalar tol_ = 0;
    Index max_iter_ = -1;
    bool tol_set_ = false;

public:
    ConjugateGradient() = default;
    explicit ConjugateGradient(const MatrixType& A) { compute(A); }

    // shallow copy of the matrix; the Jacobi diagonal is extracted here
    ConjugateGradient& compute(const MatrixType& A) {
        A_ = b200::SolverMatrix<MatrixType>::get(A);
        h_ = std::make_shared<SolverHandle>();
        b200::check(cmcg_cg_create(A_.handle(), _Preconditioner::id, &h_->s));
        if (tol_set_) b200::check(cmcg_cg_set_tolerance(h_->s, tol_));
        if (max_iter_ >= 0) b200::check(cmcg_cg_set_max_iterations(h_->s, max_iter_));
        return *this;
    }
    // default tolerance: machine epsilon of the scalar type (IterativeSolverBase.h:131)
    RealScalar tolerance() const {
        return tol_set_ ? tol_ : (std::is_same<Scalar, double>::value ? 2.220446049250313e-16 : 1.1920928955078125e-07);
    }
    ConjugateGradient& setTolerance(RealScalar t) {
        tol_ = t;
        tol_set_ = true;
        if (h_) b200::check(cmcg_cg_set_tolerance(h_->s, t));
        return *this;
    }
    // default: 2 * columns (IterativeSolverBase.h:83-86)
    Index maxIterations() const { return max_iter_ < 0 ? 2 * A_.cols() : max_iter_; }
    ConjugateGradient& setMaxIterations(Index m) {
        max_iter_ = m;
        if (h_) b200::check(cmcg_cg_set_max_iterations(h_->s, m));
        return *this;
    }
    // execution path (CMCG_PATH_*) and mixed-precision method (no reference counterpart)
    ConjugateGradient& setPath(int32_t path) {
        b200::check(cmcg_cg_set_path(solver(), path));
        return *this;
    }
    cmcg_solver solver() const {
        if (!h_) throw std::runtime_error("ConjugateGradient: compute() was not called");
        return h_->s;
    }

    template <typename Vec>
    Vec solve(const Vec& b) const {
        return solveWithGuessImpl(b, nullptr);
    }
    template <typename Vec, typename Guess>
    Vec solveWithGuess(const Vec& b, const Guess& x0) const {
        static_assert(std::is_same<typename Vec::Scalar, typename Guess::Scalar>::value, "guess type differs");
        const Index ob = A_.batches() > b.batches() ? A_.batches() : b.batches();
        if (x0.rows() * x0.cols() != b.rows() * b.cols() || x0.batches() != ob)
            throw std::invalid_argument("solveWithGuess: guess size mismatch");
        return solveWithGuessImpl(b, x0.data());
    }

    // FP64 solution of a float or BF16-valued system, refined to outer_tol
    // (residual replacement in FP64, no reference counterpart). outer: the
    // matrix whose values define the FP64 residual (default: this matrix).
    template <typename Vec>
    Vec solveRefined(const Vec& b, double outer_tol, int32_t max_outer = 100, const SMatrix* outer = nullptr) const {
        static_assert(std::is_same<typename Vec::Scalar, double>::value, "solveRefined: FP64 right-hand side");
        const Index ob = A_.batches() > b.batches() ? A_.batches() : b.batches();
        Vec x(b.rows(), b.cols(), ob);
        (void)A_.handle();
        b200::check(cmcg_cg_solve_refined(solver(), outer ? outer->handle() : nullptr, b.data(),
                                          static_cast<int32_t>(b.batches()), x.data(), outer_tol, max_outer));
        return x;
    }

    // largest iteration count / error over all systems of the last solve
    Index iterations() const {
        int64_t it = 0;
        b200::check(cmcg_cg_iterations(solver(), &it));
        return static_cast<Index>(it);
    }
    RealScalar error() const {
        double e = 0;
        b200::check(cmcg_cg_error(solver(), &e));
        return e;
    }
    SystemStats systemStats(Index instances) const {
        SystemStats st;
        st.iterations.resize(static_cast<size_t>(instances));
        st.status.resize(static_cast<size_t>(instances));
        st.outer.resize(static_cast<size_t>(instances));
        st.error.resize(static_cast<size_t>(instances));
        b200::check(cmcg_cg_system_stats(solver(), st.iterations.data(), st.error.data(), st.status.data(),
                                         st.outer.data()));
        return st;
    }

private:
    template <typename Vec>
    Vec solveWithGuessImpl(const Vec& b, const void* guess) const {
        static_assert(std::is_same<typename Vec::Scalar, float>::value || std::is_same<typename Vec::Scalar, double>::value,
                      "solve: float or double vectors");
        if (b.rows() * b.cols() != A_.rows()) throw std::invalid_argument("solve: rhs size mismatch");
        const Index ob = A_.batches() > b.batches() ? A_.batches() : b.batches();
        Vec x(b.rows(), b.cols(), ob);
        (void)A_.handle();   // values changed through getData() reach the library
        b200::check(cmcg_cg_solve(solver(), b200::DType<typename Vec::Scalar>::id, b.data(),
                                  static_cast<int32_t>(b.batches()), guess, x.data()));
        return x;
    }
};

}  // namespace cuMat
