// Seeded synthetic problem generators for the batched sparse CG path.
//
// These build the same matrices the reference's benchmark drivers assemble on
// the host before uploading (benchmarks/conjugate_gradient/Implementation_cuMat.cu:29-41,
// benchmarks/csrmv/Implementation_cuMat_ELLPACK.cu:33-62): row index
// IDX(x, y) = y + x*g, Eigen RowMajor compressed storage (columns sorted within
// a row), int32 indices. The variable-coefficient finite-volume families extend
// the 5-point Poisson stencil: every cell face carries kappa = exp(g),
// g ~ N(0, sigma^2); an interior face couples its two cells with -kappa and adds
// kappa to both diagonals, a boundary face (Dirichlet 0) adds kappa to the
// diagonal of its one cell. kappa == 1 reproduces the Poisson matrix exactly.
//
// All values are generated in double and stored rounded to FP32: the FP32 matrix
// is the problem definition, so an FP64 residual computed from upcast FP32
// values is exact.
//
// Random streams: std::mt19937 seeded with the config seed;
// std::uniform_real_distribution<float>(-1, 1) for right-hand sides,
// std::uniform_int_distribution<int>(lo, hi) for grid sides,
// std::normal_distribution<double>(0, sigma) for face log-coefficients and
// std::normal_distribution<double>(0, 1) for targets. Draw order for a batch:
// all sides, then the face coefficients system by system (x-faces, then
// y-faces), then the right-hand sides system by system, then the targets.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

inline float rnd_f32(double v) { return static_cast<float>(v); }

// Faces of an s x s cell grid. xf[x*s + y] for x in [0, s] is the face between
// cells (x-1, y) and (x, y); yf[x*(s+1) + y] for y in [0, s] is the face
// between (x, y-1) and (x, y).
struct Faces2D {
    int s;
    std::vector<double> xf, yf;
};

void draw_faces_2d(std::mt19937& rng, int s, double sigma, Faces2D& f) {
    f.s = s;
    f.xf.resize(static_cast<size_t>(s + 1) * s);
    f.yf.resize(static_cast<size_t>(s) * (s + 1));
    if (sigma == 0.0) {
        std::fill(f.xf.begin(), f.xf.end(), 1.0);
        std::fill(f.yf.begin(), f.yf.end(), 1.0);
        return;
    }
    std::normal_distribution<double> N(0.0, sigma);
    for (auto& v : f.xf) v = std::exp(N(rng));
    for (auto& v : f.yf) v = std::exp(N(rng));
}

// Writes the rows of one s x s system. row_ptr receives s*s+1 entries relative
// to nnz_base; col receives global column indices (col_base + local).
int64_t fill_fv2d(const Faces2D& f, int64_t col_base, int64_t nnz_base,
                  int32_t* row_ptr, int32_t* col, float* val) {
    const int s = f.s;
    auto IDX = [s](int x, int y) -> int64_t { return static_cast<int64_t>(y) + static_cast<int64_t>(x) * s; };
    auto KX = [&f, s](int x, int y) { return f.xf[static_cast<size_t>(x) * s + y]; };
    auto KY = [&f, s](int x, int y) { return f.yf[static_cast<size_t>(x) * (s + 1) + y]; };
    int64_t k = nnz_base;
    for (int x = 0; x < s; ++x) {
        for (int y = 0; y < s; ++y) {
            const int64_t r = IDX(x, y);
            row_ptr[r] = static_cast<int32_t>(k);
            const double kw = KX(x, y), ke = KX(x + 1, y), ks = KY(x, y), kn = KY(x, y + 1);
            const double diag = kw + ks + kn + ke;
            if (x > 0) { col[k] = static_cast<int32_t>(col_base + IDX(x - 1, y)); val[k] = rnd_f32(-kw); ++k; }
            if (y > 0) { col[k] = static_cast<int32_t>(col_base + IDX(x, y - 1)); val[k] = rnd_f32(-ks); ++k; }
            col[k] = static_cast<int32_t>(col_base + r); val[k] = rnd_f32(diag); ++k;
            if (y < s - 1) { col[k] = static_cast<int32_t>(col_base + IDX(x, y + 1)); val[k] = rnd_f32(-kn); ++k; }
            if (x < s - 1) { col[k] = static_cast<int32_t>(col_base + IDX(x + 1, y)); val[k] = rnd_f32(-ke); ++k; }
        }
    }
    return k;
}

inline int64_t nnz_fv2d(int64_t s) { return 5 * s * s - 4 * s; }
inline int64_t nnz_fv3d(int64_t s) { return 7 * s * s * s - 6 * s * s; }

}  // namespace

extern "C" {

// ---- 5-point Poisson (kappa == 1) -----------------------------------------

int64_t cmgen_poisson2d_nnz(int32_t g) { return nnz_fv2d(g); }

// row_ptr: g*g+1, col/val: cmgen_poisson2d_nnz(g).
int cmgen_poisson2d(int32_t g, int32_t* row_ptr, int32_t* col, float* val) {
    if (g <= 0 || static_cast<int64_t>(g) * g > INT32_MAX) return 1;
    std::mt19937 unused(0);
    Faces2D f;
    draw_faces_2d(unused, g, 0.0, f);
    const int64_t end = fill_fv2d(f, 0, 0, row_ptr, col, val);
    row_ptr[static_cast<int64_t>(g) * g] = static_cast<int32_t>(end);
    return 0;
}

// n draws of U[lo, hi] as float from mt19937(seed).
int cmgen_uniform_f32(uint32_t seed, int64_t n, float lo, float hi, float* out) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> U(lo, hi);
    for (int64_t i = 0; i < n; ++i) out[i] = U(rng);
    return 0;
}

// ---- batches of 2D variable-coefficient systems ---------------------------

// Draws the sides of n_sys systems (the first draws of the stream). When
// side_lo == side_hi no draw is made. Returns total rows / nnz.
int cmgen_fv2d_batch_dims(int64_t n_sys, int32_t side_lo, int32_t side_hi, uint32_t seed,
                          int32_t* sides, int64_t* n_rows, int64_t* nnz) {
    if (n_sys <= 0 || side_lo <= 0 || side_hi < side_lo) return 1;
    std::mt19937 rng(seed);
    std::uniform_int_distribution<int> S(side_lo, side_hi);
    int64_t rows = 0, nz = 0;
    for (int64_t i = 0; i < n_sys; ++i) {
        const int s = (side_lo == side_hi) ? side_lo : S(rng);
        sides[i] = s;
        rows += static_cast<int64_t>(s) * s;
        nz += nnz_fv2d(s);
    }
    *n_rows = rows;
    *nnz = nz;
    if (rows > INT32_MAX || nz > INT32_MAX) return 2;
    return 0;
}

// Packs the systems as one block-diagonal CSR matrix. row_off has n_sys+1
// entries (system i owns rows [row_off[i], row_off[i+1])). b gets one U[-1,1]
// right-hand side per system; xstar (may be NULL) gets N(0,1) targets.
int cmgen_fv2d_batch(int64_t n_sys, int32_t side_lo, int32_t side_hi, double sigma, uint32_t seed,
                     int32_t* row_ptr, int32_t* col, float* val, int64_t* row_off,
                     float* b, float* xstar) {
    if (n_sys <= 0 || side_lo <= 0 || side_hi < side_lo) return 1;
    std::mt19937 rng(seed);
    std::vector<int> sides(static_cast<size_t>(n_sys));
    {
        std::uniform_int_distribution<int> S(side_lo, side_hi);
        for (auto& s : sides) s = (side_lo == side_hi) ? side_lo : S(rng);
    }
    int64_t r0 = 0, k = 0;
    Faces2D f;
    for (int64_t i = 0; i < n_sys; ++i) {
        row_off[i] = r0;
        draw_faces_2d(rng, sides[i], sigma, f);
        k = fill_fv2d(f, r0, k, row_ptr + r0, col, val);
        r0 += static_cast<int64_t>(sides[i]) * sides[i];
    }
    row_off[n_sys] = r0;
    row_ptr[r0] = static_cast<int32_t>(k);
    std::uniform_real_distribution<float> U(-1.0f, 1.0f);
    for (int64_t i = 0; i < r0; ++i) b[i] = U(rng);
    if (xstar) {
        std::normal_distribution<double> N(0.0, 1.0);
        for (int64_t i = 0; i < r0; ++i) xstar[i] = static_cast<float>(N(rng));
    }
    return 0;
}

// ---- 3D 7-point variable-coefficient system --------------------------------

int64_t cmgen_fv3d_nnz(int32_t s) { return nnz_fv3d(s); }

// s^3 cells, row = z + s*(y + s*x); faces drawn x-faces, y-faces, z-faces, each
// in (x, y, z) lexicographic order of the face position; then n U[-1,1] rhs.
int cmgen_fv3d(int32_t s, double sigma, uint32_t seed,
               int32_t* row_ptr, int32_t* col, float* val, float* b) {
    if (s <= 0) return 1;
    const int64_t S = s, n = S * S * S;
    if (n > INT32_MAX || nnz_fv3d(s) > INT32_MAX) return 2;
    std::mt19937 rng(seed);
    std::normal_distribution<double> N(0.0, sigma);
    // kappa stored as float (exp in double, then rounded) to keep memory modest.
    std::vector<float> kx(static_cast<size_t>((S + 1) * S * S)), ky(static_cast<size_t>(S * (S + 1) * S)),
        kz(static_cast<size_t>(S * S * (S + 1)));
    for (auto& v : kx) v = static_cast<float>(std::exp(N(rng)));
    for (auto& v : ky) v = static_cast<float>(std::exp(N(rng)));
    for (auto& v : kz) v = static_cast<float>(std::exp(N(rng)));
    auto IX = [S](int64_t x, int64_t y, int64_t z) { return (x * S + y) * S + z; };          // (S+1) x S x S
    auto IY = [S](int64_t x, int64_t y, int64_t z) { return (x * (S + 1) + y) * S + z; };    // S x (S+1) x S
    auto IZ = [S](int64_t x, int64_t y, int64_t z) { return (x * S + y) * (S + 1) + z; };    // S x S x (S+1)
    auto ROW = [S](int64_t x, int64_t y, int64_t z) { return z + S * (y + S * x); };
    int64_t k = 0;
    for (int64_t x = 0; x < S; ++x)
        for (int64_t y = 0; y < S; ++y)
            for (int64_t z = 0; z < S; ++z) {
                const int64_t r = ROW(x, y, z);
                row_ptr[r] = static_cast<int32_t>(k);
                const double kw = kx[IX(x, y, z)], ke = kx[IX(x + 1, y, z)];
                const double ks = ky[IY(x, y, z)], kn = ky[IY(x, y + 1, z)];
                const double kd = kz[IZ(x, y, z)], ku = kz[IZ(x, y, z + 1)];
                const double diag = kw + ke + ks + kn + kd + ku;
                if (x > 0) { col[k] = static_cast<int32_t>(ROW(x - 1, y, z)); val[k] = rnd_f32(-kw); ++k; }
                if (y > 0) { col[k] = static_cast<int32_t>(ROW(x, y - 1, z)); val[k] = rnd_f32(-ks); ++k; }
                if (z > 0) { col[k] = static_cast<int32_t>(ROW(x, y, z - 1)); val[k] = rnd_f32(-kd); ++k; }
                col[k] = static_cast<int32_t>(r); val[k] = rnd_f32(diag); ++k;
                if (z < S - 1) { col[k] = static_cast<int32_t>(ROW(x, y, z + 1)); val[k] = rnd_f32(-ku); ++k; }
                if (y < S - 1) { col[k] = static_cast<int32_t>(ROW(x, y + 1, z)); val[k] = rnd_f32(-kn); ++k; }
                if (x < S - 1) { col[k] = static_cast<int32_t>(ROW(x + 1, y, z)); val[k] = rnd_f32(-ke); ++k; }
            }
    row_ptr[n] = static_cast<int32_t>(k);
    std::uniform_real_distribution<float> U(-1.0f, 1.0f);
    for (int64_t i = 0; i < n; ++i) b[i] = U(rng);
    return 0;
}

// ---- CSR -> column-major ELLPACK ------------------------------------------

// Width = longest row. indices/values are rows x width column-major
// (entry (row, slot) at row + slot*rows); slot j of a row holds its j-th CSR
// entry, so the 5-point stencil lands in slot order W, S, C, N, E as in the
// reference ELLPACK benchmark. Padding: index -1, value 0.
int32_t cmgen_ell_width(int32_t rows, const int32_t* row_ptr) {
    int32_t w = 0;
    for (int32_t r = 0; r < rows; ++r) w = std::max(w, row_ptr[r + 1] - row_ptr[r]);
    return w;
}

int cmgen_csr_to_ell(int32_t rows, const int32_t* row_ptr, const int32_t* col, const float* val,
                     int32_t width, int32_t* ell_idx, float* ell_val) {
    const int64_t R = rows;
    for (int64_t r = 0; r < R; ++r) {
        const int32_t a = row_ptr[r], e = row_ptr[r + 1];
        if (e - a > width) return 1;
        for (int32_t j = 0; j < width; ++j) {
            const int64_t o = r + static_cast<int64_t>(j) * R;
            if (a + j < e) { ell_idx[o] = col[a + j]; if (ell_val) ell_val[o] = val[a + j]; }
            else { ell_idx[o] = -1; if (ell_val) ell_val[o] = 0.0f; }
        }
    }
    return 0;
}

}  // extern "C"
