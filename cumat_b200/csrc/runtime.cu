// Runtime half of the C ABI: errors, contexts, sparsity patterns, matrices.
//
// Replaces, for the sparse CG path, the reference's Context / DevicePointer /
// SparsityPattern / SparseMatrix storage (cuMat/src/Context.h:132-446,
// DevicePointer.h:12-152, SparseMatrixBase.h:29-206, SparseMatrix.h:48-414):
// device memory is owned by explicit handles instead of reference-counted
// shared pointers, and patterns are validated on the host when created (the
// reference only asserts sizes, SparseMatrixBase.h:112-119).

#include <atomic>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>

#include "common.cuh"
#include "objects.h"

namespace cmcg {

namespace {
thread_local std::string g_last_error;
thread_local int64_t g_launches = 0;
}  // namespace

// ---- log hook ---------------------------------------------------------------------
namespace {
std::mutex g_log_mu;
std::atomic<cmcg_log_fn> g_log_cb{nullptr};
std::atomic<int> g_log_level{-1};
void* g_log_user = nullptr;
// CUMAT_LOG=<level>: messages up to that level go to stderr when no callback is set
int env_log_level() {
    static const int lv = [] {
        const char* e = std::getenv("CUMAT_LOG");
        return e ? std::atoi(e) : -1;
    }();
    return lv;
}
}  // namespace

bool log_on(int level) {
    return g_log_cb.load() ? level <= g_log_level.load() : level <= env_log_level();
}

void log_msg(int level, const char* fmt, ...) {
    if (!log_on(level)) return;
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    std::lock_guard<std::mutex> lk(g_log_mu);
    if (cmcg_log_fn cb = g_log_cb.load()) cb(level, buf, g_log_user);
    else std::fprintf(stderr, "[cumat_b200:%d] %s\n", level, buf);
}

void set_error(const std::string& msg) {
    g_last_error = msg;
    log_msg(0, "%s", msg.c_str());
}

cmcg_status fail(cmcg_status code, const std::string& msg) {
    g_last_error = msg;
    log_msg(0, "%s", msg.c_str());
    return code;
}

cmcg_status cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    const char* base = std::strrchr(file, '/');
    g_last_error = std::string("CUDA error '") + cudaGetErrorString(e) + "' in " + what + " (" +
                   (base ? base + 1 : file) + ":" + std::to_string(line) + ")";
    log_msg(0, "%s", g_last_error.c_str());
    return e == cudaErrorMemoryAllocation ? CMCG_ERR_OUT_OF_MEMORY : CMCG_ERR_CUDA;
}

void count_launch(int n) { g_launches += n; }

// ---- device memory ----------------------------------------------------------------
//
// A process-wide cache of freed device blocks, in place of the reference's
// caching device allocator behind Context::mallocDevice / freeDevice
// (cuMat/src/Context.h:271-320): building and releasing solvers, matrices
// and work buffers per call (as the reference's CG benchmark does) then costs
// no driver allocation. Sizes are rounded to classes (powers of two from
// 512 B to 1 MiB, multiples of 2 MiB above); a freed block joins the cache
// only after a device synchronisation (cudaFree synchronises the device as
// well), so no kernel still in flight can read it once it is handed out
// again. Cached bytes per process are capped by CUMAT_CACHE_MB (default
// 1024; 0 turns the cache off); a block above a quarter of the cap goes back
// to the driver, and an allocation that fails empties the cache and retries.
namespace {
struct MemBlock {
    int device;
    size_t bytes;
};
std::mutex g_mem_mu;
// (never destroyed: no CUDA call may run from a static destructor)
std::unordered_map<void*, MemBlock>& live_blocks() {
    static auto* m = new std::unordered_map<void*, MemBlock>();
    return *m;
}
std::multimap<std::pair<int, size_t>, void*>& free_blocks() {
    static auto* m = new std::multimap<std::pair<int, size_t>, void*>();
    return *m;
}
size_t g_cached_bytes = 0;

size_t cache_cap() {
    static const size_t cap = [] {
        const char* e = std::getenv("CUMAT_CACHE_MB");
        return static_cast<size_t>(e ? std::max(0, std::atoi(e)) : 1024) << 20;
    }();
    return cap;
}

size_t size_class(size_t b) {
    if (b > (size_t(1) << 20)) return (b + (size_t(2) << 20) - 1) / (size_t(2) << 20) * (size_t(2) << 20);
    size_t c = 512;
    while (c < b) c <<= 1;
    return c;
}

// returns every cached block to the driver (lock held)
void trim_cache_locked() {
    for (auto& kv : free_blocks()) cudaFree(kv.second);
    free_blocks().clear();
    g_cached_bytes = 0;
}
}  // namespace

cmcg_status dev_alloc(void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return CMCG_OK;
    int dev = 0;
    CMCG_CUDA(cudaGetDevice(&dev));
    const size_t cls = size_class(bytes);
    std::lock_guard<std::mutex> lk(g_mem_mu);
    auto it = free_blocks().find({dev, cls});
    if (it != free_blocks().end()) {
        *p = it->second;
        free_blocks().erase(it);
        g_cached_bytes -= cls;
        live_blocks()[*p] = MemBlock{dev, cls};
        return CMCG_OK;
    }
    cudaError_t e = cudaMalloc(p, cls);
    if (e == cudaErrorMemoryAllocation && !free_blocks().empty()) {
        cudaGetLastError();
        trim_cache_locked();
        e = cudaMalloc(p, cls);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    }
    live_blocks()[*p] = MemBlock{dev, cls};
    return CMCG_OK;
}

void dev_free(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_mem_mu);
    auto it = live_blocks().find(p);
    if (it == live_blocks().end()) {   // (not from dev_alloc)
        cudaFree(p);
        return;
    }
    const MemBlock b = it->second;
    live_blocks().erase(it);
    int cur = -1;
    if (b.bytes > cache_cap() / 4 || cudaGetDevice(&cur) != cudaSuccess || cur != b.device ||
        cudaDeviceSynchronize() != cudaSuccess) {
        cudaFree(p);
        return;
    }
    free_blocks().emplace(std::make_pair(b.device, b.bytes), p);
    g_cached_bytes += b.bytes;
    // over the cap: return the largest cached blocks first
    while (g_cached_bytes > cache_cap() && !free_blocks().empty()) {
        auto big = std::max_element(free_blocks().begin(), free_blocks().end(),
                                    [](const auto& x, const auto& y) { return x.first.second < y.first.second; });
        cudaFree(big->second);
        g_cached_bytes -= big->first.second;
        free_blocks().erase(big);
    }
}

cmcg_status ensure_buffer(void** p, size_t* cur, size_t need) {
    if (*cur >= need && *p) return CMCG_OK;
    dev_free(*p);
    *p = nullptr;
    *cur = 0;
    CMCG_TRY(dev_alloc(p, need));
    *cur = need;
    return CMCG_OK;
}

// entries are padded to a multiple of 8 (16 bytes of BF16) and at least 8, so
// every 16-byte aligned bulk copy of a row range stays inside the allocation
int64_t csr_padded_nnz(int64_t nnz) { return (nnz + 7) / 8 * 8 + 8; }

void ctx_release(cmcg_ctx c) {
    if (!c) return;
    if (--c->refs > 0) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    dev_free(c->red_partial);
    dev_free(c->red_ticket);
    dev_free(c->d_err);
    if (c->capture_stream) cudaStreamDestroy(c->capture_stream);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

void pattern_release(cmcg_pattern p) {
    if (!p) return;
    if (--p->refs > 0) return;
    dev_free(p->d_row_ptr);
    dev_free(p->d_col);
    dev_free(p->d_ell);
    dev_free(p->d_row_off);
    dev_free(p->d_spmv_tiles);
    free_sell(p->sell);
    free_dia(p->dia);
    free_declared(p);
    cmcg_ctx c = p->ctx;
    delete p;
    ctx_release(c);
}

void matrix_release(cmcg_matrix m) {
    if (!m) return;
    if (--m->refs > 0) return;
    cudaSetDevice(m->pat->ctx->device);
    cudaStreamSynchronize(m->pat->ctx->stream);
    dev_free(m->d_vals);
    dev_free(m->d_sell_vals);
    dev_free(m->d_t_vals);
    cmcg_pattern p = m->pat;
    delete m;
    pattern_release(p);
}

namespace {

template <typename S, typename D>
__global__ void k_convert(const S* __restrict__ src, D* __restrict__ dst, int64_t n);

template <>
__global__ void k_convert<float, float>(const float* __restrict__ s, float* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = s[i];
}
template <>
__global__ void k_convert<double, float>(const double* __restrict__ s, float* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = (float)s[i];
}
template <>
__global__ void k_convert<float, double>(const float* __restrict__ s, double* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = (double)s[i];
}
template <>
__global__ void k_convert<double, double>(const double* __restrict__ s, double* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = s[i];
}
template <>
__global__ void k_convert<float, __nv_bfloat16>(const float* __restrict__ s, __nv_bfloat16* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = __float2bfloat16_rn(s[i]);
}
template <>
__global__ void k_convert<double, __nv_bfloat16>(const double* __restrict__ s, __nv_bfloat16* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = __double2bfloat16(s[i]);
}
template <>
__global__ void k_convert<__nv_bfloat16, __nv_bfloat16>(const __nv_bfloat16* __restrict__ s, __nv_bfloat16* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = s[i];
}
template <>
__global__ void k_convert<__nv_bfloat16, float>(const __nv_bfloat16* __restrict__ s, float* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = __bfloat162float(s[i]);
}
template <>
__global__ void k_convert<__nv_bfloat16, double>(const __nv_bfloat16* __restrict__ s, double* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = (double)__bfloat162float(s[i]);
}

template <typename S, typename D>
cmcg_status launch_convert(cmcg_ctx ctx, const void* src, void* dst, int64_t n) {
    if (n == 0) return CMCG_OK;
    const int threads = 256;
    const int64_t want = (n + threads - 1) / threads;
    const int blocks = static_cast<int>(std::min<int64_t>(want, static_cast<int64_t>(ctx->sm_count) * 16));
    k_convert<S, D><<<blocks, threads, 0, ctx->stream>>>(static_cast<const S*>(src), static_cast<D*>(dst), n);
    count_launch();
    CMCG_CHECK_LAUNCH();
    return CMCG_OK;
}

template <typename S>
cmcg_status convert_from(cmcg_ctx ctx, int dst_dt, const void* src, void* dst, int64_t n) {
    switch (dst_dt) {
        case CMCG_F32: return launch_convert<S, float>(ctx, src, dst, n);
        case CMCG_F64: return launch_convert<S, double>(ctx, src, dst, n);
        case CMCG_BF16: return launch_convert<S, __nv_bfloat16>(ctx, src, dst, n);
    }
    return fail(CMCG_ERR_INVALID_ARGUMENT, "unknown destination dtype");
}

}  // namespace

// Converts n elements between element types on the context stream.
cmcg_status convert(cmcg_ctx ctx, int src_dt, const void* src, int dst_dt, void* dst, int64_t n) {
    switch (src_dt) {
        case CMCG_F32: return convert_from<float>(ctx, dst_dt, src, dst, n);
        case CMCG_F64: return convert_from<double>(ctx, dst_dt, src, dst, n);
        case CMCG_BF16: return convert_from<__nv_bfloat16>(ctx, dst_dt, src, dst, n);
    }
    return fail(CMCG_ERR_INVALID_ARGUMENT, "unknown source dtype");
}

}  // namespace cmcg

using namespace cmcg;

extern "C" {

const char* cmcg_last_error_string(void) { return g_last_error.c_str(); }

int32_t cmcg_version(void) { return 10000; }

int64_t cmcg_launch_count(void) { return g_launches; }

cmcg_status cmcg_ctx_create(int32_t device, void* stream, cmcg_ctx* out) {
    CMCG_REQUIRE(out != nullptr, "cmcg_ctx_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    CMCG_CUDA(cudaGetDeviceCount(&ndev));
    CMCG_REQUIRE(device >= 0 && device < ndev, "cmcg_ctx_create: device index out of range");
    CMCG_CUDA(cudaSetDevice(device));
    auto* c = new cmcg_ctx_s();
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete c;
            return cuda_fail(e, "cudaStreamCreateWithFlags", __FILE__, __LINE__);
        }
        c->own_stream = true;
    }
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&c->d_err), 16);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_err, 0, 16, c->stream);
    if (e != cudaSuccess) {
        ctx_release(c);
        return cuda_fail(e, "device error word", __FILE__, __LINE__);
    }
    *out = c;
    return CMCG_OK;
}

cmcg_status cmcg_ctx_destroy(cmcg_ctx ctx) {
    // patterns still alive keep the context (and its stream) until they go
    ctx_release(ctx);
    return CMCG_OK;
}

cmcg_status cmcg_ctx_device_errors(cmcg_ctx ctx, int32_t* flags) {
    CMCG_REQUIRE(ctx && flags, "cmcg_ctx_device_errors: NULL argument");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    CMCG_CUDA(cudaStreamSynchronize(ctx->stream));
    CMCG_CUDA(cudaMemcpy(flags, ctx->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost));
    CMCG_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int32_t), ctx->stream));
    CMCG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CMCG_OK;
}

cmcg_status cmcg_ctx_synchronize(cmcg_ctx ctx) {
    CMCG_REQUIRE(ctx, "cmcg_ctx_synchronize: NULL context");
    CMCG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CMCG_OK;
}

cmcg_status cmcg_ctx_stream(cmcg_ctx ctx, void** stream) {
    CMCG_REQUIRE(ctx && stream, "cmcg_ctx_stream: NULL argument");
    *stream = ctx->stream;
    return CMCG_OK;
}

// ---- device memory for callers without a CUDA runtime of their own ---------------

cmcg_status cmcg_device_alloc(cmcg_ctx ctx, int64_t bytes, void** out) {
    CMCG_REQUIRE(ctx && out, "cmcg_device_alloc: NULL argument");
    CMCG_REQUIRE(bytes >= 0, "cmcg_device_alloc: negative size");
    *out = nullptr;
    CMCG_CUDA(cudaSetDevice(ctx->device));
    return dev_alloc(out, static_cast<size_t>(bytes));
}

cmcg_status cmcg_device_free(cmcg_ctx ctx, void* p) {
    CMCG_REQUIRE(ctx, "cmcg_device_free: NULL context");
    if (!p) return CMCG_OK;
    CMCG_CUDA(cudaSetDevice(ctx->device));
    // work queued on the context may still read the buffer
    CMCG_CUDA(cudaStreamSynchronize(ctx->stream));
    CMCG_CUDA(cudaFree(p));
    return CMCG_OK;
}

cmcg_status cmcg_memcpy(cmcg_ctx ctx, void* dst, const void* src, int64_t bytes, int32_t kind) {
    CMCG_REQUIRE(ctx && (bytes == 0 || (dst && src)), "cmcg_memcpy: NULL argument");
    CMCG_REQUIRE(bytes >= 0, "cmcg_memcpy: negative size");
    CMCG_REQUIRE(kind == CMCG_HOST_TO_DEVICE || kind == CMCG_DEVICE_TO_HOST || kind == CMCG_DEVICE_TO_DEVICE,
                 "cmcg_memcpy: bad kind");
    if (bytes == 0) return CMCG_OK;
    const cudaMemcpyKind k = kind == CMCG_HOST_TO_DEVICE   ? cudaMemcpyHostToDevice
                             : kind == CMCG_DEVICE_TO_HOST ? cudaMemcpyDeviceToHost
                                                           : cudaMemcpyDeviceToDevice;
    CMCG_CUDA(cudaMemcpyAsync(dst, src, static_cast<size_t>(bytes), k, ctx->stream));
    // host buffers are the caller's again when the call returns
    if (kind != CMCG_DEVICE_TO_DEVICE) CMCG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CMCG_OK;
}

cmcg_status cmcg_memset_zero(cmcg_ctx ctx, void* dst, int64_t bytes) {
    CMCG_REQUIRE(ctx && (bytes == 0 || dst), "cmcg_memset_zero: NULL argument");
    CMCG_REQUIRE(bytes >= 0, "cmcg_memset_zero: negative size");
    if (bytes) CMCG_CUDA(cudaMemsetAsync(dst, 0, static_cast<size_t>(bytes), ctx->stream));
    return CMCG_OK;
}

// ---- patterns -----------------------------------------------------------------

static cmcg_status upload_default_systems(cmcg_pattern p) {
    p->row_off = {0, p->rows};
    dev_free(p->d_row_off);
    p->d_row_off = nullptr;
    CMCG_TRY(dev_alloc(reinterpret_cast<void**>(&p->d_row_off), 2 * sizeof(int32_t)));
    const int32_t h[2] = {0, p->rows};
    CMCG_CUDA(cudaMemcpyAsync(p->d_row_off, h, sizeof(h), cudaMemcpyHostToDevice, p->ctx->stream));
    CMCG_CUDA(cudaStreamSynchronize(p->ctx->stream));
    return CMCG_OK;
}

cmcg_status cmcg_set_log_callback(cmcg_log_fn callback, int32_t max_level, void* user) {
    std::lock_guard<std::mutex> lk(g_log_mu);
    g_log_user = user;
    g_log_level.store(max_level);
    g_log_cb.store(callback);
    return CMCG_OK;
}

cmcg_status cmcg_pattern_create_csr(cmcg_ctx ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                                    const int32_t* col_idx, int32_t is_device, cmcg_pattern* out) {
    CMCG_REQUIRE(ctx && out, "cmcg_pattern_create_csr: NULL context or output");
    *out = nullptr;
    CMCG_REQUIRE(rows > 0 && cols > 0, "cmcg_pattern_create_csr: rows and cols must be positive");
    CMCG_REQUIRE(nnz >= 0 && nnz <= INT32_MAX, "cmcg_pattern_create_csr: nnz must be in [0, 2^31)");
    CMCG_REQUIRE(row_ptr != nullptr, "cmcg_pattern_create_csr: row_ptr is NULL");
    CMCG_REQUIRE(nnz == 0 || col_idx != nullptr, "cmcg_pattern_create_csr: col_idx is NULL");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    auto* p = new cmcg_pattern_s();
    p->ctx = ctx;
    ctx->refs++;
    p->format = CMCG_CSR;
    p->rows = rows;
    p->cols = cols;
    p->nnz = nnz;
    p->h_row_ptr.resize(static_cast<size_t>(rows) + 1);
    p->h_col.resize(static_cast<size_t>(nnz));
    auto cleanup = [p](cmcg_status st) { pattern_release(p); return st; };
    const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    if (cudaMemcpy(p->h_row_ptr.data(), row_ptr, (rows + 1) * sizeof(int32_t), kind) != cudaSuccess ||
        (nnz && cudaMemcpy(p->h_col.data(), col_idx, nnz * sizeof(int32_t), kind) != cudaSuccess))
        return cleanup(fail(CMCG_ERR_CUDA, "cmcg_pattern_create_csr: copying the index arrays failed"));
    // validation (bit-exact CSR semantics of the reference's JA / IA)
    if (p->h_row_ptr[0] != 0) return cleanup(fail(CMCG_ERR_INVALID_ARGUMENT, "CSR row_ptr[0] must be 0"));
    for (int32_t r = 0; r < rows; ++r)
        if (p->h_row_ptr[r + 1] < p->h_row_ptr[r])
            return cleanup(fail(CMCG_ERR_INVALID_ARGUMENT, "CSR row_ptr must be non-decreasing (row " + std::to_string(r) + ")"));
    if (p->h_row_ptr[rows] != nnz) return cleanup(fail(CMCG_ERR_INVALID_ARGUMENT, "CSR row_ptr[rows] must equal nnz"));
    for (int64_t k = 0; k < nnz; ++k)
        if (p->h_col[k] < 0 || p->h_col[k] >= cols)
            return cleanup(fail(CMCG_ERR_INVALID_ARGUMENT, "CSR column index out of range at entry " + std::to_string(k)));
    cmcg_status st;
    // row_ptr padded with 8 copies of nnz and col with zeros to a multiple of 8
    // entries, so 16-byte aligned vector loads and bulk copies of any row range
    // stay inside the arrays
    std::vector<int32_t> rp_pad(p->h_row_ptr);
    rp_pad.resize(static_cast<size_t>(rows) + 1 + 8, static_cast<int32_t>(nnz));
    if ((st = dev_alloc(reinterpret_cast<void**>(&p->d_row_ptr), rp_pad.size() * sizeof(int32_t))) != CMCG_OK) return cleanup(st);
    const int64_t npad = csr_padded_nnz(nnz);
    if ((st = dev_alloc(reinterpret_cast<void**>(&p->d_col), npad * sizeof(int32_t))) != CMCG_OK) return cleanup(st);
    if (cudaMemsetAsync(p->d_col, 0, npad * sizeof(int32_t), ctx->stream) != cudaSuccess ||
        cudaMemcpy(p->d_row_ptr, rp_pad.data(), rp_pad.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        (nnz && cudaMemcpyAsync(p->d_col, p->h_col.data(), nnz * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess))
        return cleanup(fail(CMCG_ERR_CUDA, "cmcg_pattern_create_csr: upload failed"));
    if ((st = upload_default_systems(p)) != CMCG_OK) return cleanup(st);
    *out = p;
    return CMCG_OK;
}

cmcg_status cmcg_pattern_create_ell(cmcg_ctx ctx, int32_t rows, int32_t cols, int32_t nnz_per_row,
                                    const int32_t* indices, int32_t is_device, cmcg_pattern* out) {
    CMCG_REQUIRE(ctx && out, "cmcg_pattern_create_ell: NULL context or output");
    *out = nullptr;
    CMCG_REQUIRE(rows > 0 && cols > 0, "cmcg_pattern_create_ell: rows and cols must be positive");
    CMCG_REQUIRE(nnz_per_row > 0 && nnz_per_row <= cols, "cmcg_pattern_create_ell: need 0 < nnz_per_row <= cols");
    CMCG_REQUIRE(indices != nullptr, "cmcg_pattern_create_ell: indices is NULL");
    CMCG_REQUIRE(static_cast<int64_t>(rows) * nnz_per_row <= INT32_MAX, "cmcg_pattern_create_ell: rows * width too large");
    CMCG_CUDA(cudaSetDevice(ctx->device));
    auto* p = new cmcg_pattern_s();
    p->ctx = ctx;
    ctx->refs++;
    p->format = CMCG_ELLPACK;
    p->rows = rows;
    p->cols = cols;
    p->width = nnz_per_row;
    p->rows_pad = (rows + 3) / 4 * 4;
    p->nnz = static_cast<int64_t>(rows) * nnz_per_row;
    auto cleanup = [p](cmcg_status st) { pattern_release(p); return st; };
    std::vector<int32_t> src(static_cast<size_t>(p->nnz));
    const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    if (cudaMemcpy(src.data(), indices, p->nnz * sizeof(int32_t), kind) != cudaSuccess)
        return cleanup(fail(CMCG_ERR_CUDA, "cmcg_pattern_create_ell: copying indices failed"));
    for (int64_t k = 0; k < p->nnz; ++k)
        if (src[k] < -1 || src[k] >= cols)
            return cleanup(fail(CMCG_ERR_INVALID_ARGUMENT, "ELLPACK index out of range at entry " + std::to_string(k)));
    p->h_col.assign(static_cast<size_t>(p->rows_pad) * nnz_per_row, -1);
    for (int32_t j = 0; j < nnz_per_row; ++j)
        std::memcpy(&p->h_col[static_cast<size_t>(j) * p->rows_pad], &src[static_cast<size_t>(j) * rows], rows * sizeof(int32_t));
    cmcg_status st;
    if ((st = dev_alloc(reinterpret_cast<void**>(&p->d_ell), p->h_col.size() * sizeof(int32_t))) != CMCG_OK) return cleanup(st);
    if (cudaMemcpyAsync(p->d_ell, p->h_col.data(), p->h_col.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return cleanup(fail(CMCG_ERR_CUDA, "cmcg_pattern_create_ell: upload failed"));
    if ((st = upload_default_systems(p)) != CMCG_OK) return cleanup(st);
    *out = p;
    return CMCG_OK;
}

cmcg_status cmcg_pattern_set_systems(cmcg_pattern p, int64_t n_sys, const int64_t* row_off) {
    CMCG_REQUIRE(p && row_off, "cmcg_pattern_set_systems: NULL argument");
    CMCG_REQUIRE(p->rows == p->cols, "cmcg_pattern_set_systems: pattern must be square");
    CMCG_REQUIRE(n_sys >= 1 && n_sys <= p->rows, "cmcg_pattern_set_systems: need 1 <= n_sys <= rows");
    CMCG_REQUIRE(row_off[0] == 0 && row_off[n_sys] == p->rows, "cmcg_pattern_set_systems: row_off must span [0, rows]");
    for (int64_t s = 0; s < n_sys; ++s)
        CMCG_REQUIRE(row_off[s + 1] > row_off[s], "cmcg_pattern_set_systems: systems must be non-empty and ordered");
    // every stored entry must stay inside its system's diagonal block
    for (int64_t s = 0; s < n_sys; ++s) {
        const int64_t a = row_off[s], e = row_off[s + 1];
        for (int64_t r = a; r < e; ++r) {
            if (p->format == CMCG_CSR) {
                for (int32_t k = p->h_row_ptr[r]; k < p->h_row_ptr[r + 1]; ++k)
                    if (p->h_col[k] < a || p->h_col[k] >= e)
                        return fail(CMCG_ERR_INVALID_ARGUMENT, "entry (" + std::to_string(r) + ", " + std::to_string(p->h_col[k]) +
                                                                   ") couples system " + std::to_string(s) + " with another system");
            } else {
                for (int32_t j = 0; j < p->width; ++j) {
                    const int32_t c = p->h_col[static_cast<size_t>(j) * p->rows_pad + r];
                    if (c >= 0 && (c < a || c >= e))
                        return fail(CMCG_ERR_INVALID_ARGUMENT, "ELLPACK entry of row " + std::to_string(r) + " couples two systems");
                }
            }
        }
    }
    p->row_off.assign(row_off, row_off + n_sys + 1);
    // the sliced layout depends on the systems: rebuild it on next use
    cudaStreamSynchronize(p->ctx->stream);
    free_sell(p->sell);
    p->sell.plan_id++;
    free_dia(p->dia);
    p->dia.plan_id++;
    p->systems_version++;
    std::vector<int32_t> h(row_off, row_off + n_sys + 1);
    dev_free(p->d_row_off);
    p->d_row_off = nullptr;
    CMCG_TRY(dev_alloc(reinterpret_cast<void**>(&p->d_row_off), h.size() * sizeof(int32_t)));
    CMCG_CUDA(cudaMemcpyAsync(p->d_row_off, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice, p->ctx->stream));
    CMCG_CUDA(cudaStreamSynchronize(p->ctx->stream));
    return CMCG_OK;
}

cmcg_status cmcg_pattern_info(cmcg_pattern p, int32_t* rows, int32_t* cols, int64_t* nnz, int32_t* format,
                              int64_t* n_sys, int32_t* width) {
    CMCG_REQUIRE(p, "cmcg_pattern_info: NULL pattern");
    if (rows) *rows = p->rows;
    if (cols) *cols = p->cols;
    if (nnz) *nnz = p->nnz;
    if (format) *format = p->declared >= 0 ? p->declared : p->format;
    if (n_sys) *n_sys = static_cast<int64_t>(p->row_off.size()) - 1;
    if (width) *width = p->declared == CMCG_BSR ? p->block : p->width;
    return CMCG_OK;
}

cmcg_status cmcg_pattern_download(cmcg_pattern p, int32_t* a, int32_t* b) {
    CMCG_REQUIRE(p && a, "cmcg_pattern_download: NULL argument");
    CMCG_CUDA(cudaSetDevice(p->ctx->device));
    CMCG_CUDA(cudaStreamSynchronize(p->ctx->stream));
    if (p->declared >= 0) {
        // the caller's CSC / BSR arrays, as given
        std::copy(p->h_decl_ptr.begin(), p->h_decl_ptr.end(), a);
        if (b) std::copy(p->h_decl_idx.begin(), p->h_decl_idx.end(), b);
    } else if (p->format == CMCG_CSR) {
        CMCG_CUDA(cudaMemcpy(a, p->d_row_ptr, (p->rows + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (b && p->nnz) CMCG_CUDA(cudaMemcpy(b, p->d_col, p->nnz * sizeof(int32_t), cudaMemcpyDeviceToHost));
    } else {
        CMCG_CUDA(cudaMemcpy2D(a, p->rows * sizeof(int32_t), p->d_ell, p->rows_pad * sizeof(int32_t),
                               p->rows * sizeof(int32_t), p->width, cudaMemcpyDeviceToHost));
    }
    return CMCG_OK;
}

cmcg_status cmcg_pattern_destroy(cmcg_pattern p) {
    if (!p) return CMCG_OK;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    pattern_release(p);
    return CMCG_OK;
}

// ---- matrices -------------------------------------------------------------------

cmcg_status cmcg_matrix_create(cmcg_pattern p, int32_t dtype, int32_t batches, cmcg_matrix* out) {
    CMCG_REQUIRE(p && out, "cmcg_matrix_create: NULL pattern or output");
    *out = nullptr;
    CMCG_REQUIRE(dtype_size(dtype) != 0, "cmcg_matrix_create: dtype must be F32, F64 or BF16");
    CMCG_REQUIRE(batches >= 1, "cmcg_matrix_create: batches must be >= 1");
    CMCG_CUDA(cudaSetDevice(p->ctx->device));
    auto* m = new cmcg_matrix_s();
    m->pat = p;
    m->dtype = dtype;
    m->batches = batches;
    m->stride = (p->format == CMCG_CSR) ? csr_padded_nnz(p->nnz) : static_cast<int64_t>(p->width) * p->rows_pad;
    const size_t bytes = static_cast<size_t>(m->stride) * batches * dtype_size(dtype);
    cmcg_status st = dev_alloc(&m->d_vals, bytes);
    if (st != CMCG_OK) { delete m; return st; }
    if (cudaMemsetAsync(m->d_vals, 0, bytes, p->ctx->stream) != cudaSuccess) {
        dev_free(m->d_vals);
        delete m;
        return fail(CMCG_ERR_CUDA, "cmcg_matrix_create: memset failed");
    }
    p->refs++;
    *out = m;
    return CMCG_OK;
}

cmcg_status cmcg_matrix_set_values(cmcg_matrix m, int32_t src_dtype, const void* values, int32_t is_device) {
    CMCG_REQUIRE(m && values, "cmcg_matrix_set_values: NULL argument");
    CMCG_REQUIRE(dtype_size(src_dtype) != 0, "cmcg_matrix_set_values: bad source dtype");
    cmcg_pattern p = m->pat;
    cmcg_ctx ctx = p->ctx;
    CMCG_CUDA(cudaSetDevice(ctx->device));
    const size_t es = dtype_size(src_dtype);
    // stage the user's dense batch-major layout on the device, then convert into
    // the padded internal layout batch by batch (and slot by slot for ELL)
    const int64_t per_batch = p->nnz;
    const size_t total = static_cast<size_t>(per_batch) * m->batches * es;
    void* stage = nullptr;
    const void* src = values;
    if (!is_device) {
        CMCG_TRY(dev_alloc(&stage, total));
        cudaError_t e = cudaMemcpyAsync(stage, values, total, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) { dev_free(stage); return cuda_fail(e, "upload values", __FILE__, __LINE__); }
        src = stage;
    }
    cmcg_status st = CMCG_OK;
    const size_t ed = dtype_size(m->dtype);
    if (p->d_val_perm) {
        // CSC / BSR: convert in the caller's order, then gather into CSR order
        void* conv = nullptr;
        st = dev_alloc(&conv, std::max<size_t>(static_cast<size_t>(per_batch) * m->batches * ed, 16));
        if (st == CMCG_OK) st = convert(ctx, src_dtype, src, m->dtype, conv, per_batch * m->batches);
        if (st == CMCG_OK) st = permute_values(p, m->dtype, conv, per_batch, m->d_vals, m->stride, m->batches, true);
        cudaStreamSynchronize(ctx->stream);
        dev_free(conv);
        if (stage) dev_free(stage);
        m->version++;
        return st;
    }
    for (int32_t b = 0; b < m->batches && st == CMCG_OK; ++b) {
        const char* sb = static_cast<const char*>(src) + static_cast<size_t>(b) * per_batch * es;
        char* db = static_cast<char*>(m->d_vals) + static_cast<size_t>(b) * m->stride * ed;
        if (p->format == CMCG_CSR) {
            st = convert(ctx, src_dtype, sb, m->dtype, db, per_batch);
        } else {
            for (int32_t j = 0; j < p->width && st == CMCG_OK; ++j)
                st = convert(ctx, src_dtype, sb + static_cast<size_t>(j) * p->rows * es, m->dtype,
                             db + static_cast<size_t>(j) * p->rows_pad * ed, p->rows);
        }
    }
    if (stage) {
        cudaStreamSynchronize(ctx->stream);
        dev_free(stage);
    }
    m->version++;
    return st;
}

cmcg_status cmcg_matrix_get_values(cmcg_matrix m, void* host_values) {
    CMCG_REQUIRE(m && host_values, "cmcg_matrix_get_values: NULL argument");
    cmcg_pattern p = m->pat;
    CMCG_CUDA(cudaSetDevice(p->ctx->device));
    CMCG_CUDA(cudaStreamSynchronize(p->ctx->stream));
    const size_t ed = dtype_size(m->dtype);
    if (p->d_val_perm) {
        // CSC / BSR: scatter from CSR order into the caller's order
        void* tmp = nullptr;
        const size_t bytes = std::max<size_t>(static_cast<size_t>(p->nnz) * m->batches * ed, 16);
        CMCG_TRY(dev_alloc(&tmp, bytes));
        cmcg_status st = permute_values(p, m->dtype, m->d_vals, m->stride, tmp, p->nnz, m->batches, false);
        if (st == CMCG_OK && cudaMemcpy(host_values, tmp, static_cast<size_t>(p->nnz) * m->batches * ed,
                                        cudaMemcpyDeviceToHost) != cudaSuccess)
            st = fail(CMCG_ERR_CUDA, "cmcg_matrix_get_values: download failed");
        dev_free(tmp);
        return st;
    }
    for (int32_t b = 0; b < m->batches; ++b) {
        char* hb = static_cast<char*>(host_values) + static_cast<size_t>(b) * p->nnz * ed;
        const char* db = static_cast<const char*>(m->d_vals) + static_cast<size_t>(b) * m->stride * ed;
        if (p->format == CMCG_CSR) {
            if (p->nnz) CMCG_CUDA(cudaMemcpy(hb, db, p->nnz * ed, cudaMemcpyDeviceToHost));
        } else {
            CMCG_CUDA(cudaMemcpy2D(hb, p->rows * ed, db, p->rows_pad * ed, p->rows * ed, p->width, cudaMemcpyDeviceToHost));
        }
    }
    return CMCG_OK;
}

cmcg_status cmcg_matrix_info(cmcg_matrix m, int32_t* dtype, int32_t* batches) {
    CMCG_REQUIRE(m, "cmcg_matrix_info: NULL matrix");
    if (dtype) *dtype = m->dtype;
    if (batches) *batches = m->batches;
    return CMCG_OK;
}

cmcg_status cmcg_matrix_destroy(cmcg_matrix m) {
    // solvers still alive keep the matrix until they are destroyed
    matrix_release(m);
    return CMCG_OK;
}

}  // extern "C"
