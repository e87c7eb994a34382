// Context, grid descriptors, scratch and error reporting of the C ABI.
#include "gb_common.cuh"

#include <cstdarg>
#include <cstring>

namespace gb {

namespace {
thread_local std::string g_error;
}

void set_error(const char* fmt, ...)
{
    char buf[4096];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

void clear_error() { g_error.clear(); }

gb_status check_cuda(const char* op)
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) { return GB_OK; }
    set_error("gust: %s: CUDA error %s (%s)", op, cudaGetErrorName(e), cudaGetErrorString(e));
    return (e == cudaErrorMemoryAllocation) ? GB_OOM : GB_CUDA;
}

void* scratch(gb_ctx* ctx, int slot, size_t bytes)
{
    if (slot >= static_cast<int>(ctx->slot_ptr.size())) {
        ctx->slot_ptr.resize(slot + 1, nullptr);
        ctx->slot_bytes.resize(slot + 1, 0);
    }
    if (ctx->slot_bytes[slot] >= bytes && ctx->slot_ptr[slot] != nullptr) { return ctx->slot_ptr[slot]; }
    if (ctx->slot_ptr[slot] != nullptr) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->slot_ptr[slot]);
        ctx->slot_ptr[slot] = nullptr;
        ctx->slot_bytes[slot] = 0;
    }
    void* p = nullptr;
    const size_t want = (bytes + 255) & ~static_cast<size_t>(255);
    if (cudaMalloc(&p, want) != cudaSuccess) {
        cudaGetLastError();
        set_error("gust: scratch: cannot allocate %zu bytes of device memory", want);
        return nullptr;
    }
    ctx->slot_ptr[slot] = p;
    ctx->slot_bytes[slot] = want;
    return p;
}

gb_status read_words(gb_ctx* ctx, int first, int count, unsigned long long* out)
{
    cudaMemcpyAsync(ctx->h_words + first, ctx->d_words + first, sizeof(unsigned long long) * count,
                    cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("read_words"); }
    std::memcpy(out, ctx->h_words + first, sizeof(unsigned long long) * count);
    return GB_OK;
}

namespace {
cudaEvent_t take_event(gb_ctx* ctx)
{
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

void span_begin(gb_ctx* ctx, int family)
{
    if (!ctx->profiling) { return; }
    if (((ctx->profile_mask >> family) & 1u) == 0) {
        ctx->open_spans.push_back(-1);
        return;
    }
    gb_ctx::Span s{family, take_event(ctx), take_event(ctx)};
    cudaEventRecord(s.start, ctx->stream);
    ctx->open_spans.push_back(static_cast<int>(ctx->spans.size()));
    ctx->spans.push_back(s);
}

void span_end(gb_ctx* ctx)
{
    if (!ctx->profiling || ctx->open_spans.empty()) { return; }
    const int n = ctx->open_spans.back();
    ctx->open_spans.pop_back();
    if (n >= 0) { cudaEventRecord(ctx->spans[n].stop, ctx->stream); }
}

gb_status check_grid(const char* op, const gb_grid* g)
{
    if (g == nullptr) {
        set_error("gust: %s: grid is null", op);
        return GB_BAD_ARG;
    }
    if (g->nx < 1 || g->ny < 1 || g->nz < 2 || g->ng < 2) {
        set_error("gust: %s: grid needs nx, ny >= 1, nz >= 2 and ng >= 2 (got %d x %d x %d, ng %d)", op, g->nx, g->ny,
                  g->nz, g->ng);
        return GB_BAD_ARG;
    }
    if (g->sy < g->nx + 1 + 2 * g->ng || g->sz < g->sy * (g->ny + 1 + 2 * g->ng)) {
        set_error("gust: %s: grid strides too small for its extents", op);
        return GB_BAD_ARG;
    }
    if (!(g->dx > 0) || !(g->dy > 0) || !(g->dzeta > 0)) {
        set_error("gust: %s: grid cell sizes must be > 0", op);
        return GB_BAD_ARG;
    }
    if (volume(*g) > INT32_MAX) {
        set_error("gust: %s: grid of %lld padded points (at most 2^31 - 1: 32-bit point offsets)", op,
                  static_cast<long long>(volume(*g)));
        return GB_BAD_ARG;
    }
    return GB_OK;
}

gb_status check_loc(const char* op, int loc)
{
    if (loc == GB_LOC_CELL || loc == GB_LOC_XFACE || loc == GB_LOC_YFACE || loc == GB_LOC_ZFACE) { return GB_OK; }
    set_error("gust: %s: loc must be cell (0), xface (1), yface (2) or zface (4) (got %d)", op, loc);
    return GB_BAD_ARG;
}

}  // namespace gb

namespace gb {

//! The FP64 pipe's rate: 8 independent chains of dependent fused
//! multiply-adds per thread (a = a * b + c with b just below 1, so the
//! values stay finite), the chains' sum written out.
__global__ void __launch_bounds__(256) k_probe_fp64(int iters, double* __restrict__ sink)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { a[q] = 1.0 + 1e-3 * (t + q); }
    const double b = 0.999999, c = 1e-7;
    for (int n = 0; n < iters; ++n) {
#pragma unroll
        for (int q = 0; q < 8; ++q) { a[q] = fma(a[q], b, c); }
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) { s += a[q]; }
    sink[t] = s;
}

}  // namespace gb

extern "C" {

gb_status gb_grid_init(gb_grid* g, int32_t nx, int32_t ny, int32_t nz, int32_t ng, double dx, double dy,
                       double dzeta, int32_t periodic_x, int32_t periodic_y)
{
    gb::clear_error();
    if (g == nullptr) {
        gb::set_error("gust: gb_grid_init: grid is null");
        return GB_BAD_ARG;
    }
    g->nx = nx;
    g->ny = ny;
    g->nz = nz;
    g->ng = ng;
    g->periodic_x = periodic_x ? 1 : 0;
    g->periodic_y = periodic_y ? 1 : 0;
    g->sy = static_cast<int64_t>(nx) + 1 + 2 * ng;
    g->sz = g->sy * (static_cast<int64_t>(ny) + 1 + 2 * ng);
    g->dx = dx;
    g->dy = dy;
    g->dzeta = dzeta;
    return gb::check_grid("gb_grid_init", g);
}

int64_t gb_grid_volume(const gb_grid* g) { return g == nullptr ? 0 : gb::volume(*g); }

gb_status gb_ctx_create(void* stream, gb_ctx** out)
{
    gb::clear_error();
    if (out == nullptr) {
        gb::set_error("gust: gb_ctx_create: out is null");
        return GB_BAD_ARG;
    }
    *out = nullptr;
    auto* ctx = new gb_ctx;
    ctx->stream = static_cast<cudaStream_t>(stream);
    if (cudaGetDevice(&ctx->device) != cudaSuccess) {
        delete ctx;
        return gb::check_cuda("gb_ctx_create");
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (cudaMalloc(&ctx->d_words, sizeof(unsigned long long) * gb_ctx::n_words) != cudaSuccess
        || cudaMallocHost(&ctx->h_words, sizeof(unsigned long long) * gb_ctx::n_words) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->d_words) { cudaFree(ctx->d_words); }
        delete ctx;
        gb::set_error("gust: gb_ctx_create: cannot allocate the result words");
        return GB_OOM;
    }
    *out = ctx;
    return GB_OK;
}

gb_status gb_ctx_destroy(gb_ctx* ctx)
{
    gb::clear_error();
    if (ctx == nullptr) { return GB_OK; }
    cudaStreamSynchronize(ctx->stream);
    for (void* p : ctx->slot_ptr) {
        if (p) { cudaFree(p); }
    }
    cudaFree(ctx->d_words);
    cudaFreeHost(ctx->h_words);
    delete ctx;
    return gb::check_cuda("gb_ctx_destroy");
}

int64_t gb_ctx_launches(const gb_ctx* ctx) { return ctx == nullptr ? 0 : ctx->launches; }

gb_status gb_ctx_tune(gb_ctx* ctx, int32_t key, int32_t value)
{
    gb::clear_error();
    if (ctx == nullptr || key < 0 || key >= GB_N_TUNE) {
        gb::set_error("gust: gb_ctx_tune: unknown context or key %d", key);
        return GB_BAD_ARG;
    }
    ctx->tune[key] = value;
    return GB_OK;
}

gb_status gb_ctx_profile(gb_ctx* ctx, int32_t enable)
{
    gb::clear_error();
    if (ctx == nullptr) {
        gb::set_error("gust: gb_ctx_profile: ctx is null");
        return GB_BAD_ARG;
    }
    cudaStreamSynchronize(ctx->stream);
    for (auto& s : ctx->spans) {
        ctx->event_pool.push_back(s.start);
        ctx->event_pool.push_back(s.stop);
    }
    ctx->spans.clear();
    ctx->open_spans.clear();
    ctx->profiling = enable != 0;
    return gb::check_cuda("gb_ctx_profile");
}

gb_status gb_ctx_profile_mask(gb_ctx* ctx, uint32_t mask)
{
    gb::clear_error();
    if (ctx == nullptr) {
        gb::set_error("gust: gb_ctx_profile_mask: ctx is null");
        return GB_BAD_ARG;
    }
    ctx->profile_mask = mask;
    return GB_OK;
}

gb_status gb_ctx_profile_read(gb_ctx* ctx, int32_t family, double* total_ms, int64_t* spans)
{
    gb::clear_error();
    if (ctx == nullptr || total_ms == nullptr || spans == nullptr) {
        gb::set_error("gust: gb_ctx_profile_read: null argument");
        return GB_BAD_ARG;
    }
    cudaStreamSynchronize(ctx->stream);
    double t = 0;
    int64_t n = 0;
    for (const auto& s : ctx->spans) {
        if (s.family != family) { continue; }
        float ms = 0;
        if (cudaEventElapsedTime(&ms, s.start, s.stop) == cudaSuccess) {
            t += ms;
            ++n;
        }
    }
    cudaGetLastError();
    *total_ms = t;
    *spans = n;
    return GB_OK;
}

gb_status gb_probe_fp64(gb_ctx* ctx, int32_t iters, double* sink, int64_t* threads)
{
    gb::clear_error();
    if (ctx == nullptr || sink == nullptr || threads == nullptr || iters < 1) {
        gb::set_error("gust: gb_probe_fp64: null argument or iters < 1");
        return GB_BAD_ARG;
    }
    const int blocks = 4 * ctx->num_sms;
    gb::k_probe_fp64<<<blocks, 256, 0, ctx->stream>>>(iters, sink);
    *threads = static_cast<int64_t>(blocks) * 256;
    return gb::check_cuda("gb_probe_fp64");
}

const char* gb_last_error(void) { return gb::g_error.c_str(); }

}  // extern "C"
