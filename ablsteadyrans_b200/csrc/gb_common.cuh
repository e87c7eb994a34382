// Shared device and host helpers of the B200 SIMPLEC hot path: the grid
// layout (one index space for every location type), the context with its
// stream and scratch, error reporting and the warp reductions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gust_b200.h"

namespace gb {

// ---------------------------------------------------------------- layout ---

//! Element offset of point (i, j, k) of any location type. The arithmetic is
//! 32-bit (an accepted grid has fewer than 2^31 points, check_grid), widened
//! once: the offsets of a stencil's points from one (i, j, k) then differ by
//! constants the compiler folds, where 64-bit products of each point's
//! indices cost several instructions per load.
__host__ __device__ __forceinline__ int64_t at(const gb_grid& g, int i, int j, int k)
{
    return static_cast<int64_t>((i + g.ng) + (j + g.ng) * static_cast<int32_t>(g.sy)
                                + (k + g.ng) * static_cast<int32_t>(g.sz));
}

__host__ __device__ __forceinline__ int64_t volume(const gb_grid& g)
{
    return g.sz * static_cast<int64_t>(g.nz + 1 + 2 * g.ng);
}

//! Valid extents of a location: cells, plus one point in each nodal direction.
__host__ __device__ __forceinline__ int ext_x(const gb_grid& g, int loc) { return g.nx + (loc & 1); }
__host__ __device__ __forceinline__ int ext_y(const gb_grid& g, int loc) { return g.ny + ((loc >> 1) & 1); }
__host__ __device__ __forceinline__ int ext_z(const gb_grid& g, int loc) { return g.nz + ((loc >> 2) & 1); }

//! The periodic image of a lateral index outside the valid range [0, n_valid),
//! or -1 (outside a non-periodic face: the caller reads zero). n is the number
//! of cells, the period.
__host__ __device__ __forceinline__ int lateral_image(int i, int n_valid, int n, bool periodic)
{
    if (i >= 0 && i < n_valid) { return i; }
    if (!periodic) { return -1; }
    return (i < 0) ? i + n : i - n;
}

// ---------------------------------------------------------- reductions ---

__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) { v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o)); }
    return v;
}
//! Warp max that keeps a NaN (fmax drops it): a diverged field reports NaN.
__device__ __forceinline__ double warp_max_nan(double v)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = (w > v || w != w) ? w : v;
    }
    return v;
}
__device__ __forceinline__ float warp_max(float v)
{
    for (int o = 16; o > 0; o >>= 1) { v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o)); }
    return v;
}
__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) { v += __shfl_xor_sync(0xffffffffu, v, o); }
    return v;
}

//! atomic max of a non-negative value (NaN propagates: its bits order above
//! every finite value and inf). Slot holds the value's bit pattern.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double v)
{
    if (v != v) { atomicMax(slot, 0x7ff8000000000000ull); return; }
    atomicMax(slot, static_cast<unsigned long long>(__double_as_longlong(v)));
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, float v)
{
    atomic_max_nonneg(slot, static_cast<double>(v));
}

// ------------------------------------------------------ asynchronous copy ---

//! Asynchronous global -> shared copy of one element (cp.async, LDGSTS):
//! the copy completes in the background; cp_async_wait<N>() waits until at
//! most N of this thread's committed groups are still in flight.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* gmem_src)
{
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    if constexpr (sizeof(T) == 8) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

//! 1 / v rounded to nearest, the value IEEE division 1 / v gives, by the
//! reciprocal intrinsic (which skips the general quotient's numerator
//! handling).
__device__ __forceinline__ double recip_rn(double v) { return __drcp_rn(v); }
__device__ __forceinline__ float recip_rn(float v) { return __frcp_rn(v); }

// ------------------------------------------- programmatic dependent launch ---
//
// A kernel launched by launch_pdl may begin while the kernel before it on the
// stream is finishing (its launch and block scheduling overlap the previous
// kernel's tail). Such a kernel calls pdl_entry() first: griddepcontrol.wait
// blocks until the previous grid has completed and its memory operations
// are visible (it returns at once for a launch without that dependency),
// then griddepcontrol.launch_dependents lets the next programmatic launch
// be scheduled. Every access of global memory follows the wait, so a
// kernel neither reads before its producer's writes land nor writes what
// its predecessor may still read. Launches between other stream operations
// (a memset, an event) are serialised as usual.

__device__ __forceinline__ void pdl_entry()
{
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

//! A launch with programmatic stream serialisation (the kernel must call
//! pdl_entry() before touching global memory); a plain launch when pdl is false.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args&&... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ------------------------------------------ bulk copies (TMA) and mbarriers ---
//
// A bulk copy (cp.async.bulk, executed by the TMA unit) moves a contiguous
// run of bytes from global to shared memory and reports its bytes to an
// mbarrier of the block; the block waits on the barrier's phase. Both
// addresses must be 16-byte aligned and the size a multiple of 16.

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

//! Makes the barriers' initialisation visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

//! Orders this thread's earlier generic accesses of shared memory before
//! later bulk copies into it (a slot's readers, then its next fill).
__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

//! The one arrival of a phase, announcing the bytes its copies will bring.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

//! Waits for the barrier's phase of the given parity for at most `limit`
//! polls (each poll may suspend the thread briefly); false: gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit)
{
    for (int n = 0; n < limit; ++n) {
        if (mbar_try_wait(bar, parity)) { return true; }
    }
    return false;
}

//! Bulk copy of `bytes` from global src to shared dst, completing on bar.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// ---------------------------------------------------------------- errors ---

void set_error(const char* fmt, ...);
void clear_error();

//! Record a CUDA error (if any) of the last launch or call; returns the status.
gb_status check_cuda(const char* op);

}  // namespace gb

// ------------------------------------------------------------- context ---

struct gb_ctx {
    cudaStream_t stream{nullptr};
    int device{0};
    int num_sms{148};
    int64_t launches{0};
    //! Scratch slots, grown on demand (device memory).
    std::vector<void*> slot_ptr;
    std::vector<size_t> slot_bytes;
    //! Device and pinned-host result words (reductions read back).
    unsigned long long* d_words{nullptr};
    unsigned long long* h_words{nullptr};
    static constexpr int n_words = 64;
    //! Per-kernel-family timing (CUDA events on the stream around each launch),
    //! on while profiling is enabled.
    bool profiling{false};
    struct Span { int family; cudaEvent_t start, stop; };
    std::vector<Span> spans;
    std::vector<int> open_spans;        // per open Span: its index in spans, or -1 (family not timed)
    uint32_t profile_mask{0xffffffffu};  // families timed while profiling (bit = GB_KERNEL_*)
    std::vector<cudaEvent_t> event_pool;
    //! Tuning knobs (GB_TUNE_*), 0 = default.
    int tune[GB_N_TUNE] = {};
};

namespace gb {

//! Scratch slot `slot` of at least `bytes` (contents undefined); nullptr and
//! GB_OOM recorded on failure.
void* scratch(gb_ctx* ctx, int slot, size_t bytes);

//! Open / close a timed span of a kernel family (no-ops unless profiling).
void span_begin(gb_ctx* ctx, int family);
void span_end(gb_ctx* ctx);

//! RAII span around the launches of one kernel family.
struct Span {
    gb_ctx* ctx;
    Span(gb_ctx* c, int family) : ctx(c) { span_begin(c, family); }
    ~Span() { span_end(ctx); }
};

//! Device pointer of result word n of the context.
inline unsigned long long* dword(gb_ctx* ctx, int n) { return ctx->d_words + n; }

//! Copy `count` result words to the host (synchronises the stream).
gb_status read_words(gb_ctx* ctx, int first, int count, unsigned long long* out);

gb_status check_grid(const char* op, const gb_grid* g);
gb_status check_loc(const char* op, int loc);

inline double bits_to_double(unsigned long long b)
{
    double d;
    static_assert(sizeof(d) == sizeof(b), "");
    __builtin_memcpy(&d, &b, sizeof(d));
    return d;
}

}  // namespace gb
