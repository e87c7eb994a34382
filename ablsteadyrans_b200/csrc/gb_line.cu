// z-line relaxation: the exact tridiagonal solve of every (i, j) column with
// the x/y neighbour terms of the lagged iterate on the right-hand side
// (gust::solve_column, Source/LineSolve_K.H:22-45), swept `sweeps` times as a
// z-line Jacobi iteration (gust::zline_jacobi, Source/Predictor.cpp:87-127).
//
// B200 mapping: one thread per column, a warp over 32 consecutive i of one j,
// so every k step of the Thomas recurrences reads and writes coalesced rows of
// each k-plane. The recurrence scratch c', e' lives in shared memory (one
// column per thread, [k][thread] so a warp's accesses are consecutive) when
// the column fits, else in a global scratch array that stays in L2 for the
// tile sizes here. The max |change| of the last sweep is a warp-shuffle max
// and one atomic per warp. Iterates ping-pong between the caller's delta and
// one scratch array so the last sweep lands in delta.
#include "gb_line.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

namespace gb {

namespace {

template <typename T>
struct LineArgs {
    gb_grid g;
    int ni, nj, nk;
    const T* __restrict__ A;
    int64_t cs;  // component stride of A
    const T* __restrict__ ap;
    const T* __restrict__ rhs;
    const T* __restrict__ dold;  // lagged iterate (ghosts unread: images by index)
    T* __restrict__ dnew;
    T* __restrict__ cbuf;  // global scratch (SMEM == false)
    T* __restrict__ ebuf;
    int first;  // dold == 0: no neighbour terms, change against 0
    unsigned long long* change;  // max |dnew - dold| (nullptr: not wanted)
    const T* __restrict__ rfold;  // rhs with the lagged lateral terms folded in (the split sweep)
};

template <typename T, bool SMEM>
__global__ void __launch_bounds__(128) zline_sweep_kernel(LineArgs<T> a)
{
    extern __shared__ unsigned char smem_raw[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const bool active = (i < a.ni) && (j < a.nj);
    T chg = T(0);
    if (active) {
        const gb_grid& g = a.g;
        const int im = lateral_image(i - 1, a.ni, g.nx, g.periodic_x != 0);
        const int ip = lateral_image(i + 1, a.ni, g.nx, g.periodic_x != 0);
        const int jm = lateral_image(j - 1, a.nj, g.ny, g.periodic_y != 0);
        const int jp = lateral_image(j + 1, a.nj, g.ny, g.periodic_y != 0);
        const int64_t o0 = at(g, i, j, 0);
        const int64_t oxm = (im >= 0) ? at(g, im, j, 0) : -1;
        const int64_t oxp = (ip >= 0) ? at(g, ip, j, 0) : -1;
        const int64_t oym = (jm >= 0) ? at(g, i, jm, 0) : -1;
        const int64_t oyp = (jp >= 0) ? at(g, i, jp, 0) : -1;
        const T* __restrict__ axm = a.A + GB_COEF_XM * a.cs;
        const T* __restrict__ axp = a.A + GB_COEF_XP * a.cs;
        const T* __restrict__ aym = a.A + GB_COEF_YM * a.cs;
        const T* __restrict__ ayp = a.A + GB_COEF_YP * a.cs;
        const T* __restrict__ azm = a.A + GB_COEF_ZM * a.cs;
        const T* __restrict__ azp = a.A + GB_COEF_ZP * a.cs;
        const int nthr = blockDim.x * blockDim.y;
        const int tid = threadIdx.y * blockDim.x + threadIdx.x;
        T* cs = SMEM ? reinterpret_cast<T*>(smem_raw) + tid : a.cbuf + o0;
        T* es = SMEM ? reinterpret_cast<T*>(smem_raw) + static_cast<int64_t>(a.nk) * nthr + tid : a.ebuf + o0;
        const int64_t sstep = SMEM ? nthr : g.sz;
        T cprev = T(0), eprev = T(0);
        int64_t ko = 0, ks = 0;
#pragma unroll 4
        for (int k = 0; k < a.nk; ++k, ko += g.sz, ks += sstep) {
            const int64_t o = o0 + ko;
            T rk = a.rhs[o];
            if (!a.first) {
                const T dxm = (oxm >= 0) ? a.dold[oxm + ko] : T(0);
                const T dxp = (oxp >= 0) ? a.dold[oxp + ko] : T(0);
                const T dym = (oym >= 0) ? a.dold[oym + ko] : T(0);
                const T dyp = (oyp >= 0) ? a.dold[oyp + ko] : T(0);
                rk = rk + axm[o] * dxm + axp[o] * dxp + aym[o] * dym + ayp[o] * dyp;
            }
            const T lower = -azm[o], upper = -azp[o];
            const T m = (k == 0) ? a.ap[o] : a.ap[o] - lower * cprev;
            cprev = upper / m;
            eprev = ((k == 0) ? rk : rk - lower * eprev) / m;
            cs[ks] = cprev;
            es[ks] = eprev;
        }
        // Back substitution from the top of the column.
        T x = eprev;
        ks -= sstep;
        ko -= g.sz;
        a.dnew[o0 + ko] = x;
        if (a.change) { chg = fabs(x - (a.first ? T(0) : a.dold[o0 + ko])); }
        for (int k = a.nk - 2; k >= 0; --k) {
            ks -= sstep;
            ko -= g.sz;
            x = es[ks] - cs[ks] * x;
            a.dnew[o0 + ko] = x;
            if (a.change) {
                const T d = fabs(x - (a.first ? T(0) : a.dold[o0 + ko]));
                chg = (d > chg || d != d) ? d : chg;
            }
        }
    }
    if (a.change != nullptr) {
        chg = warp_max(chg);
        if ((threadIdx.x & 31) == 0) { atomic_max_nonneg(a.change, chg); }
    }
}

//! The pipelined sweep: the same column solve, with the inputs of the next
//! R-1 k-levels in flight. Each thread stages its own column's values of level
//! k + R - 1 into a shared-memory ring with asynchronous copies (cp.async),
//! then waits only for level k, so the memory latency of one level overlaps
//! the recurrence of R-1 others. A column is a thread's private data: no
//! block barrier is needed. c', e' stay in shared memory ([k][thread]).
template <typename T, bool FIRST, int R>
__global__ void __launch_bounds__(128) zline_pipe_kernel(LineArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NV = FIRST ? 4 : 12;
    const int nthr = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const bool active = (i < a.ni) && (j < a.nj);
    const gb_grid& g = a.g;
    T* ring = reinterpret_cast<T*>(smem_raw);
    T* cs = ring + R * NV * nthr;
    T* es = cs + static_cast<int64_t>(a.nk) * nthr;
    int64_t o0 = 0, oxm = -1, oxp = -1, oym = -1, oyp = -1;
    if (active) {
        const int im = lateral_image(i - 1, a.ni, g.nx, g.periodic_x != 0);
        const int ip = lateral_image(i + 1, a.ni, g.nx, g.periodic_x != 0);
        const int jm = lateral_image(j - 1, a.nj, g.ny, g.periodic_y != 0);
        const int jp = lateral_image(j + 1, a.nj, g.ny, g.periodic_y != 0);
        o0 = at(g, i, j, 0);
        oxm = (im >= 0) ? at(g, im, j, 0) : -1;
        oxp = (ip >= 0) ? at(g, ip, j, 0) : -1;
        oym = (jm >= 0) ? at(g, i, jm, 0) : -1;
        oyp = (jp >= 0) ? at(g, i, jp, 0) : -1;
    }
    const T* __restrict__ azm = a.A + GB_COEF_ZM * a.cs + o0;
    const T* __restrict__ azp = a.A + GB_COEF_ZP * a.cs + o0;
    const T* __restrict__ axm = a.A + GB_COEF_XM * a.cs + o0;
    const T* __restrict__ axp = a.A + GB_COEF_XP * a.cs + o0;
    const T* __restrict__ aym = a.A + GB_COEF_YM * a.cs + o0;
    const T* __restrict__ ayp = a.A + GB_COEF_YP * a.cs + o0;
    auto issue = [&](int k) {
        if (active && k < a.nk) {
            const int64_t ko = static_cast<int64_t>(k) * g.sz;
            T* s = ring + (k % R) * NV * nthr + tid;
            cp_async_elem(s, a.rhs + o0 + ko);
            cp_async_elem(s + nthr, a.ap + o0 + ko);
            cp_async_elem(s + 2 * nthr, azm + ko);
            cp_async_elem(s + 3 * nthr, azp + ko);
            if (!FIRST) {
                cp_async_elem(s + 4 * nthr, axm + ko);
                cp_async_elem(s + 5 * nthr, axp + ko);
                cp_async_elem(s + 6 * nthr, aym + ko);
                cp_async_elem(s + 7 * nthr, ayp + ko);
                if (oxm >= 0) { cp_async_elem(s + 8 * nthr, a.dold + oxm + ko); } else { s[8 * nthr] = T(0); }
                if (oxp >= 0) { cp_async_elem(s + 9 * nthr, a.dold + oxp + ko); } else { s[9 * nthr] = T(0); }
                if (oym >= 0) { cp_async_elem(s + 10 * nthr, a.dold + oym + ko); } else { s[10 * nthr] = T(0); }
                if (oyp >= 0) { cp_async_elem(s + 11 * nthr, a.dold + oyp + ko); } else { s[11 * nthr] = T(0); }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int k = 0; k < R - 1; ++k) { issue(k); }
    T cprev = T(0), eprev = T(0);
    for (int k = 0; k < a.nk; ++k) {
        issue(k + R - 1);
        cp_async_wait<R - 1>();
        if (active) {
            const T* s = ring + (k % R) * NV * nthr + tid;
            T rk = s[0];
            if (!FIRST) {
                rk = rk + s[4 * nthr] * s[8 * nthr] + s[5 * nthr] * s[9 * nthr] + s[6 * nthr] * s[10 * nthr]
                   + s[7 * nthr] * s[11 * nthr];
            }
            const T lower = -s[2 * nthr], upper = -s[3 * nthr];
            const T m = (k == 0) ? s[nthr] : s[nthr] - lower * cprev;
            cprev = upper / m;
            eprev = ((k == 0) ? rk : rk - lower * eprev) / m;
            cs[k * nthr + tid] = cprev;
            es[k * nthr + tid] = eprev;
        }
    }
    cp_async_wait<0>();
    T chg = T(0);
    if (active) {
        T x = eprev;
        int64_t ko = static_cast<int64_t>(a.nk - 1) * g.sz;
        a.dnew[o0 + ko] = x;
        if (a.change) { chg = fabs(x - (FIRST ? T(0) : a.dold[o0 + ko])); }
#pragma unroll 4
        for (int k = a.nk - 2; k >= 0; --k) {
            ko -= g.sz;
            x = es[k * nthr + tid] - cs[k * nthr + tid] * x;
            a.dnew[o0 + ko] = x;
            if (a.change) {
                const T d = fabs(x - (FIRST ? T(0) : a.dold[o0 + ko]));
                chg = (d > chg || d != d) ? d : chg;
            }
        }
    }
    if (a.change != nullptr) {
        chg = warp_max(chg);
        if ((threadIdx.x & 31) == 0) { atomic_max_nonneg(a.change, chg); }
    }
}

//! The pipelined sweep with the column factorisation kept between sweeps.
//! The system (a_P, a_ZM, a_ZP) is the same in every sweep of a solve, so the
//! first sweep stores the reciprocal pivots 1/m_k and the eliminated uppers
//! c'_k = -a_ZP,k / m_k (m_0 = a_P,0, m_k = a_P,k + a_ZM,k c'_{k-1}) in
//! scratch, and every later sweep runs the forward recurrence
//! e_k = (r_k + a_ZM,k e_{k-1}) / m_k as a multiply by the stored 1/m_k:
//! no division on the k chain. Inputs are staged R levels ahead with cp.async
//! as in zline_pipe_kernel.
//! BACK, where the back substitution finds c' and e': 0 both in shared
//! memory; 1 both in global memory (c' in its stored array, e' in the output
//! array, which the back substitution overwrites level by level), so shared
//! memory holds the ring alone; 2 e' in shared memory and c' read again from
//! its stored array (this sweep's reads or writes of it, still in L2), which
//! halves the column's shared memory without e''s extra traffic. Less shared
//! memory per column puts more warps on an SM.
template <typename T, bool FIRST, int R, int BACK = 0>
__device__ __forceinline__ void zline_fact_body(const LineArgs<T>& a, T* __restrict__ im_out,
                                                const T* __restrict__ im_in, T* __restrict__ cp_out,
                                                const T* __restrict__ cp_in)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NV = FIRST ? 4 : 12;
    const int nthr = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const bool active = (i < a.ni) && (j < a.nj);
    const gb_grid& g = a.g;
    T* ring = reinterpret_cast<T*>(smem_raw);
    T* cs = ring + R * NV * nthr;
    T* es = (BACK == 2) ? cs : cs + static_cast<int64_t>(a.nk) * nthr;
    int64_t o0 = 0, oxm = -1, oxp = -1, oym = -1, oyp = -1;
    if (active) {
        const int im = lateral_image(i - 1, a.ni, g.nx, g.periodic_x != 0);
        const int ip = lateral_image(i + 1, a.ni, g.nx, g.periodic_x != 0);
        const int jm = lateral_image(j - 1, a.nj, g.ny, g.periodic_y != 0);
        const int jp = lateral_image(j + 1, a.nj, g.ny, g.periodic_y != 0);
        o0 = at(g, i, j, 0);
        oxm = (im >= 0) ? at(g, im, j, 0) : -1;
        oxp = (ip >= 0) ? at(g, ip, j, 0) : -1;
        oym = (jm >= 0) ? at(g, i, jm, 0) : -1;
        oyp = (jp >= 0) ? at(g, i, jp, 0) : -1;
    }
    const T* __restrict__ azm = a.A + GB_COEF_ZM * a.cs + o0;
    const T* __restrict__ azp = a.A + GB_COEF_ZP * a.cs + o0;
    const T* __restrict__ axm = a.A + GB_COEF_XM * a.cs + o0;
    const T* __restrict__ axp = a.A + GB_COEF_XP * a.cs + o0;
    const T* __restrict__ aym = a.A + GB_COEF_YM * a.cs + o0;
    const T* __restrict__ ayp = a.A + GB_COEF_YP * a.cs + o0;
    // slots: 0 rhs, 1 a_P (first) or 1/m, 2 a_ZM, 3 a_ZP (first) or c', 4-7 lateral
    // coefficients, 8-11 the lagged neighbours
    auto issue = [&](int k) {
        if (active && k < a.nk) {
            const int64_t ko = static_cast<int64_t>(k) * g.sz;
            T* s = ring + (k % R) * NV * nthr + tid;
            cp_async_elem(s, a.rhs + o0 + ko);
            cp_async_elem(s + nthr, FIRST ? a.ap + o0 + ko : im_in + o0 + ko);
            cp_async_elem(s + 2 * nthr, azm + ko);
            cp_async_elem(s + 3 * nthr, FIRST ? azp + ko : cp_in + o0 + ko);
            if (!FIRST) {
                cp_async_elem(s + 4 * nthr, axm + ko);
                cp_async_elem(s + 5 * nthr, axp + ko);
                cp_async_elem(s + 6 * nthr, aym + ko);
                cp_async_elem(s + 7 * nthr, ayp + ko);
                if (oxm >= 0) { cp_async_elem(s + 8 * nthr, a.dold + oxm + ko); } else { s[8 * nthr] = T(0); }
                if (oxp >= 0) { cp_async_elem(s + 9 * nthr, a.dold + oxp + ko); } else { s[9 * nthr] = T(0); }
                if (oym >= 0) { cp_async_elem(s + 10 * nthr, a.dold + oym + ko); } else { s[10 * nthr] = T(0); }
                if (oyp >= 0) { cp_async_elem(s + 11 * nthr, a.dold + oyp + ko); } else { s[11 * nthr] = T(0); }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int k = 0; k < R - 1; ++k) { issue(k); }
    T cprev = T(0), eprev = T(0);
    for (int k = 0; k < a.nk; ++k) {
        issue(k + R - 1);
        cp_async_wait<R - 1>();
        if (active) {
            const T* s = ring + (k % R) * NV * nthr + tid;
            T rk = s[0];
            const T lower = -s[2 * nthr];
            T inv, c;
            if (FIRST) {
                const T m = (k == 0) ? s[nthr] : s[nthr] - lower * cprev;
                inv = recip_rn(m);
                c = -s[3 * nthr] * inv;
                const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
                im_out[o] = inv;
                cp_out[o] = c;
            } else {
                inv = s[nthr];
                c = s[3 * nthr];
                rk = rk + s[4 * nthr] * s[8 * nthr] + s[5 * nthr] * s[9 * nthr] + s[6 * nthr] * s[10 * nthr]
                   + s[7 * nthr] * s[11 * nthr];
            }
            cprev = c;
            eprev = ((k == 0) ? rk : rk - lower * eprev) * inv;
            if (BACK == 1) {
                a.dnew[o0 + static_cast<int64_t>(k) * g.sz] = eprev;
            } else {
                if (BACK == 0) { cs[k * nthr + tid] = c; }
                es[k * nthr + tid] = eprev;
            }
        }
    }
    cp_async_wait<0>();
    T chg = T(0);
    if (BACK == 1 && active) {
        // x_k = e'_k - c'_k x_{k+1} in place over e' (this thread's own writes)
        const T* cpk = FIRST ? cp_out : cp_in;
        T x = eprev;
        int64_t ko = static_cast<int64_t>(a.nk - 1) * g.sz;
        if (a.change) { chg = fabs(x - (FIRST ? T(0) : a.dold[o0 + ko])); }
#pragma unroll 8
        for (int k = a.nk - 2; k >= 0; --k) {
            ko -= g.sz;
            x = a.dnew[o0 + ko] - cpk[o0 + ko] * x;
            a.dnew[o0 + ko] = x;
            if (a.change) {
                const T d = fabs(x - (FIRST ? T(0) : a.dold[o0 + ko]));
                chg = (d > chg || d != d) ? d : chg;
            }
        }
    }
    if (BACK != 1 && active) {
        const T* cpk = FIRST ? cp_out : cp_in;
        T x = eprev;
        int64_t ko = static_cast<int64_t>(a.nk - 1) * g.sz;
        a.dnew[o0 + ko] = x;
        if (a.change) { chg = fabs(x - (FIRST ? T(0) : a.dold[o0 + ko])); }
#pragma unroll 4
        for (int k = a.nk - 2; k >= 0; --k) {
            ko -= g.sz;
            const T ck = (BACK == 2) ? cpk[o0 + ko] : cs[k * nthr + tid];
            x = es[k * nthr + tid] - ck * x;
            a.dnew[o0 + ko] = x;
            if (a.change) {
                const T d = fabs(x - (FIRST ? T(0) : a.dold[o0 + ko]));
                chg = (d > chg || d != d) ? d : chg;
            }
        }
    }
    if (a.change != nullptr) {
        chg = warp_max(chg);
        if ((threadIdx.x & 31) == 0) { atomic_max_nonneg(a.change, chg); }
    }
}

template <typename T, bool FIRST, int R>
__global__ void __launch_bounds__(128) zline_fact_kernel(LineArgs<T> a, T* __restrict__ im_out,
                                                         const T* __restrict__ im_in, T* __restrict__ cp_out,
                                                         const T* __restrict__ cp_in)
{
    zline_fact_body<T, FIRST, R>(a, im_out, im_in, cp_out, cp_in);
}

//! Several independent systems (up to kMaxLineSystems, each at its own
//! location) swept by one launch: blockIdx.z picks the system, the grid
//! covers the largest one and a block past a system's extents idles. More
//! columns in flight per launch than one system gives.
constexpr int kMaxLineSystems = 3;

template <typename T>
struct MultiLineArgs {
    LineArgs<T> a[kMaxLineSystems];
    T* inv[kMaxLineSystems];
    T* cp[kMaxLineSystems];
    T* fold[kMaxLineSystems];  // the split sweep's folded right-hand sides
};

template <typename T, bool FIRST, int R, int S, int BACK>
__device__ __forceinline__ void zline_fact_system(const MultiLineArgs<T>& m)
{
    if (FIRST) {
        zline_fact_body<T, true, R, BACK>(m.a[S], m.inv[S], nullptr, m.cp[S], nullptr);
    } else {
        zline_fact_body<T, false, R, BACK>(m.a[S], nullptr, m.inv[S], nullptr, m.cp[S]);
    }
}

template <typename T, bool FIRST, int R, int BACK>
__global__ void __launch_bounds__(128) zline_fact_multi_kernel(MultiLineArgs<T> m)
{
    // constant indices into the parameter block (no dynamic parameter indexing)
    switch (blockIdx.z) {
    case 0: zline_fact_system<T, FIRST, R, 0, BACK>(m); break;
    case 1: zline_fact_system<T, FIRST, R, 1, BACK>(m); break;
    default: zline_fact_system<T, FIRST, R, 2, BACK>(m); break;
    }
}

//! The segmented sweep: the column's levels split among the warps of a block.
//! A block holds 32 consecutive columns in (j, i) order and ceil(nk / L) warps;
//! warp w owns levels [w L, w L + L) of every column, loads all of them at
//! once into registers (every load of a thread is independent, so the memory
//! latency is paid once per segment, not once per level) and runs the Thomas
//! recurrences of gust::solve_column (Source/LineSolve_K.H:22-45) over its
//! own levels. What crosses a segment boundary is one value per recurrence
//! (c' on the first sweep, e' and x on every sweep): each warp composes its
//! segment into one map of that value (a 2x2 projective map for c', which
//! is a continued fraction; an affine map for e' and x), the maps go through
//! shared memory, and each warp applies the maps of the segments before it
//! to find its own starting value. Inside a segment the recurrences are the
//! sequential ones, in the sequential operation order; only the values
//! carried in across a boundary are evaluated through the composed maps, so
//! the results agree with the sequential solve to rounding.
//! FIRST: the first sweep of a solve (zero iterate, no lateral terms): it
//! also stores the column factors 1/m and c' for the later sweeps, which read
//! them in place of a_P and a_ZP (as zline_fact_body).
//! 2^-e for a finite positive normal s = m 2^e (m in [1, 2)), from the
//! exponent bits (1 for 0, a subnormal, inf or NaN): the scale that brings s
//! into [1, 2) by an exact multiplication.
__device__ __forceinline__ double pow2_inverse_scale(double s)
{
    const long long b = __double_as_longlong(s);
    const int eb = static_cast<int>((b >> 52) & 0x7ff);
    if (eb == 0 || eb == 0x7ff) { return 1.0; }
    return __longlong_as_double(static_cast<long long>(2046 - eb) << 52);
}

__device__ __forceinline__ float pow2_inverse_scale(float s)
{
    const int b = __float_as_int(s);
    const int eb = (b >> 23) & 0xff;
    if (eb == 0 || eb == 0xff) { return 1.0f; }
    return __int_as_float((254 - eb) << 23);
}

//! The four entries of a projective map scaled by one power of two (exact)
//! so that the largest magnitude lies in [1, 2): the map is unchanged and
//! the entries neither overflow nor underflow along a segment's product.
template <typename T>
__device__ __forceinline__ void seg_pow2_normalise(T& a, T& b, T& c, T& d)
{
    const T s = fmax(fmax(fabs(a), fabs(b)), fmax(fabs(c), fabs(d)));
    const T f = pow2_inverse_scale(s);
    a *= f;
    b *= f;
    c *= f;
    d *= f;
}

template <typename T, bool FIRST, int L, bool PREF = false>
__device__ __forceinline__ void zline_seg_body(const LineArgs<T>& a, T* __restrict__ inv_io, T* __restrict__ cp_io,
                                               int cblock)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const int w = threadIdx.y;
    const int W = blockDim.y;
    // 32 consecutive columns in (j, i) order: a block is never mostly past
    // the end of a row (a face system's rows are one column longer than 32 k)
    const int c = cblock * 32 + lane;
    const int i = c % a.ni;
    const int j = c / a.ni;
    const bool col = c < a.ni * a.nj;
    const int k0 = w * L;
    const int nk = a.nk;
    const gb_grid& g = a.g;
    T* carry_c = reinterpret_cast<T*>(smem_raw);      // [4][W][32]: the projective map of c'
    T* carry_e = carry_c + 4 * W * 32;                 // [2][W][32]: the affine map of e'
    T* carry_x = carry_e + 2 * W * 32;                 // [2][W][32]: the affine map of x
    const int cs = W * 32;
    const int me = w * 32 + lane;
    // Every lane reads an in-range column and level (a lane past the columns
    // reads the last one, a level past the column its top; their results are
    // discarded), so no load sits behind a branch and a segment's loads can
    // all be in flight together; a missing lateral neighbour reads the
    // column itself and its term is selected away.
    const int ic = min(i, a.ni - 1), jc = min(j, a.nj - 1);
    const int im = lateral_image(ic - 1, a.ni, g.nx, g.periodic_x != 0);
    const int ip = lateral_image(ic + 1, a.ni, g.nx, g.periodic_x != 0);
    const int jm = lateral_image(jc - 1, a.nj, g.ny, g.periodic_y != 0);
    const int jp = lateral_image(jc + 1, a.nj, g.ny, g.periodic_y != 0);
    const int64_t o0 = at(g, ic, jc, 0);
    const bool hxm = im >= 0, hxp = ip >= 0, hym = jm >= 0, hyp = jp >= 0;
    const int64_t oxm = hxm ? at(g, im, jc, 0) : o0;
    const int64_t oxp = hxp ? at(g, ip, jc, 0) : o0;
    const int64_t oym = hym ? at(g, ic, jm, 0) : o0;
    const int64_t oyp = hyp ? at(g, ic, jp, 0) : o0;
    const T* __restrict__ azm = a.A + GB_COEF_ZM * a.cs;
    const T* __restrict__ azp = a.A + GB_COEF_ZP * a.cs;
    const T* __restrict__ axm = a.A + GB_COEF_XM * a.cs;
    const T* __restrict__ axp = a.A + GB_COEF_XP * a.cs;
    const T* __restrict__ aym = a.A + GB_COEF_YM * a.cs;
    const T* __restrict__ ayp = a.A + GB_COEF_YP * a.cs;
    // r: the right-hand side with the lagged lateral terms; lo: a_ZM; dg: a_P
    // (FIRST) or 1/m; up: a_ZP (FIRST) or c'
    T r[L], lo[L], dg[L], up[L];
#pragma unroll
    for (int q = 0; q < L; ++q) {
        const int k = min(k0 + q, nk - 1);
        const int64_t ko = static_cast<int64_t>(k) * g.sz;
        const int64_t o = o0 + ko;
        r[q] = a.rhs[o];
        lo[q] = azm[o];
        if (FIRST) {
            dg[q] = a.ap[o];
            up[q] = azp[o];
        } else if (PREF) {
            r[q] = a.rfold[o];
            dg[q] = inv_io[o];
            up[q] = cp_io[o];
        } else {
            dg[q] = inv_io[o];
            up[q] = cp_io[o];
            const T vxm = a.dold[oxm + ko], vxp = a.dold[oxp + ko], vym = a.dold[oym + ko], vyp = a.dold[oyp + ko];
            const T dxm = hxm ? vxm : T(0);
            const T dxp = hxp ? vxp : T(0);
            const T dym = hym ? vym : T(0);
            const T dyp = hyp ? vyp : T(0);
            r[q] = r[q] + axm[o] * dxm + axp[o] * dxp + aym[o] * dym + ayp[o] * dyp;
        }
    }
    if (FIRST) {
        // c'_k = -a_ZP,k / (a_P,k + a_ZM,k c'_{k-1}): the segment's map of c' as
        // the product of [[0, -a_ZP], [a_ZM, a_P]] acting on (numerator, denominator)
        T p00 = T(1), p01 = T(0), p10 = T(0), p11 = T(1);
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nk) {
                const T l = (k == 0) ? T(0) : lo[q];
                const T n00 = -up[q] * p10, n01 = -up[q] * p11;
                const T n10 = l * p00 + dg[q] * p10, n11 = l * p01 + dg[q] * p11;
                p00 = n00;
                p01 = n01;
                p10 = n10;
                p11 = n11;
                if (sizeof(T) == 4) { seg_pow2_normalise(p00, p01, p10, p11); }
            }
        }
        // Scaling by a power of two is exact, so the map normalised once per
        // segment is the per-level normalised one times a power of two, and
        // c' (its ratio) is bit for bit the same; FP64's range holds L levels'
        // products of the coefficients, FP32's normalises every level.
        if (sizeof(T) == 8) { seg_pow2_normalise(p00, p01, p10, p11); }
        carry_c[me] = p00;
        carry_c[cs + me] = p01;
        carry_c[2 * cs + me] = p10;
        carry_c[3 * cs + me] = p11;
        __syncthreads();
        // c' at the level below this segment: the maps of the segments below applied to c' = 0
        T num = T(0), den = T(1);
        for (int s = 0; s < w; ++s) {
            const int m = s * 32 + lane;
            const T n2 = carry_c[m] * num + carry_c[cs + m] * den;
            const T d2 = carry_c[2 * cs + m] * num + carry_c[3 * cs + m] * den;
            num = n2;
            den = d2;
            // (an exact common power of two: every 4th segment in FP64, whose
            // range holds 4 normalised maps' growth; c' = num / den unchanged)
            if (sizeof(T) == 4 || (s & 3) == 3) {
                T z0 = T(0), z1 = T(0);
                seg_pow2_normalise(num, den, z0, z1);
            }
        }
        T cprev = (w == 0) ? T(0) : num / den;
        // the sequential factorisation over the segment (zline_fact_body's order)
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nk) {
                const T lower = -lo[q];
                const T m = (k == 0) ? dg[q] : dg[q] - lower * cprev;
                const T inv = recip_rn(m);
                const T c = -up[q] * inv;
                dg[q] = inv;
                up[q] = c;
                cprev = c;
                if (col) {
                    const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
                    inv_io[o] = inv;
                    cp_io[o] = c;
                }
            }
        }
    }
    // forward substitution e_k = (r_k + a_ZM,k e_{k-1}) / m_k: the segment's affine map
    {
        T al = T(0), be = T(1);
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nk) {
                if (k == 0) {
                    al = r[q] * dg[q];
                    be = T(0);
                } else {
                    al = (r[q] + lo[q] * al) * dg[q];
                    be = (lo[q] * be) * dg[q];
                }
            }
        }
        carry_e[me] = al;
        carry_e[cs + me] = be;
    }
    __syncthreads();
    {
        T eprev = T(0);
        for (int s = 0; s < w; ++s) {
            const int m = s * 32 + lane;
            eprev = carry_e[m] + carry_e[cs + m] * eprev;
        }
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nk) {
                const T lower = -lo[q];
                eprev = ((k == 0) ? r[q] : r[q] - lower * eprev) * dg[q];
                r[q] = eprev;  // e' in place of r
            }
        }
    }
    // back substitution x_k = e'_k - c'_k x_{k+1} (x_{nk-1} = e'_{nk-1}): the
    // segment's affine map of x from the level above it
    {
        T ga = T(0), de = T(1);
#pragma unroll
        for (int q = L - 1; q >= 0; --q) {
            const int k = k0 + q;
            if (k < nk) {
                if (k == nk - 1) {
                    ga = r[q];
                    de = T(0);
                } else {
                    ga = r[q] - up[q] * ga;
                    de = -up[q] * de;
                }
            }
        }
        carry_x[me] = ga;
        carry_x[cs + me] = de;
    }
    __syncthreads();
    T chg = T(0);
    {
        T x = T(0);
        for (int s = W - 1; s > w; --s) {
            const int m = s * 32 + lane;
            x = carry_x[m] + carry_x[cs + m] * x;
        }
#pragma unroll
        for (int q = L - 1; q >= 0; --q) {
            const int k = k0 + q;
            if (k < nk) {
                x = (k == nk - 1) ? r[q] : r[q] - up[q] * x;
                if (col) {
                    const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
                    a.dnew[o] = x;
                    if (a.change) {
                        const T d = fabs(x - (FIRST ? T(0) : a.dold[o]));
                        chg = (d > chg || d != d) ? d : chg;
                    }
                }
            }
        }
    }
    if (a.change != nullptr) {
        chg = warp_max(chg);
        if (lane == 0) { atomic_max_nonneg(a.change, chg); }
    }
}

template <typename T, bool FIRST, int L>
__global__ void __launch_bounds__(512) zline_seg_kernel(LineArgs<T> a, T* __restrict__ inv_io, T* __restrict__ cp_io)
{
    zline_seg_body<T, FIRST, L>(a, inv_io, cp_io, blockIdx.x);
}

//! The split sweep's first half: the right-hand side with the lagged lateral
//! terms, r' = rhs + a_XM d_XM + a_XP d_XP + a_YM d_YM + a_YP d_YP (the
//! segmented sweep's fold, in its operation order), one thread per point,
//! for every system of the launch (blockIdx.z = system * nk + k). The column
//! solves then read r' in place of the nine values the fold needs: a fully
//! parallel pass and a light one instead of one with a heavy load phase.
template <typename T>
__device__ __forceinline__ void line_fold_point(const LineArgs<T>& a, T* __restrict__ out, int i, int j, int k)
{
    if (i >= a.ni || j >= a.nj || k >= a.nk) { return; }
    const gb_grid& g = a.g;
    const int im = lateral_image(i - 1, a.ni, g.nx, g.periodic_x != 0);
    const int ip = lateral_image(i + 1, a.ni, g.nx, g.periodic_x != 0);
    const int jm = lateral_image(j - 1, a.nj, g.ny, g.periodic_y != 0);
    const int jp = lateral_image(j + 1, a.nj, g.ny, g.periodic_y != 0);
    const int64_t o = at(g, i, j, k);
    const T dxm = (im >= 0) ? a.dold[at(g, im, j, k)] : T(0);
    const T dxp = (ip >= 0) ? a.dold[at(g, ip, j, k)] : T(0);
    const T dym = (jm >= 0) ? a.dold[at(g, i, jm, k)] : T(0);
    const T dyp = (jp >= 0) ? a.dold[at(g, i, jp, k)] : T(0);
    out[o] = a.rhs[o] + a.A[GB_COEF_XM * a.cs + o] * dxm + a.A[GB_COEF_XP * a.cs + o] * dxp
           + a.A[GB_COEF_YM * a.cs + o] * dym + a.A[GB_COEF_YP * a.cs + o] * dyp;
}

template <typename T>
__global__ void __launch_bounds__(128) k_line_fold(MultiLineArgs<T> m, int nkmax)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int s = blockIdx.z / nkmax, k = blockIdx.z % nkmax;
    switch (s) {
    case 0: line_fold_point<T>(m.a[0], m.fold[0], i, j, k); break;
    case 1: line_fold_point<T>(m.a[1], m.fold[1], i, j, k); break;
    default: line_fold_point<T>(m.a[2], m.fold[2], i, j, k); break;
    }
}

template <typename T, int L>
__global__ void __launch_bounds__(512) zline_seg_pref_multi_kernel(MultiLineArgs<T> m)
{
    switch (blockIdx.z) {
    case 0: zline_seg_body<T, false, L, true>(m.a[0], m.inv[0], m.cp[0], blockIdx.x); break;
    case 1: zline_seg_body<T, false, L, true>(m.a[1], m.inv[1], m.cp[1], blockIdx.x); break;
    default: zline_seg_body<T, false, L, true>(m.a[2], m.inv[2], m.cp[2], blockIdx.x); break;
    }
}

//! The segmented sweep's register cap per thread for L levels a warp. Two
//! blocks of nk / L warps share an SM; each of its 4 schedulers holds 16 K
//! registers, so the warps one scheduler takes times 32 lanes times the cap
//! must fit 16 K: 96 for L = 8 (9 warps a block on 65 levels), 64 for L = 5
//! (13 warps), 56 for L = 4 (17 warps).
constexpr int seg_reg_cap(int L)
{
    return L == 4 ? 56 : (L == 5 ? 64 : 96);
}

//! The segmented sweep over several systems (MultiLineArgs; blockIdx.z picks
//! the system, with constant indices into the parameter block). The register
//! cap (seg_reg_cap, no spills at any L) lets two blocks share an SM: its
//! register file is split among its 4 schedulers, and two blocks of W warps
//! place ceil(W / 2) warps on one of them. At L = 5 (the default) a block of
//! 13 warps at 64 registers gives 26 warps an SM to hide the segment loads'
//! latency, against 18 at L = 8 and 96 registers (the 104 the compiler picks
//! unbounded would fit one block only).
template <typename T, bool FIRST, int L>
__global__ void __maxnreg__(seg_reg_cap(L)) zline_seg_multi_kernel(MultiLineArgs<T> m)
{
    pdl_entry();
    switch (blockIdx.z) {
    case 0: zline_seg_body<T, FIRST, L>(m.a[0], m.inv[0], m.cp[0], blockIdx.x); break;
    case 1: zline_seg_body<T, FIRST, L>(m.a[1], m.inv[1], m.cp[1], blockIdx.x); break;
    default: zline_seg_body<T, FIRST, L>(m.a[2], m.inv[2], m.cp[2], blockIdx.x); break;
    }
}

//! Shared memory of the segmented sweep's carries: 8 values per thread.
template <typename T>
constexpr size_t seg_smem_bytes(int warps)
{
    return static_cast<size_t>(8) * warps * 32 * sizeof(T);
}

//! Levels per segment of the segmented sweep (GB_TUNE_LINE_SEGMENT: 4, 5 or 8,
//! default 5) and its warps per block for nk levels; 0 when the column is too
//! tall (more segments than seg_max_warps), which the callers then sweep with
//! the factored kernel. The split form's solves (zline_seg_pref_multi_kernel,
//! 512 threads a block) take at most kSegMaxWarps segments.
constexpr int kSegMaxWarps = 16;

inline int seg_levels(const gb_ctx* ctx)
{
    const int v = ctx->tune[GB_TUNE_LINE_SEGMENT];
    return (v == 4 || v == 8) ? v : 5;
}


//! The segmented multi-system kernel's warps a block at most for L levels a
//! warp: a block's registers (warps x 32 x the cap) within the SM's 64 K, and
//! 32 warps.
constexpr int seg_max_warps(int L)
{
    return (65536 / (32 * seg_reg_cap(L)) < 32) ? 65536 / (32 * seg_reg_cap(L)) : 32;
}

inline int seg_warps(int nk, int L)
{
    const int w = (nk + L - 1) / L;
    return (w >= 1 && w <= seg_max_warps(L)) ? w : 0;
}

//! The two copies of a periodic seam face take the low copy's value.
template <typename T>
__global__ void seam_sync_kernel(gb_grid g, int loc, T* __restrict__ f)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int ni = ext_x(g, loc), nj = ext_y(g, loc), nk = ext_z(g, loc);
    const bool sx = (loc & 1) && g.periodic_x, sy = ((loc >> 1) & 1) && g.periodic_y;
    if (sx) {
        if (n < nj * nk) {
            const int j = n % nj, k = n / nj;
            f[at(g, g.nx, j, k)] = f[at(g, 0, j, k)];
        }
    }
    if (sy) {
        if (n < ni * nk) {
            const int i = n % ni, k = n / ni;
            f[at(g, i, g.ny, k)] = f[at(g, i, 0, k)];
        }
    }
}

}  // namespace

template <typename T>
void seam_sync(gb_ctx* ctx, const gb_grid& g, int loc, T* f)
{
    const bool sx = (loc & 1) && g.periodic_x, sy = ((loc >> 1) & 1) && g.periodic_y;
    if (!sx && !sy) { return; }
    const int n = std::max(ext_y(g, loc), ext_x(g, loc)) * ext_z(g, loc);
    seam_sync_kernel<T><<<(n + 255) / 256, 256, 0, ctx->stream>>>(g, loc, f);
    ++ctx->launches;
}

template <typename T>
size_t line_smem_bytes(int nk)
{
    return static_cast<size_t>(2) * nk * 64 * sizeof(T);
}

template <typename T>
gb_status zline_sweeps(gb_ctx* ctx, const gb_grid& g, int loc, const T* A, const T* ap, const T* rhs, int sweeps,
                       T* delta, unsigned long long* change_word, LineScratch scratch_kind)
{
    const int ni = ext_x(g, loc), nj = ext_y(g, loc), nk = ext_z(g, loc);
    const int64_t vol = volume(g);
    // Ping-pong: sweep s writes buf[(sweeps - 1 - s) & 1], so the last sweep lands in delta.
    T* tmp = static_cast<T*>(scratch(ctx, kSlotLineNext, sizeof(T) * vol));
    if (tmp == nullptr) { return GB_OOM; }
    const size_t smem = line_smem_bytes<T>(nk);
    const int segL = seg_levels(ctx);
    const int segW = seg_warps(nk, segL);
    if (scratch_kind == LineScratch::automatic) {
        const int v = ctx->tune[GB_TUNE_LINE_VARIANT];
        scratch_kind = (v == 1)   ? LineScratch::pipelined
                       : (v == 2) ? LineScratch::shared
                       : (v == 3) ? LineScratch::global
                       : (v == 4) ? LineScratch::factored
                                  : LineScratch::segmented;
    }
    if (scratch_kind == LineScratch::segmented && segW == 0) { scratch_kind = LineScratch::factored; }
    if (scratch_kind == LineScratch::segmented) {
        // one system through the batched form (the segmented kernels, and the
        // split form with GB_TUNE_LINE_VARIANT 6)
        const int locs[1] = {loc};
        const T* As[1] = {A};
        const T* aps[1] = {ap};
        const T* rhss[1] = {rhs};
        T* deltas[1] = {delta};
        unsigned long long* words[1] = {change_word};
        return zline_sweeps_multi<T>(ctx, g, 1, locs, As, aps, rhss, sweeps, deltas, words);
    }
    const bool factored = (scratch_kind == LineScratch::factored);
    const bool pipelined = factored || (scratch_kind == LineScratch::pipelined);
    T* inv = nullptr;
    T* cpr = nullptr;
    if (factored) {
        inv = static_cast<T*>(scratch(ctx, kSlotLineInv, sizeof(T) * vol));
        cpr = static_cast<T*>(scratch(ctx, kSlotLineCp, sizeof(T) * vol));
        if (inv == nullptr || cpr == nullptr) { return GB_OOM; }
    }
    bool use_smem = (scratch_kind == LineScratch::shared);
    T* cbuf = nullptr;
    T* ebuf = nullptr;
    // The pipelined kernel: one warp per block, R levels in flight (4 in FP64, 8 in FP32).
    constexpr int R = (sizeof(T) == 8) ? 4 : 8;
    const int pipe_thr = (ctx->tune[GB_TUNE_LINE_BLOCK] == 64 || ctx->tune[GB_TUNE_LINE_BLOCK] == 128)
                           ? ctx->tune[GB_TUNE_LINE_BLOCK] : 32;
    const size_t pipe_smem_first = static_cast<size_t>(R * 4 + 2 * nk) * pipe_thr * sizeof(T);
    const size_t pipe_smem = static_cast<size_t>(R * 12 + 2 * nk) * pipe_thr * sizeof(T);
    // the factored sweep with twice the levels in flight (GB_TUNE_LINE_DEPTH = 2)
    constexpr int R2 = 2 * R;
    const bool deep = factored && ctx->tune[GB_TUNE_LINE_DEPTH] == 2;
    const size_t deep_smem_first = static_cast<size_t>(R2 * 4 + 2 * nk) * pipe_thr * sizeof(T);
    const size_t deep_smem = static_cast<size_t>(R2 * 12 + 2 * nk) * pipe_thr * sizeof(T);
    if (pipelined) {
        static std::atomic<bool> attr_done[2];  // set once per process (one device per process)
        const int ti = sizeof(T) == 8 ? 1 : 0;
        if (!attr_done[ti].load()) {
            cudaFuncSetAttribute(zline_pipe_kernel<T, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(zline_pipe_kernel<T, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(zline_fact_kernel<T, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(zline_fact_kernel<T, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(zline_fact_kernel<T, true, R2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(zline_fact_kernel<T, false, R2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            attr_done[ti].store(true);
        }
    } else if (!use_smem) {
        cbuf = static_cast<T*>(scratch(ctx, kSlotLineC, sizeof(T) * vol));
        ebuf = static_cast<T*>(scratch(ctx, kSlotLineE, sizeof(T) * vol));
        if (cbuf == nullptr || ebuf == nullptr) { return GB_OOM; }
    } else {
        static std::atomic<bool> attr_set[2];
        const int ti = sizeof(T) == 8 ? 1 : 0;
        if (!attr_set[ti].load()) {
            cudaFuncSetAttribute(zline_sweep_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            attr_set[ti].store(true);
        }
    }
    T* buf[2] = {delta, tmp};
    if (change_word != nullptr) { cudaMemsetAsync(change_word, 0, sizeof(unsigned long long), ctx->stream); }
    for (int s = 0; s < sweeps; ++s) {
        LineArgs<T> a;
        a.g = g;
        a.ni = ni;
        a.nj = nj;
        a.nk = nk;
        a.A = A;
        a.cs = vol;
        a.ap = ap;
        a.rhs = rhs;
        a.dold = buf[(sweeps - s) & 1];
        a.dnew = buf[(sweeps - 1 - s) & 1];
        a.cbuf = cbuf;
        a.ebuf = ebuf;
        a.first = (s == 0) ? 1 : 0;
        a.change = (s == sweeps - 1) ? change_word : nullptr;
        Span span(ctx, GB_KERNEL_LINE_SWEEP);
        if (deep) {
            const dim3 block(pipe_thr, 1);
            const dim3 grid((ni + pipe_thr - 1) / pipe_thr, nj);
            if (a.first) {
                zline_fact_kernel<T, true, R2><<<grid, block, deep_smem_first, ctx->stream>>>(a, inv, nullptr, cpr,
                                                                                            nullptr);
            } else {
                zline_fact_kernel<T, false, R2><<<grid, block, deep_smem, ctx->stream>>>(a, nullptr, inv, nullptr, cpr);
            }
        } else if (factored) {
            const dim3 block(pipe_thr, 1);
            const dim3 grid((ni + pipe_thr - 1) / pipe_thr, nj);
            if (a.first) {
                zline_fact_kernel<T, true, R><<<grid, block, pipe_smem_first, ctx->stream>>>(a, inv, nullptr, cpr,
                                                                                           nullptr);
            } else {
                zline_fact_kernel<T, false, R><<<grid, block, pipe_smem, ctx->stream>>>(a, nullptr, inv, nullptr, cpr);
            }
        } else if (pipelined) {
            const dim3 block(pipe_thr, 1);
            const dim3 grid((ni + pipe_thr - 1) / pipe_thr, nj);
            if (a.first) {
                zline_pipe_kernel<T, true, R><<<grid, block, pipe_smem_first, ctx->stream>>>(a);
            } else {
                zline_pipe_kernel<T, false, R><<<grid, block, pipe_smem, ctx->stream>>>(a);
            }
        } else if (use_smem) {
            const dim3 block(32, 2);
            const dim3 grid((ni + 31) / 32, (nj + 1) / 2);
            zline_sweep_kernel<T, true><<<grid, block, smem, ctx->stream>>>(a);
        } else {
            const dim3 block(32, 4);
            const dim3 grid((ni + 31) / 32, (nj + 3) / 4);
            zline_sweep_kernel<T, false><<<grid, block, 0, ctx->stream>>>(a);
        }
        ++ctx->launches;
    }
    seam_sync<T>(ctx, g, loc, delta);
    return check_cuda("zline_jacobi");
}

template <typename T>
gb_status zline_sweeps_multi(gb_ctx* ctx, const gb_grid& g, int n, const int* locs, const T* const* A,
                             const T* const* ap, const T* const* rhs, int sweeps, T* const* delta,
                             unsigned long long* const* change_words)
{
    if (n < 1 || n > kMaxLineSystems) {
        set_error("gust: zline_sweeps_multi: 1 to %d systems (got %d)", kMaxLineSystems, n);
        return GB_BAD_ARG;
    }
    const int64_t vol = volume(g);
    constexpr int R = (sizeof(T) == 8) ? 4 : 8;
    constexpr int kThr = 32;
    int ni[kMaxLineSystems], nj[kMaxLineSystems], nk[kMaxLineSystems];
    T* tmp[kMaxLineSystems];
    T* inv[kMaxLineSystems];
    T* cpr[kMaxLineSystems];
    int max_ni = 0, max_nj = 0, max_nk = 0;
    for (int s = 0; s < n; ++s) {
        ni[s] = ext_x(g, locs[s]);
        nj[s] = ext_y(g, locs[s]);
        nk[s] = ext_z(g, locs[s]);
        max_ni = std::max(max_ni, ni[s]);
        max_nj = std::max(max_nj, nj[s]);
        max_nk = std::max(max_nk, nk[s]);
        tmp[s] = static_cast<T*>(scratch(ctx, kSlotMultiBase + 3 * s, sizeof(T) * vol));
        inv[s] = static_cast<T*>(scratch(ctx, kSlotMultiBase + 3 * s + 1, sizeof(T) * vol));
        cpr[s] = static_cast<T*>(scratch(ctx, kSlotMultiBase + 3 * s + 2, sizeof(T) * vol));
        if (!tmp[s] || !inv[s] || !cpr[s]) { return GB_OOM; }
        if (change_words != nullptr && change_words[s] != nullptr) {
            cudaMemsetAsync(change_words[s], 0, sizeof(unsigned long long), ctx->stream);
        }
    }
    // the segmented sweep (the default; GB_TUNE_LINE_VARIANT 4 selects the factored one below)
    const int segL = seg_levels(ctx);
    const int segW = seg_warps(max_nk, segL);
    if (ctx->tune[GB_TUNE_LINE_VARIANT] != 4 && segW > 0) {
        const dim3 block(32, segW);
        int max_cols = 0;
        for (int s = 0; s < n; ++s) { max_cols = std::max(max_cols, ni[s] * nj[s]); }
        const dim3 grid((max_cols + 31) / 32, 1, n);
        const size_t sm = seg_smem_bytes<T>(segW);
        if (sm > 48 * 1024) {
            // more than 24 FP64 segments (tall columns at L = 4 or 5): the carries need the opt-in
            static std::atomic<bool> big_attr[2];  // set once per process (one device per process)
            const int ti = sizeof(T) == 8 ? 1 : 0;
            if (!big_attr[ti].load()) {
                const int big = static_cast<int>(seg_smem_bytes<T>(32));
                cudaFuncSetAttribute(zline_seg_multi_kernel<T, true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
                cudaFuncSetAttribute(zline_seg_multi_kernel<T, false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
                cudaFuncSetAttribute(zline_seg_multi_kernel<T, true, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
                cudaFuncSetAttribute(zline_seg_multi_kernel<T, false, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
                big_attr[ti].store(true);
            }
        }
        // GB_TUNE_LINE_VARIANT 6: the later sweeps split into the fold and light column solves
        const bool split = ctx->tune[GB_TUNE_LINE_VARIANT] == 6 && sweeps > 1 && segW <= kSegMaxWarps;
        // GB_TUNE_LINE_FIRST 2: the first sweep (the factorisation) by the sequential factored kernel,
        // which stores the same factors (1/m, c') the segmented later sweeps read
        constexpr int RF = (sizeof(T) == 8) ? 4 : 8;
        const bool fact_first = ctx->tune[GB_TUNE_LINE_FIRST] == 2;
        const size_t fsm = static_cast<size_t>(RF * 4 + 2 * max_nk) * 32 * sizeof(T);
        if (fact_first) {
            static std::atomic<bool> ff_attr[2];
            const int ti = sizeof(T) == 8 ? 1 : 0;
            if (!ff_attr[ti].load()) {
                cudaFuncSetAttribute(zline_fact_multi_kernel<T, true, RF, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024);
                ff_attr[ti].store(true);
            }
            if (fsm > 200 * 1024) { return GB_BAD_ARG; }
        }
        T* fold[kMaxLineSystems] = {};
        if (split) {
            for (int s = 0; s < n; ++s) {
                fold[s] = static_cast<T*>(scratch(ctx, kSlotMultiBase + 3 * kMaxLineSystems + s, sizeof(T) * vol));
                if (!fold[s]) { return GB_OOM; }
            }
        }
        for (int k = 0; k < sweeps; ++k) {
            MultiLineArgs<T> m{};
            for (int s = 0; s < n; ++s) {
                T* buf[2] = {delta[s], tmp[s]};
                LineArgs<T>& a = m.a[s];
                a.g = g;
                a.ni = ni[s];
                a.nj = nj[s];
                a.nk = nk[s];
                a.A = A[s];
                a.cs = vol;
                a.ap = ap[s];
                a.rhs = rhs[s];
                a.dold = buf[(sweeps - k) & 1];
                a.dnew = buf[(sweeps - 1 - k) & 1];
                a.first = (k == 0) ? 1 : 0;
                a.change = (k == sweeps - 1 && change_words != nullptr) ? change_words[s] : nullptr;
                a.rfold = fold[s];
                m.inv[s] = inv[s];
                m.cp[s] = cpr[s];
                m.fold[s] = fold[s];
            }
            Span span(ctx, GB_KERNEL_LINE_SWEEP);
            if (fact_first && k == 0) {
                const dim3 fgrid((max_ni + 31) / 32, max_nj, n);
                zline_fact_multi_kernel<T, true, RF, 0><<<fgrid, 32, fsm, ctx->stream>>>(m);
                ++ctx->launches;
                continue;
            }
            if (split && k > 0) {
                const dim3 fgrid((max_ni + 127) / 128, max_nj, max_nk * n);
                k_line_fold<T><<<fgrid, 128, 0, ctx->stream>>>(m, max_nk);
                if (segL == 4) {
                    zline_seg_pref_multi_kernel<T, 4><<<grid, block, sm, ctx->stream>>>(m);
                } else if (segL == 5) {
                    zline_seg_pref_multi_kernel<T, 5><<<grid, block, sm, ctx->stream>>>(m);
                } else {
                    zline_seg_pref_multi_kernel<T, 8><<<grid, block, sm, ctx->stream>>>(m);
                }
                ctx->launches += 2;
                continue;
            }
            const bool pdl = ctx->tune[GB_TUNE_PDL] != 1;
            if (segL == 4) {
                if (k == 0) {
                    launch_pdl(pdl, zline_seg_multi_kernel<T, true, 4>, grid, block, sm, ctx->stream, m);
                } else {
                    launch_pdl(pdl, zline_seg_multi_kernel<T, false, 4>, grid, block, sm, ctx->stream, m);
                }
            } else if (segL == 5) {
                if (k == 0) {
                    launch_pdl(pdl, zline_seg_multi_kernel<T, true, 5>, grid, block, sm, ctx->stream, m);
                } else {
                    launch_pdl(pdl, zline_seg_multi_kernel<T, false, 5>, grid, block, sm, ctx->stream, m);
                }
            } else {
                if (k == 0) {
                    launch_pdl(pdl, zline_seg_multi_kernel<T, true, 8>, grid, block, sm, ctx->stream, m);
                } else {
                    launch_pdl(pdl, zline_seg_multi_kernel<T, false, 8>, grid, block, sm, ctx->stream, m);
                }
            }
            ++ctx->launches;
        }
        for (int s = 0; s < n; ++s) { seam_sync<T>(ctx, g, locs[s], delta[s]); }
        return check_cuda("zline_sweeps_multi");
    }
    static std::atomic<bool> attr_done[2];  // set once per process (one device per process)
    const int ti = sizeof(T) == 8 ? 1 : 0;
    if (!attr_done[ti].load()) {
        cudaFuncSetAttribute(zline_fact_multi_kernel<T, true, R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
        cudaFuncSetAttribute(zline_fact_multi_kernel<T, false, R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
        cudaFuncSetAttribute(zline_fact_multi_kernel<T, true, R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
        cudaFuncSetAttribute(zline_fact_multi_kernel<T, false, R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
        attr_done[ti].store(true);
    }
    // where the back substitution finds c' and e' (zline_fact_body's BACK):
    // GB_TUNE_LINE_BACK 1 -> 0 (shared), 2 -> 1 (global), 3 -> 2 (e' shared, c' again from L2)
    const int knob = ctx->tune[GB_TUNE_LINE_BACK];
    const int back_mode = (knob == 2) ? 1 : (knob == 3) ? 2 : 0;
    const size_t back = (back_mode == 1) ? 0 : (back_mode == 2) ? static_cast<size_t>(max_nk) : static_cast<size_t>(2 * max_nk);
    const size_t smem_first = static_cast<size_t>(R * 4 + back) * kThr * sizeof(T);
    const size_t smem = static_cast<size_t>(R * 12 + back) * kThr * sizeof(T);
    const dim3 grid((max_ni + kThr - 1) / kThr, max_nj, n);
    for (int k = 0; k < sweeps; ++k) {
        MultiLineArgs<T> m{};
        for (int s = 0; s < n; ++s) {
            T* buf[2] = {delta[s], tmp[s]};
            LineArgs<T>& a = m.a[s];
            a.g = g;
            a.ni = ni[s];
            a.nj = nj[s];
            a.nk = nk[s];
            a.A = A[s];
            a.cs = vol;
            a.ap = ap[s];
            a.rhs = rhs[s];
            a.dold = buf[(sweeps - k) & 1];
            a.dnew = buf[(sweeps - 1 - k) & 1];
            a.cbuf = nullptr;
            a.ebuf = nullptr;
            a.first = (k == 0) ? 1 : 0;
            a.change = (k == sweeps - 1 && change_words != nullptr) ? change_words[s] : nullptr;
            m.inv[s] = inv[s];
            m.cp[s] = cpr[s];
        }
        Span span(ctx, GB_KERNEL_LINE_SWEEP);
        const size_t sm = (k == 0) ? smem_first : smem;
        if (k == 0) {
            switch (back_mode) {
            case 1: zline_fact_multi_kernel<T, true, R, 1><<<grid, kThr, sm, ctx->stream>>>(m); break;
            case 2: zline_fact_multi_kernel<T, true, R, 2><<<grid, kThr, sm, ctx->stream>>>(m); break;
            default: zline_fact_multi_kernel<T, true, R, 0><<<grid, kThr, sm, ctx->stream>>>(m); break;
            }
        } else {
            switch (back_mode) {
            case 1: zline_fact_multi_kernel<T, false, R, 1><<<grid, kThr, sm, ctx->stream>>>(m); break;
            case 2: zline_fact_multi_kernel<T, false, R, 2><<<grid, kThr, sm, ctx->stream>>>(m); break;
            default: zline_fact_multi_kernel<T, false, R, 0><<<grid, kThr, sm, ctx->stream>>>(m); break;
            }
        }
        ++ctx->launches;
    }
    for (int s = 0; s < n; ++s) { seam_sync<T>(ctx, g, locs[s], delta[s]); }
    return check_cuda("zline_sweeps_multi");
}

// ---- Sweeps of many uneven systems in one launch per sweep ----------------
//
// The batched form of the segmented sweep: systems of different grids (the
// tiles of a batch, each with its own nx, ny, nz and location) are swept
// together. The host lays out one column work-list for all of them: an entry
// per 32-column block of a system, (system, block within the system). Each
// launch is persistent: at most the blocks the SMs hold at once, each walking
// the list with a stride of the grid size and running the segmented sweep's
// body on the entry's columns. Systems whose columns need the same number of
// warps share a launch (a block's warps are its segments; the warps above a
// column's top are identity maps, so a block taller than a column gives the
// same values bit for bit, but wastes its slots).

template <typename T>
struct BatchLineSys {
    LineArgs<T> a;               // sweep-independent fields (dold, dnew, first, change set per sweep)
    T* buf[2];                   // delta, its ping-pong partner
    T* inv;                      // 1/m of the first sweep's factorisation
    T* cp;                       // c'
    unsigned long long* change;  // this system's max |change| word (null: not wanted)
};

//! Systems one batched launch takes: their descriptors travel in the launch's
//! parameter block (the constant bank, read as instruction operands like a
//! single system's arguments, not loaded into registers), 26 KB of the 32 KB
//! a launch may carry.
constexpr int kBatchLaunchSystems = 120;

template <typename T>
struct BatchLineParams {
    BatchLineSys<T> sys[kBatchLaunchSystems];
    //! The work-list: entry e is column block e - first_block[s] of the system
    //! s with first_block[s] <= e < first_block[s + 1].
    int first_block[kBatchLaunchSystems + 1];
    int nsys;
};

//! The batched sweep's register cap: the segmented sweep's, but 72 at L = 5
//! (the descriptors' fields taken from the constant bank by a runtime index
//! need registers the single-system kernel folds into its instructions; 64
//! spills). Two blocks of up to 14 warps still share an SM (7 warps x 32
//! lanes x 72 within a scheduler's 16 K registers).
constexpr int batch_reg_cap(int L)
{
    return L == 5 ? 72 : seg_reg_cap(L);
}

//! The batched sweep's warps a block at most (its registers within the SM's 64 K).
constexpr int batch_max_warps(int L)
{
    return (65536 / (32 * batch_reg_cap(L)) < 32) ? 65536 / (32 * batch_reg_cap(L)) : 32;
}

template <typename T, bool FIRST, int L>
__global__ void __maxnreg__(batch_reg_cap(L))
    zline_seg_batch_kernel(const __grid_constant__ BatchLineParams<T> p, int sweep, int sweeps)
{
    const int items = p.first_block[p.nsys];
    for (int it = blockIdx.x; it < items; it += gridDim.x) {
        // the entry's system by bisection of the block offsets (values uniform
        // over the block, so they stay out of the per-thread registers)
        int lo = 0, hi = p.nsys - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.first_block[mid] <= it) {
                lo = mid;
            } else {
                hi = mid - 1;
            }
        }
        const BatchLineSys<T>& d = p.sys[lo];
        LineArgs<T> a = d.a;
        a.dold = d.buf[(sweeps - sweep) & 1];
        a.dnew = d.buf[(sweeps - 1 - sweep) & 1];
        a.first = FIRST ? 1 : 0;
        a.change = (sweep == sweeps - 1) ? d.change : nullptr;
        zline_seg_body<T, FIRST, L>(a, d.inv, d.cp, it - p.first_block[lo]);
        // the next entry's carries reuse the shared memory
        __syncthreads();
    }
}

template <typename T, bool FIRST, int L>
cudaError_t launch_seg_batch(const BatchLineParams<T>& sys, int warps, int sweep, int sweeps, cudaStream_t stream)
{
    auto kern = zline_seg_batch_kernel<T, FIRST, L>;
    const size_t sm = seg_smem_bytes<T>(warps);
    if (sm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(seg_smem_bytes<T>(32)));
        if (e != cudaSuccess) { return e; }
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, sm);
    const int resident = std::max(1, sms) * std::max(1, per_sm);
    const int blocks = std::min(sys.first_block[sys.nsys], resident);
    kern<<<blocks, dim3(32, warps), sm, stream>>>(sys, sweep, sweeps);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_seg_batch_any(int L, bool first, const BatchLineParams<T>& sys, int warps, int sweep, int sweeps,
                                 cudaStream_t stream)
{
    if (L == 4) {
        return first ? launch_seg_batch<T, true, 4>(sys, warps, sweep, sweeps, stream)
                     : launch_seg_batch<T, false, 4>(sys, warps, sweep, sweeps, stream);
    }
    if (L == 8) {
        return first ? launch_seg_batch<T, true, 8>(sys, warps, sweep, sweeps, stream)
                     : launch_seg_batch<T, false, 8>(sys, warps, sweep, sweeps, stream);
    }
    return first ? launch_seg_batch<T, true, 5>(sys, warps, sweep, sweeps, stream)
                 : launch_seg_batch<T, false, 5>(sys, warps, sweep, sweeps, stream);
}

template <typename T>
gb_status zline_sweeps_batch(gb_ctx* ctx, int n, const gb_grid* grids, const int* locs, const T* const* A,
                             const T* const* ap, const T* const* rhs, int sweeps, T* const* delta, double* change)
{
    const int L = seg_levels(ctx);
    // scratch: the ping-pong partners, 1/m and c' of every system (offsets in
    // 256-byte units), then the change words
    std::vector<int64_t> off(n + 1, 0);
    std::vector<int> warps(n);
    for (int s = 0; s < n; ++s) {
        const int64_t vol = volume(grids[s]);
        off[s + 1] = off[s] + ((vol * static_cast<int64_t>(sizeof(T)) + 255) / 256) * 256;
        warps[s] = (ext_z(grids[s], locs[s]) + L - 1) / L;
        if (warps[s] > batch_max_warps(L)) {
            set_error("gust: zline_jacobi_batch: system %d has %d z-levels, more than the batched sweep's %d",
                      s, ext_z(grids[s], locs[s]), batch_max_warps(L) * L);
            return GB_BAD_ARG;
        }
    }
    const size_t field_bytes = static_cast<size_t>(off[n]);
    char* pool = static_cast<char*>(scratch(ctx, kSlotBatchBase, 3 * field_bytes + sizeof(unsigned long long) * n));
    if (pool == nullptr) { return GB_OOM; }
    unsigned long long* d_words = reinterpret_cast<unsigned long long*>(pool + 3 * field_bytes);

    // One launch per run of systems with the same warps a block, at most
    // kBatchLaunchSystems of them: its descriptors (indexed from 0 in the
    // launch) and their column blocks' offsets in its work-list.
    struct Launch {
        int warps;
    };
    std::vector<Launch> launches;
    std::vector<BatchLineParams<T>> params;
    {
        std::vector<int> order(n);
        for (int s = 0; s < n; ++s) { order[s] = s; }
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return warps[x] < warps[y]; });
        for (int q = 0; q < n; ++q) {
            const int s = order[q];
            if (launches.empty() || launches.back().warps != warps[s] || params.back().nsys == kBatchLaunchSystems) {
                launches.push_back(Launch{warps[s]});
                params.emplace_back();
                std::memset(static_cast<void*>(&params.back()), 0, sizeof(BatchLineParams<T>));
            }
            BatchLineParams<T>& pr = params.back();
            const int local = pr.nsys;
            BatchLineSys<T>& d = pr.sys[local];
            LineArgs<T>& a = d.a;
            a.g = grids[s];
            a.ni = ext_x(grids[s], locs[s]);
            a.nj = ext_y(grids[s], locs[s]);
            a.nk = ext_z(grids[s], locs[s]);
            a.A = A[s];
            a.cs = volume(grids[s]);
            a.ap = ap[s];
            a.rhs = rhs[s];
            d.buf[0] = delta[s];
            d.buf[1] = reinterpret_cast<T*>(pool + off[s]);
            d.inv = reinterpret_cast<T*>(pool + field_bytes + off[s]);
            d.cp = reinterpret_cast<T*>(pool + 2 * field_bytes + off[s]);
            d.change = d_words + s;
            const int64_t blocks = (static_cast<int64_t>(a.ni) * a.nj + 31) / 32;
            if (pr.first_block[local] + blocks > (int64_t(1) << 30)) {
                set_error("gust: zline_jacobi_batch: more than 2^30 column blocks in one launch");
                return GB_BAD_ARG;
            }
            pr.first_block[local + 1] = pr.first_block[local] + static_cast<int>(blocks);
            pr.nsys = local + 1;
        }
    }
    for (int s = 0; s < n; ++s) { cudaMemsetAsync(delta[s], 0, sizeof(T) * volume(grids[s]), ctx->stream); }
    cudaMemsetAsync(d_words, 0, sizeof(unsigned long long) * n, ctx->stream);
    for (int k = 0; k < sweeps; ++k) {
        for (size_t q = 0; q < launches.size(); ++q) {
            Span span(ctx, GB_KERNEL_LINE_SWEEP);
            const cudaError_t e = launch_seg_batch_any<T>(L, k == 0, params[q], launches[q].warps, k, sweeps,
                                                          ctx->stream);
            if (e != cudaSuccess) {
                set_error("gust: zline_jacobi_batch: launch failed: %s", cudaGetErrorString(e));
                return GB_CUDA;
            }
            ++ctx->launches;
        }
    }
    for (int s = 0; s < n; ++s) { seam_sync<T>(ctx, grids[s], locs[s], delta[s]); }
    gb_status st = check_cuda("zline_jacobi_batch");
    if (st != GB_OK || change == nullptr) { return st; }
    std::vector<unsigned long long> w(n);
    cudaMemcpyAsync(w.data(), d_words, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("zline_jacobi_batch"); }
    for (int s = 0; s < n; ++s) { change[s] = bits_to_double(w[s]); }
    return GB_OK;
}

template gb_status zline_sweeps_batch<double>(gb_ctx*, int, const gb_grid*, const int*, const double* const*,
                                              const double* const*, const double* const*, int, double* const*,
                                              double*);
template gb_status zline_sweeps_batch<float>(gb_ctx*, int, const gb_grid*, const int*, const float* const*,
                                             const float* const*, const float* const*, int, float* const*, double*);

template gb_status zline_sweeps_multi<double>(gb_ctx*, const gb_grid&, int, const int*, const double* const*,
                                              const double* const*, const double* const*, int, double* const*,
                                              unsigned long long* const*);
template gb_status zline_sweeps_multi<float>(gb_ctx*, const gb_grid&, int, const int*, const float* const*,
                                             const float* const*, const float* const*, int, float* const*,
                                             unsigned long long* const*);
template gb_status zline_sweeps<double>(gb_ctx*, const gb_grid&, int, const double*, const double*, const double*, int,
                                        double*, unsigned long long*, LineScratch);
template gb_status zline_sweeps<float>(gb_ctx*, const gb_grid&, int, const float*, const float*, const float*, int,
                                       float*, unsigned long long*, LineScratch);
template void seam_sync<double>(gb_ctx*, const gb_grid&, int, double*);
template void seam_sync<float>(gb_ctx*, const gb_grid&, int, float*);

}  // namespace gb

namespace {

template <typename T>
gb_status zline_jacobi_api(gb_ctx* ctx, const gb_grid* g, int32_t loc, const T* A, const T* ap, const T* rhs,
                           int32_t sweeps, T* delta, T* change)
{
    gb::clear_error();
    const char* op = "zline_jacobi";
    if (ctx == nullptr) {
        gb::set_error("gust: %s: ctx is null", op);
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_grid(op, g);
    if (st != GB_OK) { return st; }
    if ((st = gb::check_loc(op, loc)) != GB_OK) { return st; }
    if (sweeps < 1) {
        gb::set_error("gust: zline_jacobi: sweeps must be >= 1 (got %d)", sweeps);
        return GB_BAD_ARG;
    }
    if (A == nullptr || ap == nullptr || rhs == nullptr || delta == nullptr) {
        gb::set_error("gust: zline_jacobi: A, ap, rhs and delta must be device arrays of the grid");
        return GB_BAD_ARG;
    }
    // delta.setVal(0): the ghosts outside the domain stay 0 (the couplings are folded).
    cudaMemsetAsync(delta, 0, sizeof(T) * gb::volume(*g), ctx->stream);
    st = gb::zline_sweeps<T>(ctx, *g, loc, A, ap, rhs, sweeps, delta, gb::dword(ctx, 0), gb::LineScratch::automatic);
    if (st != GB_OK) { return st; }
    unsigned long long w = 0;
    if ((st = gb::read_words(ctx, 0, 1, &w)) != GB_OK) { return st; }
    if (change != nullptr) { *change = static_cast<T>(gb::bits_to_double(w)); }
    return GB_OK;
}

template <typename Sys>
struct LineSystemOf;
template <>
struct LineSystemOf<double> { using type = gb_line_system; };
template <>
struct LineSystemOf<float> { using type = gb_line_system_f32; };

template <typename T>
gb_status zline_jacobi_batch_api(gb_ctx* ctx, int32_t n, const typename LineSystemOf<T>::type* systems,
                                 int32_t sweeps, double* change)
{
    gb::clear_error();
    const char* op = "zline_jacobi_batch";
    if (ctx == nullptr) {
        gb::set_error("gust: %s: ctx is null", op);
        return GB_BAD_ARG;
    }
    if (n < 1 || systems == nullptr) {
        gb::set_error("gust: zline_jacobi_batch: n must be >= 1 with a systems array (got %d)", n);
        return GB_BAD_ARG;
    }
    if (sweeps < 1) {
        gb::set_error("gust: zline_jacobi_batch: sweeps must be >= 1 (got %d)", sweeps);
        return GB_BAD_ARG;
    }
    std::vector<gb_grid> grids(n);
    std::vector<int> locs(n);
    std::vector<const T*> A(n), ap(n), rhs(n);
    std::vector<T*> delta(n);
    for (int s = 0; s < n; ++s) {
        const auto& y = systems[s];
        gb_status st = gb::check_grid(op, &y.grid);
        if (st != GB_OK) { return st; }
        if ((st = gb::check_loc(op, y.loc)) != GB_OK) { return st; }
        if (y.A == nullptr || y.ap == nullptr || y.rhs == nullptr || y.delta == nullptr) {
            gb::set_error("gust: zline_jacobi_batch: system %d: A, ap, rhs and delta must be device arrays of its "
                          "grid", s);
            return GB_BAD_ARG;
        }
        grids[s] = y.grid;
        locs[s] = y.loc;
        A[s] = y.A;
        ap[s] = y.ap;
        rhs[s] = y.rhs;
        delta[s] = y.delta;
    }
    return gb::zline_sweeps_batch<T>(ctx, n, grids.data(), locs.data(), A.data(), ap.data(), rhs.data(), sweeps,
                                     delta.data(), change);
}

}  // namespace

extern "C" {

gb_status gb_zline_jacobi(gb_ctx* ctx, const gb_grid* g, int32_t loc, const double* A, const double* ap,
                          const double* rhs, int32_t sweeps, double* delta, double* change)
{
    return zline_jacobi_api<double>(ctx, g, loc, A, ap, rhs, sweeps, delta, change);
}

gb_status gb_zline_jacobi_f32(gb_ctx* ctx, const gb_grid* g, int32_t loc, const float* A, const float* ap,
                              const float* rhs, int32_t sweeps, float* delta, float* change)
{
    return zline_jacobi_api<float>(ctx, g, loc, A, ap, rhs, sweeps, delta, change);
}

gb_status gb_zline_jacobi_batch(gb_ctx* ctx, int32_t n, const gb_line_system* systems, int32_t sweeps,
                                double* change)
{
    return zline_jacobi_batch_api<double>(ctx, n, systems, sweeps, change);
}

gb_status gb_zline_jacobi_batch_f32(gb_ctx* ctx, int32_t n, const gb_line_system_f32* systems, int32_t sweeps,
                                    double* change)
{
    return zline_jacobi_batch_api<float>(ctx, n, systems, sweeps, change);
}

}  // extern "C"

// ---- The allocation-free z-line solve ------------------------------------
//
// gb_zline_jacobi_noalloc runs the same FP64 column solves as gb_zline_jacobi
// (the pipelined kernel with one-warp blocks; the context path also keeps the
// column factors between sweeps, so the two agree to rounding) for a caller
// that may not allocate device memory at all: no
// gb_ctx (creating one allocates), no cudaMalloc or cudaFree behind its back.
// Its only scratch, the ping-pong iterate and the change word, live in the
// fixed array below, which the CUDA runtime reserves on each device when it
// loads this library's device code.
namespace {

//! Largest padded grid volume (points) the allocation-free solve accepts:
//! 2^21 points, 16 MiB of FP64 iterate (a 128 x 128 x 64 cell grid with two
//! ghost layers is 1.22 M points).
constexpr int64_t kNoAllocMaxPoints = int64_t(1) << 21;
//! The change word sits one 256-byte block past the iterate.
constexpr int64_t kNoAllocWords = kNoAllocMaxPoints + 32;

//! Shared by every call on a device. The iterate part needs no initial value:
//! each sweep writes every point the next sweep reads. The change word must be
//! zero when the last sweep starts; each call zeroes it on its own stream.
static __device__ __align__(256) double g_line_noalloc_scratch[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_addr[kNoAllocMaxDevices] = {};

//! Per-device set-up, once, with that device current: the array's device
//! address and the shared-memory limit of the two sweep kernels. The address
//! is kept for the life of the process, so a cudaDeviceReset of the device
//! after its first call is not supported (the address would be stale).
gb_status noalloc_setup(int dev, double** out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_line_noalloc_scratch);
        if (e == cudaSuccess) {
            e = cudaFuncSetAttribute(gb::zline_pipe_kernel<double, true, 4>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        }
        if (e == cudaSuccess) {
            e = cudaFuncSetAttribute(gb::zline_pipe_kernel<double, false, 4>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            gb::set_error("gust: zline_jacobi_noalloc: set-up on device %d failed: %s (%s)", dev,
                          cudaGetErrorName(e), cudaGetErrorString(e));
            return GB_CUDA;
        }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return GB_OK;
}

}  // namespace

extern "C" gb_status gb_zline_jacobi_noalloc(const gb_grid* g, int32_t loc, const double* A, const double* ap,
                                             const double* rhs, int32_t sweeps, double* delta, double* change,
                                             void* stream)
{
    gb::clear_error();
    const char* op = "zline_jacobi_noalloc";
    gb_status st = gb::check_grid(op, g);
    if (st != GB_OK) { return st; }
    if ((st = gb::check_loc(op, loc)) != GB_OK) { return st; }
    if (sweeps < 1) {
        gb::set_error("gust: zline_jacobi_noalloc: sweeps must be >= 1 (got %d)", sweeps);
        return GB_BAD_ARG;
    }
    if (A == nullptr || ap == nullptr || rhs == nullptr || delta == nullptr) {
        gb::set_error("gust: zline_jacobi_noalloc: A, ap, rhs and delta must be device arrays of the grid");
        return GB_BAD_ARG;
    }
    const int64_t vol = gb::volume(*g);
    if (vol > kNoAllocMaxPoints) {
        gb::set_error("gust: zline_jacobi_noalloc: the grid has %lld padded points, more than the fixed scratch "
                      "of %lld points (16 MiB); use gb_zline_jacobi with a context",
                      static_cast<long long>(vol), static_cast<long long>(kNoAllocMaxPoints));
        return GB_BAD_ARG;
    }
    constexpr int R = 4, NTHR = 32;
    const int ni = gb::ext_x(*g, loc), nj = gb::ext_y(*g, loc), nk = gb::ext_z(*g, loc);
    const size_t smem_first = static_cast<size_t>(R * 4 + 2 * nk) * NTHR * sizeof(double);
    const size_t smem = static_cast<size_t>(R * 12 + 2 * nk) * NTHR * sizeof(double);
    if (smem > 200 * 1024) {
        gb::set_error("gust: zline_jacobi_noalloc: %d z-levels need %zu bytes of shared memory per block, more than "
                      "200 KiB", nk, smem);
        return GB_BAD_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
        cudaGetLastError();
        gb::set_error("gust: zline_jacobi_noalloc: no usable current CUDA device");
        return GB_CUDA;
    }
    double* base = nullptr;
    if ((st = noalloc_setup(dev, &base)) != GB_OK) { return st; }
    double* next = base;
    unsigned long long* word = reinterpret_cast<unsigned long long*>(base + kNoAllocMaxPoints);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(delta, 0, sizeof(double) * vol, s);
    cudaMemsetAsync(word, 0, sizeof(unsigned long long), s);
    double* buf[2] = {delta, next};
    for (int k = 0; k < sweeps; ++k) {
        gb::LineArgs<double> a;
        a.g = *g;
        a.ni = ni;
        a.nj = nj;
        a.nk = nk;
        a.A = A;
        a.cs = vol;
        a.ap = ap;
        a.rhs = rhs;
        a.dold = buf[(sweeps - k) & 1];
        a.dnew = buf[(sweeps - 1 - k) & 1];
        a.cbuf = nullptr;
        a.ebuf = nullptr;
        a.first = (k == 0) ? 1 : 0;
        a.change = (k == sweeps - 1) ? word : nullptr;
        const dim3 grid((ni + NTHR - 1) / NTHR, nj);
        if (a.first) {
            gb::zline_pipe_kernel<double, true, R><<<grid, NTHR, smem_first, s>>>(a);
        } else {
            gb::zline_pipe_kernel<double, false, R><<<grid, NTHR, smem, s>>>(a);
        }
    }
    const bool sx = (loc & 1) && g->periodic_x, sy = ((loc >> 1) & 1) && g->periodic_y;
    if (sx || sy) {
        const int n = std::max(nj, ni) * nk;
        gb::seam_sync_kernel<double><<<(n + 255) / 256, 256, 0, s>>>(*g, loc, delta);
    }
    if ((st = gb::check_cuda(op)) != GB_OK) { return st; }
    if (change != nullptr) {
        unsigned long long w = 0;
        cudaMemcpyAsync(&w, word, sizeof(w), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) { return gb::check_cuda(op); }
        *change = gb::bits_to_double(w);
    }
    return GB_OK;
}
