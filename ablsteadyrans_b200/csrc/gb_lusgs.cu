// The line LU-SGS solve (gust::zline_lusgs with steady.line_ghosts = lagged,
// Source/LineSweeps.cpp:183-210, 415-428): `sweeps` symmetric passes of
// in-place z-line solves, each column solved with its x/y neighbours as they
// stand at that moment of the pass: the lower neighbours already updated in
// the pass's direction, the upper ones not; across a periodic seam the values
// the pass started from (FillBoundary before every pass).
//
// B200 mapping. Within a pass a column depends on the two columns before it
// in both directions, so the pass walks the wavefront planes
// (i - ilo) + (j - jlo) = s (the reference's diagonal order, which gives the
// values of its sequential order): no two columns of a plane are neighbours,
// so a plane's columns are solved in parallel, and the planes follow one
// another. The system is the same in every pass of a solve, so its column
// factors (1/m, c') are computed once, in parallel over all columns, and each
// column solve is division-free.
//
// The pass is ONE launch of one thread-block cluster (up to 8 CTAs, on as
// many SMs): each CTA takes 32 columns of the plane at a time, its warps
// splitting the column's levels into segments (the segmented recurrences of
// the z-line sweep: each warp's levels loaded at once, the values crossing a
// segment boundary carried through shared memory as composed affine maps),
// and the cluster's hardware barrier (barrier.cluster, release/acquire)
// separates the planes. The iterate is read through L2 (ld.global.cg), since
// other CTAs of the cluster wrote it on other SMs.
#include "gb_line.cuh"

#include <cooperative_groups.h>

#include <algorithm>

namespace cg = cooperative_groups;

namespace gb {

namespace {

enum LusgsSlot : int { kSlotLusgsInv = 16, kSlotLusgsCp, kSlotLusgsE, kSlotLusgsBefore };

struct LusgsArgs {
    gb_grid g;
    int ni, nj, nk;
    const double* __restrict__ A;  // 7 components, stride cs
    int64_t cs;
    const double* __restrict__ rhs;
    const double* __restrict__ inv;  // 1/m
    const double* __restrict__ cp;   // c'
    double* e;                       // forward recurrence scratch
    double* d;                       // the iterate, in place
};

//! The column factors of (-a_ZM, a_P, -a_ZP): m_0 = a_P,0, m_k = a_P,k +
//! a_ZM,k c'_{k-1}; 1/m_k and c'_k = -a_ZP,k / m_k. One thread per column.
__global__ void k_lusgs_factor(gb_grid g, int ni, int nj, int nk, const double* __restrict__ A, int64_t cs,
                               const double* __restrict__ ap, double* __restrict__ inv, double* __restrict__ cp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= ni || j >= nj) { return; }
    const int64_t o0 = at(g, i, j, 0);
    const double* azm = A + GB_COEF_ZM * cs;
    const double* azp = A + GB_COEF_ZP * cs;
    double c = 0;
    for (int k0 = 0; k0 < nk; k0 += 8) {
        double P[8], L[8], U[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (k0 + q < nk) {
                const int64_t o = o0 + static_cast<int64_t>(k0 + q) * g.sz;
                P[q] = ap[o];
                L[q] = -azm[o];
                U[q] = -azp[o];
            }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = k0 + q;
            if (k < nk) {
                const double m = (k == 0) ? P[q] : P[q] - L[q] * c;
                const double im = 1.0 / m;
                c = U[q] * im;
                const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
                inv[o] = im;
                cp[o] = c;
            }
        }
    }
}

//! FillBoundary of the ghost layer of d that the column solves read: the
//! periodic images of the x ghosts (valid j) and the y ghosts (valid i); the
//! corners are never read. Ghosts outside a non-periodic face stay 0.
__global__ void k_lusgs_images(gb_grid g, int ni, int nj, int nk, int per_x, int per_y, double* __restrict__ d)
{
    const int k = blockIdx.y;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) { return; }
    if (per_x && t < nj) {
        d[at(g, -1, t, k)] = d[at(g, g.nx - 1, t, k)];
        d[at(g, ni, t, k)] = d[at(g, ni - g.nx, t, k)];
    }
    if (per_y && t < ni) {
        d[at(g, t, -1, k)] = d[at(g, t, g.ny - 1, k)];
        d[at(g, t, nj, k)] = d[at(g, t, nj - g.ny, k)];
    }
}

//! One pass: the wavefront planes in order (ascending forward, descending
//! backward), one column per thread inside a plane, a block barrier between
//! planes. JREV: the j-reversed pair (planes (i - ilo) + (jhi - j) = s).
template <bool JREV>
__global__ void __launch_bounds__(256) k_lusgs_pass(LusgsArgs a, int forward)
{
    const gb_grid& g = a.g;
    const int last = a.ni + a.nj - 2;
    const double* axm = a.A + GB_COEF_XM * a.cs;
    const double* axp = a.A + GB_COEF_XP * a.cs;
    const double* aym = a.A + GB_COEF_YM * a.cs;
    const double* ayp = a.A + GB_COEF_YP * a.cs;
    const double* azm = a.A + GB_COEF_ZM * a.cs;
    const int64_t sy = g.sy;
    for (int q = 0; q <= last; ++q) {
        const int s = forward ? q : last - q;
        const int amin = max(0, s - (a.nj - 1)), amax = min(s, a.ni - 1);
        for (int m = threadIdx.x; m <= amax - amin; m += blockDim.x) {
            const int i = amin + m;
            const int j = JREV ? a.nj - 1 - (s - i) : s - i;
            const int64_t o0 = at(g, i, j, 0);
            double ep = 0;
            for (int k0 = 0; k0 < a.nk; k0 += 8) {
                double R[8], L[8], IM[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (k0 + r < a.nk) {
                        const int64_t o = o0 + static_cast<int64_t>(k0 + r) * g.sz;
                        R[r] = a.rhs[o] + axm[o] * a.d[o - 1] + axp[o] * a.d[o + 1] + aym[o] * a.d[o - sy]
                             + ayp[o] * a.d[o + sy];
                        L[r] = -azm[o];
                        IM[r] = a.inv[o];
                    }
                }
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const int k = k0 + r;
                    if (k < a.nk) {
                        ep = ((k == 0) ? R[r] : R[r] - L[r] * ep) * IM[r];
                        a.e[o0 + static_cast<int64_t>(k) * g.sz] = ep;
                    }
                }
            }
            double x = 0;
            for (int k1 = a.nk - 1; k1 >= 0; k1 -= 8) {
                double E[8], C[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (k1 - r >= 0) {
                        const int64_t o = o0 + static_cast<int64_t>(k1 - r) * g.sz;
                        E[r] = a.e[o];
                        C[r] = a.cp[o];
                    }
                }
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const int k = k1 - r;
                    if (k >= 0) {
                        x = (k == a.nk - 1) ? E[r] : E[r] - C[r] * x;
                        a.d[o0 + static_cast<int64_t>(k) * g.sz] = x;
                    }
                }
            }
        }
        __syncthreads();
    }
}

//! One pass as one cluster launch (see the file's header): planes in order
//! (ascending forward, descending backward), 32 columns per CTA at a time,
//! L levels per warp, a cluster barrier between planes. JREV: the j-reversed
//! pair. Shared memory: the carries of e' and x, [4][W][32].
template <bool JREV, int L>
__global__ void __launch_bounds__(512) k_lusgs_pass_cluster(LusgsArgs a, int forward)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = static_cast<int>(cluster.num_blocks());
    const int cta = static_cast<int>(cluster.block_rank());
    const gb_grid& g = a.g;
    const int lane = threadIdx.x, w = threadIdx.y, W = blockDim.y;
    const int cs = W * 32;
    const int me = w * 32 + lane;
    double* carry_e = reinterpret_cast<double*>(smem_raw);
    double* carry_x = carry_e + 2 * cs;
    const int k0 = w * L;
    const int nk = a.nk;
    const int last = a.ni + a.nj - 2;
    const double* axm = a.A + GB_COEF_XM * a.cs;
    const double* axp = a.A + GB_COEF_XP * a.cs;
    const double* aym = a.A + GB_COEF_YM * a.cs;
    const double* ayp = a.A + GB_COEF_YP * a.cs;
    const double* azm = a.A + GB_COEF_ZM * a.cs;
    const int64_t sy = g.sy;
    for (int q = 0; q <= last; ++q) {
        const int s = forward ? q : last - q;
        const int amin = max(0, s - (a.nj - 1)), amax = min(s, a.ni - 1);
        const int count = amax - amin + 1;
        for (int base = cta * 32; base < count; base += C * 32) {   // the same trip count for every thread of a CTA
            const int m = base + lane;
            const bool col = m < count;
            const int i = amin + m;
            const int j = JREV ? a.nj - 1 - (s - i) : s - i;
            const int64_t o0 = col ? at(g, i, j, 0) : 0;
            double R[L], LO[L], IM[L], CP[L];
#pragma unroll
            for (int r = 0; r < L; ++r) {
                const int k = k0 + r;
                R[r] = 0.0;
                LO[r] = 0.0;
                IM[r] = 0.0;
                CP[r] = 0.0;
                if (col && k < nk) {
                    const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
                    R[r] = a.rhs[o] + axm[o] * __ldcg(a.d + o - 1) + axp[o] * __ldcg(a.d + o + 1)
                         + aym[o] * __ldcg(a.d + o - sy) + ayp[o] * __ldcg(a.d + o + sy);
                    LO[r] = -azm[o];
                    IM[r] = a.inv[o];
                    CP[r] = a.cp[o];
                }
            }
            // e_k = (R_k - L_k e_{k-1}) / m_k: the segment's affine map
            double al = 0.0, be = 1.0;
#pragma unroll
            for (int r = 0; r < L; ++r) {
                const int k = k0 + r;
                if (k < nk) {
                    if (k == 0) {
                        al = R[r] * IM[r];
                        be = 0.0;
                    } else {
                        al = (R[r] - LO[r] * al) * IM[r];
                        be = (-LO[r] * be) * IM[r];
                    }
                }
            }
            carry_e[me] = al;
            carry_e[cs + me] = be;
            __syncthreads();
            double ep = 0.0;
            for (int t = 0; t < w; ++t) { ep = carry_e[t * 32 + lane] + carry_e[cs + t * 32 + lane] * ep; }
#pragma unroll
            for (int r = 0; r < L; ++r) {
                const int k = k0 + r;
                if (k < nk) {
                    ep = ((k == 0) ? R[r] : R[r] - LO[r] * ep) * IM[r];
                    R[r] = ep;
                }
            }
            // x_k = e_k - c'_k x_{k+1} (x_{nk-1} = e_{nk-1}): the segment's affine map from above
            double ga = 0.0, de = 1.0;
#pragma unroll
            for (int r = L - 1; r >= 0; --r) {
                const int k = k0 + r;
                if (k < nk) {
                    if (k == nk - 1) {
                        ga = R[r];
                        de = 0.0;
                    } else {
                        ga = R[r] - CP[r] * ga;
                        de = -CP[r] * de;
                    }
                }
            }
            carry_x[me] = ga;
            carry_x[cs + me] = de;
            __syncthreads();
            double x = 0.0;
            for (int t = W - 1; t > w; --t) { x = carry_x[t * 32 + lane] + carry_x[cs + t * 32 + lane] * x; }
#pragma unroll
            for (int r = L - 1; r >= 0; --r) {
                const int k = k0 + r;
                if (k < nk) {
                    x = (k == nk - 1) ? R[r] : R[r] - CP[r] * x;
                    if (col) { a.d[o0 + static_cast<int64_t>(k) * g.sz] = x; }
                }
            }
        }
        cluster.sync();
    }
}

//! max |b - d| over the valid points into a result word (rows of the box
//! over the warps, one atomic per block).
__global__ void __launch_bounds__(256) k_lusgs_change(gb_grid g, int ni, int nj, int nk, const double* __restrict__ b,
                                                      const double* __restrict__ d, unsigned long long* word)
{
    __shared__ double red[8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * 8 + warp;
    double v = 0;
    if (r < nj * nk) {
        const int64_t o0 = at(g, 0, r % nj, r / nj);
        for (int i = lane; i < ni; i += 32) {
            const double x = fabs(b[o0 + i] - d[o0 + i]);
            v = (x > v || x != x) ? x : v;
        }
    }
    v = warp_max_nan(v);
    if (lane == 0) { red[warp] = v; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < 8) ? red[threadIdx.x] : 0.0;
        t = warp_max_nan(t);
        if (threadIdx.x == 0) { atomic_max_nonneg(word, t); }
    }
}

}  // namespace

gb_status zline_lusgs(gb_ctx* ctx, const gb_grid& g, int loc, const double* A, const double* ap, const double* rhs,
                      int sweeps, int alternate, double* delta, unsigned long long* change_word)
{
    const int ni = ext_x(g, loc), nj = ext_y(g, loc), nk = ext_z(g, loc);
    const int64_t vol = volume(g);
    double* inv = static_cast<double*>(scratch(ctx, kSlotLusgsInv, sizeof(double) * vol));
    double* cp = static_cast<double*>(scratch(ctx, kSlotLusgsCp, sizeof(double) * vol));
    double* e = static_cast<double*>(scratch(ctx, kSlotLusgsE, sizeof(double) * vol));
    double* before = static_cast<double*>(scratch(ctx, kSlotLusgsBefore, sizeof(double) * vol));
    if (!inv || !cp || !e || !before) { return GB_OOM; }
    const bool per_x = g.periodic_x != 0, per_y = g.periodic_y != 0;
    {
        Span span(ctx, GB_KERNEL_LINE_SWEEP);
        k_lusgs_factor<<<dim3((ni + 31) / 32, (nj + 3) / 4), dim3(32, 4), 0, ctx->stream>>>(g, ni, nj, nk, A, vol, ap,
                                                                                         inv, cp);
        ++ctx->launches;
    }
    LusgsArgs a{g, ni, nj, nk, A, vol, rhs, inv, cp, e, delta};
    const int plane = std::min(ni, nj);
    const int nthr = std::min(256, std::max(32, (plane + 31) / 32 * 32));
    const int ext = std::max(ni, nj);
    // the cluster pass: 8 levels per warp (columns of at most 128 levels), a
    // CTA per 32 columns of the widest plane, at most 8 CTAs (the portable
    // cluster size); taller columns take the single-block pass
    const int cl_warps = ((nk + 7) / 8 <= 16 && ctx->tune[GB_TUNE_LINE_VARIANT] != 4) ? (nk + 7) / 8 : 0;
    const int cl_ctas = std::min(8, std::max(1, (plane + 31) / 32));
    if (change_word != nullptr) { cudaMemsetAsync(change_word, 0, sizeof(unsigned long long), ctx->stream); }
    for (int s = 0; s < sweeps; ++s) {
        const bool jrev = alternate && (s % 2 == 1);
        for (int forward = 1; forward >= 0; --forward) {
            if (s == sweeps - 1 && !forward && change_word != nullptr) {
                cudaMemcpyAsync(before, delta, sizeof(double) * vol, cudaMemcpyDeviceToDevice, ctx->stream);
            }
            Span span(ctx, GB_KERNEL_LINE_SWEEP);
            if (per_x || per_y) {
                k_lusgs_images<<<dim3((ext + 127) / 128, nk), 128, 0, ctx->stream>>>(g, ni, nj, nk, per_x, per_y,
                                                                                     delta);
                ++ctx->launches;
            }
            if (cl_warps > 0) {
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3(cl_ctas, 1, 1);
                cfg.blockDim = dim3(32, cl_warps, 1);
                cfg.dynamicSmemBytes = static_cast<size_t>(4) * cl_warps * 32 * sizeof(double);
                cfg.stream = ctx->stream;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = cl_ctas;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                if (jrev) {
                    cudaLaunchKernelEx(&cfg, k_lusgs_pass_cluster<true, 8>, a, static_cast<int>(forward));
                } else {
                    cudaLaunchKernelEx(&cfg, k_lusgs_pass_cluster<false, 8>, a, static_cast<int>(forward));
                }
            } else if (jrev) {
                k_lusgs_pass<true><<<1, nthr, 0, ctx->stream>>>(a, forward);
            } else {
                k_lusgs_pass<false><<<1, nthr, 0, ctx->stream>>>(a, forward);
            }
            ++ctx->launches;
        }
    }
    if (change_word != nullptr) {
        k_lusgs_change<<<(nj * nk + 7) / 8, 256, 0, ctx->stream>>>(g, ni, nj, nk, before, delta, change_word);
        ++ctx->launches;
    }
    seam_sync<double>(ctx, g, loc, delta);
    return check_cuda("zline_lusgs");
}

}  // namespace gb

extern "C" gb_status gb_zline_lusgs(gb_ctx* ctx, const gb_grid* g, int32_t loc, const double* A, const double* ap,
                                    const double* rhs, int32_t sweeps, int32_t alternate, double* delta,
                                    double* change)
{
    gb::clear_error();
    const char* op = "zline_lusgs";
    if (ctx == nullptr) {
        gb::set_error("gust: %s: ctx is null", op);
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_grid(op, g);
    if (st != GB_OK) { return st; }
    if ((st = gb::check_loc(op, loc)) != GB_OK) { return st; }
    if (sweeps < 1) {
        gb::set_error("gust: zline_lusgs: sweeps must be >= 1 (got %d)", sweeps);
        return GB_BAD_ARG;
    }
    if (alternate != 0 && alternate != 1) {
        gb::set_error("gust: zline_lusgs: steady.line_alternate = %d: must be 0 or 1", alternate);
        return GB_BAD_ARG;
    }
    if (A == nullptr || ap == nullptr || rhs == nullptr || delta == nullptr) {
        gb::set_error("gust: zline_lusgs: A, ap, rhs and delta must be device arrays of the grid");
        return GB_BAD_ARG;
    }
    // delta.setVal(0): ghosts outside the domain stay 0 (the couplings are folded)
    cudaMemsetAsync(delta, 0, sizeof(double) * gb::volume(*g), ctx->stream);
    st = gb::zline_lusgs(ctx, *g, loc, A, ap, rhs, sweeps, alternate, delta, gb::dword(ctx, 0));
    if (st != GB_OK) { return st; }
    unsigned long long w = 0;
    if ((st = gb::read_words(ctx, 0, 1, &w)) != GB_OK) { return st; }
    if (change != nullptr) { *change = gb::bits_to_double(w); }
    return GB_OK;
}
