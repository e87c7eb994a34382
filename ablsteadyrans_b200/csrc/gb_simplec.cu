// The SIMPLEC outer iteration on the GPU (gust::SimplecStage::iterate,
// Source/Simplec.cpp:452-506): boundary ghost fills (the wall law's ground
// gradient on a surface_layer ground), the FP64 residual (convection,
// full-stress terrain diffusion with the given diffusivities or the k-L
// closure's, the wall model's ground fluxes, pressure gradient, forcing,
// continuity, the k sources and wall-k rows), the implicit rows, the momentum
// predictor with z-line sweeps, the pressure correction through the Poisson
// layer, the theta and k sweeps and the stage norms. Every reduction is
// deterministic (block partials summed in a fixed order, maxima by bit
// pattern), so a run repeats to the bit.
#include "gb_line.cuh"
#include "gb_poisson_api.cuh"
#include "gb_simplec.cuh"
#include "gb_stencil.cuh"
#include "gb_turbulence.cuh"

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>

namespace gb {

using namespace st;

namespace {

enum { R_EVEN = 0, R_ODD, R_VALUE, R_PROFILE, R_GRADIENT };
enum { F_U = 0, F_V, F_W, F_P, F_THETA, F_TKE };

constexpr int kRedBlocks = 512;
//! The result word that counts the ground columns without a positive, finite u*.
constexpr int W_SURFACE_BAD = 40;
constexpr int W_CONF_BAD = 41, W_CONF_TOP = 42;   // the confidence test's count and height

// ------------------------------------------------------------- heights ---

__device__ __forceinline__ double node_z(const double* __restrict__ z, const gb_grid& g, int i, int j, int k)
{
    const int lo = -1, hix = g.nx + 1, hiy = g.ny + 1, hiz = g.nz + 1;
    i = i < lo ? lo : (i > hix ? hix : i);
    j = j < lo ? lo : (j > hiy ? hiy : j);
    if (k < lo) { return z[at(g, i, j, lo)] + (lo - k) * (z[at(g, i, j, lo)] - z[at(g, i, j, lo + 1)]); }
    if (k > hiz) { return z[at(g, i, j, hiz)] + (k - hiz) * (z[at(g, i, j, hiz)] - z[at(g, i, j, hiz - 1)]); }
    return z[at(g, i, j, k)];
}

//! Height of point (i, j, k) of type t above its column's ground (Heights_K.H:40-56).
__device__ __forceinline__ double height_above_ground(const double* z, const gb_grid& g, int t, int i, int j, int k)
{
    const int nx = nodal(t, 0) ? 1 : 2, ny = nodal(t, 1) ? 1 : 2, nz = nodal(t, 2) ? 1 : 2;
    double zp = 0, zg = 0;
    for (int a = 0; a < nx; ++a) {
        for (int b = 0; b < ny; ++b) {
            zg += node_z(z, g, i + a, j + b, 0);
            for (int c = 0; c < nz; ++c) { zp += node_z(z, g, i + a, j + b, k + c); }
        }
    }
    return zp / (nx * ny * nz) - zg / (nx * ny);
}

//! Node-mean height of point (i, j, k) of type t (Heights_K.H:60-71).
__device__ __forceinline__ double point_z(const double* z, const gb_grid& g, int t, int i, int j, int k)
{
    const int nx = nodal(t, 0) ? 1 : 2, ny = nodal(t, 1) ? 1 : 2, nz = nodal(t, 2) ? 1 : 2;
    double zp = 0;
    for (int a = 0; a < nx; ++a) {
        for (int b = 0; b < ny; ++b) {
            for (int c = 0; c < nz; ++c) { zp += node_z(z, g, i + a, j + b, k + c); }
        }
    }
    return zp / (nx * ny * nz);
}

//! The log-law inflow profile's value of field f at height h (InflowProfile.H eval).
struct Profile {
    double ustar, z0, kappa, Cmu0, inv_lmax, cosd, sind;
    int rn;
    double rz[GB_MAX_PROFILE], rt[GB_MAX_PROFILE];
    __device__ double value(int f, double h) const
    {
        h = fmax(h, 0.0);
        const double c = 1.0 / (1.0 + kappa * (h + z0) * inv_lmax);
        const double S = ustar / kappa * log((h + z0) / z0);
        const double ul = ustar * c;
        switch (f) {
        case F_U: return S * cosd;
        case F_V: return S * sind;
        case F_THETA: {
            if (rn == 1 || h <= rz[0]) { return rt[0]; }
            if (h >= rz[rn - 1]) { return rt[rn - 1]; }
            int m = 1;
            while (m < rn - 1 && !(h < rz[m])) { ++m; }
            const double w = (h - rz[m - 1]) / (rz[m] - rz[m - 1]);
            return rt[m - 1] + w * (rt[m] - rt[m - 1]);
        }
        case F_TKE: return ul * ul / (Cmu0 * Cmu0);
        default: return 0;
        }
    }
};

int rule_for(int f, int t, int d, bool lo)
{
    const bool normal_vel = (f == F_U && d == 0) || (f == F_V && d == 1) || (f == F_W && d == 2);
    const bool vel = (f == F_U || f == F_V || f == F_W);
    switch (t) {
    case GB_FACE_INFLOW: return (f == F_P) ? R_EVEN : R_PROFILE;
    case GB_FACE_OUTFLOW: return (f == F_P) ? R_ODD : R_EVEN;
    case GB_FACE_SLIP_WALL:
        if (normal_vel) { return R_VALUE; }
        return (f == F_THETA && d == 2 && !lo) ? R_GRADIENT : R_EVEN;
    case GB_FACE_NO_SLIP_WALL: return vel ? R_VALUE : R_EVEN;
    case GB_FACE_SURFACE_LAYER:
        if (normal_vel) { return R_VALUE; }
        return (vel || f == F_THETA) ? R_GRADIENT : R_EVEN;
    default: return R_EVEN;
    }
}

bool dirichlet_normal(const gb_bc& bc, int face)
{
    const int t = bc.face[face];
    return t == GB_FACE_INFLOW || t == GB_FACE_SLIP_WALL || t == GB_FACE_NO_SLIP_WALL || t == GB_FACE_SURFACE_LAYER;
}

inline bool is_per(const gb_grid& g, int d) { return d == 0 ? g.periodic_x : d == 1 ? g.periodic_y : false; }
const int kLoc[6] = {XF, YF, ZF, CC, CC, CC};

// ------------------------------------------------------ deterministic sums ---

__global__ void k_sumsq_partial(gb_grid g, Box b, const double* __restrict__ f, double* __restrict__ partial, int mode)
{
    // mode 0: sum of squares, 1: sum
    __shared__ double red[8];
    double s = 0;
    const int64_t n_tot = b.count();
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
    for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < n_tot;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int i = b.lo[0] + static_cast<int>(n % nx);
        const int j = b.lo[1] + static_cast<int>((n / nx) % ny);
        const int k = b.lo[2] + static_cast<int>(n / (static_cast<int64_t>(nx) * ny));
        const double v = f[at(g, i, j, k)];
        s += (mode == 0) ? v * v : v;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = s; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < 8) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) { partial[blockIdx.x] = t; }
    }
}

__global__ void k_sum_partials(const double* __restrict__ partial, int n, double* __restrict__ out)
{
    __shared__ double red[8];
    double s = 0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) { s += partial[t]; }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = s; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < 8) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) { *out = t; }
    }
}

//! The mean of f over one k-plane of box b per block (block k: level k),
//! summed in a fixed order (Predictor.cpp:286-306: the horizontal mean of the
//! other component's residual per level, every face once).
//! One block per level (blockDim.x = kLevelThreads): each thread sums its
//! points in four independent partial sums (loads in flight together, a
//! fixed order), then the block reduces them in a fixed tree.
constexpr int kLevelThreads = 1024;

__global__ void __launch_bounds__(kLevelThreads) k_level_mean(gb_grid g, Box b, const double* __restrict__ f,
                                                              double npts_level, double* __restrict__ mean)
{
    __shared__ double red[kLevelThreads / 32];
    const int k = blockIdx.x;
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
    const int np = nx * ny;
    double s4[4] = {0, 0, 0, 0};
    for (int n0 = threadIdx.x; n0 < np; n0 += 4 * kLevelThreads) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int n = n0 + u * kLevelThreads;
            if (n < np) { s4[u] += f[at(g, b.lo[0] + n % nx, b.lo[1] + n / nx, k)]; }
        }
    }
    double s = (s4[0] + s4[1]) + (s4[2] + s4[3]);
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = s; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = red[threadIdx.x];
        t = warp_sum(t);
        if (threadIdx.x == 0) { mean[k] = t / npts_level; }
    }
}

__global__ void __launch_bounds__(256) k_maxabs(gb_grid g, Box b, const double* __restrict__ f,
                                                const double* __restrict__ mul, unsigned long long* __restrict__ slot)
{
    // one warp per row (j, k) of the box, the lanes over i (a row's loads all
    // in flight at once); a block max, then one atomic per block (one per
    // warp on a single word serialises)
    __shared__ double red[8];
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + warp;
    double v = 0;
    if (r < ny * nz) {
        const int64_t o0 = at(g, b.lo[0], b.lo[1] + r % ny, b.lo[2] + r / ny);
#pragma unroll 4
        for (int i = lane; i < nx; i += 32) {
            const double a = fabs(mul ? f[o0 + i] * mul[o0 + i] : f[o0 + i]);
            v = (a > v || a != a) ? a : v;
        }
    }
    v = warp_max_nan(v);
    if (lane == 0) { red[warp] = v; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        t = warp_max_nan(t);
        if (threadIdx.x == 0) { atomic_max_nonneg(slot, t); }
    }
}

//! Several reductions in one launch (blockIdx.y picks the item): each item
//! reduces exactly as its single launch does (the same blocks, threads and
//! order), so the sums are the same bits.
constexpr int kMaxRed = 8;
struct RedItem {
    Box b;
    const double* f;
    const double* mul;
    int mode;   // sums: 0 squares, 1 values
    int slot;   // sums: the result slot; maxima: the result word
};
struct RedPack {
    RedItem it[kMaxRed];
    int n;
};

__global__ void k_sumsq_partial_many(gb_grid g, const __grid_constant__ RedPack P, double* __restrict__ partial)
{
    pdl_entry();
    const RedItem& it = P.it[blockIdx.y];
    const Box b = it.b;
    const double* __restrict__ f = it.f;
    const int mode = it.mode;
    __shared__ double red[8];
    double s = 0;
    const int64_t n_tot = b.count();
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
    for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < n_tot;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int i = b.lo[0] + static_cast<int>(n % nx);
        const int j = b.lo[1] + static_cast<int>((n / nx) % ny);
        const int k = b.lo[2] + static_cast<int>(n / (static_cast<int64_t>(nx) * ny));
        const double v = f[at(g, i, j, k)];
        s += (mode == 0) ? v * v : v;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = s; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < 8) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) { partial[it.slot * gridDim.x + blockIdx.x] = t; }
    }
}

__global__ void k_sum_partials_many(const __grid_constant__ RedPack P, const double* __restrict__ partial, int nb,
                                    double* __restrict__ out)
{
    pdl_entry();
    const int slot = P.it[blockIdx.x].slot;
    __shared__ double red[8];
    double s = 0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) { s += partial[slot * nb + t]; }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = s; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < 8) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) { out[slot] = t; }
    }
}

__global__ void __launch_bounds__(256) k_maxabs_many(gb_grid g, const __grid_constant__ RedPack P,
                                                     unsigned long long* __restrict__ words)
{
    pdl_entry();
    const RedItem& it = P.it[blockIdx.y];
    const Box b = it.b;
    const double* __restrict__ f = it.f;
    const double* __restrict__ mul = it.mul;
    __shared__ double red[8];
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + warp;
    double v = 0;
    if (r < ny * nz) {
        const int64_t o0 = at(g, b.lo[0], b.lo[1] + r % ny, b.lo[2] + r / ny);
#pragma unroll 4
        for (int i = lane; i < nx; i += 32) {
            const double a = fabs(mul ? f[o0 + i] * mul[o0 + i] : f[o0 + i]);
            v = (a > v || a != a) ? a : v;
        }
    }
    v = warp_max_nan(v);
    if (lane == 0) { red[warp] = v; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        t = warp_max_nan(t);
        if (threadIdx.x == 0) { atomic_max_nonneg(words + it.slot, t); }
    }
}

}  // namespace

// ================================================================ host ===

struct SimplecWork {
    double* R[6];
    double* F[3];
    double* G[9];
    double* Gd[9];   // the momentum diffusive fluxes, component C through its faces along D at [3 C + D]
    double* tmp;
    double* A;
    double* At;
    double* ap[3];
    double* dd[3];
    double* mask;
    double* rhs;
    double* delta;
    double* dtf[3];
    double* beta[3];
    double* keep[3];
    double* phi;
    double* om;
    double* theta_ref;
    double* conv0;
    double* conv1;
    double* og;
    double* level_sum;
    double* partial;
    double* sums;
    float* A32;
    float* ap32;
    float* rhs32;
    float* delta32;
    // per system of the batched line solves (index 0 = A, rhs, delta, and the FP32 arrays above)
    double* Am[3];
    double* rhsm[3];
    double* deltam[3];
    float* A32m[3];
    float* ap32m[3];
    float* rhs32m[3];
    float* delta32m[3];
};

}  // namespace gb

struct gb_simplec {
    gb_ctx* ctx{nullptr};
    gb_grid g{};
    gb_bc bc{};
    gb_physics ph{};
    gb_simplec_opts opt{};
    gb_mesh_fields mesh{};
    gb_diffusivities df{};
    // the diffusivities the stencils read: df, or the closure's fields
    // (0 before the first residual: the first local dtau's, Simplec.cpp:328)
    gb_diffusivities dfe{};
    bool wall{false};                    // bc.zlo = surface_layer
    double* cf[gb::kClosureFields]{};    // the closure's fields at the last residual
    double* dist{nullptr};               // the cells' height above the ground (closure)
    // nu the next local dtau reads: the closure's of the last iteration's
    // residual (SimplecStage::nu, Simplec.H:214; 0 before the first)
    double* nu_dtau{nullptr};
    double* agl{nullptr};                // height above the ground for the confidence test (made on first use)
    // the closure's nu_t history (Closure::accept, Closure.cpp:471-479): the
    // nu_t of the last iteration's residual, blended by turb.nut_relax < 1
    double* nut_hist{nullptr};
    bool has_hist{false};
    double* ss[gb::kSsPlanes]{};         // the surface state of the iteration's first fill
    double* ssr[gb::kSsPlanes]{};        // the residual's own surface state
    double* sst[gb::kSsPlanes]{};        // the later fills' surface state
    double* gg[3]{};                     // the wall law's ground gradient (u, v, theta)
    const double* z{nullptr};
    gb::SimplecWork w{};
    gb::Profile prof{};
    gb_poisson* poisson{nullptr};
    gb_poisson* init_poisson{nullptr};  // the initializer's projection (its own BC), made on use
    double jmin{0};
    std::vector<void*> owned;
    unsigned long long* h_words{nullptr};
    // The iteration's two launch sequences without a host synchronisation
    // (before and after the Krylov solve of the pressure correction) as CUDA
    // graphs: captured on the stage's own stream on an iteration after the
    // first, launched on the context's stream, rebuilt when what their kernels'
    // arguments depend on changes (the state and dtau pointers, the nu_t
    // history's presence, the tuning knobs).
    // the Newton stage's SIMPLEC preconditioner (simplec_linear_setup/apply),
    // allocated on first use: the increment state, q + sigma du, the transport
    // at q and at q + sigma du, theta's convection at q, the setup's cell step
    double* lin_d[6]{};
    double* lin_qn[6]{};
    double* lin_F0[3]{};
    double* lin_F1[3]{};
    double* lin_conv0{nullptr};
    double* lin_dtau{nullptr};
    double lin_speed{1};
    bool lin_ready{false};
    cudaStream_t capture_stream{nullptr};
    cudaGraphExec_t seg_exec[2]{nullptr, nullptr};
    int64_t seg_launches[2]{0, 0};
    uint64_t seg_key[2]{0, 0};
    int iterations{0};
    ~gb_simplec();
};

gb_simplec::~gb_simplec()
{
    if (poisson) { gb_poisson_destroy(poisson); }
    if (init_poisson) { gb_poisson_destroy(init_poisson); }
    for (void* p : owned) { cudaFree(p); }
}

namespace gb {

namespace {

double* dbuf(gb_simplec* S, int64_t n)
{
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * std::max<int64_t>(n, 1)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    // zeroed on the stage's stream: ordered before the stage's kernels (a plain
    // cudaMemset is not ordered against non-blocking streams)
    cudaMemsetAsync(p, 0, sizeof(double) * std::max<int64_t>(n, 1), S->ctx->stream);
    S->owned.push_back(p);
    return static_cast<double*>(p);
}

float* fbuf(gb_simplec* S, int64_t n)
{
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(float) * std::max<int64_t>(n, 1)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaMemsetAsync(p, 0, sizeof(float) * std::max<int64_t>(n, 1), S->ctx->stream);
    S->owned.push_back(p);
    return static_cast<float*>(p);
}

// --------------------------------------------------------- reductions ---

//! Sum (mode 1) or sum of squares (mode 0) of f over box b into S->w.sums[slot].
void dsum(gb_simplec* S, const Box& b, const double* f, int mode, int slot)
{
    gb_ctx* ctx = S->ctx;
    Span span(ctx, GB_KERNEL_VECTOR);
    k_sumsq_partial<<<kRedBlocks, 256, 0, ctx->stream>>>(S->g, b, f, S->w.partial + slot * kRedBlocks, mode);
    k_sum_partials<<<1, 256, 0, ctx->stream>>>(S->w.partial + slot * kRedBlocks, kRedBlocks, S->w.sums + slot);
    ctx->launches += 2;
}

//! max |f (* mul)| over box b into result word `word` of the context (bits).
void dmax(gb_simplec* S, const Box& b, const double* f, const double* mul, int word)
{
    gb_ctx* ctx = S->ctx;
    const int rows = (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
    Span span(ctx, GB_KERNEL_VECTOR);
    k_maxabs<<<std::max(1, (rows + 7) / 8), 256, 0, ctx->stream>>>(S->g, b, f, mul, dword(ctx, word));
    ++ctx->launches;
}

//! dsum of several arrays in two launches (the items' slots into w.sums).
void dsum_many(gb_simplec* S, const RedPack& P)
{
    gb_ctx* ctx = S->ctx;
    if (P.n <= 0) { return; }
    Span span(ctx, GB_KERNEL_VECTOR);
    const bool pdl = ctx->tune[GB_TUNE_PDL] != 1;
    launch_pdl(pdl, k_sumsq_partial_many, dim3(kRedBlocks, P.n), dim3(256), 0, ctx->stream, S->g, P, S->w.partial);
    launch_pdl(pdl, k_sum_partials_many, dim3(P.n), dim3(256), 0, ctx->stream, P,
               static_cast<const double*>(S->w.partial), static_cast<int>(kRedBlocks), S->w.sums);
    ctx->launches += 2;
}

//! dmax of several arrays in one launch (the items' slots are result words).
void dmax_many(gb_simplec* S, const RedPack& P)
{
    gb_ctx* ctx = S->ctx;
    if (P.n <= 0) { return; }
    int rows = 1;
    for (int q = 0; q < P.n; ++q) {
        const Box& b = P.it[q].b;
        rows = std::max(rows, (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1));
    }
    Span span(ctx, GB_KERNEL_VECTOR);
    launch_pdl(ctx->tune[GB_TUNE_PDL] != 1, k_maxabs_many, dim3((rows + 7) / 8, P.n), dim3(256), 0, ctx->stream,
               S->g, P, dword(ctx, 0));
    ++ctx->launches;
}

//! A reduction item.
RedItem red_item(const Box& b, const double* f, const double* mul, int mode, int slot)
{
    RedItem it{};
    it.b = b;
    it.f = f;
    it.mul = mul;
    it.mode = mode;
    it.slot = slot;
    return it;
}

//! The three velocity components' max |.| into words w0, w0 + 1, w0 + 2.
void dmax_velocity(gb_simplec* S, const double* u, const double* v, const double* w, int w0)
{
    const gb_grid& g = S->g;
    RedPack P{};
    P.it[0] = red_item(valid_box(g, XF), u, nullptr, 0, w0);
    P.it[1] = red_item(valid_box(g, YF), v, nullptr, 0, w0 + 1);
    P.it[2] = red_item(valid_box(g, ZF), w, nullptr, 0, w0 + 2);
    P.n = 3;
    dmax_many(S, P);
}

// ---------------------------------------------------------- ghost fills ---

struct FieldPtrs {
    double* p[6];
    int t[6];
    int n;
};
struct FieldFill {
    double* a;
    int t, f, rule;
    double V;
    const double* gg;   // the wall law's gradient per column (null: the constant G)
};
struct FillPack {
    FieldFill F[6];
};
struct FillPack2 {
    FieldFill F[2][6];   // per side of the launch
};

//! FillBoundary of the lateral ghosts (two layers) of every field for the
//! periodic directions: x over the valid y and z, then y over the x ghosts.
void fill_periodic_all(gb_simplec* S, double* const* f, const int* t, int nf)
{
    const gb_grid g = S->g;
    const int ng = g.ng;
    FieldPtrs P{};
    for (int n = 0; n < nf; ++n) {
        P.p[n] = f[n];
        P.t[n] = t[n];
    }
    P.n = nf;
    if (g.periodic_x) {
        Box b{{0, 0, 0}, {2 * ng - 1, g.ny, g.nz}};
        for_box(S->ctx, b, [=] __device__(int l2, int j, int k) {
            const int l = (l2 % ng) + 1;
            const bool hi = l2 >= ng;
            for (int n = 0; n < P.n; ++n) {
                const int t = P.t[n];
                const int nvx = g.nx + (t & 1), nvy = g.ny + ((t >> 1) & 1), nvz = g.nz + ((t >> 2) & 1);
                if (j >= nvy || k >= nvz) { continue; }
                double* a = P.p[n];
                if (!hi) { a[at(g, -l, j, k)] = a[at(g, g.nx - l, j, k)]; }
                else { a[at(g, nvx - 1 + l, j, k)] = a[at(g, nvx - 1 + l - g.nx, j, k)]; }
            }
        }, GB_KERNEL_BC);
    }
    if (g.periodic_y) {
        const int ilo = g.periodic_x ? -ng : 0;
        Box b{{ilo, 0, 0}, {g.nx + ng, 2 * ng - 1, g.nz}};
        const bool px = g.periodic_x;
        for_box(S->ctx, b, [=] __device__(int i, int l2, int k) {
            const int l = (l2 % ng) + 1;
            const bool hi = l2 >= ng;
            for (int n = 0; n < P.n; ++n) {
                const int t = P.t[n];
                const int nvx = g.nx + (t & 1), nvy = g.ny + ((t >> 1) & 1), nvz = g.nz + ((t >> 2) & 1);
                const int ihi = px ? nvx - 1 + ng : nvx - 1;
                if (i > ihi || k >= nvz) { continue; }
                double* a = P.p[n];
                if (!hi) { a[at(g, i, -l, k)] = a[at(g, i, g.ny - l, k)]; }
                else { a[at(g, i, nvy - 1 + l, k)] = a[at(g, i, nvy - 1 + l - g.ny, k)]; }
            }
        }, GB_KERNEL_BC);
    }
}

//! The face fills of every field along d on one side (fill_face / fill_gradient_z,
//! BoundaryConditions.cpp:418-517), fields in the reference's order. homog:
//! the homogeneous fill of an increment (every boundary value, inflow
//! profile and gradient taken as 0, BoundaryConditions.cpp:421-517).
void fill_side(gb_simplec* S, const gb_state& q, int d, int sides, bool homog = false)
{
    const gb_grid g = S->g;
    const int ng = g.ng;
    // the sides this launch fills: bit 0 the low side, bit 1 the high side
    int nsides = 0;
    bool side_lo[2] = {true, false};
    FillPack2 P{};
    double* arr[6] = {q.u, q.v, q.w, q.p, q.theta, q.tke};
    for (int sd = 0; sd < 2; ++sd) {
        if (!(sides & (1 << sd))) { continue; }
        const bool lo = (sd == 0);
        const int face = d + (lo ? 0 : 3);
        const int ft = S->bc.face[face];
        for (int f = 0; f < 6; ++f) {
            FieldFill& F = P.F[nsides][f];
            F.a = arr[f];
            F.t = kLoc[f];
            F.f = f;
            F.rule = rule_for(f, ft, d, lo);
            F.V = (ft == GB_FACE_NO_SLIP_WALL && f <= F_W && !homog) ? S->bc.wall_velocity[face][f] : 0.0;
            F.gg = nullptr;
            if (ft == GB_FACE_SURFACE_LAYER && F.rule == R_GRADIENT && !homog) {
                F.gg = S->gg[f == F_U ? 0 : f == F_V ? 1 : 2];
            }
        }
        side_lo[nsides] = lo;
        ++nsides;
    }
    if (nsides == 0) { return; }
    const bool lo0 = side_lo[0], lo1 = side_lo[1];
    const Profile prof = S->prof;
    const double* z = S->z;
    const double G = homog ? 0.0 : S->bc.zhi_theta_grad;
    const int per[3] = {g.periodic_x, g.periodic_y, 0};
    // union box over the slab: layers 0..ng along d, the grown extents elsewhere
    Box b{};
    for (int e = 0; e < 3; ++e) {
        if (e == d) { continue; }
        const bool grow = (e < d) || per[e];
        b.lo[e] = grow ? -ng : 0;
        b.hi[e] = ((e == 0) ? g.nx : (e == 1) ? g.ny : g.nz) + (grow ? ng : 0);
    }
    // one thread per (point, field, side): the fields' fills are independent
    // (each reads only its own array), and so are the two sides' (they write
    // and read disjoint points: the caller merges them only when the extent
    // along d is at least 2 ng + 2); the layer index along d carries the
    // field and the side (layer + (ng + 1) (field + 6 side))
    b.lo[d] = 0;
    b.hi[d] = nsides * 6 * (ng + 1) - 1;
    const int pe0 = per[0], pe1 = per[1];
    // launched with the (layer, field, side) index slowest: a warp then takes
    // one field's rule on one side along a row of the slab (for d = 0 the
    // rows run along y), not twelve rules in turn
    const int q0 = (d == 0) ? 1 : 0, q1 = (d == 2) ? 1 : 2;
    const Box pb{{b.lo[q0], b.lo[q1], b.lo[d]}, {b.hi[q0], b.hi[q1], b.hi[d]}};
    for_box(S->ctx, pb, [=] __device__(int a0, int a1, int a2) {
        int c[3];
        c[q0] = a0;
        c[q1] = a1;
        c[d] = a2;
        const int fs = c[d] / (ng + 1);
        c[d] -= fs * (ng + 1);
        const int sd = fs / 6, n = fs % 6;
        const bool lo = (sd == 0) ? lo0 : lo1;
        const int layer = c[d];
        const int i = c[0], j = c[1], k = c[2];
        {
            const FieldFill& F = P.F[sd][n];
            const int t = F.t;
            // this field's slab extent in the other directions
            bool inside = true;
            for (int e = 0; e < 3 && inside; ++e) {
                if (e == d) { continue; }
                const bool grow = (e < d) || (e == 0 ? pe0 : (e == 1 ? pe1 : 0));
                const int nv = ((e == 0) ? g.nx : (e == 1) ? g.ny : g.nz) + nodal(t, e);
                const int lo_e = grow ? -ng : 0, hi_e = nv - 1 + (grow ? ng : 0);
                if (c[e] < lo_e || c[e] > hi_e) { inside = false; }
            }
            if (!inside) { return; }
            const int nd = (d == 0) ? g.nx : (d == 1) ? g.ny : g.nz;
            const bool nod = nodal(t, d);
            double* a = F.a;
            if (F.rule == R_GRADIENT) {
                // the top or a surface_layer ground (d == 2): one thread per column does both layers
                if (layer != 1) { return; }
                const int edge = lo ? 0 : nd - 1 + nod;
                const int c1 = lo ? edge + 1 : edge - 1, g1 = lo ? edge - 1 : edge + 1, g2 = lo ? edge - 2 : edge + 2;
                const double zc1 = point_z(z, g, t, i, j, c1), zg1 = point_z(z, g, t, i, j, g1),
                             zg2 = point_z(z, g, t, i, j, g2);
                const double Gp = F.gg ? ground_gradient_at(g, F.gg, t, i, j) : G;
                const double v1 = a[at(g, i, j, c1)] + (zg1 - zc1) * Gp;
                a[at(g, i, j, g1)] = v1;
                a[at(g, i, j, g2)] = v1 + (zg2 - zg1) * Gp;
                return;
            }
            const int edge = lo ? 0 : (nod ? nd : nd - 1);
            if (layer == 0) {
                if (!(nod && (F.rule == R_VALUE || F.rule == R_PROFILE))) { return; }
                int p[3] = {i, j, k};
                p[d] = edge;
                a[at(g, p[0], p[1], p[2])] = (F.rule == R_PROFILE && !homog)
                    ? prof.value(F.f, height_above_ground(z, g, t, p[0], p[1], p[2])) : F.V;
                return;
            }
            const int gidx = lo ? edge - layer : edge + layer;
            const int mirror = nod ? 2 * edge : (lo ? 2 * edge - 1 : 2 * edge + 1);
            int p[3] = {i, j, k}, s[3] = {i, j, k};
            p[d] = gidx;
            s[d] = mirror - gidx;
            double* dst = &a[at(g, p[0], p[1], p[2])];
            if (F.rule == R_PROFILE) {
                *dst = homog ? 0.0 : prof.value(F.f, height_above_ground(z, g, t, p[0], p[1], p[2]));
            } else if (F.rule == R_VALUE) {
                *dst = 2 * F.V - a[at(g, s[0], s[1], s[2])];
            } else {
                const double v = a[at(g, s[0], s[1], s[2])];
                *dst = (F.rule == R_ODD) ? -v : v;
            }
        }
    }, GB_KERNEL_BC);
}

//! fill_no_flux_w (BoundaryConditions.cpp:754-799).
void fill_no_flux_w(gb_simplec* S, const gb_state& q)
{
    const gb_grid g = S->g;
    const bool lo_on = dirichlet_normal(S->bc, 2), hi_on = dirichlet_normal(S->bc, 5);
    if (!lo_on && !hi_on) { return; }
    double* w = q.w;
    const double* u = q.u;
    const double* v = q.v;
    const double* z = S->z;
    const int ng = g.ng;
    Box b{{-1, -1, 0}, {g.nx, g.ny, 1}};
    for_box(S->ctx, b, [=] __device__(int i, int j, int side) {
        const bool lo = (side == 0);
        if ((lo && !lo_on) || (!lo && !hi_on)) { return; }
        const int face = lo ? 0 : g.nz;
        const int sgn = lo ? -1 : 1;
        const double V = deriv<NODE, ZF, 0>(z, g, i, j, face) * (1.0 / g.dx) * interp<XF, ZF>(u, g, i, j, face)
                       + deriv<NODE, ZF, 1>(z, g, i, j, face) * (1.0 / g.dy) * interp<YF, ZF>(v, g, i, j, face);
        w[at(g, i, j, face)] = V;
        for (int m = 1; m <= ng; ++m) { w[at(g, i, j, face + sgn * m)] = 2 * V - w[at(g, i, j, face - sgn * m)]; }
    }, GB_KERNEL_BC);
}

}  // namespace

//! BoundaryConditions::fill_ghosts (BoundaryConditions.cpp:597-663); a
//! surface_layer ground: the surface state from the laterally filled state
//! into ss and the wall law's gradient for the ground fills.
void fill_ghosts_into(gb_simplec* S, const gb_state& q, double* const* ss, bool homog = false)
{
    double* f[6] = {q.u, q.v, q.w, q.p, q.theta, q.tke};
    fill_periodic_all(S, f, kLoc, 6);
    for (int d = 0; d < 3; ++d) {
        if (d == 2 && S->wall && !homog) {
            turb_surface_state(S->ctx, S->g, S->bc, S->ph, q, S->z, S->mesh.z0, ss, dword(S->ctx, W_SURFACE_BAD));
            turb_ground_gradients(S->ctx, S->g, S->bc, ss, S->mesh.z0, S->gg);
        }
        if (is_per(S->g, d)) { continue; }
        const int nd = (d == 0) ? S->g.nx : (d == 1) ? S->g.ny : S->g.nz;
        if (nd >= 2 * S->g.ng + 2) {
            fill_side(S, q, d, 3, homog);
        } else {
            fill_side(S, q, d, 1, homog);
            fill_side(S, q, d, 2, homog);
        }
        if (d == 2) {
            // the no-flux w faces after u, v, w (p, theta, k do not read w)
            fill_no_flux_w(S, q);
        }
    }
    fill_periodic_all(S, f, kLoc, 6);
}

void simplec_fill_ghosts(gb_simplec* S, const gb_state& q) { fill_ghosts_into(S, q, S->ss); }

// ------------------------------------------------------------ stencils ---

namespace {

//! transport_fluxes (MassFlux.cpp:101-127): a_x u, a_y v, Omega, valid + one ghost.
void transport_fluxes(gb_simplec* S, const gb_state& q, double* F0, double* F1, double* F2)
{
    const gb_grid g = S->g;
    const double* u = q.u;
    const double* v = q.v;
    const double* w = q.w;
    const double* ax = S->mesh.ax;
    const double* ay = S->mesh.ay;
    const double* z = S->z;
    for_box(S->ctx, Box{{-1, -1, -1}, {g.nx + 1, g.ny + 1, g.nz + 1}}, [=] __device__(int i, int j, int k) {
        if (k <= g.nz) {
            if (j <= g.ny) { F0[at(g, i, j, k)] = ax[at(g, i, j, k)] * u[at(g, i, j, k)]; }
            if (i <= g.nx) { F1[at(g, i, j, k)] = ay[at(g, i, j, k)] * v[at(g, i, j, k)]; }
        }
        if (i <= g.nx && j <= g.ny) {
            F2[at(g, i, j, k)] = w[at(g, i, j, k)]
                               - deriv<NODE, ZF, 0>(z, g, i, j, k) * (1.0 / g.dx) * interp<XF, ZF>(u, g, i, j, k)
                               - deriv<NODE, ZF, 1>(z, g, i, j, k) * (1.0 / g.dy) * interp<YF, ZF>(v, g, i, j, k);
        }
    }, GB_KERNEL_MASSFLUX);
}

//! omega_from_w on the valid z-faces.
void omega_from_w(gb_simplec* S, const double* u, const double* v, const double* w, double* om)
{
    const gb_grid g = S->g;
    const double* z = S->z;
    for_box(S->ctx, valid_box(g, ZF), [=] __device__(int i, int j, int k) {
        om[at(g, i, j, k)] = w[at(g, i, j, k)]
                           - deriv<NODE, ZF, 0>(z, g, i, j, k) * (1.0 / g.dx) * interp<XF, ZF>(u, g, i, j, k)
                           - deriv<NODE, ZF, 1>(z, g, i, j, k) * (1.0 / g.dy) * interp<YF, ZF>(v, g, i, j, k);
    }, GB_KERNEL_MASSFLUX);
}

//! velocity_divergence (MassFlux.cpp:129-136): Omega on the fly, then the face divergence.
void velocity_divergence(gb_simplec* S, const double* u, const double* v, const double* w, double* div)
{
    const gb_grid g = S->g;
    const double* z = S->z;
    const double* ax = S->mesh.ax;
    const double* ay = S->mesh.ay;
    const double* az = S->mesh.az;
    const double* J = S->mesh.detJ;
    // a thread takes kDivLevels levels of a column: each z-face's Omega is
    // evaluated once and serves the cells below and above it
    constexpr int kDivLevels = 4;
    const Box b{{0, 0, 0}, {g.nx - 1, g.ny - 1, (g.nz + kDivLevels - 1) / kDivLevels - 1}};
    for_box(S->ctx, b, [=] __device__(int i, int j, int seg) {
        auto om = [&](int kk) {
            return w[at(g, i, j, kk)] - deriv<NODE, ZF, 0>(z, g, i, j, kk) * (1.0 / g.dx) * interp<XF, ZF>(u, g, i, j, kk)
                 - deriv<NODE, ZF, 1>(z, g, i, j, kk) * (1.0 / g.dy) * interp<YF, ZF>(v, g, i, j, kk);
        };
        const int k0 = seg * kDivLevels;
        double om_lo = om(k0);
        for (int q = 0; q < kDivLevels; ++q) {
            const int k = k0 + q;
            if (k >= g.nz) { break; }
            const double om_hi = om(k + 1);
            const int64_t o = at(g, i, j, k), ox = at(g, i + 1, j, k), oy = at(g, i, j + 1, k), oz = at(g, i, j, k + 1);
            div[o] = ((ax[ox] * u[ox] - ax[o] * u[o]) * (1.0 / g.dx) + (ay[oy] * v[oy] - ay[o] * v[o]) * (1.0 / g.dy)
                      + (az[oz] * om_hi - az[o] * om_lo) * (1.0 / g.dzeta))
                   / J[o];
            om_lo = om_hi;
        }
    }, GB_KERNEL_MASSFLUX);
}

template <int D>
__device__ __forceinline__ double slope_dp(const double* z, const double* p, const gb_grid& g, int i, int j, int k)
{
    const double s = (D == 0) ? deriv<NODE, ZF, 0>(z, g, i, j, k) * (1.0 / g.dx) : deriv<NODE, ZF, 1>(z, g, i, j, k) * (1.0 / g.dy);
    const double dp = (k == 0) ? 3.0 * p[at(g, i, j, k + 1)] - 2.0 * p[at(g, i, j, k)] - p[at(g, i, j, k + 2)]
                               : p[at(g, i, j, k)] - p[at(g, i, j, k - 1)];
    return s * dp * (1.0 / g.dzeta);
}

//! Component C of the pressure gradient (G p)_C at a valid point of its
//! face type (MassFlux.cpp:138-179).
template <int C>
__device__ __forceinline__ double pressure_gradient_at(const double* __restrict__ p, const double* __restrict__ z,
                                                       const double* __restrict__ J, const double* __restrict__ ax,
                                                       const double* __restrict__ ay, const gb_grid& g, int i, int j,
                                                       int k)
{
    if (C == 0) {
        const double cross = 0.25 * ((slope_dp<0>(z, p, g, i - 1, j, k) + slope_dp<0>(z, p, g, i, j, k))
                                     + (slope_dp<0>(z, p, g, i - 1, j, k + 1) + slope_dp<0>(z, p, g, i, j, k + 1)));
        return (ax[at(g, i, j, k)] * (p[at(g, i, j, k)] - p[at(g, i - 1, j, k)]) * (1.0 / g.dx) - cross)
             / interp<CC, XF>(J, g, i, j, k);
    }
    if (C == 1) {
        const double cross = 0.25 * ((slope_dp<1>(z, p, g, i, j - 1, k) + slope_dp<1>(z, p, g, i, j, k))
                                     + (slope_dp<1>(z, p, g, i, j - 1, k + 1) + slope_dp<1>(z, p, g, i, j, k + 1)));
        return (ay[at(g, i, j, k)] * (p[at(g, i, j, k)] - p[at(g, i, j - 1, k)]) * (1.0 / g.dy) - cross)
             / interp<CC, YF>(J, g, i, j, k);
    }
    return (p[at(g, i, j, k)] - p[at(g, i, j, k - 1)]) * (1.0 / g.dzeta) / interp<CC, ZF>(J, g, i, j, k);
}

//! R_c += (G p)_c (MassFlux.cpp:138-179) on the valid points of each component.
void add_pressure_gradient(gb_simplec* S, const double* p, double* Ru, double* Rv, double* Rw)
{
    const gb_grid g = S->g;
    const double* z = S->z;
    const double* J = S->mesh.detJ;
    const double* ax = S->mesh.ax;
    const double* ay = S->mesh.ay;
    for_box(S->ctx, Box{{0, 0, 0}, {g.nx, g.ny, g.nz}}, [=] __device__(int i, int j, int k) {
        if (j < g.ny && k < g.nz) { Ru[at(g, i, j, k)] += pressure_gradient_at<0>(p, z, J, ax, ay, g, i, j, k); }
        if (i < g.nx && k < g.nz) { Rv[at(g, i, j, k)] += pressure_gradient_at<1>(p, z, J, ax, ay, g, i, j, k); }
        if (i < g.nx && j < g.ny) { Rw[at(g, i, j, k)] += pressure_gradient_at<2>(p, z, J, ax, ay, g, i, j, k); }
    }, GB_KERNEL_RESIDUAL);
}

// ----------------------------------------------------------- convection ---

__device__ __forceinline__ double limited_slope(int lim, double a, double b, double eps2)
{
    if (lim == GB_LIMITER_VAN_LEER) {
        const double ab = a * b;
        return (ab > 0) ? 2.0 * ab / (a + b) : 0.0;
    }
    if (lim == GB_LIMITER_VAN_ALBADA) { return ((b * b + eps2) * a + (a * a + eps2) * b) / (a * a + b * b + 2.0 * eps2); }
    return 0.0;
}

__device__ __forceinline__ double muscl_face(int lim, double tr, double qm, double q0, double q1, double qp, double eps2)
{
    if (lim == GB_LIMITER_UPWIND) { return (tr >= 0) ? q0 : q1; }
    return (tr >= 0) ? q0 + 0.5 * limited_slope(lim, q0 - qm, q1 - q0, eps2)
                     : q1 - 0.5 * limited_slope(lim, q1 - q0, qp - q1, eps2);
}

//! The box of the control-volume fluxes of a field at T along D (CVFluxes.cpp:52-66).
template <int T>
Box flux_box(const gb_grid& g, int D)
{
    Box b = valid_box(g, T);
    const int n = (D == 0) ? g.nx : (D == 1) ? g.ny : g.nz;
    if (nodal(T, D)) {
        b.lo[D] = -1;
        b.hi[D] = n;
    } else {
        b.lo[D] = 0;
        b.hi[D] = n;
    }
    return b;
}

//! The convective flux of q (at T) through its control volume's face along D
//! at the flux point (i, j, k): Convection.cpp:17-43 flux_kernel<T, D, L>.
template <int T, int D>
__device__ __forceinline__ double conv_face(const double* __restrict__ q, const double* __restrict__ F, int lim,
                                            double eps2, const gb_grid& g, int i, int j, int k)
{
    constexpr int Sx = T ^ (1 << D);
    constexpr int TF = 1 << D;
    constexpr int l = lo_off(T, Sx, D);
    constexpr int ex = (D == 0), ey = (D == 1), ez = (D == 2);
    const double tr = interp<TF, Sx>(F, g, i, j, k);
    const int i0 = i + l * ex, j0 = j + l * ey, k0 = k + l * ez;
    return tr * muscl_face(lim, tr, q[at(g, i0 - ex, j0 - ey, k0 - ez)], q[at(g, i0, j0, k0)],
                           q[at(g, i0 + ex, j0 + ey, k0 + ez)], q[at(g, i0 + 2 * ex, j0 + 2 * ey, k0 + 2 * ez)], eps2);
}

template <int T, int D>
void conv_fluxes(gb_simplec* S, const double* q, const double* F, int lim, double eps2, double* G)
{
    const gb_grid g = S->g;
    for_box(S->ctx, flux_box<T>(g, D), [=] __device__(int i, int j, int k) {
        G[at(g, i, j, k)] = conv_face<T, D>(q, F, lim, eps2, g, i, j, k);
    }, GB_KERNEL_RESIDUAL);
}

//! out (op)= the control-volume divergence of G (CVFluxes.cpp:16-39); sign +1: =, -1: -=.
template <int T>
void flux_divergence(gb_simplec* S, const double* gx, const double* gy, const double* gz, double* out, int mode)
{
    const gb_grid g = S->g;
    const double* J = S->mesh.detJ;
    constexpr int lx = flux_lo(T, 0), ly = flux_lo(T, 1), lz = flux_lo(T, 2);
    for_box(S->ctx, valid_box(g, T), [=] __device__(int i, int j, int k) {
        const double v = ((gx[at(g, i + lx + 1, j, k)] - gx[at(g, i + lx, j, k)]) * (1.0 / g.dx)
                          + (gy[at(g, i, j + ly + 1, k)] - gy[at(g, i, j + ly, k)]) * (1.0 / g.dy)
                          + (gz[at(g, i, j, k + lz + 1)] - gz[at(g, i, j, k + lz)]) * (1.0 / g.dzeta))
                       / interp<CC, T>(J, g, i, j, k);
        const int64_t o = at(g, i, j, k);
        if (mode == 0) { out[o] = v; } else { out[o] -= v; }
    }, GB_KERNEL_RESIDUAL);
}

//! The bounded form's - q (transport divergence) (Convection.cpp:65-90).
template <int T>
void subtract_transport_divergence(gb_simplec* S, const double* q, const double* F0, const double* F1, const double* F2,
                                   double* out)
{
    const gb_grid g = S->g;
    const double* J = S->mesh.detJ;
    constexpr int SX = T ^ XF, SY = T ^ YF, SZ = T ^ ZF;
    constexpr int lx = flux_lo(T, 0), ly = flux_lo(T, 1), lz = flux_lo(T, 2);
    for_box(S->ctx, valid_box(g, T), [=] __device__(int i, int j, int k) {
        const double div = (interp<XF, SX>(F0, g, i + lx + 1, j, k) - interp<XF, SX>(F0, g, i + lx, j, k)) * (1.0 / g.dx)
                         + (interp<YF, SY>(F1, g, i, j + ly + 1, k) - interp<YF, SY>(F1, g, i, j + ly, k)) * (1.0 / g.dy)
                         + (interp<ZF, SZ>(F2, g, i, j, k + lz + 1) - interp<ZF, SZ>(F2, g, i, j, k + lz)) * (1.0 / g.dzeta);
        out[at(g, i, j, k)] -= q[at(g, i, j, k)] * div / interp<CC, T>(J, g, i, j, k);
    }, GB_KERNEL_RESIDUAL);
}

template <int T>
void convection(gb_simplec* S, const double* q, double* const* F, int lim, double eps, bool bounded, double* out)
{
    const double eps2 = eps * eps;
    double** G = S->w.G;
    conv_fluxes<T, 0>(S, q, F[0], lim, eps2, G[0]);
    conv_fluxes<T, 1>(S, q, F[1], lim, eps2, G[1]);
    conv_fluxes<T, 2>(S, q, F[2], lim, eps2, G[2]);
    flux_divergence<T>(S, G[0], G[1], G[2], out, 0);
    if (bounded) { subtract_transport_divergence<T>(S, q, F[0], F[1], F[2], out); }
}

// ------------------------------------------------------------ diffusion ---

__device__ __forceinline__ double log_mean(double a, double b)
{
    const double tiny = 2.2250738585072014e-308;
    const double sum = a + b;
    const double x = (a - b) / (sum + tiny);
    const double s = (fabs(x) < 0.01) ? 1.0 : 0.0;
    const double x2 = x * x;
    const double series = 0.5 * sum * (1.0 - x2 * (1.0 / 3 + x2 * (4.0 / 45 + x2 * (44.0 / 945))));
    const double direct = (a - b) / (log(a + tiny) - log(b + tiny) + s);
    return (1.0 - s) * direct + s * series;
}

template <int Sx>
__device__ __forceinline__ double face_gamma(const double* gm, const gb_grid& g, int i, int j, int k, int logz)
{
    if (!logz || !nodal(Sx, 2)) { return interp<CC, Sx>(gm, g, i, j, k); }
    constexpr int lx = lo_off(CC, Sx, 0), ly = lo_off(CC, Sx, 1);
    constexpr int nx = npts(CC, Sx, 0), ny = npts(CC, Sx, 1);
    double sum = 0;
    for (int b = 0; b < ny; ++b) {
        for (int a = 0; a < nx; ++a) { sum += log_mean(gm[at(g, i + lx + a, j + ly + b, k - 1)], gm[at(g, i + lx + a, j + ly + b, k)]); }
    }
    return sum * (1.0 / (nx * ny));
}

template <int D>
__device__ __forceinline__ double area_dot(const Metric<double>& m, const double v[3])
{
    if (D == 0) { return m.zz * v[0]; }
    if (D == 1) { return m.zz * v[1]; }
    return v[2] - m.zx * v[0] - m.zy * v[1];
}

//! The diffusive flux of a cell scalar q through the face along D at the flux
//! point (i, j, k) (Diffusion.cpp:10-57).
template <int D>
__device__ __forceinline__ double scalar_diff_face(const double* __restrict__ q, const double* __restrict__ gamma,
                                                   const double* __restrict__ z, int logz, const gb_grid& g, int i,
                                                   int j, int k)
{
    constexpr int Sx = 1 << D;
    const Metric<double> m = metric_at<Sx>(z, g, i, j, k);
    double gr[3];
    grad_at<CC, Sx>(q, g, i, j, k, m, gr);
    return face_gamma<Sx>(gamma, g, i, j, k, logz) * area_dot<D>(m, gr);
}

//! The diffusive flux of velocity component C through its control volume's
//! face along D at the flux point (i, j, k) (Diffusion.cpp:59-127).
template <int C, int D>
__device__ __forceinline__ double momentum_diff_face(const double* __restrict__ u, const double* __restrict__ v,
                                                     const double* __restrict__ w, const double* __restrict__ nu,
                                                     const double* __restrict__ z, int logz, const gb_grid& g, int i,
                                                     int j, int k)
{
    constexpr int T = 1 << C;
    constexpr int Sx = T ^ (1 << D);
    const Metric<double> m = metric_at<Sx>(z, g, i, j, k);
    double gu[3], gv[3], gw[3];
    grad_at<XF, Sx>(u, g, i, j, k, m, gu);
    grad_at<YF, Sx>(v, g, i, j, k, m, gv);
    grad_at<ZF, Sx>(w, g, i, j, k, m, gw);
    const double* gc = (C == 0) ? gu : (C == 1) ? gv : gw;
    const double tau[3] = {gc[0] + gu[C], gc[1] + gv[C], gc[2] + gw[C]};
    return face_gamma<Sx>(nu, g, i, j, k, logz) * area_dot<D>(m, tau);
}

template <int D>
void scalar_diffusive_flux(gb_simplec* S, const double* q, const double* gamma, double* G)
{
    const gb_grid g = S->g;
    const double* z = S->z;
    const int logz = S->ph.log_mean;
    for_box(S->ctx, flux_box<CC>(g, D), [=] __device__(int i, int j, int k) {
        G[at(g, i, j, k)] = scalar_diff_face<D>(q, gamma, z, logz, g, i, j, k);
    }, GB_KERNEL_RESIDUAL);
}

template <int C, int D>
void momentum_diffusive_flux(gb_simplec* S, const gb_state& q, const double* nu, double* G)
{
    const gb_grid g = S->g;
    const double* z = S->z;
    const double* u = q.u;
    const double* v = q.v;
    const double* w = q.w;
    const int logz = S->ph.log_mean;
    for_box(S->ctx, flux_box<1 << C>(g, D), [=] __device__(int i, int j, int k) {
        G[at(g, i, j, k)] = momentum_diff_face<C, D>(u, v, w, nu, z, logz, g, i, j, k);
    }, GB_KERNEL_RESIDUAL);
}

//! The diffusion of velocity component C subtracted from R; a surface_layer
//! ground sets the u and v control volumes' ground fluxes to the wall
//! stress first (set_ground_fluxes; w's ground row is a boundary row).
template <int C>
void momentum_diffusion_subtract(gb_simplec* S, const gb_state& q, double* R)
{
    double** G = S->w.G;
    momentum_diffusive_flux<C, 0>(S, q, S->dfe.nu, G[0]);
    momentum_diffusive_flux<C, 1>(S, q, S->dfe.nu, G[1]);
    momentum_diffusive_flux<C, 2>(S, q, S->dfe.nu, G[2]);
    if (S->wall && C < 2) { turb_ground_flux(S->ctx, S->g, S->bc, S->ssr, C, G[2]); }
    flux_divergence<1 << C>(S, G[0], G[1], G[2], R, 1);
}

//! The diffusion of a cell scalar subtracted from R; field 2 theta, 3 k (the
//! wall model's ground flux on a surface_layer ground).
void scalar_diffusion_subtract(gb_simplec* S, const double* q, const double* gamma, double* R, int field)
{
    double** G = S->w.G;
    scalar_diffusive_flux<0>(S, q, gamma, G[0]);
    scalar_diffusive_flux<1>(S, q, gamma, G[1]);
    scalar_diffusive_flux<2>(S, q, gamma, G[2]);
    if (S->wall) { turb_ground_flux(S->ctx, S->g, S->bc, S->ssr, field, G[2]); }
    flux_divergence<CC>(S, G[0], G[1], G[2], R, 1);
}

// ------------------------------------------------------- fused residual ---
//
// The convection, diffusion and pressure-gradient terms of one equation in
// one launch. A block holds 32 x 8 columns of the equation's points and
// marches up kc levels of them. At each level every thread evaluates the
// convective and diffusive fluxes through the low x, y faces of its control
// volume into shared memory (the block's last row and column also the high
// faces) and through its upper z face into registers (the lower one is the
// level below's upper face), then takes the divergences from there. Each
// face flux is evaluated once per block (twice on the block's edges and at
// its first level), by the same device functions as the separate flux
// launches, and no flux array goes through memory.

constexpr int kFusedTx = 32, kFusedTy = 8;
// levels per block: config 1's residual measured 0.856 ms with 2, 0.886 with
// 4, 1.036 with 8 and 1.806 with 32 (one launch per flux direction: 1.017):
// the face evaluations are latency-bound, and more, shorter blocks keep more
// of them in flight than the z faces saved by longer ones are worth
constexpr int kFusedLevels = 2;

//! The momentum diffusive fluxes at one location type L (a cell centre or
//! an edge): the face flux of every velocity component C whose control
//! volume has its faces along D at L (L = (1 << C) ^ (1 << D)), from one
//! evaluation of the terrain metric, the face diffusivity and the
//! gradients of u, v and w at the point (momentum_diff_face's operations,
//! shared by the two or three fluxes that need them), each within its own
//! flux box (CVFluxes.cpp:52-66); a surface_layer ground's u and v ground
//! faces take the wall stress (set_ground_fluxes, SurfaceLayer.cpp:418-450).
struct StressArgs {
    gb_grid g;
    Box b;                  // the union of the pairs' flux boxes
    Box pb[3];              // each pair's flux box
    double* G[3];           // each pair's flux array
    const double* u;
    const double* v;
    const double* w;
    const double* nu;
    const double* z;
    int logz;
    int wall;
    const double* taux;
    const double* tauy;
};

//! (Four 256-thread blocks an SM, at most 64 registers a thread, as the fused
//! residual and coefficient launches: each is bound by its loads' latency,
//! and the fourth block's warps cut the residual evaluation's time by 12 %
//! against three blocks at 72-84 registers, a few bytes of spills included.)
template <int L>
__global__ void __launch_bounds__(256, 4) k_momentum_stress(const StressArgs a)
{
    pdl_entry();
    // the (component, direction) pairs at L in increasing C
    constexpr int C0 = (L == CC) ? 0 : (L == (XF ^ YF)) ? 0 : (L == (XF ^ ZF)) ? 0 : 1;
    constexpr int D0 = (L == CC) ? 0 : (L == (XF ^ YF)) ? 1 : 2;
    constexpr int C1 = (L == CC) ? 1 : (L == (XF ^ YF)) ? 1 : 2;
    constexpr int D1 = (L == CC) ? 1 : (L == (XF ^ YF)) ? 0 : (L == (XF ^ ZF)) ? 0 : 1;
    constexpr int NP = (L == CC) ? 3 : 2;
    const Box& b = a.b;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= b.count()) { return; }
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
    const int i = b.lo[0] + static_cast<int>(n % nx);
    const int j = b.lo[1] + static_cast<int>((n / nx) % ny);
    const int k = b.lo[2] + static_cast<int>(n / (static_cast<int64_t>(nx) * ny));
    auto inside = [&](const Box& p) {
        return i >= p.lo[0] && i <= p.hi[0] && j >= p.lo[1] && j <= p.hi[1] && k >= p.lo[2] && k <= p.hi[2];
    };
    bool in[3] = {inside(a.pb[0]), inside(a.pb[1]), NP == 3 ? inside(a.pb[2]) : false};
    if (!in[0] && !in[1] && !in[2]) { return; }
    const gb_grid& g = a.g;
    const Metric<double> m = metric_at<L>(a.z, g, i, j, k);
    double gu[3], gv[3], gw[3];
    grad_at<XF, L>(a.u, g, i, j, k, m, gu);
    grad_at<YF, L>(a.v, g, i, j, k, m, gv);
    grad_at<ZF, L>(a.w, g, i, j, k, m, gw);
    const double gam = face_gamma<L>(a.nu, g, i, j, k, a.logz);
    const int64_t o = at(g, i, j, k);
    auto flux = [&](auto Cc, auto Dc) {
        constexpr int C = decltype(Cc)::value, D = decltype(Dc)::value;
        const double* gc = (C == 0) ? gu : (C == 1) ? gv : gw;
        const double tau[3] = {gc[0] + gu[C], gc[1] + gv[C], gc[2] + gw[C]};
        return gam * area_dot<D>(m, tau);
    };
    using I2 = std::integral_constant<int, 2>;
    if (in[0]) {
        double f = flux(std::integral_constant<int, C0>{}, std::integral_constant<int, D0>{});
        if (D0 == 2 && a.wall && k == 0) {
            if (C0 == 0) { f = 0.5 * (a.taux[plane_at(g, i - 1, j)] + a.taux[plane_at(g, i, j)]); }
            if (C0 == 1) { f = 0.5 * (a.tauy[plane_at(g, i, j - 1)] + a.tauy[plane_at(g, i, j)]); }
        }
        a.G[0][o] = f;
    }
    if (in[1]) {
        double f = flux(std::integral_constant<int, C1>{}, std::integral_constant<int, D1>{});
        if (D1 == 2 && a.wall && k == 0) {
            if (C1 == 0) { f = 0.5 * (a.taux[plane_at(g, i - 1, j)] + a.taux[plane_at(g, i, j)]); }
            if (C1 == 1) { f = 0.5 * (a.tauy[plane_at(g, i, j - 1)] + a.tauy[plane_at(g, i, j)]); }
        }
        a.G[1][o] = f;
    }
    if (NP == 3 && in[2]) { a.G[2][o] = flux(I2{}, I2{}); }
}

//! The nine momentum diffusive fluxes into w.Gd in four launches.
void momentum_stress(gb_simplec* S, const gb_state& q)
{
    const gb_grid g = S->g;
    double** Gd = S->w.Gd;
    auto launch = [&](auto Lc, int c0, int d0, int c1, int d1, int c2, int d2) {
        constexpr int L = decltype(Lc)::value;
        StressArgs a{};
        a.g = g;
        const int cs[3] = {c0, c1, c2}, ds[3] = {d0, d1, d2};
        const int np = (c2 >= 0) ? 3 : 2;
        for (int p = 0; p < np; ++p) {
            const int T = 1 << cs[p];
            a.pb[p] = (T == XF) ? flux_box<XF>(g, ds[p]) : (T == YF) ? flux_box<YF>(g, ds[p]) : flux_box<ZF>(g, ds[p]);
            a.G[p] = Gd[3 * cs[p] + ds[p]];
        }
        a.b = a.pb[0];
        for (int p = 1; p < np; ++p) {
            for (int e = 0; e < 3; ++e) {
                a.b.lo[e] = std::min(a.b.lo[e], a.pb[p].lo[e]);
                a.b.hi[e] = std::max(a.b.hi[e], a.pb[p].hi[e]);
            }
        }
        a.u = q.u;
        a.v = q.v;
        a.w = q.w;
        a.nu = S->dfe.nu;
        a.z = S->z;
        a.logz = S->ph.log_mean;
        a.wall = S->wall ? 1 : 0;
        a.taux = S->ssr[kSsTauX];
        a.tauy = S->ssr[kSsTauY];
        const int64_t n = a.b.count();
        span_begin(S->ctx, GB_KERNEL_RESIDUAL);
        launch_pdl(S->ctx->tune[GB_TUNE_PDL] != 1, k_momentum_stress<L>, dim3(static_cast<unsigned>((n + 255) / 256)),
                   dim3(256), 0, S->ctx->stream, a);
        span_end(S->ctx);
        ++S->ctx->launches;
    };
    launch(std::integral_constant<int, CC>{}, 0, 0, 1, 1, 2, 2);
    launch(std::integral_constant<int, XF ^ YF>{}, 0, 1, 1, 0, -1, -1);
    launch(std::integral_constant<int, XF ^ ZF>{}, 0, 2, 2, 0, -1, -1);
    launch(std::integral_constant<int, YF ^ ZF>{}, 1, 2, 2, 1, -1, -1);
}

struct FusedResidualArgs {
    gb_grid g;
    int ni, nj, nk, kc;          // the equation's valid points; levels per block
    const double* gd[3];         // a velocity component's diffusive fluxes along x, y, z (momentum_stress)
    const double* q;             // the transported field
    const double* u;
    const double* v;
    const double* w;
    const double* p;
    const double* F0;            // the transport fluxes
    const double* F1;
    const double* F2;
    const double* gamma;         // nu (momentum) or the scalar's diffusivity
    const double* z;
    const double* J;
    const double* ax;
    const double* ay;
    int lim;
    double eps2;
    int logz;
    int wall;                    // a surface_layer ground: its z faces carry the wall's flux
    const double* plane;         // the wall stress (u, v) or the cell area (theta) per column
    double qs;                   // the surface heat flux (theta)
    const double* ps;            // k's shear and buoyancy production and dissipation (null: none)
    const double* pb;
    const double* eps;
    double* R;
};

//! The convective and diffusive fluxes of equation E (0-2 the velocity
//! components, 3 theta, 4 k) through the face along D at flux point (i, j, k),
//! the ground faces of a surface_layer ground replaced by the wall's flux
//! (set_ground_fluxes, SurfaceLayer.cpp:418-450).
template <int E, int D>
__device__ __forceinline__ void fused_face(const FusedResidualArgs& a, int i, int j, int k, double& gc, double& gd)
{
    constexpr int T = (E < 3) ? (1 << E) : CC;
    const double* F = (D == 0) ? a.F0 : (D == 1) ? a.F1 : a.F2;
    gc = conv_face<T, D>(a.q, F, a.lim, a.eps2, a.g, i, j, k);
    if (E < 3) {
        gd = a.gd[D][at(a.g, i, j, k)];
        return;
    }
    if (D == 2 && a.wall && k == 0) {
        if (E == 0) {
            gd = 0.5 * (a.plane[plane_at(a.g, i - 1, j)] + a.plane[plane_at(a.g, i, j)]);
        } else if (E == 1) {
            gd = 0.5 * (a.plane[plane_at(a.g, i, j - 1)] + a.plane[plane_at(a.g, i, j)]);
        } else if (E == 3) {
            gd = -a.qs * a.plane[plane_at(a.g, i, j)];
        } else {
            gd = 0;
        }
        return;
    }
    gd = scalar_diff_face<D>(a.q, a.gamma, a.z, a.logz, a.g, i, j, k);
}

//! R = div(convective flux) - div(diffusive flux) (+ the pressure gradient
//! for a velocity component; for k the bounded form's - k div(transport) and
//! the sources), in the operation order of the separate launches
//! (Residual.cpp:159-256).
template <int E>
__global__ void __launch_bounds__(kFusedTx* kFusedTy, 4) k_fused_residual(const FusedResidualArgs a)
{
    pdl_entry();
    constexpr int T = (E < 3) ? (1 << E) : CC;
    constexpr int lx = flux_lo(T, 0), ly = flux_lo(T, 1), lz = flux_lo(T, 2);
    __shared__ double xc[kFusedTy][kFusedTx + 1], xd[kFusedTy][kFusedTx + 1];
    __shared__ double yc[kFusedTy + 1][kFusedTx], yd[kFusedTy + 1][kFusedTx];
    const gb_grid& g = a.g;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * kFusedTx + tx, j = blockIdx.y * kFusedTy + ty;
    const bool active = i < a.ni && j < a.nj;
    const bool xhi = active && (tx == kFusedTx - 1 || i == a.ni - 1);
    const bool yhi = active && (ty == kFusedTy - 1 || j == a.nj - 1);
    const int kb = blockIdx.z * a.kc, ke = min(kb + a.kc, a.nk);
    double zc_lo = 0, zd_lo = 0;
    if (active && kb < ke) { fused_face<E, 2>(a, i, j, kb + lz, zc_lo, zd_lo); }
    for (int k = kb; k < ke; ++k) {
        double zc_hi = 0, zd_hi = 0;
        if (active) {
            fused_face<E, 0>(a, i + lx, j, k, xc[ty][tx], xd[ty][tx]);
            if (xhi) { fused_face<E, 0>(a, i + lx + 1, j, k, xc[ty][tx + 1], xd[ty][tx + 1]); }
            fused_face<E, 1>(a, i, j + ly, k, yc[ty][tx], yd[ty][tx]);
            if (yhi) { fused_face<E, 1>(a, i, j + ly + 1, k, yc[ty + 1][tx], yd[ty + 1][tx]); }
            fused_face<E, 2>(a, i, j, k + lz + 1, zc_hi, zd_hi);
        }
        __syncthreads();
        if (active) {
            const int64_t o = at(g, i, j, k);
            const double Jt = interp<CC, T>(a.J, g, i, j, k);
            double r = ((xc[ty][tx + 1] - xc[ty][tx]) * (1.0 / g.dx) + (yc[ty + 1][tx] - yc[ty][tx]) * (1.0 / g.dy)
                        + (zc_hi - zc_lo) * (1.0 / g.dzeta))
                     / Jt;
            if (E == 4) {
                constexpr int SX = T ^ XF, SY = T ^ YF, SZ = T ^ ZF;
                const double div = (interp<XF, SX>(a.F0, g, i + lx + 1, j, k) - interp<XF, SX>(a.F0, g, i + lx, j, k)) * (1.0 / g.dx)
                                 + (interp<YF, SY>(a.F1, g, i, j + ly + 1, k) - interp<YF, SY>(a.F1, g, i, j + ly, k)) * (1.0 / g.dy)
                                 + (interp<ZF, SZ>(a.F2, g, i, j, k + lz + 1) - interp<ZF, SZ>(a.F2, g, i, j, k + lz)) * (1.0 / g.dzeta);
                r -= a.q[o] * div / Jt;
            }
            r -= ((xd[ty][tx + 1] - xd[ty][tx]) * (1.0 / g.dx) + (yd[ty + 1][tx] - yd[ty][tx]) * (1.0 / g.dy)
                  + (zd_hi - zd_lo) * (1.0 / g.dzeta))
               / Jt;
            if (E < 3) { r += pressure_gradient_at<(E < 3 ? E : 0)>(a.p, a.z, a.J, a.ax, a.ay, g, i, j, k); }
            if (E == 4 && a.ps != nullptr) { r = ((r - a.ps[o]) - a.pb[o]) + a.eps[o]; }
            a.R[o] = r;
        }
        zc_lo = zc_hi;
        zd_lo = zd_hi;
        __syncthreads();
    }
}

//! One fused residual launch for equation E into R.
template <int E>
void fused_residual(gb_simplec* S, const gb_state& q, double* R)
{
    constexpr int T = (E < 3) ? (1 << E) : CC;
    const gb_grid g = S->g;
    const gb_physics& ph = S->ph;
    FusedResidualArgs a{};
    a.g = g;
    a.ni = g.nx + (T & 1);
    a.nj = g.ny + ((T >> 1) & 1);
    a.nk = g.nz + ((T >> 2) & 1);
    const int knob = S->ctx->tune[GB_TUNE_RESIDUAL];
    a.kc = (knob >= 2) ? knob : kFusedLevels;
    const double* fields[5] = {q.u, q.v, q.w, q.theta, q.tke};
    a.q = fields[E];
    a.u = q.u;
    a.v = q.v;
    a.w = q.w;
    a.p = q.p;
    a.F0 = S->w.F[0];
    a.F1 = S->w.F[1];
    a.F2 = S->w.F[2];
    a.gamma = (E < 3) ? S->dfe.nu : (E == 3) ? S->dfe.gamma_theta : S->dfe.gamma_tke;
    a.z = S->z;
    a.J = S->mesh.detJ;
    a.ax = S->mesh.ax;
    a.ay = S->mesh.ay;
    a.lim = (E == 4) ? GB_LIMITER_UPWIND : ph.limiter;
    const double eps = (E < 3) ? ph.smooth_eps_velocity : (E == 3) ? ph.smooth_eps_theta : 1e-5;
    a.eps2 = eps * eps;
    a.logz = ph.log_mean;
    a.wall = S->wall ? 1 : 0;
    a.plane = (E == 0) ? S->ssr[kSsTauX] : (E == 1) ? S->ssr[kSsTauY] : (E == 3) ? S->ssr[kSsArea] : nullptr;
    a.qs = (S->bc.surface_stability == GB_SURFACE_HEAT_FLUX) ? S->bc.surface_heat_flux : 0.0;
    if (E == 4 && ph.closure) {
        a.ps = S->cf[kClosurePs];
        a.pb = S->cf[kClosurePb];
        a.eps = S->cf[kClosureEps];
    }
    if (E < 3) {
        for (int d = 0; d < 3; ++d) { a.gd[d] = S->w.Gd[3 * E + d]; }
    }
    a.R = R;
    const dim3 block(kFusedTx, kFusedTy);
    const dim3 grid((a.ni + kFusedTx - 1) / kFusedTx, (a.nj + kFusedTy - 1) / kFusedTy, (a.nk + a.kc - 1) / a.kc);
    span_begin(S->ctx, GB_KERNEL_RESIDUAL);
    launch_pdl(S->ctx->tune[GB_TUNE_PDL] != 1, k_fused_residual<E>, grid, block, 0, S->ctx->stream, a);
    span_end(S->ctx);
    ++S->ctx->launches;
}

// ------------------------------------------------------------- forcing ---

void forcing(gb_simplec* S, const gb_state& q, double** R)
{
    const gb_grid g = S->g;
    const gb_physics ph = S->ph;
    if (ph.gravity > 0) {
        const double gt = ph.gravity / ph.theta0;
        const double* th = q.theta;
        const double* tr = S->w.theta_ref;
        double* Rw = R[2];
        for_box(S->ctx, valid_box(g, ZF), [=] __device__(int i, int j, int k) {
            Rw[at(g, i, j, k)] -= gt * 0.5 * ((th[at(g, i, j, k - 1)] - tr[at(g, i, j, k - 1)]) + (th[at(g, i, j, k)] - tr[at(g, i, j, k)]));
        }, GB_KERNEL_RESIDUAL);
    }
    if (ph.coriolis) {
        const double pi = 3.14159265358979323846;
        const double phi = ph.latitude * pi / 180;
        const double fc = 4 * pi / ph.rotation_period;
        const double fs = fc * std::sin(phi);
        const double fcos = ph.coriolis_3d ? fc * std::cos(phi) : 0.0;
        const double ug = ph.geostrophic ? ph.ug : 0.0, vg = ph.geostrophic ? ph.vg : 0.0;
        const double* u = q.u;
        const double* v = q.v;
        const double* w = q.w;
        double* Ru = R[0];
        double* Rv = R[1];
        double* Rw = R[2];
        const bool three_d = ph.coriolis_3d;
        for_box(S->ctx, Box{{0, 0, 0}, {g.nx, g.ny, g.nz}}, [=] __device__(int i, int j, int k) {
            if (j < g.ny && k < g.nz) {
                Ru[at(g, i, j, k)] -= fs * (interp<YF, XF>(v, g, i, j, k) - vg) - fcos * interp<ZF, XF>(w, g, i, j, k);
            }
            if (i < g.nx && k < g.nz) { Rv[at(g, i, j, k)] += fs * (interp<XF, YF>(u, g, i, j, k) - ug); }
            if (three_d && i < g.nx && j < g.ny) { Rw[at(g, i, j, k)] -= fcos * interp<XF, ZF>(u, g, i, j, k); }
        }, GB_KERNEL_RESIDUAL);
    }
    for (int c = 0; c < 3; ++c) {
        if (ph.pressure_gradient[c] == 0) { continue; }
        const double f = -ph.pressure_gradient[c];
        double* Rc = R[c];
        for_box(S->ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) { Rc[at(g, i, j, k)] += f; },
                GB_KERNEL_RESIDUAL);
    }
}

void fill_theta_ref(gb_simplec* S)
{
    const gb_grid g = S->g;
    const Profile prof = S->prof;
    const double* z = S->z;
    double* tr = S->w.theta_ref;
    for_box(S->ctx, Box{{-1, -1, -1}, {g.nx, g.ny, g.nz}}, [=] __device__(int i, int j, int k) {
        const double zc = interp<NODE, CC>(z, g, i, j, k);
        const int n = prof.rn;
        double v = prof.rt[0];
        if (zc >= prof.rz[n - 1]) {
            v = prof.rt[n - 1];
        } else {
            for (int m = 1; m < n; ++m) {
                if (zc < prof.rz[m]) {
                    if (zc > prof.rz[m - 1]) {
                        const double wgt = (zc - prof.rz[m - 1]) / (prof.rz[m] - prof.rz[m - 1]);
                        v = prof.rt[m - 1] + wgt * (prof.rt[m] - prof.rt[m - 1]);
                    } else {
                        v = prof.rt[m - 1];
                    }
                    break;
                }
            }
        }
        tr[at(g, i, j, k)] = v;
    }, GB_KERNEL_RESIDUAL);
}

// ------------------------------------------------------------- damping ---

//! The Rayleigh layer and the sponge (DampingCoef, BoundaryConditions.cpp:945-1008).
struct Damping {
    double zd, rc, sw, ss, inv_w, lx, ly;
    int fields, above;
    int lateral[4];   // xlo, xhi, ylo, yhi hold an inflow or outflow
    bool on;
};

Damping damping_of(const gb_simplec* S)
{
    const gb_bc& bc = S->bc;
    Damping d{};
    d.zd = bc.rayleigh_zdamp;
    d.rc = bc.rayleigh_dampcoef;
    d.sw = bc.sponge_width;
    d.ss = bc.sponge_strength;
    d.inv_w = d.sw > 0 ? 1 / d.sw : 0.0;
    d.lx = S->g.nx * S->g.dx;
    d.ly = S->g.ny * S->g.dy;
    d.fields = bc.rayleigh_fields;
    d.above = bc.rayleigh_above_ground;
    const int faces[4] = {0, 3, 1, 4};
    for (int n = 0; n < 4; ++n) {
        const int t = bc.face[faces[n]];
        d.lateral[n] = (t == GB_FACE_INFLOW || t == GB_FACE_OUTFLOW) ? 1 : 0;
    }
    d.on = d.zd > 0 || d.sw > 0;
    return d;
}

//! The Rayleigh (cr) and sponge (cs) coefficients of point (i, j, k) of
//! type t for field n (0 u .. 4 k), its heights above the ground (h) and
//! absolute (zc); z_top is the top node height.
__device__ __forceinline__ void damping_at(const Damping& d, const double* z, const gb_grid& g, int n, int t, int i,
                                           int j, int k, double& cr, double& cs, double& h, double& zc)
{
    h = height_above_ground(z, g, t, i, j, k);
    zc = point_z(z, g, t, i, j, k);
    const double ztop = z[at(g, 0, 0, g.nz)];
    const double x = (i + (nodal(t, 0) ? 0 : 0.5)) * g.dx;
    const double y = (j + (nodal(t, 1) ? 0 : 0.5)) * g.dy;
    const double zr = d.above ? h : zc;
    cr = 0;
    if (((d.fields >> n) & 1) && d.zd > 0 && zr > d.zd) {
        const double pi = 3.14159265358979323846;
        const double sn = sin(0.5 * pi * (zr - d.zd) / (ztop - d.zd));
        cr = d.rc * sn * sn;
    }
    cs = 0;
    if (d.sw > 0) {
        const double dist[4] = {x - 0.0, d.lx - x, y - 0.0, d.ly - y};
        for (int m = 0; m < 4; ++m) {
            if (d.lateral[m] && dist[m] < d.sw) {
                const double r = 1 - dist[m] * d.inv_w;
                cs += d.ss * r * r;
            }
        }
    }
}

//! BoundaryConditions::add_damping (BoundaryConditions.cpp:1022-1071):
//! R += c (q - q_ref) on the valid points of u, v, w, theta, k.
void add_damping(gb_simplec* S, const gb_state& q, double** R)
{
    const Damping d = damping_of(S);
    if (!d.on) { return; }
    const gb_grid g = S->g;
    const Profile prof = S->prof;
    const double* z = S->z;
    const double* qf[5] = {q.u, q.v, q.w, q.theta, q.tke};
    double* rf[5] = {R[0], R[1], R[2], R[4], R[5]};
    const int ff[5] = {F_U, F_V, F_W, F_THETA, F_TKE};
    for (int n = 0; n < 5; ++n) {
        const int f = ff[n];
        const int t = (n < 3) ? (1 << n) : CC;
        const double* a = qf[n];
        double* r = rf[n];
        for_box(S->ctx, valid_box(g, t), [=] __device__(int i, int j, int k) {
            double cr, cs, h, zc;
            damping_at(d, z, g, n, t, i, j, k, cr, cs, h, zc);
            const int64_t o = at(g, i, j, k);
            if (cr > 0) {
                const double zr = d.above ? h : zc;
                const double ref = (f == F_W) ? 0.0 : prof.value(f, (f == F_THETA) ? zr : h);
                r[o] += cr * (a[o] - ref);
            }
            if (cs > 0) {
                const double ref = (f == F_W) ? 0.0 : prof.value(f, h);
                r[o] += cs * (a[o] - ref);
            }
        }, GB_KERNEL_RESIDUAL);
    }
}

//! add_damping_to_implicit (BoundaryConditions.cpp:1073-1099): a_P += c.
void add_damping_to_implicit(gb_simplec* S, int f, int t, double* A)
{
    const Damping d = damping_of(S);
    if (!d.on) { return; }
    const gb_grid g = S->g;
    const double* z = S->z;
    const int64_t cs_ = volume(g);
    const int n = (f == F_THETA) ? 3 : (f == F_TKE) ? 4 : f;
    for_box(S->ctx, valid_box(g, t), [=] __device__(int i, int j, int k) {
        double cr, cs, h, zc;
        damping_at(d, z, g, n, t, i, j, k, cr, cs, h, zc);
        A[GB_COEF_P * cs_ + at(g, i, j, k)] += cr + cs;
    }, GB_KERNEL_COEFS);
}

//! apply_rows (BoundaryConditions.cpp:801-852).
void apply_rows(gb_simplec* S, const gb_state& q, double** R)
{
    const gb_grid g = S->g;
    const Profile prof = S->prof;
    const double* z = S->z;
    const double* qv[3] = {q.u, q.v, q.w};
    for (int d = 0; d < 3; ++d) {
        if (is_per(g, d)) { continue; }
        for (int lo = 1; lo >= 0; --lo) {
            const int fc = d + (lo ? 0 : 3);
            if (!dirichlet_normal(S->bc, fc)) { continue; }
            const bool is_profile = S->bc.face[fc] == GB_FACE_INFLOW;
            const int t = 1 << d;
            Box b = valid_box(g, t);
            const int face = lo ? 0 : ((d == 0) ? g.nx : (d == 1) ? g.ny : g.nz);
            b.lo[d] = b.hi[d] = face;
            double* Rd = R[d];
            const double* qd = qv[d];
            const double* u = q.u;
            const double* v = q.v;
            const int dd = d;
            for_box(S->ctx, b, [=] __device__(int i, int j, int k) {
                double V;
                if (dd < 2) {
                    V = is_profile ? prof.value(dd, height_above_ground(z, g, 1 << dd, i, j, k)) : 0.0;
                } else {
                    V = deriv<NODE, ZF, 0>(z, g, i, j, k) * (1.0 / g.dx) * interp<XF, ZF>(u, g, i, j, k)
                      + deriv<NODE, ZF, 1>(z, g, i, j, k) * (1.0 / g.dy) * interp<YF, ZF>(v, g, i, j, k);
                }
                Rd[at(g, i, j, k)] = qd[at(g, i, j, k)] - V;
            }, GB_KERNEL_BC);
        }
    }
}

}  // namespace

// ------------------------------------------------------------ residual ---

void simplec_residual(gb_simplec* S, const gb_state& q, double** R)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    const int64_t vol = volume(g);
    for (int n = 0; n < 6; ++n) { cudaMemsetAsync(R[n], 0, sizeof(double) * vol, ctx->stream); }
    // the closure's fields and the wall state at q (Residual.cpp:166-176, 205-208)
    if (S->ph.closure) {
        turb_closure(ctx, g, S->bc, S->ph, q, S->z, S->dist, S->mesh.z0, S->cf, S->has_hist ? S->nut_hist : nullptr);
    }
    if (S->wall) { turb_surface_state(ctx, g, S->bc, S->ph, q, S->z, S->mesh.z0, S->ssr, dword(ctx, W_SURFACE_BAD)); }
    double** F = S->w.F;
    transport_fluxes(S, q, F[0], F[1], F[2]);
    const gb_physics& ph = S->ph;
    const bool fused = ctx->tune[GB_TUNE_RESIDUAL] != 1;
    if (fused) {
        momentum_stress(S, q);
        fused_residual<0>(S, q, R[0]);
        fused_residual<1>(S, q, R[1]);
        fused_residual<2>(S, q, R[2]);
    } else {
        convection<XF>(S, q.u, F, ph.limiter, ph.smooth_eps_velocity, false, R[0]);
        convection<YF>(S, q.v, F, ph.limiter, ph.smooth_eps_velocity, false, R[1]);
        convection<ZF>(S, q.w, F, ph.limiter, ph.smooth_eps_velocity, false, R[2]);
        momentum_diffusion_subtract<0>(S, q, R[0]);
        momentum_diffusion_subtract<1>(S, q, R[1]);
        momentum_diffusion_subtract<2>(S, q, R[2]);
        add_pressure_gradient(S, q.p, R[0], R[1], R[2]);
    }
    forcing(S, q, R);
    velocity_divergence(S, q.u, q.v, q.w, R[3]);
    if (fused) {
        fused_residual<3>(S, q, R[4]);
        fused_residual<4>(S, q, R[5]);
    } else {
        convection<CC>(S, q.theta, F, ph.limiter, ph.smooth_eps_theta, false, R[4]);
        scalar_diffusion_subtract(S, q.theta, S->dfe.gamma_theta, R[4], 2);
        convection<CC>(S, q.tke, F, GB_LIMITER_UPWIND, 1e-5, true, R[5]);
        scalar_diffusion_subtract(S, q.tke, S->dfe.gamma_tke, R[5], 3);
        if (S->ph.closure) { turb_k_sources(ctx, g, S->cf, R[5]); }
    }
    if (S->wall) { turb_apply_wall_k(ctx, g, S->bc, S->ssr, q.tke, R[5]); }
    add_damping(S, q, R);
    apply_rows(S, q, R);
    seam_sync<double>(ctx, g, XF, R[0]);
    seam_sync<double>(ctx, g, YF, R[1]);
    seam_sync<double>(ctx, g, ZF, R[2]);
}

// -------------------------------------------------------- implicit rows ---

namespace {

//! The two parts of an implicit face weight shared by the control volumes on
//! either side of the face (ImplicitOperator.cpp:13-37): the diffusive
//! conductance and the transport flux at the face.
template <int T, int C, int D>
__device__ __forceinline__ void face_parts(int i, int j, int k, const double* f, const double* gm, const double* z,
                                           const gb_grid& g, int logz, double& dif, double& tr)
{
    constexpr int Sx = T ^ (1 << D);
    const double dxinv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dzeta};
    const Metric<double> m = metric_at<Sx>(z, g, i, j, k);
    const double gs = face_gamma<Sx>(gm, g, i, j, k, logz);
    tr = interp<(1 << D), Sx>(f, g, i, j, k);
    if (D < 2) {
        const double own = (C == D) ? 2.0 : 1.0;
        dif = gs * m.zz * own * dxinv[D];
    } else {
        double nc2 = 0;
        if (C == 0) { nc2 = m.zx * m.zx; }
        if (C == 1) { nc2 = m.zy * m.zy; }
        if (C == 2) { nc2 = 1; }
        dif = gs * (1 + m.zx * m.zx + m.zy * m.zy + nc2) / m.zz * dxinv[2];
    }
}

//! The face weight of the control volume on side 0 (above the face: its low
//! face) or side 1 (below: its high face): the conductance plus the inflow.
__device__ __forceinline__ double weight_of(int side, double dif, double tr, double dxinv)
{
    const double inflow = (side == 0) ? fmax(tr, 0.0) : fmax(-tr, 0.0);
    return (dif + inflow) * dxinv;
}

template <int T, int C, int D>
__device__ __forceinline__ double face_weight(int side, int i, int j, int k, const double* f, const double* gm,
                                              const double* z, const gb_grid& g, int logz)
{
    double dif, tr;
    face_parts<T, C, D>(i, j, k, f, gm, z, g, logz, dif, tr);
    const double dxinv = (D == 0) ? 1.0 / g.dx : (D == 1) ? 1.0 / g.dy : 1.0 / g.dzeta;
    return weight_of(side, dif, tr, dxinv);
}

//! The implicit coefficients with each face's parts evaluated once per block
//! (the layout of k_fused_residual: 32 x 8 columns marching kc levels, the
//! low x and y faces in shared memory, the z faces in registers).
template <int C>
__global__ void __launch_bounds__(kFusedTx* kFusedTy, 4)
    k_fused_coefficients(const gb_grid g, int ni, int nj, int nk, int kc, const double* __restrict__ z,
                         const double* __restrict__ J, int logz, const double* __restrict__ F0,
                         const double* __restrict__ F1, const double* __restrict__ F2, const double* __restrict__ gm,
                         double* __restrict__ A)
{
    pdl_entry();
    constexpr int T = (C < 0) ? CC : (1 << C);
    constexpr int lx = flux_lo(T, 0), ly = flux_lo(T, 1), lz = flux_lo(T, 2);
    __shared__ double xdif[kFusedTy][kFusedTx + 1], xtr[kFusedTy][kFusedTx + 1];
    __shared__ double ydif[kFusedTy + 1][kFusedTx], ytr[kFusedTy + 1][kFusedTx];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * kFusedTx + tx, j = blockIdx.y * kFusedTy + ty;
    const bool active = i < ni && j < nj;
    const bool xhi = active && (tx == kFusedTx - 1 || i == ni - 1);
    const bool yhi = active && (ty == kFusedTy - 1 || j == nj - 1);
    const int kb = blockIdx.z * kc, ke = min(kb + kc, nk);
    const int64_t cs = volume(g);
    const double dxinv = 1.0 / g.dx, dyinv = 1.0 / g.dy, dzinv = 1.0 / g.dzeta;
    double zdif_lo = 0, ztr_lo = 0;
    if (active && kb < ke) { face_parts<T, C, 2>(i, j, kb + lz, F2, gm, z, g, logz, zdif_lo, ztr_lo); }
    for (int k = kb; k < ke; ++k) {
        double zdif_hi = 0, ztr_hi = 0;
        if (active) {
            face_parts<T, C, 0>(i + lx, j, k, F0, gm, z, g, logz, xdif[ty][tx], xtr[ty][tx]);
            if (xhi) { face_parts<T, C, 0>(i + lx + 1, j, k, F0, gm, z, g, logz, xdif[ty][tx + 1], xtr[ty][tx + 1]); }
            face_parts<T, C, 1>(i, j + ly, k, F1, gm, z, g, logz, ydif[ty][tx], ytr[ty][tx]);
            if (yhi) { face_parts<T, C, 1>(i, j + ly + 1, k, F1, gm, z, g, logz, ydif[ty + 1][tx], ytr[ty + 1][tx]); }
            face_parts<T, C, 2>(i, j, k + lz + 1, F2, gm, z, g, logz, zdif_hi, ztr_hi);
        }
        __syncthreads();
        if (active) {
            const double Jinv = 1.0 / interp<CC, T>(J, g, i, j, k);
            const double xm = weight_of(0, xdif[ty][tx], xtr[ty][tx], dxinv) * Jinv;
            const double xp = weight_of(1, xdif[ty][tx + 1], xtr[ty][tx + 1], dxinv) * Jinv;
            const double ym = weight_of(0, ydif[ty][tx], ytr[ty][tx], dyinv) * Jinv;
            const double yp = weight_of(1, ydif[ty + 1][tx], ytr[ty + 1][tx], dyinv) * Jinv;
            const double zm = weight_of(0, zdif_lo, ztr_lo, dzinv) * Jinv;
            const double zp = weight_of(1, zdif_hi, ztr_hi, dzinv) * Jinv;
            const int64_t o = at(g, i, j, k);
            A[GB_COEF_XM * cs + o] = xm;
            A[GB_COEF_XP * cs + o] = xp;
            A[GB_COEF_YM * cs + o] = ym;
            A[GB_COEF_YP * cs + o] = yp;
            A[GB_COEF_ZM * cs + o] = zm;
            A[GB_COEF_ZP * cs + o] = zp;
            A[GB_COEF_P * cs + o] = ((xm + xp) + (ym + yp)) + (zm + zp);
        }
        zdif_lo = zdif_hi;
        ztr_lo = ztr_hi;
        __syncthreads();
    }
}

//! ImplicitOperator.cpp:39-74 coefficients<C> (C = -1: a cell scalar) on
//! the grid g with node heights z and detJ J.
template <int C>
void implicit_coefficients_on(gb_ctx* ctx, const gb_grid g, const double* z, const double* J, int logz,
                              double* const* F, const double* gm, double* A)
{
    constexpr int T = (C < 0) ? CC : (1 << C);
    constexpr int lx = flux_lo(T, 0), ly = flux_lo(T, 1), lz = flux_lo(T, 2);
    const int64_t cs = volume(g);
    const double* F0 = F[0];
    const double* F1 = F[1];
    const double* F2 = F[2];
    const int knob = ctx->tune[GB_TUNE_RESIDUAL];
    if (knob != 1) {
        const int ni = g.nx + (T & 1), nj = g.ny + ((T >> 1) & 1), nk = g.nz + ((T >> 2) & 1);
        const int kc = (knob >= 2) ? knob : kFusedLevels;
        const dim3 block(kFusedTx, kFusedTy);
        const dim3 grid((ni + kFusedTx - 1) / kFusedTx, (nj + kFusedTy - 1) / kFusedTy, (nk + kc - 1) / kc);
        span_begin(ctx, GB_KERNEL_COEFS);
        launch_pdl(ctx->tune[GB_TUNE_PDL] != 1, k_fused_coefficients<C>, grid, block, 0, ctx->stream, g, ni, nj, nk,
                   kc, z, J, logz, F0, F1, F2, gm, A);
        span_end(ctx);
        ++ctx->launches;
        return;
    }
    for_box(ctx, valid_box(g, T), [=] __device__(int i, int j, int k) {
        const double Jinv = 1.0 / interp<CC, T>(J, g, i, j, k);
        const double xm = face_weight<T, C, 0>(0, i + lx, j, k, F0, gm, z, g, logz) * Jinv;
        const double xp = face_weight<T, C, 0>(1, i + lx + 1, j, k, F0, gm, z, g, logz) * Jinv;
        const double ym = face_weight<T, C, 1>(0, i, j + ly, k, F1, gm, z, g, logz) * Jinv;
        const double yp = face_weight<T, C, 1>(1, i, j + ly + 1, k, F1, gm, z, g, logz) * Jinv;
        const double zm = face_weight<T, C, 2>(0, i, j, k + lz, F2, gm, z, g, logz) * Jinv;
        const double zp = face_weight<T, C, 2>(1, i, j, k + lz + 1, F2, gm, z, g, logz) * Jinv;
        const int64_t o = at(g, i, j, k);
        A[GB_COEF_XM * cs + o] = xm;
        A[GB_COEF_XP * cs + o] = xp;
        A[GB_COEF_YM * cs + o] = ym;
        A[GB_COEF_YP * cs + o] = yp;
        A[GB_COEF_ZM * cs + o] = zm;
        A[GB_COEF_ZP * cs + o] = zp;
        A[GB_COEF_P * cs + o] = ((xm + xp) + (ym + yp)) + (zm + zp);
    }, GB_KERNEL_COEFS);
}

template <int C>
void implicit_coefficients(gb_simplec* S, double* const* F, const double* gm, double* A)
{
    implicit_coefficients_on<C>(S->ctx, S->g, S->z, S->mesh.detJ, S->ph.log_mean, F, gm, A);
}

//! One boundary face's fold of the implicit rows (apply_to_implicit).
struct FoldFace {
    int d;              // the face's direction
    int edge;           // its points' index along d
    int dirichlet_pt;   // a Dirichlet point: the row becomes the identity
    int ghost_coef;     // the coefficient towards the ghost
    int other_coef;     // the opposite coefficient (to_other)
    int to_other;       // the ghost coefficient moves to the opposite one
    double fold;        // else a_P += fold a_ghost
};
struct FoldPack {
    FoldFace f[6];
    int n;
    Box vb;               // the valid points of the rows' location
    int64_t start[7];     // face q's points are [start[q], start[q + 1]) of the launch
};

__device__ __forceinline__ void apply_fold(const FoldFace& F, double* A, int64_t cs, int64_t o)
{
    if (F.dirichlet_pt) {
        for (int n = 0; n < GB_N_COEFS; ++n) { A[n * cs + o] = 0; }
        A[GB_COEF_P * cs + o] = 1;
    } else {
        const double ag = A[F.ghost_coef * cs + o];
        A[F.ghost_coef * cs + o] = 0;
        if (F.to_other) { A[F.other_coef * cs + o] += ag; } else { A[GB_COEF_P * cs + o] += F.fold * ag; }
    }
}

//! Every face's folds in one launch: a thread per point of each face plane;
//! a point on several faces (an edge or a corner) is taken by the thread of
//! its first face in the order of the folds, which applies all of that
//! point's folds in that order (the order of the per-face launches).
__global__ void k_fold_rows(const gb_grid g, const __grid_constant__ FoldPack P, double* __restrict__ A)
{
    pdl_entry();
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= P.start[P.n]) { return; }
    int q = 0;
    while (n >= P.start[q + 1]) { ++q; }
    // the point of face q's plane (the valid box with index d fixed at the edge), i fastest
    Box b = P.vb;
    b.lo[P.f[q].d] = b.hi[P.f[q].d] = P.f[q].edge;
    const int64_t m = n - P.start[q];
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
    const int c[3] = {b.lo[0] + static_cast<int>(m % nx), b.lo[1] + static_cast<int>((m / nx) % ny),
                      b.lo[2] + static_cast<int>(m / (static_cast<int64_t>(nx) * ny))};
    for (int e = 0; e < q; ++e) {
        if (c[P.f[e].d] == P.f[e].edge) { return; }  // an earlier face's thread takes it
    }
    const int64_t cs = volume(g);
    const int64_t o = at(g, c[0], c[1], c[2]);
    for (int e = 0; e < P.n; ++e) {
        if (c[P.f[e].d] == P.f[e].edge) { apply_fold(P.f[e], A, cs, o); }
    }
}

//! apply_to_implicit (BoundaryConditions.cpp:885-941): the damping first,
//! then the folds (a Dirichlet face point's row becomes the identity), the
//! faces in the order d = x, y, z, low side then high side.
void apply_to_implicit(gb_simplec* S, int f, int t, double* A)
{
    add_damping_to_implicit(S, f, t, A);
    const gb_grid g = S->g;
    FoldPack P{};
    P.vb = valid_box(g, t);
    P.n = 0;
    P.start[0] = 0;
    for (int d = 0; d < 3; ++d) {
        if (is_per(g, d)) { continue; }
        for (int lo = 1; lo >= 0; --lo) {
            const int fc = d + (lo ? 0 : 3);
            const int rule = rule_for(f, S->bc.face[fc], d, lo);
            const bool nod = nodal(t, d);
            const int nd = (d == 0) ? g.nx : (d == 1) ? g.ny : g.nz;
            FoldFace& F = P.f[P.n];
            F.d = d;
            F.edge = lo ? 0 : (nod ? nd : nd - 1);
            F.dirichlet_pt = (nod && (rule == R_VALUE || rule == R_PROFILE)) ? 1 : 0;
            const int cm = (d == 0) ? GB_COEF_XM : (d == 1) ? GB_COEF_YM : GB_COEF_ZM;
            const int cp = (d == 0) ? GB_COEF_XP : (d == 1) ? GB_COEF_YP : GB_COEF_ZP;
            F.ghost_coef = lo ? cm : cp;
            F.other_coef = lo ? cp : cm;
            F.fold = 0;
            F.to_other = 0;
            if (nod) { F.to_other = 1; }
            else if (rule == R_EVEN) { F.fold = -1; }
            else if (rule == R_ODD || rule == R_VALUE) { F.fold = 1; }
            else if (rule == R_GRADIENT) { F.to_other = 1; }
            Box b = P.vb;
            b.lo[d] = b.hi[d] = F.edge;
            P.start[P.n + 1] = P.start[P.n] + b.count();
            ++P.n;
        }
    }
    const int64_t total = P.start[P.n];
    if (total == 0) { return; }
    span_begin(S->ctx, GB_KERNEL_COEFS);
    launch_pdl(S->ctx->tune[GB_TUNE_PDL] != 1, k_fold_rows, dim3(static_cast<unsigned>((total + 255) / 256)),
               dim3(256), 0, S->ctx->stream, g, P, A);
    span_end(S->ctx);
    ++S->ctx->launches;
}

void dirichlet_rows(gb_simplec* S, int f, int t, double* mask)
{
    const gb_grid g = S->g;
    cudaMemsetAsync(mask, 0, sizeof(double) * volume(g), S->ctx->stream);
    for (int d = 0; d < 3; ++d) {
        if (is_per(g, d)) { continue; }
        for (int lo = 1; lo >= 0; --lo) {
            const int fc = d + (lo ? 0 : 3);
            const int rule = rule_for(f, S->bc.face[fc], d, lo);
            if (!(nodal(t, d) && (rule == R_VALUE || rule == R_PROFILE))) { continue; }
            const int edge = lo ? 0 : ((d == 0) ? g.nx : (d == 1) ? g.ny : g.nz);
            Box b = valid_box(g, t);
            b.lo[d] = b.hi[d] = edge;
            for_box(S->ctx, b, [=] __device__(int i, int j, int k) { mask[at(g, i, j, k)] = 1.0; }, GB_KERNEL_COEFS);
        }
    }
}

}  // namespace

//! implicit_rows (Residual.cpp:272-304): the coefficients with the
//! effective diffusivity, the Patankar diagonal of k with the closure, the
//! first cells' wall rows (the surface state of the iteration's first fill)
//! for every equation but w, then the boundary folds.
void simplec_implicit_rows(gb_simplec* S, int eq, double* const* F, double* A)
{
    switch (eq) {
    case F_U: implicit_coefficients<0>(S, F, S->dfe.nu, A); break;
    case F_V: implicit_coefficients<1>(S, F, S->dfe.nu, A); break;
    case F_W: implicit_coefficients<2>(S, F, S->dfe.nu, A); break;
    case F_THETA: implicit_coefficients<-1>(S, F, S->dfe.gamma_theta, A); break;
    default: implicit_coefficients<-1>(S, F, S->dfe.gamma_tke, A); break;
    }
    const int t = (eq <= F_W) ? (1 << eq) : CC;
    if (S->ph.closure && eq == F_TKE) { turb_patankar(S->ctx, S->g, S->cf[kClosureDSdk], A); }
    if (S->wall && eq != F_W) {
        turb_wall_rows(S->ctx, S->g, S->ss, t, S->mesh.detJ, A);
        if (eq == F_TKE) { turb_wall_k_rows(S->ctx, S->g, S->bc, S->ss, A); }
    }
    apply_to_implicit(S, eq, t, A);
}

// ------------------------------------------------------------ face dtau ---

namespace {

void face_dtau(gb_simplec* S, const double* dc, double** f)
{
    const gb_grid g = S->g;
    double* fx = f[0];
    double* fy = f[1];
    double* fz = f[2];
    const bool px = g.periodic_x, py = g.periodic_y;
    for_box(S->ctx, Box{{0, 0, 0}, {g.nx, g.ny, g.nz}}, [=] __device__(int i, int j, int k) {
        auto D = [&](int a, int b, int c) {
            if (px) { a = (a < 0) ? a + g.nx : (a >= g.nx ? a - g.nx : a); }
            if (py) { b = (b < 0) ? b + g.ny : (b >= g.ny ? b - g.ny : b); }
            return dc[at(g, a, b, c)];
        };
        if (j < g.ny && k < g.nz) {
            const bool lo = (!px && i == 0), hi = (!px && i == g.nx);
            fx[at(g, i, j, k)] = lo ? D(i, j, k) : hi ? D(i - 1, j, k) : 0.5 * (D(i - 1, j, k) + D(i, j, k));
        }
        if (i < g.nx && k < g.nz) {
            const bool lo = (!py && j == 0), hi = (!py && j == g.ny);
            fy[at(g, i, j, k)] = lo ? D(i, j, k) : hi ? D(i, j - 1, k) : 0.5 * (D(i, j - 1, k) + D(i, j, k));
        }
        if (i < g.nx && j < g.ny) {
            const bool lo = (k == 0), hi = (k == g.nz);
            fz[at(g, i, j, k)] = lo ? D(i, j, k) : hi ? D(i, j, k - 1) : 0.5 * (D(i, j, k - 1) + D(i, j, k));
        }
    }, GB_KERNEL_COEFS);
}

template <typename TD>
__global__ void k_convert(TD* __restrict__ dst, const double* __restrict__ src, int64_t n)
{
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t < n) { dst[t] = static_cast<TD>(src[t]); }
}

//! The z-line sweeps of one system, FP64 or (precision 1) FP32 inner solve:
//! delta (FP64) receives the correction.
gb_status line_solve(gb_simplec* S, int loc, const double* A, const double* ap, const double* rhs, double* delta,
                     int word)
{
    gb_ctx* ctx = S->ctx;
    const int64_t vol = volume(S->g);
    cudaMemsetAsync(delta, 0, sizeof(double) * vol, ctx->stream);
    if (S->opt.line_sweep == 1) {  // steady.sweep = lusgs (FP64 in either precision)
        return zline_lusgs(ctx, S->g, loc, A, ap, rhs, S->opt.zline_sweeps, S->opt.line_alternate, delta,
                           dword(ctx, word));
    }
    if (S->opt.precision == 0) {
        return zline_sweeps<double>(ctx, S->g, loc, A, ap, rhs, S->opt.zline_sweeps, delta, dword(ctx, word),
                                    LineScratch::automatic);
    }
    const unsigned nb = static_cast<unsigned>((vol + 255) / 256);
    k_convert<float><<<nb * GB_N_COEFS, 256, 0, ctx->stream>>>(S->w.A32, A, vol * GB_N_COEFS);
    k_convert<float><<<nb, 256, 0, ctx->stream>>>(S->w.ap32, ap, vol);
    k_convert<float><<<nb, 256, 0, ctx->stream>>>(S->w.rhs32, rhs, vol);
    ctx->launches += 3;
    cudaMemsetAsync(S->w.delta32, 0, sizeof(float) * vol, ctx->stream);
    gb_status st = zline_sweeps<float>(ctx, S->g, loc, S->w.A32, S->w.ap32, S->w.rhs32, S->opt.zline_sweeps,
                                       S->w.delta32, dword(ctx, word), LineScratch::automatic);
    const float* d32 = S->w.delta32;
    const gb_grid g = S->g;
    for_box(ctx, valid_box(g, loc), [=] __device__(int i, int j, int k) {
        delta[at(g, i, j, k)] = static_cast<double>(d32[at(g, i, j, k)]);
    });
    return st;
}

//! n <= 3 independent systems (each at its own location) solved by the z-line
//! sweeps in one launch per sweep (zline_sweeps_multi), FP64 or (precision 1)
//! FP32; line LU-SGS solves them one after another. delta[s] (FP64) receives
//! each correction, words[s] the change of its last sweep.
gb_status line_solve_multi(gb_simplec* S, int n, const int* locs, double* const* A, double* const* ap,
                           double* const* rhs, double* const* delta, const int* words)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    const int64_t vol = volume(g);
    if (S->opt.line_sweep == 1) {
        for (int s = 0; s < n; ++s) {
            gb_status st = line_solve(S, locs[s], A[s], ap[s], rhs[s], delta[s], words[s]);
            if (st != GB_OK) { return st; }
        }
        return GB_OK;
    }
    unsigned long long* cw[3];
    for (int s = 0; s < n; ++s) {
        cudaMemsetAsync(delta[s], 0, sizeof(double) * vol, ctx->stream);
        cw[s] = dword(ctx, words[s]);
    }
    if (S->opt.precision == 0) {
        const double* Ac[3] = {A[0], n > 1 ? A[1] : nullptr, n > 2 ? A[2] : nullptr};
        const double* apc[3] = {ap[0], n > 1 ? ap[1] : nullptr, n > 2 ? ap[2] : nullptr};
        const double* rc[3] = {rhs[0], n > 1 ? rhs[1] : nullptr, n > 2 ? rhs[2] : nullptr};
        return zline_sweeps_multi<double>(ctx, g, n, locs, Ac, apc, rc, S->opt.zline_sweeps, delta, cw);
    }
    SimplecWork& w = S->w;
    const unsigned nb = static_cast<unsigned>((vol + 255) / 256);
    const float* A32[3] = {};
    const float* ap32[3] = {};
    const float* r32[3] = {};
    float* d32[3] = {};
    for (int s = 0; s < n; ++s) {
        k_convert<float><<<nb * GB_N_COEFS, 256, 0, ctx->stream>>>(w.A32m[s], A[s], vol * GB_N_COEFS);
        k_convert<float><<<nb, 256, 0, ctx->stream>>>(w.ap32m[s], ap[s], vol);
        k_convert<float><<<nb, 256, 0, ctx->stream>>>(w.rhs32m[s], rhs[s], vol);
        ctx->launches += 3;
        cudaMemsetAsync(w.delta32m[s], 0, sizeof(float) * vol, ctx->stream);
        A32[s] = w.A32m[s];
        ap32[s] = w.ap32m[s];
        r32[s] = w.rhs32m[s];
        d32[s] = w.delta32m[s];
    }
    gb_status st = zline_sweeps_multi<float>(ctx, g, n, locs, A32, ap32, r32, S->opt.zline_sweeps, d32, cw);
    for (int s = 0; s < n; ++s) {
        const float* dsrc = d32[s];
        double* dst = delta[s];
        for_box(ctx, valid_box(g, locs[s]), [=] __device__(int i, int j, int k) {
            dst[at(g, i, j, k)] = static_cast<double>(dsrc[at(g, i, j, k)]);
        });
    }
    return st;
}

}  // namespace

// ------------------------------------------------------- predictor etc. ---

namespace {

enum Word : int {
    W_MAX_DU = 0, W_MAX_DV, W_MAX_DW, W_LAST_U, W_LAST_V, W_LAST_W, W_DIV_BEFORE, W_DIV_AFTER, W_MAX_PHI,
    W_MAX_FU, W_MAX_FV, W_MAX_FW, W_SPEED_U, W_SPEED_V, W_SPEED_W, W_MAX_DTH, W_MAX_DK, W_LAST_TH, W_LAST_K,
    W_CLIPPED, W_MON_U, W_MON_V, W_MON_W, W_COUNT
};
enum Sum : int { SUM_R0 = 0, SUM_TKE = 6, SUM_USTAR = 7, SUM_LEVEL = 8, SUM_COUNT = 8 };

//! The six residuals' sums of squares, k's sum and (a surface_layer ground)
//! the domain columns' u* sum (the u* plane is the k = -ng layer of the
//! indexing) in two launches.
void residual_sums(gb_simplec* S, const gb_state& q)
{
    const gb_grid& g = S->g;
    RedPack P{};
    for (int n = 0; n < 6; ++n) { P.it[n] = red_item(valid_box(g, kLoc[n]), S->w.R[n], nullptr, 0, SUM_R0 + n); }
    P.it[6] = red_item(valid_box(g, CC), q.tke, nullptr, 1, SUM_TKE);
    P.n = 7;
    if (S->wall) {
        P.it[7] = red_item(Box{{0, 0, -g.ng}, {g.nx - 1, g.ny - 1, -g.ng}}, S->ss[kSsUstar], nullptr, 1, SUM_USTAR);
        P.n = 8;
    }
    dsum_many(S, P);
}

gb_status momentum_predictor(gb_simplec* S, const gb_state& q, double** R)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    const int64_t cs = volume(g);
    SimplecWork& w = S->w;
    double* comps[3] = {q.u, q.v, q.w};
    const double fs = S->ph.coriolis ? 4 * 3.14159265358979323846 * std::sin(S->ph.latitude * 3.14159265358979323846 / 180)
                                         / S->ph.rotation_period
                                     : 0.0;
    for (int c = 0; c < 3; ++c) {
        const int t = 1 << c;
        simplec_implicit_rows(S, c, w.F, w.Am[c]);
        dirichlet_rows(S, c, t, w.mask);
        double* ap = w.ap[c];
        double* dd = w.dd[c];
        const double* A = w.Am[c];
        const double* mask = w.mask;
        const double* dt = w.dtf[c];
        const double* Rc = R[c];
        double* rhs = w.rhsm[c];
        const double inv_cap = S->opt.w_vnn_cap > 0 ? 1.0 / S->opt.w_vnn_cap : 0.0;
        const double s_margin = S->opt.w_vnn_cap_slope_margin;
        const bool cap = (c == 2 && S->opt.w_vnn_cap > 0);
        const double* z = S->z;
        for_box(ctx, valid_box(g, t), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            const double keep = 1.0 - mask[o];
            double p = keep / dt[o] + A[GB_COEF_P * cs + o];
            const double nb = A[GB_COEF_XM * cs + o] + A[GB_COEF_XP * cs + o] + A[GB_COEF_YM * cs + o]
                            + A[GB_COEF_YP * cs + o] + A[GB_COEF_ZM * cs + o] + A[GB_COEF_ZP * cs + o];
            double d = keep * (p - nb);
            if (cap) {
                double term = inv_cap * (A[GB_COEF_ZM * cs + o] + A[GB_COEF_ZP * cs + o]);
                if (s_margin > 0) {
                    const double hx = 0.5 * (z[at(g, i + 1, j + 1, k)] + z[at(g, i + 1, j, k)] - z[at(g, i, j + 1, k)] - z[at(g, i, j, k)]) * (1.0 / g.dx);
                    const double hy = 0.5 * (z[at(g, i + 1, j + 1, k)] + z[at(g, i, j + 1, k)] - z[at(g, i + 1, j, k)] - z[at(g, i, j, k)]) * (1.0 / g.dy);
                    const double slope2 = hx * hx + hy * hy;
                    if (slope2 > 0) {
                        const double root = sqrt(1.0 + slope2) + 1.0;
                        const double rc = slope2 / (root * root);
                        const double lim = fmax(0.0, 1.0 / (s_margin * rc) - 1.0) / dt[o];
                        term = fmin(term, lim);
                    }
                }
                p += keep * term;
                d += keep * term;
            }
            ap[o] = p;
            dd[o] = d;
            rhs[o] = -Rc[o];
        }, GB_KERNEL_COEFS);
        if (c < 2 && S->ph.coriolis && fs != 0) {
            // the other component's residual: its horizontal mean per level
            // (deterministic column-ordered sums), then the coupling
            const double* other = (c == 0) ? R[1] : R[0];
            const int to = (c == 0) ? YF : XF;
            const int d_o = 1 - c;
            const bool per_o = is_per(g, d_o);
            const int n_o = (d_o == 0) ? g.nx : g.ny, n_c = (c == 0) ? g.nx : g.ny;
            const double npts_level = static_cast<double>(n_o + (per_o ? 0 : 1)) * static_cast<double>(n_c);
            {
                // one block per level, a fixed summation order: deterministic
                Box b = valid_box(g, to);
                if (per_o) { b.hi[d_o] -= 1; }
                Span span(ctx, GB_KERNEL_VECTOR);
                k_level_mean<<<g.nz, kLevelThreads, 0, ctx->stream>>>(g, b, other, npts_level, w.level_sum);
                ++ctx->launches;
            }
            double* mean = w.level_sum;
            // the periodic images of the other residual (one ghost) for the four-face mean
            cudaMemcpyAsync(w.og, other, sizeof(double) * cs, cudaMemcpyDeviceToDevice, ctx->stream);
            double* og = w.og;
            const bool px = g.periodic_x, py = g.periodic_y;
            const double relax = S->opt.rotation_relax;
            const bool per_c = is_per(g, c);
            const int hi_edge = (c == 0) ? g.nx : g.ny;
            const int cc = c;
            for_box(ctx, valid_box(g, t), [=] __device__(int i, int j, int k) {
                const int64_t o = at(g, i, j, k);
                const double keep = 1.0 - mask[o];
                if (keep == 0) { return; }
                const int n = (cc == 0) ? i : j;
                if (!per_c && (n == 0 || n == hi_edge)) { return; }
                const double nb = A[GB_COEF_XM * cs + o] + A[GB_COEF_XP * cs + o] + A[GB_COEF_YM * cs + o]
                                + A[GB_COEF_YP * cs + o] + A[GB_COEF_ZM * cs + o] + A[GB_COEF_ZP * cs + o];
                const double net = fmax(A[GB_COEF_P * cs + o] - nb, 0.0);
                const double tau_c = 1.0 / fmax(fabs(fs) / relax, net);
                const double tau_own = 1.0 / (1.0 / dt[o] + net);
                const double stiff = fs * fs * fmax(tau_c, tau_own);
                ap[o] += stiff;
                dd[o] += stiff;
                // four-face mean with periodic images (og's ghosts resolved by index)
                auto RO = [&](int a, int b2, int kk) {
                    const int nvx = g.nx + (to & 1), nvy = g.ny + ((to >> 1) & 1);
                    if (a < 0 || a >= nvx) {
                        if (!px) { return og[at(g, a, b2, kk)]; }
                        a = (a < 0) ? a + g.nx : a - g.nx;
                    }
                    if (b2 < 0 || b2 >= nvy) {
                        if (!py) { return og[at(g, a, b2, kk)]; }
                        b2 = (b2 < 0) ? b2 + g.ny : b2 - g.ny;
                    }
                    return og[at(g, a, b2, kk)];
                };
                double avg;
                if (cc == 0) {  // interp<YF, XF>: v at (i-1..i, j..j+1)
                    avg = ((RO(i - 1, j, k) + RO(i, j, k)) + (RO(i - 1, j + 1, k) + RO(i, j + 1, k))) * 0.25;
                } else {        // interp<XF, YF>: u at (i..i+1, j-1..j)
                    avg = ((RO(i, j - 1, k) + RO(i + 1, j - 1, k)) + (RO(i, j, k) + RO(i + 1, j, k))) * 0.25;
                }
                const double m = mean[k];
                rhs[o] += ((cc == 0) ? -fs : fs) * (tau_c * m + tau_own * (avg - m));
            }, GB_KERNEL_COEFS);
        }
        if (c == 2 && S->ph.gravity > 0) {
            const double gt = S->ph.gravity / S->ph.theta0;
            simplec_implicit_rows(S, F_THETA, w.F, w.At);
            const double* At = w.At;
            const double* th = q.theta;
            const double* Rt = R[4];
            for_box(ctx, valid_box(g, ZF), [=] __device__(int i, int j, int k) {
                const int64_t o = at(g, i, j, k);
                const double keep = 1.0 - mask[o];
                if (keep == 0) { return; }
                auto zc = [&](int kk) {
                    return 0.125 * (z[at(g, i, j, kk)] + z[at(g, i + 1, j, kk)] + z[at(g, i, j + 1, kk)] + z[at(g, i + 1, j + 1, kk)]
                                    + z[at(g, i, j, kk + 1)] + z[at(g, i + 1, j, kk + 1)] + z[at(g, i, j + 1, kk + 1)]
                                    + z[at(g, i + 1, j + 1, kk + 1)]);
                };
                const double gamma = (th[at(g, i, j, k)] - th[at(g, i, j, k - 1)]) / (zc(k) - zc(k - 1));
                const double ap_theta = 0.5 * (At[GB_COEF_P * cs + at(g, i, j, k - 1)] + At[GB_COEF_P * cs + o]);
                const double tau = 1.0 / (1.0 / dt[o] + ap_theta);
                const double stiff = gt * fmax(gamma, 0.0) * tau;
                ap[o] += stiff;
                dd[o] += stiff;
                rhs[o] -= gt * tau * 0.5 * (Rt[at(g, i, j, k - 1)] + Rt[o]);
            }, GB_KERNEL_COEFS);
        }
    }
    // the three systems are independent: one batched solve
    const int locs[3] = {XF, YF, ZF};
    const int words[3] = {W_LAST_U, W_LAST_V, W_LAST_W};
    gb_status st = line_solve_multi(S, 3, locs, w.Am, w.ap, w.rhsm, w.deltam, words);
    if (st != GB_OK) { return st; }
    dmax_velocity(S, w.deltam[0], w.deltam[1], w.deltam[2], W_MAX_DU);
    for (int c = 0; c < 3; ++c) {
        const int t = 1 << c;
        double* qc = comps[c];
        const double* delta = w.deltam[c];
        for_box(ctx, valid_box(g, t), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            qc[o] += delta[o];
        });
    }
    return check_cuda("momentum_predictor");
}

//! pressure_correction's first part: beta = 1/d and the keep masks, div u*,
//! the monitors, the solver's coefficients (no host synchronisation).
gb_status pressure_prelude(gb_simplec* S, const gb_state& q, const double* source = nullptr)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    for (int c = 0; c < 3; ++c) {
        const double* dd = w.dd[c];
        double* beta = w.beta[c];
        double* keep = w.keep[c];
        for_box(ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            const bool on = dd[o] > 0;
            beta[o] = on ? 1.0 / dd[o] : 1.0;
            keep[o] = on ? 1.0 : 0.0;
        }, GB_KERNEL_COEFS);
    }
    velocity_divergence(S, q.u, q.v, q.w, w.rhs);
    if (source != nullptr) {
        // the Newton preconditioner's continuity rows: div(du) = r_p
        // (pressure_correction's source, Simplec.H:130-138)
        double* rhs = w.rhs;
        for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            rhs[o] -= source[o];
        }, GB_KERNEL_MASSFLUX);
    }
    {
        RedPack P{};
        P.it[0] = red_item(valid_box(g, CC), w.rhs, nullptr, 0, W_DIV_BEFORE);
        P.it[1] = red_item(valid_box(g, XF), q.u, nullptr, 0, W_SPEED_U);
        P.it[2] = red_item(valid_box(g, YF), q.v, nullptr, 0, W_SPEED_V);
        P.it[3] = red_item(valid_box(g, ZF), q.w, nullptr, 0, W_SPEED_W);
        P.n = 4;
        dmax_many(S, P);
    }
    return poisson_set_coeffs(S->poisson, S->mesh.ax, S->mesh.ay, S->mesh.az, w.beta[0], w.beta[1], w.beta[2]);
}

//! pressure_correction's Krylov solve (host-synchronising) and the check of
//! the singular case's removed mean.
gb_status pressure_solve(gb_simplec* S, gb_iter_info* info, bool project_net_source = false)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    gb_poisson_result pr{};
    gb_status st = poisson_solve(S->poisson, w.rhs, w.phi, &pr);
    if (st != GB_OK) { return st; }
    info->poisson_iterations = pr.iterations;
    info->poisson_removed_mean = pr.removed_mean;
    if (pr.singular && !project_net_source) {
        unsigned long long sp[3];
        if ((st = read_words(ctx, W_SPEED_U, 3, sp)) != GB_OK) { return st; }
        const double speed = std::max(std::max(bits_to_double(sp[0]), bits_to_double(sp[1])), bits_to_double(sp[2]));
        const double inv_h = 1.0 / g.dx + 1.0 / g.dy + 1.0 / (S->jmin * g.dzeta);
        if (std::fabs(pr.removed_mean) > 1.0e-8 * speed * inv_h) {
            set_error("gust: pressure_correction: the predicted velocity has a net source the boundaries cannot carry: "
                      "J-weighted mean divergence %g 1/s against the scale %g 1/s (a boundary condition or the "
                      "predictor is inconsistent)", pr.removed_mean, speed * inv_h);
            return GB_BAD_ARG;
        }
    }
    return GB_OK;
}

//! pressure_correction's last part: the fluxes, p, u, v, Omega and w, the
//! divergence after (no host synchronisation).
gb_status pressure_finish(gb_simplec* S, const gb_state& q)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    gb_status st;
    double* F[3] = {w.G[0], w.G[1], w.G[2]};
    if ((st = poisson_fluxes(S->poisson, w.phi, w.beta[0], w.beta[1], w.beta[2], F[0], F[1], F[2])) != GB_OK) { return st; }
    const double alpha = S->opt.alpha_p;
    double* p = q.p;
    const double* phi = w.phi;
    for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
        const int64_t o = at(g, i, j, k);
        p[o] += alpha * phi[o];
    });
    {
        RedPack P{};
        P.it[0] = red_item(valid_box(g, CC), w.phi, nullptr, 0, W_MAX_PHI);
        for (int c = 0; c < 3; ++c) { P.it[1 + c] = red_item(valid_box(g, kLoc[c]), F[c], w.keep[c], 0, W_MAX_FU + c); }
        P.n = 4;
        dmax_many(S, P);
    }
    omega_from_w(S, q.u, q.v, q.w, w.om);
    double* tgt[3] = {q.u, q.v, w.om};
    for (int c = 0; c < 3; ++c) {
        double* tc = tgt[c];
        const double* fc = F[c];
        const double* kc = w.keep[c];
        for_box(ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            tc[o] += fc[o] * kc[o];
        });
    }
    seam_sync<double>(ctx, g, XF, q.u);
    seam_sync<double>(ctx, g, YF, q.v);
    seam_sync<double>(ctx, g, ZF, w.om);
    {
        double* f2[2] = {q.u, q.v};
        const int t2[2] = {XF, YF};
        fill_periodic_all(S, f2, t2, 2);
    }
    // w = Omega + z_x u_f + z_y v_f
    {
        double* ww = q.w;
        const double* u = q.u;
        const double* v = q.v;
        const double* om = w.om;
        const double* z = S->z;
        for_box(ctx, valid_box(g, ZF), [=] __device__(int i, int j, int k) {
            ww[at(g, i, j, k)] = om[at(g, i, j, k)] + deriv<NODE, ZF, 0>(z, g, i, j, k) * (1.0 / g.dx) * interp<XF, ZF>(u, g, i, j, k)
                               + deriv<NODE, ZF, 1>(z, g, i, j, k) * (1.0 / g.dy) * interp<YF, ZF>(v, g, i, j, k);
        }, GB_KERNEL_MASSFLUX);
    }
    seam_sync<double>(ctx, g, ZF, q.w);
    {
        double* f1[1] = {q.w};
        const int t1[1] = {ZF};
        fill_periodic_all(S, f1, t1, 1);
    }
    velocity_divergence(S, q.u, q.v, q.w, w.rhs);
    dmax(S, valid_box(g, CC), w.rhs, nullptr, W_DIV_AFTER);
    return check_cuda("pressure_correction");
}

//! Simplec.cpp:134-220 pressure_correction on q (its ghosts filled).
gb_status pressure_correction(gb_simplec* S, const gb_state& q, gb_iter_info* info)
{
    gb_status st = pressure_prelude(S, q);
    if (st == GB_OK) { st = pressure_solve(S, info); }
    if (st == GB_OK) { st = pressure_finish(S, q); }
    return st;
}

//! A key of what a captured iteration segment's kernel arguments depend on.
uint64_t segment_key(const gb_simplec* S, const gb_state& q, const double* dtau)
{
    uint64_t k = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { k = (k ^ v) * 1099511628211ull; };
    const double* ptrs[8] = {q.u, q.v, q.w, q.p, q.theta, q.tke, q.z_nd, dtau};
    for (const double* p : ptrs) { mix(reinterpret_cast<uintptr_t>(p)); }
    mix(S->has_hist ? 1 : 0);
    for (int n = 0; n < GB_N_TUNE; ++n) { mix(static_cast<uint32_t>(S->ctx->tune[n])); }
    return k;
}

//! body() (launches on the context's stream, no host synchronisation) run
//! eagerly or as the stage's graph `id`: eagerly on the stage's first
//! iteration (it sizes the scratch and sets the kernels' attributes), while
//! profiling and with GB_TUNE_GRAPHS = 1; else the graph, captured on the
//! stage's stream when its key changed, launched on the context's stream.
//! The kernels and their order are the same either way.
template <typename F>
gb_status run_segment(gb_simplec* S, int id, uint64_t key, F&& body)
{
    gb_ctx* ctx = S->ctx;
    if (ctx->tune[GB_TUNE_GRAPHS] == 1 || ctx->profiling || S->iterations == 0) { return body(); }
    if (S->seg_exec[id] != nullptr && S->seg_key[id] != key) {
        cudaGraphExecDestroy(S->seg_exec[id]);
        S->seg_exec[id] = nullptr;
    }
    if (S->seg_exec[id] == nullptr) {
        if (S->capture_stream == nullptr
            && cudaStreamCreateWithFlags(&S->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            S->capture_stream = nullptr;
            return body();
        }
        cudaStream_t own = ctx->stream;
        const int64_t launches0 = ctx->launches;
        cudaGraph_t graph = nullptr;
        gb_status st = GB_OK;
        ctx->stream = S->capture_stream;
        bool ok = cudaStreamBeginCapture(S->capture_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            st = body();
            ok = cudaStreamEndCapture(S->capture_stream, &graph) == cudaSuccess && graph != nullptr && st == GB_OK;
        }
        ctx->stream = own;
        const int64_t n = ctx->launches - launches0;
        ctx->launches = launches0;
        if (ok) { ok = cudaGraphInstantiate(&S->seg_exec[id], graph, 0) == cudaSuccess; }
        if (graph != nullptr) { cudaGraphDestroy(graph); }
        if (!ok) {
            // a capture that failed recorded nothing that ran: run the segment eagerly
            cudaGetLastError();
            S->seg_exec[id] = nullptr;
            return body();
        }
        S->seg_launches[id] = n;
        S->seg_key[id] = key;
    }
    cudaGraphLaunch(S->seg_exec[id], ctx->stream);
    ctx->launches += S->seg_launches[id];
    return GB_OK;
}

//! Simplec.cpp:222-281 scalar_sweep for theta and for k: each system's rows
//! (the A1 rows, a_P = 1/dtau + A_P, rhs = -R), the two solved by one batched
//! line solve (the systems are independent), the increments added, k clipped
//! at the floor with the clipped points counted.
gb_status scalar_sweeps(gb_simplec* S, const gb_state& q, const double* dtau, bool clip = true)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    const int64_t cs = volume(g);
    const int eqs[2] = {F_THETA, F_TKE};
    double* fields[2] = {q.theta, q.tke};
    const double* Rq[2] = {w.R[4], w.R[5]};
    for (int e = 0; e < 2; ++e) {
        simplec_implicit_rows(S, eqs[e], w.F, w.Am[e]);
        double* rhs = w.rhsm[e];
        double* ap = w.ap[e];
        const double* A = w.Am[e];
        const double* Req = Rq[e];
        for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            rhs[o] = -Req[o];
            ap[o] = 1.0 / dtau[o] + A[GB_COEF_P * cs + o];
        }, GB_KERNEL_COEFS);
    }
    const int locs[2] = {CC, CC};
    const int words[2] = {W_LAST_TH, W_LAST_K};
    gb_status st = line_solve_multi(S, 2, locs, w.Am, w.ap, w.rhsm, w.deltam, words);
    if (st != GB_OK) { return st; }
    const int wmax[2] = {W_MAX_DTH, W_MAX_DK};
    unsigned long long* count = dword(ctx, W_CLIPPED);
    for (int e = 0; e < 2; ++e) {
        dmax(S, valid_box(g, CC), w.deltam[e], nullptr, wmax[e]);
        const double* delta = w.deltam[e];
        double* field = fields[e];
        const bool do_clip = (eqs[e] == F_TKE) && clip;
        const double floor = S->opt.tke_floor;
        for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            double v = field[o] + delta[o];
            if (do_clip && v < floor) {
                v = floor;
                atomicAdd(count, 1ull);
            }
            field[o] = v;
        });
    }
    return check_cuda("scalar_sweep");
}

}  // namespace

// ------------------------------------------------------------- iterate ---

gb_status simplec_iterate(gb_simplec* S, const gb_state& q, const double* dtau, gb_iter_info* info)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    *info = gb_iter_info{};
    const uint64_t key = segment_key(S, q, dtau);
    // 1.-3. up to the Krylov solve of the pressure correction
    gb_status st = run_segment(S, 0, key, [&]() -> gb_status {
    cudaMemsetAsync(dword(ctx, 0), 0, sizeof(unsigned long long) * W_COUNT, ctx->stream);
    cudaMemsetAsync(dword(ctx, W_SURFACE_BAD), 0, sizeof(unsigned long long), ctx->stream);
    // 1. ghosts and the wall state at q; 2. the residual (the closure at q)
    fill_ghosts_into(S, q, S->ss);
    simplec_residual(S, q, w.R);
    if (S->ph.closure) {
        cudaMemcpyAsync(S->nu_dtau, S->cf[kClosureNu], sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    }
    residual_sums(S, q);
    dmax_velocity(S, q.u, q.v, q.w, W_MON_U);
    transport_fluxes(S, q, w.F[0], w.F[1], w.F[2]);
    face_dtau(S, dtau, w.dtf);
    gb_status s1 = momentum_predictor(S, q, w.R);
    if (s1 != GB_OK) { return s1; }
    fill_ghosts_into(S, q, S->sst);
    return pressure_prelude(S, q);
    });
    if (st != GB_OK) { return st; }
    if ((st = pressure_solve(S, info)) != GB_OK) { return st; }
    // 4. the rest of the correction, 5. theta and k, 6. the nu_t history
    st = run_segment(S, 1, key, [&]() -> gb_status {
    gb_status s2 = pressure_finish(S, q);
    if (s2 != GB_OK) { return s2; }
    convection<CC>(S, q.theta, w.F, S->ph.limiter, S->ph.smooth_eps_theta, false, w.conv0);
    fill_ghosts_into(S, q, S->sst);
    transport_fluxes(S, q, w.F[0], w.F[1], w.F[2]);
    convection<CC>(S, q.theta, w.F, S->ph.limiter, S->ph.smooth_eps_theta, false, w.conv1);
    {
        double* Rt = w.R[4];
        const double* c0 = w.conv0;
        const double* c1 = w.conv1;
        for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            Rt[o] += c1[o] - c0[o];
        });
    }
    if ((s2 = scalar_sweeps(S, q, dtau)) != GB_OK) { return s2; }
    // 6. the nu_t history (Closure::accept): the fields of this iteration's residual
    if (S->ph.closure) {
        cudaMemcpyAsync(S->nut_hist, S->cf[kClosureNut], sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    }
    return GB_OK;
    });
    if (st != GB_OK) { return st; }
    if (S->ph.closure) { S->has_hist = true; }
    ++S->iterations;
    // read every result of the iteration at once
    unsigned long long words[W_COUNT];
    if ((st = read_words(ctx, 0, W_COUNT, words)) != GB_OK) { return st; }
    double sums[8];
    cudaMemcpyAsync(S->h_words, w.sums, sizeof(double) * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("simplec_iterate"); }
    std::memcpy(sums, S->h_words, sizeof(double) * 8);
    auto wd = [&](int n) { return bits_to_double(words[n]); };
    const gb_physics& ph = S->ph;
    const double U = ph.scale_velocity, H = ph.scale_height;
    const double scale[6] = {U * U / H, U * U / H, U * U / H, U / H, U * ph.scale_theta / H, U * ph.scale_tke / H};
    for (int n = 0; n < 6; ++n) {
        const Box b = valid_box(g, kLoc[n]);
        info->residual_norms[n] = std::sqrt(sums[n]) / std::sqrt(static_cast<double>(b.count())) / scale[n];
    }
    info->mean_tke = sums[SUM_TKE] / (static_cast<double>(g.nx) * g.ny * g.nz);
    info->mean_ustar = S->wall ? sums[SUM_USTAR] / (static_cast<double>(g.nx) * g.ny) : 0.0;
    info->max_speed = std::max(std::max(wd(W_MON_U), wd(W_MON_V)), wd(W_MON_W));
    info->max_du = wd(W_MAX_DU);
    info->max_dv = wd(W_MAX_DV);
    info->max_dw = wd(W_MAX_DW);
    info->last_sweep_du = wd(W_LAST_U);
    info->last_sweep_dv = wd(W_LAST_V);
    info->last_sweep_dw = wd(W_LAST_W);
    info->divergence_before = wd(W_DIV_BEFORE);
    info->divergence_after = wd(W_DIV_AFTER);
    info->max_dp = S->opt.alpha_p * wd(W_MAX_PHI);
    info->max_dtheta = wd(W_MAX_DTH);
    info->max_dtke = wd(W_MAX_DK);
    info->tke_clipped = static_cast<int64_t>(words[W_CLIPPED]);
    if (S->wall) {
        unsigned long long bad = 0;
        if ((st = read_words(ctx, W_SURFACE_BAD, 1, &bad)) != GB_OK) { return st; }
        if (bad > 0) {
            set_error("gust: compute_surface_state: no positive, finite friction velocity at %llu column fills "
                      "(surface layer heat_flux = %g)", bad, S->bc.surface_heat_flux);
            return GB_NONFINITE;
        }
    }
    for (int n = 0; n < 6; ++n) {
        if (!std::isfinite(info->residual_norms[n])) {
            set_error("gust: SimplecStage::iterate: non-finite residual (equation %d)", n);
            return GB_NONFINITE;
        }
    }
    return check_cuda("SimplecStage::iterate");
}

//! stage_norms (Simplec.cpp:385-409) at q with no iteration: the ghost fill
//! (the wall state), the residual, the six scaled RMS norms and the monitors
//! (max speed, mean k, mean u* with the surface layer).
// ------------------------------------------- the stage's steps alone ---
//
// The predictor, the pressure correction and the scalar sweep as the
// reference's callers outside SimplecStage::iterate use them
// (NewtonPreconditioner, Transfer's prolong_state): each is the same code
// the iteration runs, on the stage's workspace, with its result words read
// back at the end.

gb_status simplec_predictor_step(gb_simplec* S, const gb_state& q, double* const* R, const double* dtau,
                                 double* const* ap_out, double* const* d_out, gb_predictor_result* res)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    *res = gb_predictor_result{};
    cudaMemsetAsync(dword(ctx, 0), 0, sizeof(unsigned long long) * W_COUNT, ctx->stream);
    transport_fluxes(S, q, w.F[0], w.F[1], w.F[2]);
    face_dtau(S, dtau, w.dtf);
    double* Rl[6];
    for (int n = 0; n < 6; ++n) { Rl[n] = R[n]; }
    gb_status st = momentum_predictor(S, q, Rl);
    if (st != GB_OK) { return st; }
    for (int c = 0; c < 3; ++c) {
        if (ap_out != nullptr && ap_out[c] != nullptr) {
            cudaMemcpyAsync(ap_out[c], w.ap[c], sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
        }
        if (d_out != nullptr && d_out[c] != nullptr) {
            cudaMemcpyAsync(d_out[c], w.dd[c], sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
        }
    }
    unsigned long long words[W_COUNT];
    if ((st = read_words(ctx, 0, W_COUNT, words)) != GB_OK) { return st; }
    res->max_du = bits_to_double(words[W_MAX_DU]);
    res->max_dv = bits_to_double(words[W_MAX_DV]);
    res->max_dw = bits_to_double(words[W_MAX_DW]);
    res->last_sweep_du = bits_to_double(words[W_LAST_U]);
    res->last_sweep_dv = bits_to_double(words[W_LAST_V]);
    res->last_sweep_dw = bits_to_double(words[W_LAST_W]);
    return check_cuda("momentum_predictor");
}

gb_status simplec_pressure_step(gb_simplec* S, const gb_state& q, const double* const* d, gb_pressure_result* res)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    *res = gb_pressure_result{};
    if (d != nullptr) {
        for (int c = 0; c < 3; ++c) {
            cudaMemcpyAsync(w.dd[c], d[c], sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
        }
    }
    cudaMemsetAsync(dword(ctx, 0), 0, sizeof(unsigned long long) * W_COUNT, ctx->stream);
    // the ghosts of u* refilled first (Simplec.cpp:486), without the wall
    // state the iteration's first fill keeps for the scalar sweeps
    fill_ghosts_into(S, q, S->sst);
    gb_iter_info info{};
    gb_status st = pressure_correction(S, q, &info);
    if (st != GB_OK) { return st; }
    unsigned long long words[W_COUNT];
    if ((st = read_words(ctx, 0, W_COUNT, words)) != GB_OK) { return st; }
    res->poisson_iterations = info.poisson_iterations;
    res->poisson_removed_mean = info.poisson_removed_mean;
    res->divergence_before = bits_to_double(words[W_DIV_BEFORE]);
    res->divergence_after = bits_to_double(words[W_DIV_AFTER]);
    res->max_dp = S->opt.alpha_p * bits_to_double(words[W_MAX_PHI]);
    res->max_du = bits_to_double(words[W_MAX_FU]);
    res->max_dv = bits_to_double(words[W_MAX_FV]);
    res->max_dw = bits_to_double(words[W_MAX_FW]);
    return check_cuda("pressure_correction");
}

gb_status simplec_scalar_step(gb_simplec* S, const gb_state& q, int eq, const double* R_eq, const double* dtau,
                              int clip, gb_scalar_result* res)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    const int64_t cs = volume(g);
    *res = gb_scalar_result{};
    cudaMemsetAsync(dword(ctx, 0), 0, sizeof(unsigned long long) * W_COUNT, ctx->stream);
    // the ghosts and the transport fluxes of the current (corrected) state, as
    // the iteration refills them before the sweeps (Simplec.cpp:494-495)
    fill_ghosts_into(S, q, S->sst);
    transport_fluxes(S, q, w.F[0], w.F[1], w.F[2]);
    simplec_implicit_rows(S, eq, w.F, w.Am[0]);
    double* rhs = w.rhsm[0];
    double* ap = w.ap[0];
    const double* A = w.Am[0];
    for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
        const int64_t o = at(g, i, j, k);
        rhs[o] = -R_eq[o];
        ap[o] = 1.0 / dtau[o] + A[GB_COEF_P * cs + o];
    }, GB_KERNEL_COEFS);
    const int word = (eq == F_THETA) ? W_LAST_TH : W_LAST_K;
    gb_status st = line_solve(S, CC, w.Am[0], w.ap[0], w.rhsm[0], w.deltam[0], word);
    if (st != GB_OK) { return st; }
    const int wmax = (eq == F_THETA) ? W_MAX_DTH : W_MAX_DK;
    dmax(S, valid_box(g, CC), w.deltam[0], nullptr, wmax);
    unsigned long long* count = dword(ctx, W_CLIPPED);
    const double* delta = w.deltam[0];
    double* field = (eq == F_THETA) ? q.theta : q.tke;
    const bool do_clip = (eq == F_TKE) && clip;
    const double floor = S->opt.tke_floor;
    for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
        const int64_t o = at(g, i, j, k);
        double v = field[o] + delta[o];
        if (do_clip && v < floor) {
            v = floor;
            atomicAdd(count, 1ull);
        }
        field[o] = v;
    });
    unsigned long long words[W_COUNT];
    if ((st = read_words(ctx, 0, W_COUNT, words)) != GB_OK) { return st; }
    res->max_dq = bits_to_double(words[wmax]);
    res->last_sweep = bits_to_double(words[word]);
    res->clipped = static_cast<int64_t>(words[W_CLIPPED]);
    return check_cuda("scalar_sweep");
}

gb_status implicit_coefficients_at(gb_ctx* ctx, const gb_grid& g, int loc, double* const* F, const double* gamma,
                                   const double* z, const double* J, int logz, double* A)
{
    switch (loc) {
    case CC: implicit_coefficients_on<-1>(ctx, g, z, J, logz, F, gamma, A); break;
    case XF: implicit_coefficients_on<0>(ctx, g, z, J, logz, F, gamma, A); break;
    case YF: implicit_coefficients_on<1>(ctx, g, z, J, logz, F, gamma, A); break;
    default: implicit_coefficients_on<2>(ctx, g, z, J, logz, F, gamma, A); break;
    }
    return check_cuda("implicit_coefficients");
}

// ----------------------------------- the Newton stage's preconditioner ---
//
// gust::SimplecPreconditioner (Source/NewtonPreconditioner.H:1-108,
// NewtonPreconditioner.cpp:113-219): one SIMPLEC iteration on the Newton
// system linearized at q, (D + J) dq = r, from dq = 0, built from the stage's
// own pieces.

namespace {

gb_status lin_alloc(gb_simplec* S)
{
    if (S->lin_d[0] != nullptr) { return GB_OK; }
    const int64_t vol = volume(S->g);
    for (int f = 0; f < 6; ++f) {
        S->lin_d[f] = dbuf(S, vol);
        S->lin_qn[f] = dbuf(S, vol);
        if (!S->lin_d[f] || !S->lin_qn[f]) { return GB_OOM; }
    }
    for (int c = 0; c < 3; ++c) {
        S->lin_F0[c] = dbuf(S, vol);
        S->lin_F1[c] = dbuf(S, vol);
        if (!S->lin_F0[c] || !S->lin_F1[c]) { return GB_OOM; }
    }
    S->lin_conv0 = dbuf(S, vol);
    S->lin_dtau = dbuf(S, vol);
    if (!S->lin_conv0 || !S->lin_dtau) { return GB_OOM; }
    return GB_OK;
}

gb_state lin_state(double* const* f, const double* z)
{
    return gb_state{f[0], f[1], f[2], f[3], f[4], f[5], z};
}

}  // namespace

//! SimplecPreconditioner::setup (NewtonPreconditioner.cpp:113-150) at q:
//! the stage's fill with the wall state, the closure's fields at q (one
//! residual), the step (dtau, or local_dtau at inf_cfl when dtau is null),
//! the transport at q, the face steps, theta's convection at q and the
//! velocity scale max(1, max |u|).
gb_status simplec_linear_setup(gb_simplec* S, const gb_state& q, const double* dtau, double inf_cfl)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    gb_status st = lin_alloc(S);
    if (st != GB_OK) {
        set_error("gust: SimplecPreconditioner: out of device memory");
        return st;
    }
    fill_ghosts_into(S, q, S->ss);
    if (S->ph.closure) {
        simplec_residual(S, q, w.R);
        cudaMemcpyAsync(S->nu_dtau, S->cf[kClosureNu], sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    }
    if (dtau != nullptr) {
        cudaMemcpyAsync(S->lin_dtau, dtau, sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    } else if ((st = simplec_local_dtau(S, q, inf_cfl, S->lin_dtau)) != GB_OK) {
        return st;
    }
    transport_fluxes(S, q, S->lin_F0[0], S->lin_F0[1], S->lin_F0[2]);
    face_dtau(S, S->lin_dtau, w.dtf);
    convection<CC>(S, q.theta, S->lin_F0, S->ph.limiter, S->ph.smooth_eps_theta, false, S->lin_conv0);
    cudaMemsetAsync(dword(ctx, W_SPEED_U), 0, sizeof(unsigned long long) * 3, ctx->stream);
    dmax_velocity(S, q.u, q.v, q.w, W_SPEED_U);
    unsigned long long sp[3];
    if ((st = read_words(ctx, W_SPEED_U, 3, sp)) != GB_OK) { return st; }
    S->lin_speed = std::max(1.0, std::max(bits_to_double(sp[0]), std::max(bits_to_double(sp[1]), bits_to_double(sp[2]))));
    S->lin_ready = true;
    return check_cuda("SimplecPreconditioner::setup");
}

//! SimplecPreconditioner::apply (NewtonPreconditioner.cpp:152-219): dq from
//! r (six fields at the state's locations, valid points read). diagonal: the
//! SIMPLE denominators d = a_P (the reference's default) and theta's coupling
//! as the directional derivative along du with the scalar sweeps on q's
//! transport (linear in r); else the stage's SIMPLEC denominators with the
//! full du and the corrected transport (one iteration of the stage). The
//! wall state and the closure's fields are the stage's current ones (the
//! setup's, or the caller's refresh at q).
gb_status simplec_linear_apply(gb_simplec* S, const gb_state& q, const double* const* r, double* const* dq,
                               bool diagonal)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    const int64_t vol = volume(g);
    SimplecWork& w = S->w;
    if (!S->lin_ready) {
        set_error("gust: SimplecPreconditioner::apply: setup has not been called");
        return GB_BAD_ARG;
    }
    // -r in place of the residual (the stage's R(q) for r = -R(q))
    for (int f = 0; f < 6; ++f) {
        cudaMemsetAsync(w.R[f], 0, sizeof(double) * vol, ctx->stream);
        double* Rf = w.R[f];
        const double* rf = r[f];
        for_box(ctx, valid_box(g, kLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            Rf[o] = -rf[o];
        }, GB_KERNEL_VECTOR);
    }
    // 1. the momentum predictor on the increment from zero, theta = q's for
    // its buoyancy coupling, the transport, wall state and closure at q
    for (int f = 0; f < 6; ++f) {
        if (f == F_THETA) {
            cudaMemcpyAsync(S->lin_d[f], q.theta, sizeof(double) * vol, cudaMemcpyDeviceToDevice, ctx->stream);
        } else {
            cudaMemsetAsync(S->lin_d[f], 0, sizeof(double) * vol, ctx->stream);
        }
    }
    const gb_state d = lin_state(S->lin_d, q.z_nd);
    for (int c = 0; c < 3; ++c) {
        cudaMemcpyAsync(w.F[c], S->lin_F0[c], sizeof(double) * vol, cudaMemcpyDeviceToDevice, ctx->stream);
    }
    gb_status st = momentum_predictor(S, d, w.R);
    if (st != GB_OK) { return st; }
    // 2. the pressure correction of du*, r_p as the source, the homogeneous
    // fill giving du*'s ghosts (theta back to 0 first)
    cudaMemsetAsync(S->lin_d[F_THETA], 0, sizeof(double) * vol, ctx->stream);
    fill_ghosts_into(S, d, nullptr, true);
    if (diagonal) {
        for (int c = 0; c < 3; ++c) {
            double* dd = w.dd[c];
            const double* ap = w.ap[c];
            for_box(ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) {
                const int64_t o = at(g, i, j, k);
                dd[o] = (dd[o] > 0) ? ap[o] : 0.0;
            }, GB_KERNEL_COEFS);
        }
    }
    if ((st = pressure_prelude(S, d, r[3])) != GB_OK) { return st; }
    gb_iter_info info{};
    if ((st = pressure_solve(S, &info, true)) != GB_OK) { return st; }
    if ((st = pressure_finish(S, d)) != GB_OK) { return st; }
    // 3. theta's convection with the corrected velocity minus that at q:
    // diagonal, the directional derivative along du with the step
    // sigma = sqrt(eps) max(1, max|u|) / max|du|; else the full du
    double sigma = 1.0;
    if (diagonal) {
        cudaMemsetAsync(dword(ctx, W_MAX_DU), 0, sizeof(unsigned long long) * 3, ctx->stream);
        dmax_velocity(S, S->lin_d[F_U], S->lin_d[F_V], S->lin_d[F_W], W_MAX_DU);
        unsigned long long md[3];
        if ((st = read_words(ctx, W_MAX_DU, 3, md)) != GB_OK) { return st; }
        const double dmx = std::max(bits_to_double(md[0]), std::max(bits_to_double(md[1]), bits_to_double(md[2])));
        sigma = (dmx > 0) ? std::sqrt(std::numeric_limits<double>::epsilon()) * S->lin_speed / dmx : 1.0;
    }
    const double* qf[6] = {q.u, q.v, q.w, q.p, q.theta, q.tke};
    for (int f = 0; f < 6; ++f) {
        cudaMemcpyAsync(S->lin_qn[f], qf[f], sizeof(double) * vol, cudaMemcpyDeviceToDevice, ctx->stream);
    }
    for (int c = 0; c < 3; ++c) {
        double* qn = S->lin_qn[c];
        const double* dc = S->lin_d[c];
        for_box(ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            qn[o] += sigma * dc[o];
        }, GB_KERNEL_VECTOR);
    }
    const gb_state qn = lin_state(S->lin_qn, q.z_nd);
    fill_ghosts_into(S, qn, S->sst);
    transport_fluxes(S, qn, S->lin_F1[0], S->lin_F1[1], S->lin_F1[2]);
    convection<CC>(S, qn.theta, S->lin_F1, S->ph.limiter, S->ph.smooth_eps_theta, false, w.conv1);
    {
        double* Rt = w.R[F_THETA];
        const double* c0 = S->lin_conv0;
        const double* c1 = w.conv1;
        const double inv_sigma = 1.0 / sigma;
        for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            Rt[o] += inv_sigma * (c1[o] - c0[o]);
        }, GB_KERNEL_VECTOR);
    }
    // 4. the theta and k steps on the increments (0, ghosts included), no
    // floor on dk: diagonal, with q's transport; else the corrected one
    cudaMemsetAsync(S->lin_d[F_THETA], 0, sizeof(double) * vol, ctx->stream);
    cudaMemsetAsync(S->lin_d[F_TKE], 0, sizeof(double) * vol, ctx->stream);
    double* const* Fs = diagonal ? S->lin_F0 : S->lin_F1;
    for (int c = 0; c < 3; ++c) {
        cudaMemcpyAsync(w.F[c], Fs[c], sizeof(double) * vol, cudaMemcpyDeviceToDevice, ctx->stream);
    }
    if ((st = scalar_sweeps(S, d, S->lin_dtau, false)) != GB_OK) { return st; }
    // 5. dq: the increment's valid points; the Dirichlet rows of u, v, w are
    // identity rows of the Newton system (dq = r there); seam copies synced
    for (int f = 0; f < 6; ++f) {
        cudaMemsetAsync(dq[f], 0, sizeof(double) * vol, ctx->stream);
        double* o_ = dq[f];
        const double* src = S->lin_d[f];
        for_box(ctx, valid_box(g, kLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            o_[o] = src[o];
        }, GB_KERNEL_VECTOR);
    }
    for (int c = 0; c < 3; ++c) {
        dirichlet_rows(S, c, 1 << c, w.mask);
        double* o_ = dq[c];
        const double* rc = r[c];
        const double* mask = w.mask;
        for_box(ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            if (mask[o] > 0) { o_[o] = rc[o]; }
        }, GB_KERNEL_VECTOR);
        seam_sync<double>(ctx, g, kLoc[c], dq[c]);
    }
    return check_cuda("SimplecPreconditioner::apply");
}

gb_status simplec_norms(gb_simplec* S, const gb_state& q, double* res, double* mon)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    cudaMemsetAsync(dword(ctx, 0), 0, sizeof(unsigned long long) * W_COUNT, ctx->stream);
    fill_ghosts_into(S, q, S->ss);
    simplec_residual(S, q, w.R);
    residual_sums(S, q);
    dmax_velocity(S, q.u, q.v, q.w, W_MON_U);
    unsigned long long words[W_COUNT];
    gb_status st = read_words(ctx, 0, W_COUNT, words);
    if (st != GB_OK) { return st; }
    double sums[8];
    cudaMemcpyAsync(S->h_words, w.sums, sizeof(double) * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("stage_norms"); }
    std::memcpy(sums, S->h_words, sizeof(double) * 8);
    const gb_physics& ph = S->ph;
    const double U = ph.scale_velocity, H = ph.scale_height;
    const double scale[6] = {U * U / H, U * U / H, U * U / H, U / H, U * ph.scale_theta / H, U * ph.scale_tke / H};
    for (int n = 0; n < 6; ++n) {
        const Box b = valid_box(g, kLoc[n]);
        res[n] = std::sqrt(sums[n]) / std::sqrt(static_cast<double>(b.count())) / scale[n];
    }
    mon[0] = std::max(std::max(bits_to_double(words[W_MON_U]), bits_to_double(words[W_MON_V])), bits_to_double(words[W_MON_W]));
    mon[1] = sums[SUM_TKE] / (static_cast<double>(g.nx) * g.ny * g.nz);
    mon[2] = S->wall ? sums[SUM_USTAR] / (static_cast<double>(g.nx) * g.ny) : 0.0;
    return check_cuda("stage_norms");
}

//! SimplecStage::confidence (Simplec.cpp:411-445) on the residual of the last
//! iteration's start: the share of cells whose six residuals (both faces of
//! a velocity, the cell's p, theta and k) are within the thresholds (the
//! criterion's, per equation, times the residual scales), and the largest
//! height above the ground of a cell that is not.
gb_status simplec_confidence(gb_simplec* S, const double* thresholds, double* share, double* height)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    if (S->agl == nullptr) {
        if ((S->agl = dbuf(S, volume(g))) == nullptr) {
            set_error("gust: SimplecStage::confidence: cannot allocate the height above the ground");
            return GB_OOM;
        }
        turb_height_above_ground(ctx, g, S->z, S->agl);
    }
    const gb_physics& ph = S->ph;
    const double U = ph.scale_velocity, H = ph.scale_height;
    const double scale[6] = {U * U / H, U * U / H, U * U / H, U / H, U * ph.scale_theta / H, U * ph.scale_tke / H};
    double t[6];
    for (int n = 0; n < 6; ++n) { t[n] = thresholds[n] * scale[n]; }
    const double t0 = t[0], t1 = t[1], t2 = t[2], t3 = t[3], t4 = t[4], t5 = t[5];
    const double *ru = S->w.R[0], *rv = S->w.R[1], *rw = S->w.R[2], *rp = S->w.R[3], *rt = S->w.R[4], *rk = S->w.R[5];
    const double* d = S->agl;
    unsigned long long* bad = dword(ctx, W_CONF_BAD);
    unsigned long long* top = dword(ctx, W_CONF_TOP);
    cudaMemsetAsync(bad, 0, 2 * sizeof(unsigned long long), ctx->stream);
    for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
        const int64_t o = at(g, i, j, k);
        const bool ok = fmax(fabs(ru[o]), fabs(ru[at(g, i + 1, j, k)])) <= t0
                        && fmax(fabs(rv[o]), fabs(rv[at(g, i, j + 1, k)])) <= t1
                        && fmax(fabs(rw[o]), fabs(rw[at(g, i, j, k + 1)])) <= t2 && fabs(rp[o]) <= t3
                        && fabs(rt[o]) <= t4 && fabs(rk[o]) <= t5;
        if (!ok) {
            atomicAdd(bad, 1ull);
            atomic_max_nonneg(top, d[o]);
        }
    }, GB_KERNEL_VECTOR);
    unsigned long long words[2];
    gb_status st = read_words(ctx, W_CONF_BAD, 2, words);
    if (st != GB_OK) { return st; }
    const double cells = static_cast<double>(g.nx) * g.ny * g.nz;
    *share = 1.0 - static_cast<double>(words[0]) / cells;
    *height = bits_to_double(words[1]);
    return check_cuda("SimplecStage::confidence");
}

// ------------------------------------------------------ pseudo-time step ---

gb_status simplec_local_dtau(gb_simplec* S, const gb_state& q, double cfl, double* dtau)
{
    const gb_grid g = S->g;
    omega_from_w(S, q.u, q.v, q.w, S->w.om);
    const double* u = q.u;
    const double* v = q.v;
    const double* om = S->w.om;
    const double* J = S->mesh.detJ;
    const double* nu = S->ph.closure ? S->nu_dtau : S->df.nu;
    const double dxinv = 1.0 / g.dx, dyinv = 1.0 / g.dy, dzinv = 1.0 / g.dzeta;
    const double diff_h = 2 * (dxinv * dxinv + dyinv * dyinv);
    for_box(S->ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
        const double uc = interp<XF, CC>(u, g, i, j, k), vc = interp<YF, CC>(v, g, i, j, k), oc = interp<ZF, CC>(om, g, i, j, k);
        double rate = fabs(uc) * dxinv + fabs(vc) * dyinv + fabs(oc) * dzinv / J[at(g, i, j, k)];
        if (nu) { rate += nu[at(g, i, j, k)] * diff_h; }
        dtau[at(g, i, j, k)] = cfl / fmax(rate, 1.0e-12);
    }, GB_KERNEL_COEFS);
    return check_cuda("local_dtau");
}

// ------------------------------------------------------ initializer ---

namespace {

//! A profile component at every point of a field of type T (the valid box
//! grown by the state's two ghost layers) at the point's height above its
//! column's ground floored at h_min; k decays as exp(-(h - zi)/zi) above zi
//! (Source/Initializer.cpp:14-40 fill_from_profile).
void fill_from_profile(gb_simplec* S, int t, int f, double h_min, double zi, double* a)
{
    const gb_grid g = S->g;
    const Profile prof = S->prof;
    const double* z = S->z;
    const double zinv = 1.0 / std::max(zi, 2.2250738585072014e-308);
    Box b = valid_box(g, t);
    for (int d = 0; d < 3; ++d) {
        b.lo[d] -= 2;
        b.hi[d] += 2;
    }
    for_box(S->ctx, b, [=] __device__(int i, int j, int k) {
        const double h = fmax(height_above_ground(z, g, t, i, j, k), h_min);
        double val = prof.value(f, h);
        if (f == F_TKE && zi > 0) { val *= exp(-(fmax(h - zi, 0.0) * zinv)); }
        a[at(g, i, j, k)] = val;
    });
}

//! w = Omega + z_x u_f + z_y v_f on the valid z-faces (MassFlux.cpp w_from_omega).
void w_from_omega(gb_simplec* S, const double* u, const double* v, const double* om, double* w)
{
    const gb_grid g = S->g;
    const double* z = S->z;
    for_box(S->ctx, valid_box(g, ZF), [=] __device__(int i, int j, int k) {
        w[at(g, i, j, k)] = om[at(g, i, j, k)] + deriv<NODE, ZF, 0>(z, g, i, j, k) * (1.0 / g.dx) * interp<XF, ZF>(u, g, i, j, k)
                          + deriv<NODE, ZF, 1>(z, g, i, j, k) * (1.0 / g.dy) * interp<YF, ZF>(v, g, i, j, k);
    }, GB_KERNEL_MASSFLUX);
}

}  // namespace

gb_status simplec_initialize(gb_simplec* S, const gb_state& q, const gb_init_opts& o, gb_init_result* r)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    const int64_t vol = volume(g);
    SimplecWork& w = S->w;
    *r = gb_init_result{};
    // A new initial state starts without a nu_t history and with the first
    // local dtau's viscosity 0: in the reference each level's closure and
    // stage are new when its state is initialized (Closure::has_history,
    // Simplec.cpp:328).
    S->has_hist = false;
    if (S->ph.closure) { cudaMemsetAsync(S->nu_dtau, 0, sizeof(double) * volume(g), ctx->stream); }
    // 1. u, v at every point; w = 0 but the ground faces, which carry no flux
    fill_from_profile(S, XF, F_U, o.z_agl_min, 0.0, q.u);
    fill_from_profile(S, YF, F_V, o.z_agl_min, 0.0, q.v);
    cudaMemsetAsync(q.w, 0, sizeof(double) * vol, ctx->stream);
    omega_from_w(S, q.u, q.v, q.w, w.om);
    {
        double* om = w.om;
        Box ground = valid_box(g, ZF);
        ground.hi[2] = 0;
        for_box(ctx, ground, [=] __device__(int i, int j, int k) { om[at(g, i, j, k)] = 0.0; });
    }
    w_from_omega(S, q.u, q.v, w.om, q.w);
    // 2. k from the profile, theta the sounding (one ghost layer), p' = 0
    fill_from_profile(S, CC, F_TKE, o.z_agl_min, o.k_decay_height, q.tke);
    fill_theta_ref(S);
    cudaMemsetAsync(q.theta, 0, sizeof(double) * vol, ctx->stream);
    {
        const double* tr = w.theta_ref;
        double* th = q.theta;
        for_box(ctx, Box{{-1, -1, -1}, {g.nx, g.ny, g.nz}}, [=] __device__(int i, int j, int k) {
            th[at(g, i, j, k)] = tr[at(g, i, j, k)];
        });
    }
    cudaMemsetAsync(q.p, 0, sizeof(double) * vol, ctx->stream);
    cudaMemsetAsync(w.sums + 2, 0, sizeof(double), ctx->stream);
    if (o.obrien) {
        // O'Brien (Initializer.cpp:326-333; obrien_omega :197-274): Omega from
        // the column continuity of (a_x u, a_y v), a_z Omega_{k+1/2} =
        // a_z Omega_{k-1/2} - J Dh dzeta from 0 at the ground, the top value
        // E removed with ((z_f - z_ground) / depth)^2; one thread per column.
        cudaMemsetAsync(w.G[2], 0, sizeof(double) * vol, ctx->stream);
        gb_status st = face_divergence(ctx, g, S->mesh.ax, S->mesh.ay, S->mesh.az, S->mesh.detJ, q.u, q.v, w.G[2],
                                       w.rhs);
        if (st != GB_OK) { return st; }
        const double* az = S->mesh.az;
        const double* J = S->mesh.detJ;
        const double* dh = w.rhs;
        const double* zn = S->z;
        double* om = w.om;
        auto* worst = reinterpret_cast<unsigned long long*>(w.sums + 2);
        const double dzeta = g.dzeta;
        for_box(ctx, Box{{0, 0, 0}, {g.nx - 1, g.ny - 1, 0}}, [=] __device__(int i, int j, int) {
            om[at(g, i, j, 0)] = 0.0;
            for (int k = 0; k < g.nz; ++k) {
                om[at(g, i, j, k + 1)] = (az[at(g, i, j, k)] * om[at(g, i, j, k)]
                                          - J[at(g, i, j, k)] * dh[at(g, i, j, k)] * dzeta)
                                         / az[at(g, i, j, k + 1)];
            }
            const double E = om[at(g, i, j, g.nz)];
            // non-negative doubles order as their bit patterns (a NaN above all)
            atomicMax(worst, static_cast<unsigned long long>(__double_as_longlong(fabs(E))));
            auto zf = [&](int k) {
                return 0.25 * (zn[at(g, i, j, k)] + zn[at(g, i + 1, j, k)] + zn[at(g, i, j + 1, k)]
                               + zn[at(g, i + 1, j + 1, k)]);
            };
            const double zg = zf(0), depth = zf(g.nz) - zg;
            for (int k = 1; k <= g.nz; ++k) {
                const double frac = (zf(k) - zg) / depth;
                om[at(g, i, j, k)] -= frac * frac * E;
            }
            om[at(g, i, j, g.nz)] = 0.0;
        });
        w_from_omega(S, q.u, q.v, w.om, q.w);
    }
    // 3. the mass-consistent correction
    velocity_divergence(S, q.u, q.v, q.w, w.rhs);
    dsum(S, valid_box(g, CC), w.rhs, 0, 0);
    if (o.projection) {
        if (S->init_poisson != nullptr) {
            gb_poisson_destroy(S->init_poisson);
            S->init_poisson = nullptr;
        }
        // initializer_poisson_bc (Initializer.cpp:181-195): lambda = 0 on the
        // inflow and outflow faces, zero flux through the others
        int32_t pbc[6];
        for (int f = 0; f < 6; ++f) {
            const int d = f % 3;
            const int t = S->bc.face[f];
            pbc[f] = is_per(g, d) ? GB_POISSON_PERIODIC
                                  : ((t == GB_FACE_INFLOW || t == GB_FACE_OUTFLOW) ? GB_POISSON_DIRICHLET
                                                                                     : GB_POISSON_NEUMANN);
        }
        gb_poisson_opts po = o.poisson;
        gb_status st = gb_poisson_create(ctx, &g, pbc, S->z, S->mesh.detJ, &po, &S->init_poisson);
        if (st != GB_OK) { return st; }
        const bool unit = (o.alpha_h == 1 && o.alpha_v == 1);
        const double* beta[3] = {nullptr, nullptr, nullptr};
        if (!unit) {
            // Sigma = diag(alpha_h^2, alpha_h^2, alpha_v^2): x, y and the cross
            // part of the z-faces carry alpha_h^2, the z part alpha_v^2
            // (Initializer.cpp:380-403)
            const double ah2 = o.alpha_h * o.alpha_h, av2 = o.alpha_v * o.alpha_v;
            for (int c = 0; c < 3; ++c) {
                double* b = w.beta[c];
                const double v = (c == 2) ? av2 : ah2;
                for_box(ctx, Box{{-g.ng, -g.ng, -g.ng}, {g.nx + g.ng, g.ny + g.ng, g.nz + g.ng}},
                        [=] __device__(int i, int j, int k) { b[at(g, i, j, k)] = v; });
                beta[c] = w.beta[c];
            }
        }
        st = poisson_set_coeffs(S->init_poisson, S->mesh.ax, S->mesh.ay, S->mesh.az, beta[0], beta[1], beta[2]);
        if (st != GB_OK) { return st; }
        if (o.alpha_v != o.alpha_h) {
            // the split only where alpha_v != alpha_h: z_cross = alpha_h^2
            st = poisson_set_z_cross(S->init_poisson, S->mesh.az, beta[2], beta[0]);
            if (st != GB_OK) { return st; }
        }
        gb_poisson_result pr{};
        if ((st = poisson_solve(S->init_poisson, w.rhs, w.phi, &pr)) != GB_OK) { return st; }
        r->poisson_iterations = pr.iterations;
        r->poisson_final_residual = pr.final_residual;
        double* F[3] = {w.G[0], w.G[1], w.G[2]};
        if ((st = poisson_fluxes(S->init_poisson, w.phi, beta[0], beta[1], beta[2], F[0], F[1], F[2])) != GB_OK) {
            return st;
        }
        omega_from_w(S, q.u, q.v, q.w, w.om);
        double* tgt[3] = {q.u, q.v, w.om};
        for (int c = 0; c < 3; ++c) {
            double* tc = tgt[c];
            const double* fc = F[c];
            for_box(ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) {
                tc[at(g, i, j, k)] += fc[at(g, i, j, k)];
            });
        }
        {
            double* f2[2] = {q.u, q.v};
            const int t2[2] = {XF, YF};
            fill_periodic_all(S, f2, t2, 2);
        }
        w_from_omega(S, q.u, q.v, w.om, q.w);
        velocity_divergence(S, q.u, q.v, q.w, w.rhs);
        // the projection runs once per solve: its solver's memory goes back
        gb_poisson_destroy(S->init_poisson);
        S->init_poisson = nullptr;
    }
    dsum(S, valid_box(g, CC), w.rhs, 0, 1);
    double sums[3];
    cudaMemcpyAsync(sums, w.sums, sizeof(double) * 3, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("initialize_state"); }
    r->divergence_before = std::sqrt(sums[0]);
    r->divergence_after = std::sqrt(sums[1]);
    r->obrien_top_residual = sums[2];
    return check_cuda("initialize_state");
}

void simplec_implicit_rows_at(gb_simplec* S, const gb_state& q, int eq, double* A)
{
    transport_fluxes(S, q, S->w.F[0], S->w.F[1], S->w.F[2]);
    simplec_implicit_rows(S, eq, S->w.F, A);
}

gb_status simplec_set_wall_distance(gb_simplec* S, const double* dist)
{
    if (!S->ph.closure || S->dist == nullptr) {
        set_error("gust: SimplecStage::set_wall_distance: the stage has no closure (turb.model)");
        return GB_BAD_ARG;
    }
    cudaMemcpyAsync(S->dist, dist, sizeof(double) * volume(S->g), cudaMemcpyDeviceToDevice, S->ctx->stream);
    return check_cuda("SimplecStage::set_wall_distance");
}

gb_status simplec_turbulence(gb_simplec* S, double* const* closure, double* const* surface)
{
    gb_ctx* ctx = S->ctx;
    if (closure != nullptr) {
        if (!S->ph.closure) {
            set_error("gust: SimplecStage::closure_fields: the stage has no closure");
            return GB_BAD_ARG;
        }
        for (int n = 0; n < kClosureFields; ++n) {
            if (closure[n]) {
                cudaMemcpyAsync(closure[n], S->cf[n], sizeof(double) * volume(S->g), cudaMemcpyDeviceToDevice, ctx->stream);
            }
        }
    }
    if (surface != nullptr) {
        if (!S->wall) {
            set_error("gust: SimplecStage: the stage's ground is not a surface layer");
            return GB_BAD_ARG;
        }
        for (int n = 0; n < kSsPlanes; ++n) {
            if (surface[n]) {
                cudaMemcpyAsync(surface[n], S->ss[n], sizeof(double) * plane_size(S->g), cudaMemcpyDeviceToDevice,
                                ctx->stream);
            }
        }
    }
    return check_cuda("SimplecStage::closure_fields");
}

namespace {

//! Where a fine point sits among the coarse ones along one direction
//! (Axis, locate; Transfer.cpp:20-84): ic and the weight t, the domains
//! starting at 0.
struct Axis {
    int r, imin, imax, step;
    double lin, inv;
};

Axis make_axis(int N, bool periodic, int r, bool nod)
{
    Axis a{r, 0, 0, 1, 1.0, 0.0};
    if (nod) {
        a.imax = N - 1;
        a.inv = 1.0 / static_cast<double>(r);
    } else {
        a.inv = 1.0 / static_cast<double>(2 * r);
        if (periodic) {
            a.imin = -1;
            a.imax = N - 1;
        } else if (N >= 2) {
            a.imax = N - 2;
        } else {
            a.step = 0;
            a.lin = 0;
        }
    }
    return a;
}

__device__ __forceinline__ void locate(const Axis& a, bool nod, int i, int& ic, double& t)
{
    const int den = nod ? a.r : 2 * a.r;
    const int m = nod ? i : (2 * i + 1 - a.r);
    const int mm = nod ? m - 1 : m;
    int c = (mm >= 0) ? mm / den : -((-mm + den - 1) / den);
    c = min(max(c, a.imin), a.imax);
    t = a.lin * static_cast<double>(m - den * c) * a.inv;
    ic = c;
}

//! The bilinear interpolation per zeta-level of a coarse field at the fine
//! valid points of type t (interpolate<T>, Transfer.cpp:86-108). Only the
//! coarse valid points are read: a cell-centred index one past a periodic
//! face is its periodic image (the coarse image's ParallelCopy,
//! Transfer.cpp:316-320), so the coarse ghost cells need not be filled.
void interpolate(gb_ctx* ctx, const gb_grid& g, const gb_grid& gc, int t, const double* q, double* f, int r)
{
    const bool nx = nodal(t, 0), ny = nodal(t, 1);
    const Axis ax = make_axis(gc.nx, gc.periodic_x != 0, r, nx);
    const Axis ay = make_axis(gc.ny, gc.periodic_y != 0, r, ny);
    const bool wx = !nx && gc.periodic_x, wy = !ny && gc.periodic_y;
    const int NX = gc.nx, NY = gc.ny;
    const gb_grid gf = g, gcc = gc;
    for_box(ctx, valid_box(g, t), [=] __device__(int i, int j, int k) {
        int I, J;
        double tx, ty;
        locate(ax, nx, i, I, tx);
        locate(ay, ny, j, J, ty);
        int I1 = I + ax.step, J1 = J + ay.step;
        if (wx) {
            I = (I + NX) % NX;
            I1 = (I1 + NX) % NX;
        }
        if (wy) {
            J = (J + NY) % NY;
            J1 = (J1 + NY) % NY;
        }
        const double one = 1;
        f[at(gf, i, j, k)] = (one - ty) * ((one - tx) * q[at(gcc, I, J, k)] + tx * q[at(gcc, I1, J, k)])
                           + ty * ((one - tx) * q[at(gcc, I, J1, k)] + tx * q[at(gcc, I1, J1, k)]);
    }, GB_KERNEL_MG_TRANSFER);
}

}  // namespace

gb_status simplec_prolong(gb_simplec* S, const gb_state& q, const gb_grid& gc, const gb_state& qc, double reltol,
                          gb_prolong_result* res)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid g = S->g;
    SimplecWork& w = S->w;
    const int r = g.nx / gc.nx;
    // the prolonged state is a new level's: no nu_t history (a fresh Closure)
    // and the first local dtau's viscosity 0 (a fresh stage)
    S->has_hist = false;
    if (S->ph.closure) { cudaMemsetAsync(S->nu_dtau, 0, sizeof(double) * volume(g), ctx->stream); }
    // prolong_fields (Transfer.cpp:290-320)
    interpolate(ctx, g, gc, CC, qc.theta, q.theta, r);
    interpolate(ctx, g, gc, CC, qc.tke, q.tke, r);
    interpolate(ctx, g, gc, CC, qc.p, q.p, r);
    interpolate(ctx, g, gc, XF, qc.u, q.u, r);
    interpolate(ctx, g, gc, YF, qc.v, q.v, r);
    interpolate(ctx, g, gc, ZF, qc.w, q.w, r);
    // k >= the floor, counted
    cudaMemsetAsync(dword(ctx, 0), 0, sizeof(unsigned long long) * W_COUNT, ctx->stream);
    {
        double* tk = q.tke;
        const double floor_k = S->opt.tke_floor;
        unsigned long long* count = dword(ctx, W_CLIPPED);
        for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
            double* x = &tk[at(g, i, j, k)];
            if (*x < floor_k) {
                *x = floor_k;
                atomicAdd(count, 1ULL);
            }
        });
    }
    fill_ghosts_into(S, q, S->sst);
    // the projection: d = 1 - the Dirichlet mask, alpha_p 1, p' restored
    for (int c = 0; c < 3; ++c) {
        dirichlet_rows(S, c, kLoc[c], w.mask);
        double* dd = w.dd[c];
        const double* mk = w.mask;
        for_box(ctx, valid_box(g, kLoc[c]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            dd[o] = mk[o] * -1.0 + 1.0;
        });
    }
    cudaMemcpyAsync(w.tmp, q.p, sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    const double reltol_keep = S->poisson->opt.reltol, alpha_keep = S->opt.alpha_p;
    S->poisson->opt.reltol = reltol;
    S->opt.alpha_p = 1.0;
    gb_iter_info info{};
    gb_status st = pressure_correction(S, q, &info);
    S->poisson->opt.reltol = reltol_keep;
    S->opt.alpha_p = alpha_keep;
    if (st != GB_OK) { return st; }
    cudaMemcpyAsync(q.p, w.tmp, sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    unsigned long long words[W_COUNT];
    if ((st = read_words(ctx, 0, W_COUNT, words)) != GB_OK) { return st; }
    res->divergence_before = bits_to_double(words[W_DIV_BEFORE]);
    res->divergence_after = bits_to_double(words[W_DIV_AFTER]);
    res->poisson_iterations = info.poisson_iterations;
    res->tke_clipped = static_cast<int64_t>(words[W_CLIPPED]);
    return check_cuda("prolong_state");
}

const gb_grid& simplec_grid(const gb_simplec* S) { return S->g; }
gb_ctx* simplec_ctx(const gb_simplec* S) { return S->ctx; }
const gb_physics& simplec_physics(const gb_simplec* S) { return S->ph; }
const gb_simplec_opts& simplec_options(const gb_simplec* S) { return S->opt; }
int simplec_limiter(const gb_simplec* S) { return S->ph.limiter; }
void simplec_set_limiter(gb_simplec* S, int limiter) { S->ph.limiter = limiter; }
const double* simplec_theta_ref(const gb_simplec* S) { return S->w.theta_ref; }
void simplec_dirichlet_rows(gb_simplec* S, int c, double* mask) { dirichlet_rows(S, c, kLoc[c], mask); }
void simplec_face_dtau(gb_simplec* S, const double* dtau, double** faces) { face_dtau(S, dtau, faces); }
bool simplec_has_wall(const gb_simplec* S) { return S->wall; }

// ----------------------------------------------------------- creation ---

gb_status simplec_build(gb_simplec* S)
{
    gb_ctx* ctx = S->ctx;
    const gb_grid& g = S->g;
    const int64_t vol = volume(g);
    SimplecWork& w = S->w;
    for (int n = 0; n < 6; ++n) { w.R[n] = dbuf(S, vol); }
    for (int n = 0; n < 3; ++n) {
        w.F[n] = dbuf(S, vol);
        w.ap[n] = dbuf(S, vol);
        w.dd[n] = dbuf(S, vol);
        w.dtf[n] = dbuf(S, vol);
        w.beta[n] = dbuf(S, vol);
        w.keep[n] = dbuf(S, vol);
    }
    for (int n = 0; n < 3; ++n) { w.G[n] = dbuf(S, vol); }
    for (int n = 0; n < 9; ++n) { w.Gd[n] = dbuf(S, vol); }
    w.tmp = dbuf(S, vol);
    w.A = dbuf(S, vol * GB_N_COEFS);
    w.At = dbuf(S, vol * GB_N_COEFS);
    w.mask = dbuf(S, vol);
    w.rhs = dbuf(S, vol);
    w.delta = dbuf(S, vol);
    w.phi = dbuf(S, vol);
    w.om = dbuf(S, vol);
    w.theta_ref = dbuf(S, vol);
    w.conv0 = dbuf(S, vol);
    w.conv1 = dbuf(S, vol);
    w.og = dbuf(S, vol);
    w.level_sum = dbuf(S, g.nz + 1);
    w.partial = dbuf(S, static_cast<int64_t>(kRedBlocks) * (SUM_LEVEL + g.nz + 1));
    w.sums = dbuf(S, SUM_LEVEL + g.nz + 1);
    if (S->opt.precision == 1) {
        w.A32 = fbuf(S, vol * GB_N_COEFS);
        w.ap32 = fbuf(S, vol);
        w.rhs32 = fbuf(S, vol);
        w.delta32 = fbuf(S, vol);
    }
    w.Am[0] = w.A;
    w.rhsm[0] = w.rhs;
    w.deltam[0] = w.delta;
    w.A32m[0] = w.A32;
    w.ap32m[0] = w.ap32;
    w.rhs32m[0] = w.rhs32;
    w.delta32m[0] = w.delta32;
    for (int s = 1; s < 3; ++s) {
        w.Am[s] = dbuf(S, vol * GB_N_COEFS);
        w.rhsm[s] = dbuf(S, vol);
        w.deltam[s] = dbuf(S, vol);
        if (S->opt.precision == 1) {
            w.A32m[s] = fbuf(S, vol * GB_N_COEFS);
            w.ap32m[s] = fbuf(S, vol);
            w.rhs32m[s] = fbuf(S, vol);
            w.delta32m[s] = fbuf(S, vol);
        }
    }
    // the closure's fields and the surface state (gust::ClosureFields,
    // gust::SurfaceState), when the closure is on or the ground is a surface layer
    S->wall = S->bc.face[2] == GB_FACE_SURFACE_LAYER;
    S->dfe = S->df;
    bool turb_ok = true;
    if (S->ph.closure) {
        for (int n = 0; n < kClosureFields; ++n) { turb_ok = (S->cf[n] = dbuf(S, vol)) && turb_ok; }
        turb_ok = (S->dist = dbuf(S, vol)) && turb_ok;
        turb_ok = (S->nu_dtau = dbuf(S, vol)) && turb_ok;
        turb_ok = (S->nut_hist = dbuf(S, vol)) && turb_ok;
        S->dfe = gb_diffusivities{S->cf[kClosureNu], S->cf[kClosureGammaTheta], S->cf[kClosureGammaTke]};
    }
    if (S->wall) {
        const int64_t np = plane_size(g);
        for (int n = 0; n < kSsPlanes; ++n) {
            turb_ok = (S->ss[n] = dbuf(S, np)) && turb_ok;
            turb_ok = (S->ssr[n] = dbuf(S, np)) && turb_ok;
            turb_ok = (S->sst[n] = dbuf(S, np)) && turb_ok;
        }
        for (int n = 0; n < 3; ++n) { turb_ok = (S->gg[n] = dbuf(S, np)) && turb_ok; }
    }
    if (!turb_ok) {
        set_error("gust: SimplecStage: cannot allocate the closure's fields and the surface state");
        return GB_OOM;
    }
    if (S->ph.closure) { turb_height_above_ground(ctx, g, S->z, S->dist); }
    for (void* p : S->owned) {
        if (p == nullptr) {
            set_error("gust: SimplecStage: cannot allocate the workspace");
            return GB_OOM;
        }
    }
    if (cudaMallocHost(&S->h_words, sizeof(double) * 64) != cudaSuccess) {
        cudaGetLastError();
        return GB_OOM;
    }
    // the profile view and theta_ref
    Profile& p = S->prof;
    p.ustar = S->bc.inflow_ustar;
    p.z0 = S->bc.inflow_z0;
    p.kappa = S->bc.kappa;
    p.Cmu0 = S->bc.Cmu0;
    p.inv_lmax = S->bc.inflow_inv_lmax;
    const double pi = 3.14159265358979323846;
    p.cosd = std::cos(S->bc.inflow_direction * pi / 180.0);
    p.sind = std::sin(S->bc.inflow_direction * pi / 180.0);
    p.rn = S->bc.theta_ref_n;
    for (int n = 0; n < p.rn; ++n) {
        p.rz[n] = S->bc.theta_ref_z[n];
        p.rt[n] = S->bc.theta_ref_theta[n];
    }
    if (S->ph.gravity > 0) { fill_theta_ref(S); }
    // the Poisson solver of the correction (poisson_bc_from_faces, BoundaryConditions.cpp:362-380)
    int32_t pbc[6];
    for (int f = 0; f < 6; ++f) {
        const int d = f % 3;
        pbc[f] = is_per(g, d) ? GB_POISSON_PERIODIC
                              : (S->bc.face[f] == GB_FACE_OUTFLOW ? GB_POISSON_DIRICHLET : GB_POISSON_NEUMANN);
    }
    gb_poisson_opts po = S->opt.poisson;
    po.reltol = S->opt.pressure_reltol;
    po.precision = S->opt.precision;
    gb_status st = gb_poisson_create(ctx, &g, pbc, S->z, S->mesh.detJ, &po, &S->poisson);
    if (st != GB_OK) { return st; }
    // min J for the net-source scale (the mesh is fixed): one host pass at creation
    {
        std::vector<double> h(vol);
        cudaMemcpyAsync(h.data(), S->mesh.detJ, sizeof(double) * vol, cudaMemcpyDeviceToHost, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        double m = 1e300;
        for (int k = 0; k < g.nz; ++k) {
            for (int j = 0; j < g.ny; ++j) {
                for (int i = 0; i < g.nx; ++i) { m = std::min(m, h[at(g, i, j, k)]); }
            }
        }
        S->jmin = m;
    }
    return check_cuda("SimplecStage");
}

}  // namespace gb

namespace gb {

gb_status simplec_create_checked(gb_ctx* ctx, const gb_grid* g, const gb_bc* bc, const gb_physics* ph,
                                 const gb_simplec_opts* opt, const double* z_nd, const gb_mesh_fields* mesh,
                                 const gb_diffusivities* df, gb_simplec** out)
{
    *out = nullptr;
    auto* S = new (std::nothrow) gb_simplec;
    if (S == nullptr) { return GB_OOM; }
    S->ctx = ctx;
    S->g = *g;
    S->bc = *bc;
    S->ph = *ph;
    S->opt = *opt;
    S->z = z_nd;
    S->mesh = *mesh;
    S->df = *df;
    const gb_status st = simplec_build(S);
    if (st != GB_OK) {
        simplec_delete(S);
        return st;
    }
    *out = S;
    return GB_OK;
}

void simplec_delete(gb_simplec* S)
{
    if (S == nullptr) { return; }
    cudaStreamSynchronize(S->ctx->stream);
    for (int n = 0; n < 2; ++n) {
        if (S->seg_exec[n] != nullptr) { cudaGraphExecDestroy(S->seg_exec[n]); }
    }
    if (S->capture_stream != nullptr) { cudaStreamDestroy(S->capture_stream); }
    if (S->h_words) { cudaFreeHost(S->h_words); }
    delete S;
}

}  // namespace gb
