// The Newton-Krylov core of the finishing stage (gust::NewtonKrylov,
// gust::NewtonOperator, Source/Newton.H:1-330, Newton.cpp; gust::jvp,
// Source/Residual.cpp:324-396) on the GPU.
//
// One Newton step solves (D + J) dq = -R(q) by right-preconditioned flexible
// GMRES in scaled variables: x = S^-1 dq, rows scaled by T^-1, with S =
// diag(s_U, s_U, s_U, s_p, s_theta, s_k) and T = diag(s_U, s_U, s_U, 1,
// s_theta, s_k). D = 1/dtau on the momentum faces (the face dtau), theta and
// k, 0 on the continuity rows and on the Dirichlet rows of the normal
// velocities; no dtau is plain Newton (D = 0). Every product J v is a
// forward difference of the full residual, with the perturbed state's ghost
// cells refilled by the boundary conditions (so the wall law's ground
// gradient is differentiated too) and the step
//   eps = h (1 + mean |q~|) / rms(v~)
// over every owned point of every field, on the scaled variables (theta
// taken as theta - theta_ref). A vector is the six fields on the grid
// layout; the operations act on the valid points, and the inner products
// count a periodic seam face once (the low copy owns it). The update is
// skipped when |b| is not finite or the Krylov residual is above |b|
// (newton_update_usable).
//
// The preconditioner (steady.newton_preconditioner) is the identity or the
// SIMPLEC preconditioner of the stage (simplec_linear_setup/apply, one
// SIMPLEC iteration on the linearized system), applied in the unscaled
// variables: z = S^-1 P (T v). The reductions are block sums added on the
// host in a fixed order, so a step is deterministic.
#include "gb_simplec.cuh"
#include "gb_stencil.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <new>
#include <vector>

namespace gb {
namespace {

using namespace st;

constexpr int kNF = 6;
constexpr int kFieldLoc[kNF] = {XF, YF, ZF, CC, CC, CC};
constexpr int kRedBlocksN = 296;   // 2 x 148 SMs

using Vec = std::vector<double*>;  // six field arrays of the grid's volume

//! Whether a valid point is owned (a periodic seam face's high copy is not).
__device__ __forceinline__ bool owned(const gb_grid& g, int t, int i, int j)
{
    if ((t & 1) && g.periodic_x && i == g.nx) { return false; }
    if ((t & 2) && g.periodic_y && j == g.ny) { return false; }
    return true;
}

__device__ __forceinline__ double warp_sum_d(double v)
{
    for (int o = 16; o > 0; o >>= 1) { v += __shfl_xor_sync(0xffffffffu, v, o); }
    return v;
}

//! Block partial sums over the owned valid points of one field: mode 0
//! sum a b; mode 1 the jvp sums (|q - off| s^-1, (v s^-1)^2, 1) into three
//! partial rows.
__global__ void k_field_sums(gb_grid g, int t, int mode, const double* __restrict__ a, const double* __restrict__ b,
                             const double* __restrict__ off, double sinv, double* __restrict__ partial)
{
    __shared__ double red[3][8];
    const int nx = ext_x(g, t), ny = ext_y(g, t), nz = ext_z(g, t);
    const int64_t n_tot = static_cast<int64_t>(nx) * ny * nz;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < n_tot;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(n % nx);
        const int j = static_cast<int>((n / nx) % ny);
        const int k = static_cast<int>(n / (static_cast<int64_t>(nx) * ny));
        if (!owned(g, t, i, j)) { continue; }
        const int64_t o = at(g, i, j, k);
        if (mode == 0) {
            s0 += a[o] * b[o];
        } else {
            const double qq = off ? a[o] - off[o] : a[o];
            const double vv = b[o] * sinv;
            s0 += fabs(qq) * sinv;
            s1 += vv * vv;
            s2 += 1.0;
        }
    }
    s0 = warp_sum_d(s0);
    s1 = warp_sum_d(s1);
    s2 = warp_sum_d(s2);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = s0;
        red[1][threadIdx.x >> 5] = s1;
        red[2][threadIdx.x >> 5] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0, t1 = 0, t2 = 0;
        for (int w = 0; w < 8; ++w) {
            t0 += red[0][w];
            t1 += red[1][w];
            t2 += red[2][w];
        }
        partial[blockIdx.x] = t0;
        partial[kRedBlocksN + blockIdx.x] = t1;
        partial[2 * kRedBlocksN + blockIdx.x] = t2;
    }
}

}  // namespace
}  // namespace gb

struct gb_newton {
    gb_simplec* S{nullptr};
    gb_ctx* ctx{nullptr};                // the stage's context (outlives the stage)
    gb_newton_opts opt{};
    gb_grid g{};
    int64_t vol{0};
    double s[gb::kNF]{}, t[gb::kNF]{};
    std::vector<gb::Vec> V, Z;
    gb::Vec R0, Jv, dq, qp, inv_dtau, b, x, w, dir;
    gb::Vec dtf;                         // the face dtau (3)
    gb::Vec pr, pz;                      // the preconditioner's r = T v and its dq (with a preconditioner)
    double* partial{nullptr};            // device block sums
    double* h_partial{nullptr};          // pinned copy
    std::vector<void*> owned_mem;
    int jvp_calls{0};
    double eps_min{0}, eps_max{0};
    ~gb_newton()
    {
        for (void* p : owned_mem) { cudaFree(p); }
        if (h_partial) { cudaFreeHost(h_partial); }
    }
};

namespace gb {
namespace {

gb_ctx* nctx(gb_newton* n) { return simplec_ctx(n->S); }

double* nbuf(gb_newton* n, int64_t count)
{
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * std::max<int64_t>(count, 1)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaMemsetAsync(p, 0, sizeof(double) * std::max<int64_t>(count, 1), nctx(n)->stream);
    n->owned_mem.push_back(p);
    return static_cast<double*>(p);
}

bool make_vec(gb_newton* n, Vec& v, int fields = kNF)
{
    v.assign(fields, nullptr);
    for (int f = 0; f < fields; ++f) {
        if ((v[f] = nbuf(n, n->vol)) == nullptr) { return false; }
    }
    return true;
}

gb_state state_of(const Vec& v, const double* z)
{
    gb_state q{};
    q.u = v[0];
    q.v = v[1];
    q.w = v[2];
    q.p = v[3];
    q.theta = v[4];
    q.tke = v[5];
    q.z_nd = z;
    return q;
}

Vec vec_of(const gb_state& q)
{
    return Vec{q.u, q.v, q.w, q.p, q.theta, q.tke};
}

//! Sum of the partial rows written by k_field_sums for `launches` launches
//! (fields), each launch's three rows at its own offset; out[c] sums row c.
gb_status read_sums(gb_newton* n, int launches, double* out3)
{
    gb_ctx* ctx = nctx(n);
    const size_t bytes = sizeof(double) * 3 * kRedBlocksN * launches;
    cudaMemcpyAsync(n->h_partial, n->partial, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("Newton reduction"); }
    out3[0] = out3[1] = out3[2] = 0;
    for (int l = 0; l < launches; ++l) {
        for (int c = 0; c < 3; ++c) {
            double s = 0;
            for (int b = 0; b < kRedBlocksN; ++b) { s += n->h_partial[(3 * l + c) * kRedBlocksN + b]; }
            out3[c] += s;
        }
    }
    return GB_OK;
}

gb_status dot(gb_newton* n, const Vec& a, const Vec& b, double* out)
{
    gb_ctx* ctx = nctx(n);
    {
        Span span(ctx, GB_KERNEL_VECTOR);
        for (int f = 0; f < kNF; ++f) {
            k_field_sums<<<kRedBlocksN, 256, 0, ctx->stream>>>(n->g, kFieldLoc[f], 0, a[f], b[f], nullptr, 1.0,
                                                               n->partial + 3 * kRedBlocksN * f);
        }
        ctx->launches += kNF;
    }
    double s[3];
    gb_status st = read_sums(n, kNF, s);
    *out = s[0];
    return st;
}

//! y = a x + b y on the valid points (b = 0: y = a x; a = 0: y = b y).
void lincomb(gb_newton* n, const Vec& y, double a, const Vec& x, double b)
{
    const gb_grid g = n->g;
    for (int f = 0; f < kNF; ++f) {
        double* yf = y[f];
        const double* xf = x[f];
        for_box(nctx(n), valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            yf[o] = (b == 0.0) ? a * xf[o] : a * xf[o] + b * yf[o];
        }, GB_KERNEL_VECTOR);
    }
}

//! The jvp step and J v (refilled perturbation): Jv = (R(fill(q + eps v)) - R0) / eps.
gb_status jvp(gb_newton* n, const gb_state& q, const Vec& v, const Vec& R0, const Vec& Jv, double* eps_out)
{
    gb_simplec* S = n->S;
    gb_ctx* ctx = nctx(n);
    const gb_grid g = n->g;
    const Vec qf = vec_of(q);
    const double* tref = simplec_theta_ref(S);
    {
        Span span(ctx, GB_KERNEL_VECTOR);
        for (int f = 0; f < kNF; ++f) {
            k_field_sums<<<kRedBlocksN, 256, 0, ctx->stream>>>(g, kFieldLoc[f], 1, qf[f], v[f], f == 4 ? tref : nullptr,
                                                               1.0 / n->s[f], n->partial + 3 * kRedBlocksN * f);
        }
        ctx->launches += kNF;
    }
    double sums[3];
    gb_status st = read_sums(n, kNF, sums);
    if (st != GB_OK) { return st; }
    if (sums[1] == 0) {
        for (int f = 0; f < kNF; ++f) { cudaMemsetAsync(Jv[f], 0, sizeof(double) * n->vol, ctx->stream); }
        *eps_out = 0;
        return GB_OK;
    }
    const double mean_q = sums[0] / sums[2];
    const double rms_v = std::sqrt(sums[1] / sums[2]);
    const double eps = n->opt.fd_eps_scale * (1 + mean_q) / rms_v;
    // q + eps v on every point (v's ghost cells are 0), then the full fill
    // (the volume as one flat box of vol points: a grid of at most 2^31 points)
    const Box flat{{0, 0, 0}, {static_cast<int>(n->vol) - 1, 0, 0}};
    for (int f = 0; f < kNF; ++f) {
        double* pf = n->qp[f];
        const double* a = qf[f];
        const double* b = v[f];
        for_box(ctx, flat, [=] __device__(int i, int, int) { pf[i] = a[i] + eps * b[i]; }, GB_KERNEL_VECTOR);
    }
    const gb_state qps = state_of(n->qp, q.z_nd);
    simplec_fill_ghosts(S, qps);
    double* Rp[kNF] = {Jv[0], Jv[1], Jv[2], Jv[3], Jv[4], Jv[5]};
    simplec_residual(S, qps, Rp);
    const double einv = 1.0 / eps;
    for (int f = 0; f < kNF; ++f) {
        double* jf = Jv[f];
        const double* r0 = R0[f];
        for_box(ctx, valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            jf[o] = (jf[o] - r0[o]) * einv;
        }, GB_KERNEL_VECTOR);
    }
    ++n->jvp_calls;
    n->eps_min = (n->jvp_calls == 1) ? eps : std::min(n->eps_min, eps);
    n->eps_max = (n->jvp_calls == 1) ? eps : std::max(n->eps_max, eps);
    *eps_out = eps;
    return check_cuda("jvp");
}

//! Ax = T^-1 (D + J) S x.
gb_status apply_op(gb_newton* n, const gb_state& q, const Vec& x, const Vec& Ax, bool has_dtau)
{
    const gb_grid g = n->g;
    for (int f = 0; f < kNF; ++f) {
        double* d = n->dq[f];
        const double* xf = x[f];
        const double sf = n->s[f];
        for_box(nctx(n), valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            d[o] = sf * xf[o];
        }, GB_KERNEL_VECTOR);
    }
    double eps = 0;
    gb_status st = jvp(n, q, n->dq, n->R0, n->Jv, &eps);
    if (st != GB_OK) { return st; }
    for (int f = 0; f < kNF; ++f) {
        double* af = Ax[f];
        const double* jf = n->Jv[f];
        const double* d = n->dq[f];
        const double* id = has_dtau ? n->inv_dtau[f] : nullptr;
        const double tinv = 1.0 / n->t[f];
        for_box(nctx(n), valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            const double dj = id ? id[o] * d[o] + jf[o] : jf[o];
            af[o] = dj * tinv;
        }, GB_KERNEL_VECTOR);
    }
    return check_cuda("NewtonOperator::apply");
}

//! 1/dtau per field: the face dtau on u, v, w (0 on the Dirichlet rows),
//! the cell dtau on theta and k, 0 on p.
void setup_dtau(gb_newton* n, const double* dtau)
{
    gb_simplec* S = n->S;
    const gb_grid g = n->g;
    double* faces[3] = {n->dtf[0], n->dtf[1], n->dtf[2]};
    simplec_face_dtau(S, dtau, faces);
    for (int c = 0; c < 3; ++c) {
        simplec_dirichlet_rows(S, c, n->dir[c]);
        double* id = n->inv_dtau[c];
        const double* fd = faces[c];
        const double* m = n->dir[c];
        for_box(nctx(n), valid_box(g, kFieldLoc[c]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            id[o] = (m[o] > 0) ? 0.0 : 1.0 / fd[o];
        }, GB_KERNEL_VECTOR);
    }
    cudaMemsetAsync(n->inv_dtau[3], 0, sizeof(double) * n->vol, nctx(n)->stream);
    for (int f = 4; f < kNF; ++f) {
        double* id = n->inv_dtau[f];
        for_box(nctx(n), valid_box(g, CC), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            id[o] = 1.0 / dtau[o];
        }, GB_KERNEL_VECTOR);
    }
}

//! fill(q), R0 = R(q), b = -T^-1 R0, and |b|.
gb_status base(gb_newton* n, const gb_state& q, double* bnorm)
{
    simplec_fill_ghosts(n->S, q);
    double* R[kNF] = {n->R0[0], n->R0[1], n->R0[2], n->R0[3], n->R0[4], n->R0[5]};
    simplec_residual(n->S, q, R);
    for (int f = 0; f < kNF; ++f) {
        const double* r = n->R0[f];
        double* bf = n->b[f];
        const double m = -1.0 / n->t[f];
        const gb_grid g = n->g;
        for_box(nctx(n), valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            bf[o] = m * r[o];
        }, GB_KERNEL_VECTOR);
    }
    double bb = 0;
    gb_status st = dot(n, n->b, n->b, &bb);
    *bnorm = std::sqrt(bb);
    return st;
}

//! z = M v, the right preconditioner in the scaled variables: v itself
//! (identity), or S^-1 P (T v) with P one SIMPLEC iteration on the
//! unscaled linearized system (gust::SimplecPreconditioner::apply).
gb_status precondition(gb_newton* n, const gb_state& q, const Vec& v, const Vec& z)
{
    if (n->opt.preconditioner == 0) {
        lincomb(n, z, 1.0, v, 0.0);
        return GB_OK;
    }
    const gb_grid g = n->g;
    for (int f = 0; f < kNF; ++f) {
        double* r = n->pr[f];
        const double* vf = v[f];
        const double tf = n->t[f];
        for_box(nctx(n), valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            r[o] = tf * vf[o];
        }, GB_KERNEL_VECTOR);
    }
    // the stage's wall state and closure fields at q (the jvp's evaluations
    // in between left the perturbed state's), as the setup froze them
    simplec_fill_ghosts(n->S, q);
    if (simplec_physics(n->S).closure) {
        double* R[kNF] = {n->Jv[0], n->Jv[1], n->Jv[2], n->Jv[3], n->Jv[4], n->Jv[5]};
        simplec_residual(n->S, q, R);
    }
    const double* rr[kNF] = {n->pr[0], n->pr[1], n->pr[2], n->pr[3], n->pr[4], n->pr[5]};
    double* zz[kNF] = {n->pz[0], n->pz[1], n->pz[2], n->pz[3], n->pz[4], n->pz[5]};
    gb_status st = simplec_linear_apply(n->S, q, rr, zz, n->opt.preconditioner == 1);
    if (st != GB_OK) { return st; }
    for (int f = 0; f < kNF; ++f) {
        double* zf = z[f];
        const double* pf = n->pz[f];
        const double sinv = 1.0 / n->s[f];
        for_box(nctx(n), valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            zf[o] = sinv * pf[o];
        }, GB_KERNEL_VECTOR);
    }
    return check_cuda("NewtonPreconditioner::apply");
}

//! Restarted right-preconditioned flexible GMRES for A x = b from x = 0, to
//! |b - A x| <= rtol |b|.
gb_status fgmres(gb_newton* n, const gb_state& q, bool has_dtau, double bnorm, gb_newton_step_info* info)
{
    const int m = n->opt.gmres_restart;
    const double tol = n->opt.krylov_rtol * bnorm;
    std::vector<double> H(static_cast<size_t>(m + 1) * m), cs(m), sn(m), sv(m + 1), y(m);
    for (int f = 0; f < kNF; ++f) { cudaMemsetAsync(n->x[f], 0, sizeof(double) * n->vol, nctx(n)->stream); }
    int it = 0;
    double rnorm = bnorm;
    bool converged = !(bnorm > tol);
    gb_status st = GB_OK;
    while (!converged && it < n->opt.gmres_max_iters) {
        // r = b - A x
        if (it == 0) {
            lincomb(n, n->V[0], 1.0, n->b, 0.0);
        } else {
            if ((st = apply_op(n, q, n->x, n->w, has_dtau)) != GB_OK) { return st; }
            lincomb(n, n->V[0], 1.0, n->b, 0.0);
            lincomb(n, n->V[0], -1.0, n->w, 1.0);
        }
        double beta2 = 0;
        if ((st = dot(n, n->V[0], n->V[0], &beta2)) != GB_OK) { return st; }
        const double beta = std::sqrt(beta2);
        rnorm = beta;
        if (!(beta > tol)) {
            converged = true;
            break;
        }
        lincomb(n, n->V[0], 1.0 / beta, n->V[0], 0.0);
        std::fill(sv.begin(), sv.end(), 0.0);
        sv[0] = beta;
        int jj = 0;
        for (; jj < m && it < n->opt.gmres_max_iters; ++jj, ++it) {
            if ((st = precondition(n, q, n->V[jj], n->Z[jj])) != GB_OK) { return st; }
            if ((st = apply_op(n, q, n->Z[jj], n->w, has_dtau)) != GB_OK) { return st; }
            for (int i = 0; i <= jj; ++i) {
                double h = 0;
                if ((st = dot(n, n->w, n->V[i], &h)) != GB_OK) { return st; }
                H[static_cast<size_t>(i) * m + jj] = h;
                lincomb(n, n->w, -h, n->V[i], 1.0);
            }
            double hn2 = 0;
            if ((st = dot(n, n->w, n->w, &hn2)) != GB_OK) { return st; }
            const double hn = std::sqrt(hn2);
            H[static_cast<size_t>(jj + 1) * m + jj] = hn;
            if (hn > 0) { lincomb(n, n->V[jj + 1], 1.0 / hn, n->w, 0.0); }
            for (int i = 0; i < jj; ++i) {
                const double a = H[static_cast<size_t>(i) * m + jj], b2 = H[static_cast<size_t>(i + 1) * m + jj];
                H[static_cast<size_t>(i) * m + jj] = cs[i] * a + sn[i] * b2;
                H[static_cast<size_t>(i + 1) * m + jj] = -sn[i] * a + cs[i] * b2;
            }
            const double a = H[static_cast<size_t>(jj) * m + jj], b2 = H[static_cast<size_t>(jj + 1) * m + jj];
            const double rr = std::sqrt(a * a + b2 * b2);
            cs[jj] = (rr > 0) ? a / rr : 1.0;
            sn[jj] = (rr > 0) ? b2 / rr : 0.0;
            H[static_cast<size_t>(jj) * m + jj] = rr;
            H[static_cast<size_t>(jj + 1) * m + jj] = 0;
            sv[jj + 1] = -sn[jj] * sv[jj];
            sv[jj] = cs[jj] * sv[jj];
            rnorm = std::fabs(sv[jj + 1]);
            if (!(rnorm > tol) || !(hn > 0)) {
                converged = !(rnorm > tol);
                ++jj;
                ++it;
                break;
            }
        }
        for (int i = jj - 1; i >= 0; --i) {
            double acc = sv[i];
            for (int p = i + 1; p < jj; ++p) { acc -= H[static_cast<size_t>(i) * m + p] * y[p]; }
            y[i] = acc / H[static_cast<size_t>(i) * m + i];
        }
        for (int i = 0; i < jj; ++i) { lincomb(n, n->x, y[i], n->Z[i], 1.0); }
        if (converged) { break; }
    }
    info->gmres_iterations = it;
    info->gmres_status = converged ? 0 : 1;
    info->krylov_residual = rnorm;
    return check_cuda("FGMRES");
}

//! fill(q), R0, the solve; x holds S^-1 dq when info->applied.
gb_status solve(gb_newton* n, const gb_state& q, const double* dtau, gb_newton_step_info* info)
{
    *info = gb_newton_step_info{};
    n->jvp_calls = 0;
    n->eps_min = n->eps_max = 0;
    const bool has_dtau = dtau != nullptr;
    if (has_dtau) { setup_dtau(n, dtau); }
    double bnorm = 0;
    gb_status st = base(n, q, &bnorm);
    if (st != GB_OK) { return st; }
    info->residual_norm = bnorm;
    if (!std::isfinite(bnorm)) {
        info->applied = 0;
        return GB_OK;
    }
    if (bnorm == 0) {
        info->applied = 1;
        info->gmres_status = 0;
        for (int f = 0; f < kNF; ++f) { cudaMemsetAsync(n->x[f], 0, sizeof(double) * n->vol, nctx(n)->stream); }
        return GB_OK;
    }
    if (n->opt.preconditioner != 0 && (st = simplec_linear_setup(n->S, q, dtau, n->opt.inf_cfl)) != GB_OK) {
        return st;
    }
    if ((st = fgmres(n, q, has_dtau, bnorm, info)) != GB_OK) { return st; }
    info->krylov_relative = info->krylov_residual / bnorm;
    info->eps_min = n->eps_min;
    info->eps_max = n->eps_max;
    info->jvp_calls = n->jvp_calls;
    // newton_update_usable (Newton.cpp): the Krylov residual at most |b|
    info->applied = (std::isfinite(info->krylov_relative) && info->krylov_relative <= 1.0) ? 1 : 0;
    return GB_OK;
}

//! dst = (add ? dst : 0) + lambda S x on the valid points, k clipped at the floor when clip.
void add_scaled(gb_newton* n, const Vec& dst, const Vec& x, double lambda)
{
    const gb_grid g = n->g;
    for (int f = 0; f < kNF; ++f) {
        double* d = dst[f];
        const double* xf = x[f];
        const double sl = lambda * n->s[f];
        for_box(nctx(n), valid_box(g, kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t o = at(g, i, j, k);
            d[o] += sl * xf[o];
        }, GB_KERNEL_VECTOR);
    }
}

}  // namespace
}  // namespace gb

namespace {

gb_status check_newton(const gb_newton_opts* o)
{
    std::vector<std::string> err;
    char b[256];
    if (o->gmres_restart < 5 || o->gmres_restart > 200) {
        std::snprintf(b, sizeof(b), "steady.newton_gmres_restart = %d: must be from 5 to 200", o->gmres_restart);
        err.emplace_back(b);
    }
    if (o->gmres_max_iters < 1) {
        std::snprintf(b, sizeof(b), "steady.newton_gmres_max_iters = %d: must be >= 1", o->gmres_max_iters);
        err.emplace_back(b);
    }
    const double lo = std::pow(std::numeric_limits<double>::epsilon(), 0.75);
    if (!std::isfinite(o->fd_eps_scale) || !(o->fd_eps_scale >= lo) || !(o->fd_eps_scale <= 1e-2)) {
        std::snprintf(b, sizeof(b), "steady.newton_fd_eps_scale = %.3e: must be >= %.3e and <= 1e-2", o->fd_eps_scale, lo);
        err.emplace_back(b);
    }
    if (!std::isfinite(o->krylov_rtol) || !(o->krylov_rtol > 0) || !(o->krylov_rtol < 1)) {
        std::snprintf(b, sizeof(b), "steady.newton_krylov_rtol = %.3e: must be > 0 and < 1", o->krylov_rtol);
        err.emplace_back(b);
    }
    if (!std::isfinite(o->scale_pressure) || !(o->scale_pressure > 0)) {
        std::snprintf(b, sizeof(b), "the pressure scale = %.3e: must be finite and > 0", o->scale_pressure);
        err.emplace_back(b);
    }
    if (o->preconditioner < 0 || o->preconditioner > 2) {
        std::snprintf(b, sizeof(b), "steady.newton_preconditioner = %d: must be identity (0) or simplec (1, 2)",
                      o->preconditioner);
        err.emplace_back(b);
    }
    if (o->preconditioner != 0 && (!std::isfinite(o->inf_cfl) || !(o->inf_cfl > 0))) {
        std::snprintf(b, sizeof(b), "steady.cfl_max = %.3e: the preconditioner's CFL must be finite and > 0",
                      o->inf_cfl);
        err.emplace_back(b);
    }
    if (err.empty()) { return GB_OK; }
    std::string all = "gust: invalid inputs:";
    for (const auto& e : err) { all += "\n  " + e; }
    gb::set_error("%s", all.c_str());
    return GB_BAD_ARG;
}

}  // namespace

namespace {

//! The Newton stage's residual inputs (Smoothness.cpp:54-67,
//! newton_residual_inputs): the van Leer limiter's kink at every extremum
//! spoils forward-difference Jacobian-vector products, so every residual the
//! stage evaluates (its jvp, line search, norms and SIMPLEC preconditioner)
//! takes the smooth counterpart, van Albada; van Albada and upwind stay.
//! The stage's own limiter is restored when the call returns.
class SmoothLimiter {
public:
    explicit SmoothLimiter(gb_simplec* S) : S_(S), saved_(gb::simplec_limiter(S))
    {
        if (saved_ == GB_LIMITER_VAN_LEER) { gb::simplec_set_limiter(S_, GB_LIMITER_VAN_ALBADA); }
    }
    ~SmoothLimiter() { gb::simplec_set_limiter(S_, saved_); }
    SmoothLimiter(const SmoothLimiter&) = delete;
    SmoothLimiter& operator=(const SmoothLimiter&) = delete;

private:
    gb_simplec* S_;
    int saved_;
};

}  // namespace

extern "C" {

gb_status gb_newton_options_default(gb_newton_opts* o)
{
    gb::clear_error();
    if (o == nullptr) {
        gb::set_error("gust: gb_newton_options_default: null argument");
        return GB_BAD_ARG;
    }
    o->gmres_restart = 30;
    o->gmres_max_iters = 2000;
    o->fd_eps_scale = std::sqrt(std::numeric_limits<double>::epsilon());
    o->krylov_rtol = 1.0e-2;
    o->scale_pressure = 100.0;
    o->preconditioner = 1;
    o->inf_cfl = 10.0;
    return GB_OK;
}

gb_status gb_newton_check(const gb_newton_opts* o)
{
    gb::clear_error();
    if (o == nullptr) {
        gb::set_error("gust: check_newton_options: null argument");
        return GB_BAD_ARG;
    }
    return check_newton(o);
}

gb_status gb_newton_create(gb_simplec* s, const gb_newton_opts* o, gb_newton** out)
{
    gb::clear_error();
    if (s == nullptr || o == nullptr || out == nullptr) {
        gb::set_error("gust: NewtonKrylov: null argument");
        return GB_BAD_ARG;
    }
    gb_status st = check_newton(o);
    if (st != GB_OK) { return st; }
    if (gb::volume(gb::simplec_grid(s)) >= (static_cast<int64_t>(1) << 31)) {
        gb::set_error("gust: NewtonKrylov: the padded grid has 2^31 points or more (one flat launch per field)");
        return GB_BAD_ARG;
    }
    gb_newton* n = new (std::nothrow) gb_newton;
    if (n == nullptr) {
        gb::set_error("gust: NewtonKrylov: out of host memory");
        return GB_OOM;
    }
    n->S = s;
    n->ctx = gb::simplec_ctx(s);
    n->opt = *o;
    n->g = gb::simplec_grid(s);
    n->vol = gb::volume(n->g);
    const gb_physics& ph = gb::simplec_physics(s);
    const double U = ph.scale_velocity;
    const double sc[gb::kNF] = {U, U, U, o->scale_pressure, ph.scale_theta, ph.scale_tke};
    const double tc[gb::kNF] = {U, U, U, 1.0, ph.scale_theta, ph.scale_tke};
    for (int f = 0; f < gb::kNF; ++f) {
        n->s[f] = sc[f];
        n->t[f] = tc[f];
    }
    bool ok = true;
    n->V.resize(o->gmres_restart + 1);
    n->Z.resize(o->gmres_restart);
    for (auto& v : n->V) { ok = ok && gb::make_vec(n, v); }
    for (auto& v : n->Z) { ok = ok && gb::make_vec(n, v); }
    ok = ok && gb::make_vec(n, n->R0) && gb::make_vec(n, n->Jv) && gb::make_vec(n, n->dq) && gb::make_vec(n, n->qp)
         && gb::make_vec(n, n->inv_dtau) && gb::make_vec(n, n->b) && gb::make_vec(n, n->x) && gb::make_vec(n, n->w)
         && gb::make_vec(n, n->dir, 3) && gb::make_vec(n, n->dtf, 3);
    if (o->preconditioner != 0) { ok = ok && gb::make_vec(n, n->pr) && gb::make_vec(n, n->pz); }
    ok = ok && (n->partial = gb::nbuf(n, 3 * gb::kRedBlocksN * gb::kNF)) != nullptr;
    if (ok && cudaMallocHost(&n->h_partial, sizeof(double) * 3 * gb::kRedBlocksN * gb::kNF) != cudaSuccess) {
        cudaGetLastError();
        n->h_partial = nullptr;
        ok = false;
    }
    if (!ok) {
        delete n;
        gb::set_error("gust: NewtonKrylov: cannot allocate the Krylov vectors (%d of the grid's state, restart %d; "
                      "steady.newton_gmres_restart)", 2 * o->gmres_restart + 13, o->gmres_restart);
        return GB_OOM;
    }
    *out = n;
    return gb::check_cuda("NewtonKrylov");
}

gb_status gb_newton_destroy(gb_newton* n)
{
    gb::clear_error();
    // the context's stream, kept at creation: the stage may be gone already
    if (n) { cudaStreamSynchronize(n->ctx->stream); }
    delete n;
    return GB_OK;
}

gb_status gb_newton_jvp(gb_newton* n, const gb_state* q, double* const* v, double* const* Jv, double* eps)
{
    gb::clear_error();
    if (n == nullptr || q == nullptr || v == nullptr || Jv == nullptr || eps == nullptr) {
        gb::set_error("gust: jvp: null argument");
        return GB_BAD_ARG;
    }
    const SmoothLimiter smooth(n->S);
    double bnorm = 0;
    gb_status st = gb::base(n, *q, &bnorm);
    if (st != GB_OK) { return st; }
    gb::Vec vv(v, v + gb::kNF), jj(Jv, Jv + gb::kNF);
    n->jvp_calls = 0;
    return gb::jvp(n, *q, vv, n->R0, jj, eps);
}

gb_status gb_newton_direction(gb_newton* n, const gb_state* q, const double* dtau, double* const* dq,
                              gb_newton_step_info* info)
{
    gb::clear_error();
    if (n == nullptr || q == nullptr || dq == nullptr || info == nullptr) {
        gb::set_error("gust: NewtonKrylov::direction: null argument");
        return GB_BAD_ARG;
    }
    const SmoothLimiter smooth(n->S);
    gb_status st = gb::solve(n, *q, dtau, info);
    if (st != GB_OK) { return st; }
    gb::Vec d(dq, dq + gb::kNF);
    for (int f = 0; f < gb::kNF; ++f) { cudaMemsetAsync(d[f], 0, sizeof(double) * n->vol, gb::nctx(n)->stream); }
    if (info->applied) { gb::add_scaled(n, d, n->x, 1.0); }
    return gb::check_cuda("NewtonKrylov::direction");
}

gb_status gb_newton_step(gb_newton* n, const gb_state* q, const double* dtau, gb_newton_step_info* info)
{
    gb::clear_error();
    if (n == nullptr || q == nullptr || info == nullptr) {
        gb::set_error("gust: NewtonKrylov::step: null argument");
        return GB_BAD_ARG;
    }
    const SmoothLimiter smooth(n->S);
    gb_status st = gb::solve(n, *q, dtau, info);
    if (st != GB_OK) { return st; }
    if (info->applied) { gb::add_scaled(n, gb::vec_of(*q), n->x, 1.0); }
    gb::simplec_fill_ghosts(n->S, *q);
    return gb::check_cuda("NewtonKrylov::step");
}

gb_status gb_newton_residual_norm(gb_newton* n, const gb_state* q, double* norm)
{
    gb::clear_error();
    if (n == nullptr || q == nullptr || norm == nullptr) {
        gb::set_error("gust: NewtonKrylov::residual_norm: null argument");
        return GB_BAD_ARG;
    }
    const SmoothLimiter smooth(n->S);
    return gb::base(n, *q, norm);
}

gb_status gb_newton_trial(gb_newton* n, const gb_state* q0, double* const* dq, double lambda, const gb_state* out)
{
    gb::clear_error();
    if (n == nullptr || q0 == nullptr || dq == nullptr || out == nullptr) {
        gb::set_error("gust: continuation trial: null argument");
        return GB_BAD_ARG;
    }
    const gb::Vec a = gb::vec_of(*q0), o = gb::vec_of(*out);
    const gb_grid g = n->g;
    const double floor_k = gb::simplec_options(n->S).tke_floor;
    for (int f = 0; f < gb::kNF; ++f) {
        cudaMemcpyAsync(o[f], a[f], sizeof(double) * n->vol, cudaMemcpyDeviceToDevice, gb::nctx(n)->stream);
        double* d = o[f];
        const double* df = dq[f];
        const bool clip = (f == 5);
        gb::for_box(gb::nctx(n), gb::valid_box(g, gb::kFieldLoc[f]), [=] __device__(int i, int j, int k) {
            const int64_t p = gb::at(g, i, j, k);
            double v = d[p] + lambda * df[p];
            if (clip && v < floor_k) { v = floor_k; }
            d[p] = v;
        }, GB_KERNEL_VECTOR);
    }
    return gb::check_cuda("continuation trial");
}

}  // extern "C"
