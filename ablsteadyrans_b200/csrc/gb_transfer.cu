// The restriction of grid sequencing's transfers (gust::restrict_state,
// Source/Transfer.H:94-110, Transfer.cpp:150-286): a fine level's state onto
// the coarse level r = 2^l times coarser in x and y.
//
// One thread per coarse point: the cell fields are the detJ-weighted means of
// their r x r fine cells; u and v the coarse face's flux per unit width
// (the r fine face fluxes a q summed, over r) over the coarse face area; the
// vertical flux Omega the r x r fine z-face fluxes a_z Omega over r^2 and
// the coarse a_z, and w from it on the coarse mesh with the coarse u and v
// read with zero-gradient rows below the ground and above the top. The
// kernels are HBM-bound: each fine point is read once, each coarse point
// written once.
#include "gb_stencil.cuh"

#include <cmath>

namespace gb {

namespace {

using namespace st;

enum TransferSlot : int { kSlotRestrictU = 40, kSlotRestrictV, kSlotRestrictOmega };

//! The coarse copy of a face field with its rows below the ground and above
//! the top set to the nearest valid row (zero_gradient_rows, Transfer.cpp:177-197).
void zero_gradient_copy(gb_ctx* ctx, const gb_grid& g, int t, const double* src, double* dst)
{
    cudaMemcpyAsync(dst, src, sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    const int nz = g.nz;
    const Box rows{{0, 0, 0}, {ext_x(g, t) - 1, ext_y(g, t) - 1, 1}};
    for_box(ctx, rows, [=] __device__(int i, int j, int s) {
        if (s == 0) {
            dst[at(g, i, j, -1)] = dst[at(g, i, j, 0)];
        } else {
            dst[at(g, i, j, nz)] = dst[at(g, i, j, nz - 1)];
        }
    }, GB_KERNEL_MG_TRANSFER);
}

}  // namespace

gb_status restrict_state(gb_ctx* ctx, const gb_grid& gf, const gb_state& qf, const gb_mesh_fields& mf, const gb_grid& gc,
                         const gb_state& qc, const gb_mesh_fields& mc, double* omega_c)
{
    const int r = gf.nx / gc.nx;
    const gb_grid F = gf, C = gc;
    // cell centres: sum J q / sum J over the r x r fine cells
    {
        const double* Jf = mf.detJ;
        const double* src[3] = {qf.theta, qf.tke, qf.p};
        double* dst[3] = {qc.theta, qc.tke, qc.p};
        for (int n = 0; n < 3; ++n) {
            const double* q = src[n];
            double* o = dst[n];
            for_box(ctx, valid_box(gc, CC), [=] __device__(int I, int J, int k) {
                double sjq = 0, sj = 0;
                for (int b = 0; b < r; ++b) {
                    for (int a = 0; a < r; ++a) {
                        const double w = Jf[at(F, r * I + a, r * J + b, k)];
                        sjq += w * q[at(F, r * I + a, r * J + b, k)];
                        sj += w;
                    }
                }
                o[at(C, I, J, k)] = sjq / sj;
            }, GB_KERNEL_MG_TRANSFER);
        }
    }
    // u, v: (1/r) sum a q over the r fine faces, over the coarse area
    const double rinv = 1.0 / static_cast<double>(r);
    {
        const double* af = mf.ax;
        const double* ac = mc.ax;
        const double* q = qf.u;
        double* o = qc.u;
        for_box(ctx, valid_box(gc, XF), [=] __device__(int I, int J, int k) {
            double s = 0;
            for (int b = 0; b < r; ++b) { s += af[at(F, r * I, r * J + b, k)] * q[at(F, r * I, r * J + b, k)]; }
            const double c = s * rinv;
            o[at(C, I, J, k)] = c / ac[at(C, I, J, k)];
        }, GB_KERNEL_MG_TRANSFER);
    }
    {
        const double* af = mf.ay;
        const double* ac = mc.ay;
        const double* q = qf.v;
        double* o = qc.v;
        for_box(ctx, valid_box(gc, YF), [=] __device__(int I, int J, int k) {
            double s = 0;
            for (int b = 0; b < r; ++b) { s += af[at(F, r * I + b, r * J, k)] * q[at(F, r * I + b, r * J, k)]; }
            const double c = s * rinv;
            o[at(C, I, J, k)] = c / ac[at(C, I, J, k)];
        }, GB_KERNEL_MG_TRANSFER);
    }
    // Omega: (1/r^2) sum a_z Omega over the r x r fine z-faces (the fine
    // Omega = w - z_x u_f - z_y v_f on the fly), over the coarse a_z
    double* om = omega_c;
    if (om == nullptr) {
        om = static_cast<double*>(scratch(ctx, kSlotRestrictOmega, sizeof(double) * volume(gc)));
        if (om == nullptr) { return GB_OOM; }
    }
    {
        const double r2inv = 1.0 / static_cast<double>(r * r);
        const double* azf = mf.az;
        const double* azc = mc.az;
        const double *u = qf.u, *v = qf.v, *w = qf.w, *z = qf.z_nd;
        double* o = om;
        for_box(ctx, valid_box(gc, ZF), [=] __device__(int I, int J, int k) {
            double s = 0;
            for (int b = 0; b < r; ++b) {
                for (int a = 0; a < r; ++a) {
                    const int i = r * I + a, j = r * J + b;
                    const double omf = w[at(F, i, j, k)]
                                     - deriv<NODE, ZF, 0>(z, F, i, j, k) * (1.0 / F.dx) * interp<XF, ZF>(u, F, i, j, k)
                                     - deriv<NODE, ZF, 1>(z, F, i, j, k) * (1.0 / F.dy) * interp<YF, ZF>(v, F, i, j, k);
                    s += azf[at(F, i, j, k)] * omf;
                }
            }
            const double c = s * r2inv;
            o[at(C, I, J, k)] = c / azc[at(C, I, J, k)];
        }, GB_KERNEL_MG_TRANSFER);
    }
    // w from Omega on the coarse mesh
    double* u1 = static_cast<double*>(scratch(ctx, kSlotRestrictU, sizeof(double) * volume(gc)));
    double* v1 = static_cast<double*>(scratch(ctx, kSlotRestrictV, sizeof(double) * volume(gc)));
    if (u1 == nullptr || v1 == nullptr) { return GB_OOM; }
    zero_gradient_copy(ctx, gc, XF, qc.u, u1);
    zero_gradient_copy(ctx, gc, YF, qc.v, v1);
    {
        const double* zc = qc.z_nd;
        const double* omc = om;
        double* wc = qc.w;
        for_box(ctx, valid_box(gc, ZF), [=] __device__(int i, int j, int k) {
            wc[at(C, i, j, k)] = omc[at(C, i, j, k)]
                               + deriv<NODE, ZF, 0>(zc, C, i, j, k) * (1.0 / C.dx) * interp<XF, ZF>(u1, C, i, j, k)
                               + deriv<NODE, ZF, 1>(zc, C, i, j, k) * (1.0 / C.dy) * interp<YF, ZF>(v1, C, i, j, k);
        }, GB_KERNEL_MASSFLUX);
    }
    return check_cuda("restrict_state");
}

}  // namespace gb

extern "C" gb_status gb_restrict_state(gb_ctx* ctx, const gb_grid* gf, const gb_state* qf, const gb_mesh_fields* mf,
                                       const gb_grid* gc, const gb_state* qc, const gb_mesh_fields* mc, double* omega_c)
{
    gb::clear_error();
    if (ctx == nullptr || gf == nullptr || qf == nullptr || mf == nullptr || gc == nullptr || qc == nullptr
        || mc == nullptr) {
        gb::set_error("gust: restrict_state: null argument");
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_grid("restrict_state", gf);
    if (st != GB_OK) { return st; }
    if ((st = gb::check_grid("restrict_state", gc)) != GB_OK) { return st; }
    const int rx = gc->nx > 0 ? gf->nx / gc->nx : 0, ry = gc->ny > 0 ? gf->ny / gc->ny : 0;
    if (rx < 2 || rx != ry || rx * gc->nx != gf->nx || ry * gc->ny != gf->ny || (rx & (rx - 1)) != 0 || gc->nz != gf->nz
        || gc->periodic_x != gf->periodic_x || gc->periodic_y != gf->periodic_y) {
        gb::set_error("gust: restrict_state: the levels must satisfy 0 <= fine < coarse: the coarse grid coarser by a "
                      "power of two in x and y, the same layers and periodicity");
        return GB_BAD_ARG;
    }
    const double* need[] = {qf->u, qf->v, qf->w, qf->p, qf->theta, qf->tke, qf->z_nd, qc->u, qc->v, qc->w, qc->p,
                            qc->theta, qc->tke, qc->z_nd, mf->detJ, mf->ax, mf->ay, mf->az, mc->ax, mc->ay, mc->az};
    for (const double* p : need) {
        if (p == nullptr) {
            gb::set_error("gust: restrict_state: both states need every field and their node heights, the fine mesh "
                          "detJ and face areas, the coarse face areas");
            return GB_BAD_ARG;
        }
    }
    return gb::restrict_state(ctx, *gf, *qf, *mf, *gc, *qc, *mc, omega_c);
}
