/*
 * gust_b200.h -- C ABI of the B200-native SIMPLEC hot path of GUST
 * (hgopalan/ablsteadyrans): z-line relaxation, the terrain-following
 * pressure-correction Poisson solve and the control-volume residual stencils.
 *
 * Conventions
 *  - Plain C, POD arguments only. Field pointers are DEVICE pointers to arrays
 *    laid out by gb_grid (below); scalars and result structs live on the host.
 *  - Every call returns a gb_status and never aborts the process. On an error
 *    gb_last_error() returns a message naming the argument or the inputs key,
 *    in the reference's "gust: <op>: <what>" form.
 *  - Work is ordered on the stream of the gb_ctx passed in. A call that
 *    returns a host scalar (a norm, a change) synchronises that stream.
 *  - Location codes follow the reference's bit mask (Stencil_K.H): bit d set
 *    means nodal in direction d.
 *
 * Data layout (one layout per grid, for every location type):
 *   every array of a grid is (nz+1+2ng) k-planes of (ny+1+2ng) rows of
 *   pitch_x elements, i fastest, then j, then k ("k-plane-major SoA"). Point
 *   (i, j, k) of any location type (cell, face, node) sits at element
 *       (i + ng) + (j + ng) * sy + (k + ng) * sz,
 *   so cell, face and node arrays share one index space and one stencil
 *   arithmetic, as AMReX's Array4 does for one box. Multi-component arrays
 *   (the implicit coefficients) store component c at c * gb_grid_volume(g).
 */
#ifndef GUST_B200_H_
#define GUST_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gb_status {
    GB_OK = 0,
    GB_BAD_ARG = 1,        /* an argument or an inputs value out of range */
    GB_NONFINITE = 2,      /* a NaN or inf in an input or a result */
    GB_NOT_CONVERGED = 3,  /* an iterative solve hit its iteration limit */
    GB_TIMEOUT = 4,        /* a bounded device-side wait gave up */
    GB_OOM = 5,            /* device memory could not be allocated */
    GB_CUDA = 6            /* a CUDA runtime error */
} gb_status;

/* Location of a field's points (the reference's Loc, CVFluxes.H:20). */
enum { GB_LOC_CELL = 0, GB_LOC_XFACE = 1, GB_LOC_YFACE = 2, GB_LOC_ZFACE = 4, GB_LOC_NODE = 7 };

/* Components of the implicit coefficients (ImplicitOperator.H:57). */
enum { GB_COEF_P = 0, GB_COEF_XM, GB_COEF_XP, GB_COEF_YM, GB_COEF_YP, GB_COEF_ZM, GB_COEF_ZP, GB_N_COEFS };

typedef struct gb_grid {
    int32_t nx, ny, nz;        /* cells */
    int32_t ng;                /* ghost layers every array holds (>= 2) */
    int32_t periodic_x;        /* 1: periodic in x (amrex::Geometry::isPeriodic(0)) */
    int32_t periodic_y;
    int64_t sy, sz;            /* element strides of j and k; the i stride is 1 */
    double dx, dy, dzeta;      /* computational cell sizes, geom.CellSize() */
} gb_grid;

/* Fill g for nx x ny x nz cells with ng ghost layers and the default pitch. */
gb_status gb_grid_init(gb_grid* g, int32_t nx, int32_t ny, int32_t nz, int32_t ng, double dx, double dy,
                       double dzeta, int32_t periodic_x, int32_t periodic_y);
/* Elements of one array of the grid (one component). */
int64_t gb_grid_volume(const gb_grid* g);

/* ---- context ------------------------------------------------------------ */
typedef struct gb_ctx gb_ctx;

/* A context on the current CUDA device, ordering its work on `stream` (a
 * cudaStream_t; NULL = the legacy default stream). It owns the scratch the
 * calls below need (grown on demand, freed by gb_ctx_destroy). One context per
 * host thread. */
gb_status gb_ctx_create(void* stream, gb_ctx** out);
gb_status gb_ctx_destroy(gb_ctx* ctx);
/* Kernel launches this context has issued (all calls), for launch accounting. */
int64_t gb_ctx_launches(const gb_ctx* ctx);
/* Kernel families timed by the context's profiler. */
enum {
    GB_KERNEL_LINE_SWEEP = 0,   /* z-line Thomas sweep (one launch per sweep) */
    GB_KERNEL_POISSON_APPLY,    /* terrain Poisson operator apply / residual */
    GB_KERNEL_MG_SMOOTH,        /* multigrid z-line smoother */
    GB_KERNEL_MG_TRANSFER,      /* restriction / prolongation */
    GB_KERNEL_RESIDUAL,         /* control-volume residual stencils */
    GB_KERNEL_MASSFLUX,         /* mass-flux / divergence kernels */
    GB_KERNEL_COEFS,            /* implicit coefficients and row folds */
    GB_KERNEL_VECTOR,           /* vector ops and reductions */
    GB_KERNEL_BC,               /* ghost fills */
    GB_N_KERNEL_FAMILIES
};
/* Profiling: with enable = 1 every launch of a timed family is bracketed by
 * CUDA events on the context's stream (enable clears earlier spans).
 * gb_ctx_profile_read sums the recorded spans of one family. */
gb_status gb_ctx_profile(gb_ctx* ctx, int32_t enable);
gb_status gb_ctx_profile_read(gb_ctx* ctx, int32_t family, double* total_ms, int64_t* spans);
/* Which families profiling times: bit f set = family f (default: all). Timing
 * only the family of interest keeps the events' own cost out of a timed step. */
gb_status gb_ctx_profile_mask(gb_ctx* ctx, uint32_t mask);
/* A measurement probe, not part of the drop-in path: `iters` dependent FP64
 * fused multiply-adds in each of 8 independent chains per thread, on 4
 * blocks of 256 threads per SM, launched on the context's stream (the caller
 * times it with events there). It executes 2 * 8 * iters * threads FP64
 * operations and writes one value per thread to sink (4 * SMs * 256
 * doubles), so that none of the arithmetic is removed. *threads receives the
 * thread count. */
gb_status gb_probe_fp64(gb_ctx* ctx, int32_t iters, double* sink, int64_t* threads);
/* Tuning knobs of a context (the in-project autotuner sets them per shape). */
enum {
    GB_TUNE_LINE_VARIANT = 0,   /* z-line sweep kernel: 0 auto (= 5), 1 pipelined (cp.async ring), 2 shared,
                                   3 global scratch, 4 pipelined with the column factors kept between sweeps,
                                   5 segmented: the column's levels split among the warps of a block, the
                                   factors kept between sweeps (columns of more than 128 levels: 4), 6 the
                                   segmented sweep with each later sweep split into the fold of the lagged
                                   lateral terms (one thread per point) and the column solves */
    GB_TUNE_LINE_BLOCK,         /* threads per block of the pipelined sweep (32, 64 or 128; 0 = default) */
    GB_TUNE_MG_COARSE_KERNEL,   /* the coarsest level's relaxations: 0 auto (one single-block launch when the
                                   level has at most 64 columns), 1 the per-relaxation launches */
    GB_TUNE_LINE_DEPTH,         /* levels the factored z-line sweep keeps in flight: 0 default (4 FP64, 8 FP32),
                                   2 twice that */
    GB_TUNE_LINE_BACK,          /* where the batched factored sweep keeps c' and e' for the back substitution:
                                   0 auto (= 1), 1 shared memory, 2 the global arrays (c' stored, e' in the
                                   output array), 3 e' in shared memory and c' read again from its stored
                                   array (L2): less shared memory per warp, more warps per SM */
    GB_TUNE_MG_FUSED_RELAX,     /* one launch per colour of the zebra line relaxation: 0 auto (= 1), 1 never
                                   (the residual and the solve as two launches), 2 the residual in shared memory
                                   and one thread per column's solve, on every level, 3 that on the levels of at
                                   most 1024 columns, 4 segmented (the column's levels split among the warps of
                                   a block, the residual in registers; columns of more than 128 levels: 1) */
    GB_TUNE_GRAPHS,             /* CUDA graphs for launch sequences without a host synchronisation (the
                                   multigrid V-cycle): 0 default (on), 1 off (every kernel launched alone) */
    GB_TUNE_MG_SOLVE,           /* the column solves of the two-launch zebra relaxation: 0 default (the
                                   column's levels split among the warps of a block), 1 one thread per column */
    GB_TUNE_LINE_FIRST,         /* the first sweep of a segmented solve (the column factorisation): 0 default
                                   (= 1), 1 segmented, 2 the sequential factored kernel (the same factors) */
    GB_TUNE_LINE_SEGMENT,       /* levels per warp of the segmented z-line sweep (0 default = 5; 4 or 8: more
                                   or fewer warps per column at a lower or higher register cap) and of the
                                   segmented zebra relaxation (default 4, 8 for columns of more than 64
                                   levels): 0 default, 4 or 8 */
    GB_TUNE_RESIDUAL,           /* the SIMPLEC residual's convection, diffusion and pressure gradient and
                                   the implicit coefficients: 0 default (one launch per equation, each
                                   face evaluated once per block, 2 levels per block), 1 one thread per
                                   point (the residual's fluxes and divergences as separate launches),
                                   N >= 2 the per-equation launch with N levels per block */
    GB_TUNE_MG_TAIL,            /* the V-cycle's coarse levels as one thread-block-cluster launch: 0 default
                                   and 1 off (per-level launches), N >= 2 the levels of at most N columns
                                   (measured no faster: the cluster's 16 SMs do the levels' work) */
    GB_TUNE_MG_STENCIL,         /* the terrain operator of the Poisson apply and the zebra colour residual:
                                   0 default and 1 one thread per cell, 2 TMA-staged tiles of the iterate
                                   on every level (measured slower: the other ten words a cell stay
                                   direct loads and each level costs two block barriers) */
    GB_TUNE_PDL,                /* programmatic dependent launch of the multigrid's kernels and the stage's
                                   one-thread-per-point kernels (each one's launch overlaps its predecessor's
                                   tail): 0 default on, 1 off */
    GB_N_TUNE
};
gb_status gb_ctx_tune(gb_ctx* ctx, int32_t key, int32_t value);
/* The last error message of the calling thread ("" after success). */
const char* gb_last_error(void);

/* ---- z-line relaxation -------------------------------------------------- */

/* The z-line Jacobi solve, replacing gust::zline_jacobi (Source/Predictor.H:267-268,
 * Source/Predictor.cpp:87-127; column kernel gust::solve_column,
 * Source/LineSolve_K.H:22-45): `sweeps` sweeps of the system with the
 * off-diagonal coefficients of A (GB_N_COEFS components at loc) and the
 * diagonal ap, right-hand side rhs, into delta (set to 0 first, x/y neighbours
 * lagged, periodic images through the grid, zero outside the domain). Every
 * (i, j) column is solved exactly for (-a_zm, ap, -a_zp) by the Thomas
 * recurrences. *change receives max |change over the last sweep|. The two
 * copies of a periodic seam face are made identical afterwards (OverrideSync:
 * the low copy wins). */
gb_status gb_zline_jacobi(gb_ctx* ctx, const gb_grid* g, int32_t loc, const double* A, const double* ap,
                          const double* rhs, int32_t sweeps, double* delta, double* change);
/* The same in FP32 (the inner solver of the mixed-precision defect correction). */
gb_status gb_zline_jacobi_f32(gb_ctx* ctx, const gb_grid* g, int32_t loc, const float* A, const float* ap,
                              const float* rhs, int32_t sweeps, float* delta, float* change);
/* One system of a batched z-line solve: its own grid and location, and the
 * arrays gb_zline_jacobi takes (device arrays of that grid). */
typedef struct gb_line_system {
    gb_grid grid;
    int32_t loc;
    const double* A;
    const double* ap;
    const double* rhs;
    double* delta;
} gb_line_system;
typedef struct gb_line_system_f32 {
    gb_grid grid;
    int32_t loc;
    const float* A;
    const float* ap;
    const float* rhs;
    float* delta;
} gb_line_system_f32;
/* gust::zline_jacobi (Source/Predictor.cpp:87-127, the column solves of
 * Source/LineSolve_K.H:22-45) over n systems of different grids at once, as
 * a batch of terrain tiles and wind directions of uneven sizes brings them:
 * every system's delta is set to 0 and gets `sweeps` sweeps, each value bit
 * for bit the one gb_zline_jacobi gives that system alone on this context.
 * The columns of all systems form one work-list of 32-column blocks, walked
 * by persistent launches: one per sweep for each distinct number of
 * segments (z-levels / the segment length, GB_TUNE_LINE_SEGMENT) the
 * systems' columns have, and one more per further 120 systems of one such
 * group. change (host, n entries, or NULL) receives each
 * system's max |change over the last sweep|; with change non-NULL the call
 * waits for the context's stream. Columns taller than the segmented
 * sweep's limit are refused (GB_BAD_ARG; use gb_zline_jacobi). */
gb_status gb_zline_jacobi_batch(gb_ctx* ctx, int32_t n, const gb_line_system* systems, int32_t sweeps,
                                double* change);
/* The same in FP32. */
gb_status gb_zline_jacobi_batch_f32(gb_ctx* ctx, int32_t n, const gb_line_system_f32* systems, int32_t sweeps,
                                    double* change);
/* The line LU-SGS solve, replacing gust::zline_lusgs with steady.line_ghosts =
 * lagged (Source/LineSweeps.H:159-161, Source/LineSweeps.cpp:183-210, 415-428):
 * `sweeps` symmetric passes of in-place column solves of the system of
 * gb_zline_jacobi, each column with its x/y neighbours as they stand at that
 * moment of the pass (forward (+i, +j), backward (-i, -j); with alternate = 1
 * (steady.line_alternate) the odd sweeps take (+i, -j) then (-i, +j)); before
 * every pass the periodic ghosts take the images of the pass's starting values
 * (FillBoundary). delta is set to 0 first; *change receives max |change| over
 * the last backward pass; the seam copies are synced at the end (the low copy
 * wins). The GPU walks the wavefront planes (the reference's diagonal order,
 * which equals its sequential order value for value). FP64. */
gb_status gb_zline_lusgs(gb_ctx* ctx, const gb_grid* g, int32_t loc, const double* A, const double* ap,
                         const double* rhs, int32_t sweeps, int32_t alternate, double* delta, double* change);
/* The FP64 z-line Jacobi solve of gb_zline_jacobi for a caller that must not
 * allocate device memory. This entry point has no counterpart in the
 * reference; it exists for hosts that cannot let a library allocate: one that
 * has handed its device memory to its own arena up front (as an AMReX
 * application does), or that cannot take the device-wide synchronisation a
 * cudaMalloc/cudaFree pair brings in the middle of its step. It takes no
 * context and allocates nothing: its scratch (the ping-pong iterate and the
 * change word) is one fixed array in this library's device memory, reserved
 * by the CUDA runtime when the library's device code is loaded on a device.
 * - Limit: gb_grid_volume(g) <= 2^21 padded points (16 MiB of scratch) and
 *   at most 376 z-levels; larger grids are refused with GB_BAD_ARG and a
 *   message (use gb_zline_jacobi).
 * - Set-up: the first call on each device (that device current) looks up the
 *   array's address and sets the kernels' shared-memory limit; later calls on
 *   that device reuse it. Make that first call before any stream capture.
 *   A cudaDeviceReset of that device after its first call is not supported:
 *   the kept address would belong to the destroyed context.
 * - Sharing: every call on a device uses the same array. Calls issued one
 *   after another on one stream are safe; calls that may overlap (other
 *   streams, other threads) race on it. The iterate needs no initial value
 *   (each sweep writes every point the next one reads); the change word must
 *   start at zero, and each call zeroes it on its stream before the sweeps.
 * - stream: the caller's cudaStream_t (NULL: the default stream). With change
 *   non-NULL the call waits for the stream to read max |change|; with change
 *   NULL it returns as soon as the work is queued.
 * Results agree with those of gb_zline_jacobi to rounding (the same column
 * solves; the context path keeps the column factors between sweeps). */
gb_status gb_zline_jacobi_noalloc(const gb_grid* g, int32_t loc, const double* A, const double* ap,
                                  const double* rhs, int32_t sweeps, double* delta, double* change, void* stream);

/* ---- mesh --------------------------------------------------------------- */

/* The metric terms of the terrain-following mesh from the node heights z
 * (nodal, one ghost layer filled), replacing make_J / make_areas / make_zcc
 * (extern_erf/ERF_TerrainMetrics.cpp:680-808, called from Source/Mesh.cpp:
 * make_metrics): detJ and z_cc at cells, ax, ay at x-, y-faces, az = 1, on the
 * valid points and one ghost layer (0 below the ground). */
gb_status gb_mesh_metrics(gb_ctx* ctx, const gb_grid* g, const double* z_nd, double* detJ, double* ax, double* ay,
                          double* az, double* z_cc);

/* ---- Poisson layer ------------------------------------------------------ */

/* Boundary types of the Poisson problem per domain face, indexed xlo, ylo,
 * zlo, xhi, yhi, zhi (gust::PoissonBC, Source/Poisson.H:24-35). */
enum { GB_POISSON_PERIODIC = 0, GB_POISSON_NEUMANN = 1, GB_POISSON_DIRICHLET = 2 };

typedef struct gb_poisson_opts {
    double reltol;       /* solver.poisson_reltol (SIMPLEC: simplec.pressure_reltol) */
    double abstol;       /* solver.poisson_abstol */
    int32_t max_iter;    /* solver.poisson_max_iter */
    int32_t restart;     /* solver.poisson_restart */
    int32_t precision;   /* 0: FP64 multigrid, 1: FP32 multigrid inside the FP64 Krylov solve */
    int32_t nu1, nu2;    /* pre- and post-smoothing z-line zebra relaxations per level */
    int32_t nu_coarse;   /* relaxations on the coarsest level */
    int32_t max_levels;  /* multigrid levels (x-y 2:1 coarsening) */
    int32_t min_coarse;  /* smallest coarse extent in x and y */
} gb_poisson_opts;

typedef struct gb_poisson_result {
    int32_t iterations;
    int32_t singular;          /* no Dirichlet face: the J-weighted mean was removed */
    double initial_residual;   /* 2-norm of the (mean-free) right-hand side */
    double final_residual;     /* true residual 2-norm, recomputed */
    double removed_mean;       /* gust::PoissonResult::removed_mean */
} gb_poisson_result;

typedef struct gb_poisson gb_poisson;

/* The reference's defaults (Source/Poisson.H:41-75: reltol 1e-10, max_iter 200,
 * restart 50) with this project's multigrid settings. */
gb_status gb_poisson_options_default(gb_poisson_opts* opt);

/* gust::PoissonSolver (Source/Poisson.H:135-161) for the mesh (z_nd, detJ:
 * device arrays kept by reference, as the reference's solver keeps the mesh)
 * and the boundary types bc[6]. Builds the multigrid hierarchy. */
gb_status gb_poisson_create(gb_ctx* ctx, const gb_grid* g, const int32_t* bc, const double* z_nd, const double* detJ,
                            const gb_poisson_opts* opt, gb_poisson** out);
gb_status gb_poisson_destroy(gb_poisson* p);

/* The face coefficients (gust::FaceCoeffs without z_cross): the operator takes
 * the premultiplied areas a * beta (Source/Poisson.cpp:442-447; beta null = 1). */
gb_status gb_poisson_set_coeffs(gb_poisson* p, const double* ax, const double* ay, const double* az, const double* bx,
                                const double* by, const double* bz);

/* FaceCoeffs::z_cross (Source/Poisson.H:83-102, Source/Poisson.cpp:461-479):
 * the split z-face coefficient. The z-face gradient becomes
 * beta_z dphi/dz - z_cross (h_x dphi/dx + h_y dphi/dy): the operator adds
 * (1/J) d_zeta (a_z (beta_z - z_cross) cross) (PoissonSolver::Op::add_cross,
 * Source/Poisson.cpp:229-253) and the fluxes subtract (beta_z - z_cross) cross
 * (add_cross_flux, :255-273), on every z-face but the ground and a Neumann
 * top. The multigrid preconditioner keeps the unsplit operator. az: the raw
 * z areas; bz: the beta_z given to set_coeffs (null = 1); z_cross null
 * removes the split. A Dirichlet ground is refused, as the reference does. */
gb_status gb_poisson_set_z_cross(gb_poisson* p, const double* az, const double* bz, const double* z_cross);

/* A phi (PoissonSolver::apply / TerrainPoisson::apply with the zero-flux faces,
 * extern_erf/ERF_TerrainPoisson.cpp:74-101). Ghosts of phi are not read from
 * memory: they are resolved by index for the boundary types. */
gb_status gb_poisson_apply(gb_poisson* p, const double* phi, double* Aphi);

/* One multigrid V-cycle for A e = r from e = 0 (the preconditioner). */
gb_status gb_poisson_vcycle(gb_poisson* p, const double* r, double* e);

/* PoissonSolver::solve (Source/Poisson.cpp:540-623): removes the J-weighted
 * mean of rhs when singular (rhs is modified), solves A phi = rhs by flexible
 * GMRES(restart) preconditioned by one V-cycle to max(reltol ||rhs||, abstol),
 * removes phi's mean when singular, reports the true residual.
 * GB_NOT_CONVERGED names solver.poisson_max_iter. */
gb_status gb_poisson_solve(gb_poisson* p, double* rhs, double* phi, gb_poisson_result* res);

/* gust::tucker_wall_distance (Source/WallDistance.H:14-33; Source/WallDistance.cpp:
 * 78-94): Tucker's differential wall distance on the terrain mesh of node
 * heights z_nd. One Poisson solve of laplacian(phi) = -1 with phi = 0 on the
 * ground (tucker_bc, Source/WallDistance.cpp:65-76: periodic lateral
 * directions stay periodic, the other lateral faces and the top carry no
 * flux; opt: solver.poisson_*, null for the defaults), then in every valid
 * cell d = -|grad phi| + sqrt(|grad phi|^2 + 2 phi) with ERF's cell-centred
 * physical gradient (the first cell's vertical derivative from the
 * quadratic through phi = 0 on the ground), and the ghosts of dist from the
 * valid cells (extend_by_zero_gradient, Source/Sequencing.cpp:43-60: the
 * periodic image, else the nearest valid cell). dist: a device volume of
 * the grid. res: the Poisson solve's result. Needs nz >= 3. */
gb_status gb_tucker_wall_distance(gb_ctx* ctx, const gb_grid* g, const double* z_nd, const gb_poisson_opts* opt,
                                  double* dist, gb_poisson_result* res);

/* The coefficient-weighted face fluxes F = -beta grad phi with the terrain
 * cross terms and the zero-flux faces (TerrainPoisson::getFluxes,
 * extern_erf/ERF_TerrainPoisson.cpp:212-264, times beta; beta null = 1). */
gb_status gb_poisson_fluxes(gb_poisson* p, const double* phi, const double* bx, const double* by, const double* bz,
                            double* fx, double* fy, double* fz);

/* face_divergence (Source/Poisson.H:206-209, Source/Poisson.cpp:733-764):
 * (1/J) [d_xi (a_x F_x) + d_eta (a_y F_y) + d_zeta (a_z F_z)]. */
gb_status gb_face_divergence(gb_ctx* ctx, const gb_grid* g, const double* ax, const double* ay, const double* az,
                             const double* detJ, const double* fx, const double* fy, const double* fz, double* div);

/* ---- SIMPLEC stage ------------------------------------------------------ */

/* Domain face types (gust::FaceType, Source/BoundaryConditions.H:91):
 * periodic, inflow (profile), outflow, slip_wall, no_slip_wall and, on the
 * ground only, surface_layer (the wall model of Source/SurfaceLayer.H). */
enum {
    GB_FACE_PERIODIC = 0,
    GB_FACE_INFLOW = 1,
    GB_FACE_OUTFLOW = 2,
    GB_FACE_SLIP_WALL = 3,
    GB_FACE_NO_SLIP_WALL = 4,
    GB_FACE_SURFACE_LAYER = 5
};
/* bc.surface_stability, bc.surface_wall_k, bc.surface_denominator_floor. */
enum { GB_SURFACE_NEUTRAL = 0, GB_SURFACE_HEAT_FLUX = 1 };
enum { GB_WALL_K_DIRICHLET = 0, GB_WALL_K_SOURCE = 1 };
enum { GB_DENOMINATOR_LOG_LAW = 0, GB_DENOMINATOR_ONE = 1 };
/* convection.limiter (Source/Limiter_K.H:21). */
enum { GB_LIMITER_VAN_LEER = 0, GB_LIMITER_VAN_ALBADA = 1, GB_LIMITER_UPWIND = 2 };

#define GB_MAX_PROFILE 32

/* The boundary conditions (gust::BoundaryInputs, Source/BoundaryConditions.H:
 * 99-143) with the log-law inflow (gust::InflowProfileOptions, Source/InflowProfile.H). */
typedef struct gb_bc {
    int32_t face[6];                 /* bc.xlo, bc.ylo, bc.zlo, bc.xhi, bc.yhi, bc.zhi */
    double wall_velocity[6][3];      /* bc.<face>_wall_velocity of a no_slip_wall */
    double zhi_theta_grad;           /* bc.zhi_theta_grad (K/m) */
    double inflow_ustar;             /* bc.inflow_ustar (m/s) */
    double inflow_z0;                /* bc.inflow_z0 (m) */
    double inflow_direction;         /* bc.inflow_direction: degrees the wind blows towards, CCW from +x */
    double kappa, Cmu0;              /* the closure's constants of the inflow k */
    double inflow_inv_lmax;          /* 1 / turb.max_geom_lscale, 0 = unbounded length */
    int32_t theta_ref_n;             /* theta_ref(z): the hydrostatic reference and the inflow's theta */
    double theta_ref_z[GB_MAX_PROFILE];
    double theta_ref_theta[GB_MAX_PROFILE];
    /* bc.surface_* of a surface_layer ground (gust::SurfaceLayerOptions,
     * Source/SurfaceLayer.H:120-170, Businger-Dyer functions); kappa and Cmu0
     * above are the wall law's too. */
    double surface_z0;               /* bc.surface_z0 (m, > 0), every column's without a map (gb_mesh_fields.z0) */
    double surface_zref;             /* bc.surface_zref (m, vertical; <= 0: each column's first cell centre) */
    int32_t surface_stability;       /* GB_SURFACE_NEUTRAL or GB_SURFACE_HEAT_FLUX */
    double surface_heat_flux;        /* bc.surface_heat_flux (K m/s, upward > 0; heat_flux only) */
    int32_t surface_wall_k;          /* GB_WALL_K_DIRICHLET or GB_WALL_K_SOURCE */
    int32_t surface_denominator_floor;  /* GB_DENOMINATOR_LOG_LAW or GB_DENOMINATOR_ONE */
    /* Damping (BoundaryConditions.H:57-64, off by default): the Rayleigh layer
     * R += c(z) (q - q_ref) above z_damp, c = coef sin^2(pi/2 (z - z_damp) /
     * (z_top - z_damp)); the sponge R += c(s) (q - q_ref) within sponge_width
     * of an inflow or outflow face, c = strength (1 - s/width)^2; q_ref the
     * inflow profile (w: 0), c on the implicit diagonal. */
    double rayleigh_zdamp;           /* bc.rayleigh_zdamp (m; 0: off) */
    double rayleigh_dampcoef;        /* bc.rayleigh_dampcoef (1/s) */
    int32_t rayleigh_fields;         /* bc.rayleigh_fields: bit 0 u, 1 v, 2 w, 3 theta, 4 k */
    int32_t rayleigh_above_ground;   /* bc.rayleigh_height: 0 absolute, 1 above_ground */
    double sponge_width;             /* bc.sponge_width (m; 0: off) */
    double sponge_strength;          /* bc.sponge_strength (1/s) */
    /* bc.surface_stable_functions: 0 businger_dyer, 1 qnse (the stable side
     * phi = (1 + a zeta)/(1 + b zeta), psi = -((a - b)/b) ln(1 + b zeta) with
     * bc.surface_qnse_am, _bm, _ah, _bh; StabilityFunctions.H) */
    int32_t surface_qnse;
    double surface_qnse_am, surface_qnse_bm, surface_qnse_ah, surface_qnse_bh;
} gb_bc;

/* The residual's physics inputs (gust::ResidualInputs, Source/Residual.H:61-128;
 * gust::ForcingOptions, Source/Forcing.H; the closure's turb.* options). */
typedef struct gb_physics {
    double gravity, theta0;                       /* forcing.gravity, forcing.theta0 */
    int32_t coriolis, coriolis_3d, geostrophic;   /* forcing.coriolis, forcing.coriolis_3d, forcing.geostrophic */
    double latitude, rotation_period, ug, vg;     /* forcing.latitude, rotation_period, ug, vg */
    double pressure_gradient[3];                  /* forcing.pressure_gradient (m/s^2) */
    int32_t limiter;                              /* convection.limiter */
    double smooth_eps_velocity, smooth_eps_theta; /* convection.smooth_eps_* (van Albada) */
    int32_t log_mean;                             /* diffusivity face mean: 0 arithmetic, 1 logarithmic */
    double scale_velocity, scale_theta, scale_tke;/* residual scales U, theta_s, k_s (JvpScales) */
    double scale_height;                          /* H (gust::residual_scale_height) */
    /* The k-L closure (gust::Closure, turb.*: Source/Closure.H:87-110).
     * closure = 0: the diffusivities are given (gb_diffusivities); 1: nu,
     * gamma_theta, gamma_tke and the k sources from the closure at the state,
     * with the wall distance the height above the ground. */
    int32_t closure;
    double turb_Cmu0, turb_Cb, turb_Rt_crit, turb_Rt_min; /* turb.Cmu0, Cb, Rt_crit, Rt_min */
    double turb_max_geom_lscale;                  /* turb.max_geom_lscale (m) */
    double turb_tke_floor;                        /* turb.tke_floor (0: machine epsilon) */
    double turb_sigma_k;                          /* turb.sigma_k */
    double turb_nu_molecular, turb_alpha_molecular; /* turb.nu_molecular, turb.alpha_molecular (m^2/s) */
    double turb_kappa;                            /* turb.kappa */
    double turb_ri_gate;                          /* turb.ri_gate: 0 off, or Ri_0 in [1e-6, 1] (the stratification
                                                     gate of the length and Rt; P_b keeps N^2) */
    double turb_realizability;                    /* turb.realizability: 0 off, or C_r in [0.01, 10] (nu_t <= C_r k / S) */
    double turb_nut_relax;                        /* turb.nut_relax in (0, 1]: nu_t = w nu_t,new + (1 - w) nu_t of the
                                                     last iteration (1: no history) */
} gb_physics;

/* simplec.* and steady.zline_sweeps (gust::SimplecOptions, Source/Simplec.H:80-90). */
typedef struct gb_simplec_opts {
    double pressure_reltol;          /* simplec.pressure_reltol */
    double alpha_p;                  /* simplec.alpha_p */
    double rotation_relax;           /* simplec.rotation_relax */
    double w_vnn_cap;                /* simplec.w_vnn_cap (0 off) */
    double w_vnn_cap_slope_margin;   /* simplec.w_vnn_cap_slope_margin */
    double tke_floor;                /* turb.tke_floor */
    int32_t zline_sweeps;            /* steady.zline_sweeps */
    int32_t precision;               /* 0 plain FP64; 1 FP32 inner solves (sweeps, multigrid) in FP64 defect correction */
    gb_poisson_opts poisson;         /* the correction's Poisson solver (reltol taken from pressure_reltol) */
    int32_t line_sweep;              /* steady.sweep: 0 zjacobi (z-line Jacobi), 1 lusgs (line LU-SGS, FP64) */
    int32_t line_alternate;          /* steady.line_alternate (lusgs): 1 = odd sweeps j-reversed */
} gb_simplec_opts;

/* The solution fields (gust::State, Source/State.H:18-36): device arrays of
 * the grid with two ghost layers; z_nd the node heights. */
typedef struct gb_state {
    double *u, *v, *w, *p, *theta, *tke;
    const double* z_nd;
} gb_state;

/* The mesh metrics (gust::Mesh) and the given diffusivities (nu, gamma_theta,
 * gamma_tke: cell arrays with one ghost layer filled). */
typedef struct gb_mesh_fields {
    const double *detJ, *ax, *ay, *az;
    /* The ground's roughness per column (bc.surface_z0_file, Source/
     * SurfaceRoughness.H): a plane of (ny + 1 + 2 ng) rows of sy doubles,
     * column (i, j) at (j + ng) sy + i + ng, set on the columns -1..nx,
     * -1..ny (the ghost columns the periodic image or the nearest domain
     * column); null: bc.surface_z0 everywhere. */
    const double* z0;
} gb_mesh_fields;
typedef struct gb_diffusivities {
    const double *nu, *gamma_theta, *gamma_tke;
} gb_diffusivities;

/* What one SIMPLEC iteration reports (SimplecStage's norms and the results of
 * its parts: MomentumPredictorResult, PressureCorrectionResult, ScalarSweepResult). */
typedef struct gb_iter_info {
    double residual_norms[6];        /* scaled RMS of R_u, R_v, R_w, R_p, R_theta, R_k (stage_norms) */
    double max_speed, mean_tke;      /* monitors */
    double max_du, max_dv, max_dw;
    double last_sweep_du, last_sweep_dv, last_sweep_dw;
    double divergence_before, divergence_after, max_dp, poisson_removed_mean;
    int32_t poisson_iterations;
    double max_dtheta, max_dtke;
    int64_t tke_clipped;
    double mean_ustar;               /* monitor with a surface-layer ground: the mean u* of the wall state
                                        at the start of the iteration (0 without) */
} gb_iter_info;

/* init.* of the mass-consistent initializer (gust::InitOptions,
 * Source/Initializer.H:63-111) with init.first_guess = profile. */
typedef struct gb_init_opts {
    double z_agl_min;                /* init.z_agl_min (m, >= 0): floor of the profile's height */
    double alpha_h, alpha_v;         /* init.alpha_h, init.alpha_v (> 0); alpha_v != alpha_h: the split z-face
                                        coefficient (gb_poisson_set_z_cross) */
    double k_decay_height;           /* init.k_decay_height (m, >= 0; 0: no decay) */
    int32_t projection;              /* init.projection (0 or 1) */
    int32_t obrien;                  /* init.obrien (0 or 1): the O'Brien column correction of w0 */
    gb_poisson_opts poisson;         /* solver.poisson_* of the projection */
} gb_init_opts;

/* What the initializer reports (gust::InitResult). */
typedef struct gb_init_result {
    double divergence_before, divergence_after;   /* L2 norms of the velocity divergence (1/s) */
    int32_t poisson_iterations;
    double poisson_final_residual;
    double obrien_top_residual;   /* max |Omega_top| the O'Brien pass removed (m/s; 0 without it) */
} gb_init_result;

typedef struct gb_simplec gb_simplec;

/* gust::SimplecStage (Source/Simplec.H:185-263) for one instance: the
 * boundary conditions, physics and options, the mesh (z_nd, metrics: device
 * arrays kept by reference) and the diffusivities. Builds the workspace and
 * the correction's Poisson solver. Checks the simplec.* ranges and the face
 * types with the reference's messages. */
gb_status gb_simplec_create(gb_ctx* ctx, const gb_grid* g, const gb_bc* bc, const gb_physics* ph,
                            const gb_simplec_opts* opt, const double* z_nd, const gb_mesh_fields* mesh,
                            const gb_diffusivities* df, gb_simplec** out);
gb_status gb_simplec_destroy(gb_simplec* s);

/* BoundaryConditions::fill_ghosts (Source/BoundaryConditions.H:174-175): two
 * ghost layers of u, v, w, p, theta, k and the Dirichlet face points. */
gb_status gb_simplec_fill_ghosts(gb_simplec* s, const gb_state* q);

/* gust::residual (Source/Residual.H:133-134) at q (ghosts filled by the
 * caller): R[0..5] = R_u, R_v, R_w, R_p, R_theta, R_k (device arrays). */
gb_status gb_simplec_residual(gb_simplec* s, const gb_state* q, double* const* R);

/* implicit_rows (Source/Residual.cpp:272-304) of equation eq (0 u, 1 v, 2 w,
 * 4 theta, 5 k) at q: the coefficients of the transport fluxes of q and the
 * stage's diffusivities (the closure's at the last residual), the Patankar
 * diagonal of k, the first cells' wall rows (the surface state of the last
 * ghost fill), the damping and the boundary folds, into A (GB_N_COEFS device
 * arrays of the grid, component-major). */
gb_status gb_simplec_implicit_rows(gb_simplec* s, const gb_state* q, int32_t eq, double* A);

/* SimplecStage::iterate (Source/Simplec.cpp:452-506): one SIMPLEC outer
 * iteration of q with the local pseudo-time step dtau (cells). */
gb_status gb_simplec_iterate(gb_simplec* s, const gb_state* q, const double* dtau, gb_iter_info* info);

/* ---- the iteration's steps alone ---------------------------------------
 * The pieces of gb_simplec_iterate that the reference also calls from outside
 * SimplecStage::iterate (the Newton preconditioner and the grid-sequencing
 * transfer reuse the predictor, the pressure correction and the scalar
 * sweep). Each runs the iteration's own code on the stage's workspace, in the
 * iteration's order: gb_simplec_fill_ghosts(q), gb_simplec_residual(q, R),
 * gb_momentum_predictor(q, R, dtau), gb_pressure_correction(q),
 * gb_scalar_sweep(theta), gb_scalar_sweep(k). */

/* gust::MomentumPredictorResult (Source/Predictor.H:214-220). */
typedef struct gb_predictor_result {
    double max_du, max_dv, max_dw;                     /* max |correction| applied per component */
    double last_sweep_du, last_sweep_dv, last_sweep_dw; /* max |change over the last sweep| */
} gb_predictor_result;

/* gust::PressureCorrectionResult (Source/Simplec.H:117-124), with the
 * Poisson solve's iterations and removed mean (gust::PoissonResult). */
typedef struct gb_pressure_result {
    int32_t poisson_iterations;
    double poisson_removed_mean;
    double divergence_before, divergence_after; /* max |div u| before and after */
    double max_dp;                              /* max |alpha_p p'| */
    double max_du, max_dv, max_dw;              /* max |velocity correction| per component */
} gb_pressure_result;

/* gust::ScalarSweepResult (Source/Simplec.H:149-154). */
typedef struct gb_scalar_result {
    double max_dq;      /* max |dq| applied */
    double last_sweep;  /* max |change over the last sweep| */
    int64_t clipped;    /* cells raised to the floor (k only) */
} gb_scalar_result;

/* gust::momentum_predictor (Source/Predictor.H:242-252, Predictor.cpp:129-405)
 * on q's u, v, w: R the residual at q as gb_simplec_residual returned it (the
 * closure's fields of that evaluation and the wall state of the last
 * gb_simplec_fill_ghosts are the ones used, as the reference's caller passes
 * its residual's fields and surface state), dtau the cell pseudo-time step
 * (face_dtau is taken here), the transport fluxes of q. ap and d (three
 * device arrays each, u, v, w faces, or NULL) receive PredictorFields' a_P
 * and the SIMPLEC denominators; the stage also keeps d for
 * gb_pressure_correction. q's ghosts are not refilled. */
gb_status gb_momentum_predictor(gb_simplec* s, const gb_state* q, double* const* R, const double* dtau,
                                double* const* ap, double* const* d, gb_predictor_result* res);

/* gust::pressure_correction (Source/Simplec.H:139-141, Simplec.cpp:134-220)
 * on q's u, v, w and p: d the SIMPLEC denominators on the u, v, w faces
 * (three device arrays, finite and >= 0; NULL: those of the last
 * gb_momentum_predictor). The ghosts of q are filled first, as the iteration
 * refills them after the predictor, without touching the wall state kept for
 * the scalar sweeps. The Poisson solve uses the stage's solver and
 * simplec.pressure_reltol; a predicted velocity with a net source the
 * boundaries cannot carry is refused (GB_BAD_ARG) with the reference's
 * message. */
gb_status gb_pressure_correction(gb_simplec* s, const gb_state* q, const double* const* d, gb_pressure_result* res);

/* gust::scalar_sweep (Source/Simplec.H:156-163, Simplec.cpp:222-281) of eq
 * (4 theta, 5 k) in delta form on q's field: (1/dtau + A1) dq = -R_eq with
 * the implicit rows of the transport fluxes of q (its ghosts filled first, as
 * the iteration refills them before the sweeps), the closure's fields of the
 * last residual and the wall state of the last gb_simplec_fill_ghosts;
 * `simplec.zline_sweeps` sweeps; k clipped at simplec.tke_floor (counted)
 * unless clip is 0. */
gb_status gb_scalar_sweep(gb_simplec* s, const gb_state* q, int32_t eq, const double* R_eq, const double* dtau,
                          int32_t clip, gb_scalar_result* res);

/* gust::SimplecPreconditioner (Source/NewtonPreconditioner.H:120-186):
 * setup at q (the stage's fill with the wall state, the closure's fields at
 * q, the step dtau, or local_dtau at inf_cfl when dtau is NULL, the transport
 * and theta's convection at q), then one apply: dq for the Newton system
 * linearized at q, (D + J) dq = r, by one SIMPLEC iteration from dq = 0 (the
 * momentum predictor with -r as the residual, the pressure correction of du*
 * with r_p as the source after the homogeneous fill, theta's coupling, the
 * theta and k steps without the floor; dq = r on the Dirichlet rows of u, v,
 * w). denominators: 1 the SIMPLE d = a_P (the reference's default), 2 the
 * stage's SIMPLEC d = a_P - sum a_nb (then with r = -R(q) the result is the
 * increment of one stage iteration from q, off the Dirichlet rows). r and dq:
 * six device arrays of the grid (u, v, w, p, theta, k). */
gb_status gb_simplec_precondition(gb_simplec* s, const gb_state* q, const double* dtau, double inf_cfl,
                                  int32_t denominators, double* const* r, double* const* dq);

/* gust::implicit_coefficients (Source/ImplicitOperator.H:65-67,
 * ImplicitOperator.cpp:96-121): the 7 coefficients at loc (GB_LOC_CELL or a
 * face) of the upwind transport F (x-, y-, z-face fluxes, one ghost) and the
 * principal diffusion with the metric of the cell diffusivity gamma (one
 * ghost), the node heights z_nd and detJ; the face means of gamma are
 * arithmetic, or logarithmic with log_mean = 1 (FaceMean). A: GB_N_COEFS
 * device arrays of the grid, component-major (valid points written). */
gb_status gb_implicit_coefficients(gb_ctx* ctx, const gb_grid* g, int32_t loc, const double* F0, const double* F1,
                                   const double* F2, const double* gamma, const double* z_nd, const double* detJ,
                                   int32_t log_mean, double* A);

/* SimplecStage::closure_fields (Source/Simplec.H:216) and the wall model's
 * state: the closure's fields at the last residual (nu, gamma_theta,
 * gamma_tke, nu_t, L, Rt, P_s, P_b, eps, dS_k/dk: device volumes of the
 * grid) and the surface state of the last ghost fill (u*, U, z_ref, d0,
 * 1/L, the stress tau x, y, z, drag, k_w, |A|: device planes of one value
 * per column, gb_mesh_fields.z0's layout), copied into the given arrays;
 * null arrays (or entries) are skipped. GB_BAD_ARG when the stage has no
 * closure (closure) or no surface_layer ground (surface). */
gb_status gb_simplec_turbulence(gb_simplec* s, double* const* closure, double* const* surface);
/* ResidualInputs::wall_distance (Source/Residual.H:61-128) for
 * turb.wall_distance = tucker: the closure's wall distance from now on is a
 * copy of dist (a device volume of the grid with its ghosts, as
 * gb_tucker_wall_distance writes it) in place of the height above the ground
 * (turb.wall_distance = terrain_height, the default). GB_BAD_ARG when the
 * stage has no closure. */
gb_status gb_simplec_set_wall_distance(gb_simplec* s, const double* dist);

/* The defaults of init.* (Source/Initializer.H: z_agl_min 0, alpha_h = alpha_v
 * = 1, k_decay_height 0, projection 1, obrien 0) and solver.poisson_*. */
gb_status gb_init_options_default(gb_init_opts* o);
/* gust::initialize_state with init.first_guess = profile (Source/Initializer.cpp:
 * 281-332 first_guess_state, 344-430 the projection), on the stage's mesh and
 * boundary conditions: u, v from the inflow profile at every point's height
 * above the ground (ghosts included), w = 0 but the ground faces' kinematic w,
 * theta = theta_ref(z), k from the profile (decaying above k_decay_height),
 * p = 0; with obrien = 1, w0 from O'Brien's column correction (obrien_omega,
 * Source/Initializer.cpp:197-274); then, with projection = 1, the
 * mass-consistent correction: the divergence removed by the terrain Poisson
 * solve with lambda = 0 on the inflow and outflow faces and zero flux through
 * the others, Sigma = diag(alpha_h^2, alpha_h^2, alpha_v^2) with the split
 * z-face coefficient when alpha_v != alpha_h (u, v, Omega += the fluxes, w
 * from Omega). */
gb_status gb_simplec_initialize(gb_simplec* s, const gb_state* q, const gb_init_opts* o, gb_init_result* r);

/* What a prolongation did (gust::ProlongResult, Source/Transfer.H:112-116). */
typedef struct gb_prolong_result {
    double divergence_before, divergence_after;  /* max |div u| before and after the projection (1/s) */
    int32_t poisson_iterations;
    int64_t tke_clipped;                         /* fine cells raised to the k floor */
} gb_prolong_result;

/* prolong_state (Source/Transfer.H:118-128, Transfer.cpp:322-385) into this
 * stage's state q from a coarser level's state qc on grid gc (coarser by a
 * power of two in x and y, the same layers; only its valid points are read,
 * a periodic neighbour through its image): every field bilinear per
 * zeta-level (the linear extrapolation in the half cell next to a
 * non-periodic face), k raised to the floor, this stage's ghost fill, then
 * the projection (the pressure correction with d = 1 off the Dirichlet
 * rows, the Poisson solve to reltol: the run's solver.poisson_reltol), p'
 * restored. */
gb_status gb_simplec_prolong(gb_simplec* s, const gb_state* q, const gb_grid* gc, const gb_state* qc, double reltol,
                             gb_prolong_result* r);

/* restrict_state (Source/Transfer.H:94-110, Transfer.cpp:199-286): the fine
 * state qf on grid gf (mesh mf: detJ and the face areas) onto the coarse
 * state qc on gc (mesh mc: its face areas; coarser by a power of two in x
 * and y, the same layers and periodicity). theta, k, p': the detJ-weighted
 * means of the fine cells; u, v: the fine face fluxes a q summed over the
 * coarse face, per unit width, over the coarse area; w from the restricted
 * vertical flux Omega (a_z Omega summed over r^2 fine z-faces, over the
 * coarse a_z), the coarse u and v read with zero-gradient rows below the
 * ground and above the top. qf's u and v need one ghost layer (the
 * stage's ghost fill). omega_c (may be NULL) receives the coarse Omega. */
gb_status gb_restrict_state(gb_ctx* ctx, const gb_grid* gf, const gb_state* qf, const gb_mesh_fields* mf,
                            const gb_grid* gc, const gb_state* qc, const gb_mesh_fields* mc, double* omega_c);

/* stage_norms (Source/Simplec.cpp:385-409) at q with no iteration: the ghost
 * fill, the residual, residual_norms[6] (the scaled RMS of R_u .. R_k) and
 * monitors[3] (max speed, mean k, mean u* with a surface-layer ground, else 0). */
gb_status gb_simplec_norms(gb_simplec* s, const gb_state* q, double* residual_norms, double* monitors);

/* gust::local_dtau (Source/PseudoTime.H:32-33) with the stage's diffusivity nu. */
gb_status gb_local_dtau(gb_simplec* s, const gb_state* q, double cfl, double* dtau);

/* ---- the steady driver -------------------------------------------------- */

/* steady.* of the pseudo-time driver and the steady criterion (gust::
 * SteadyOptions, Source/Driver.H:52-110; gust::SteadyParams,
 * Source/SteadyCriterion.H:13-33). */
typedef struct gb_driver_opts {
    double cfl0, cfl_max;            /* steady.cfl0, steady.cfl_max */
    double ser_exponent;             /* steady.ser_exponent */
    double ser_max_growth;           /* steady.ser_max_growth */
    double residual_tol;             /* steady.residual_tol */
    double residual_drop_orders;     /* steady.residual_drop_orders */
    int32_t residual_ref_iterations; /* steady.residual_ref_iterations */
    double monitor_rel_tol;          /* steady.monitor_rel_tol */
    int32_t monitor_window;          /* steady.monitor_window (>= 2) */
    double confidence;               /* steady.confidence: 0 off, or (0, 1]: steady once that share of the
                                        cells meets the residual criterion cell by cell with every monitor met */
    double confidence_height;        /* steady.confidence_height: 0 anywhere, or the height above the ground
                                        (m) every failing cell must be below */
} gb_driver_opts;

/* ---- the Newton-Krylov finishing stage ---------------------------------- */

/* steady.newton_* of the Newton-Krylov core (gust::NewtonOptions, Source/
 * Newton.H:84-107) and the pressure scale of its scaled variables
 * (JvpScales::pressure, Source/Residual.H:72-80). */
typedef struct gb_newton_opts {
    int32_t gmres_restart;           /* steady.newton_gmres_restart (5..200; 30) */
    int32_t gmres_max_iters;         /* steady.newton_gmres_max_iters (>= 1; 2000) */
    double fd_eps_scale;             /* steady.newton_fd_eps_scale (eps^(3/4) .. 1e-2; sqrt(eps)) */
    double krylov_rtol;              /* steady.newton_krylov_rtol ((0, 1); 1e-2) */
    double scale_pressure;           /* s_p (100 m^2/s^2) */
    int32_t preconditioner;          /* steady.newton_preconditioner: 0 identity, 1 simplec (one SIMPLEC
                                        iteration on the linearized system with the SIMPLE denominators
                                        d = a_P, the default; gust::SimplecPreconditioner,
                                        Source/NewtonPreconditioner.H:1-108), 2 simplec with the stage's
                                        SIMPLEC denominators (PressureDenominator::stage) */
    double inf_cfl;                  /* the preconditioner's CFL when a step has no dtau (steady.cfl_max; 10) */
} gb_newton_opts;
/* What one Newton step did (gust::NewtonStepInfo, Source/Newton.H:230-248). */
typedef struct gb_newton_step_info {
    int32_t gmres_iterations;
    int32_t gmres_status;            /* 0 converged, 1 the iteration cap */
    double residual_norm;            /* |b| = |T^-1 R(q)|_2 before the step */
    double krylov_residual;          /* FGMRES's final |b - A x|_2 (its Arnoldi estimate) */
    double krylov_relative;          /* krylov_residual / residual_norm */
    double eps_min, eps_max;         /* the jvp steps used */
    int32_t jvp_calls;
    int32_t applied;                 /* the update was usable (newton_update_usable) */
} gb_newton_step_info;
typedef struct gb_newton gb_newton;
gb_status gb_newton_options_default(gb_newton_opts* o);
/* check_newton_options (Source/Newton.cpp): each violation names its key. */
gb_status gb_newton_check(const gb_newton_opts* o);
/* gust::NewtonKrylov on a stage (its residual, ghost fill and scales;
 * check_newton_options' range checks name their keys). Allocates
 * 2 restart + 13 state-sized vectors. Every residual the calls below
 * evaluate (jvp, step, direction with its preconditioner, residual_norm)
 * takes the Newton stage's residual inputs (Source/Smoothness.cpp:59-67,
 * newton_residual_inputs): a stage with convection.limiter = van_leer is
 * evaluated with van_albada for the duration of the call, and its own
 * limiter is back when the call returns. */
gb_status gb_newton_create(gb_simplec* s, const gb_newton_opts* o, gb_newton** out);
gb_status gb_newton_destroy(gb_newton* n);
/* gust::jvp with the refill (Source/Residual.cpp:324-396): Jv = (R(fill(q +
 * eps v)) - R(q)) / eps, eps = h (1 + mean |q~|) / rms(v~) over the owned
 * points of the six fields; q's ghost cells are filled first. v and Jv: six
 * device arrays each (u, v, w, p, theta, k) on the grid layout, v's ghost
 * cells 0. */
gb_status gb_newton_jvp(gb_newton* n, const gb_state* q, double* const* v, double* const* Jv, double* eps);
/* NewtonKrylov::step (Source/Newton.H:292-298): q += dq from (D + J) dq =
 * -R(q) (dtau NULL: plain Newton), skipped when the update is not usable;
 * q's ghost cells filled before and after. */
gb_status gb_newton_step(gb_newton* n, const gb_state* q, const double* dtau, gb_newton_step_info* info);
/* NewtonKrylov::direction: the same solve, dq (six device arrays) = S x on
 * the valid points (0 when not usable), q unchanged but its ghost fill. */
gb_status gb_newton_direction(gb_newton* n, const gb_state* q, const double* dtau, double* const* dq,
                              gb_newton_step_info* info);
/* NewtonKrylov::residual_norm: |T^-1 R(fill(q))|_2 (the line search's norm). */
gb_status gb_newton_residual_norm(gb_newton* n, const gb_state* q, double* norm);
/* The continuation's trial point: out = q0 + lambda dq on the valid points
 * (k clipped at the stage's tke_floor), q0's ghost cells copied. */
gb_status gb_newton_trial(gb_newton* n, const gb_state* q0, double* const* dq, double lambda, const gb_state* out);

/* ---- the steady criterion ------------------------------------------------ */

/* gust::SteadyCriterion (Source/SteadyCriterion.H:81-150): residual
 * references (the largest of the first residual_ref_iterations values, or a
 * seed they raise), the last residuals and each monitor's last
 * monitor_window + 1 values; steady when every residual is below
 * residual_tol and residual_drop_orders orders below its reference (floored
 * at residual_tol) and every monitor has a full window, changed over it by
 * at most monitor_rel_tol of max(|last|, scale) and is within that of its
 * Aitken-extrapolated limit. A NaN or infinity is Diverged for good.
 * Host only: no GPU is needed. */
typedef struct gb_criterion gb_criterion;
enum { GB_CRITERION_MAX_RESIDUALS = 8, GB_CRITERION_MAX_MONITORS = 4 };
enum { GB_NOT_STEADY = 0, GB_STEADY = 1, GB_DIVERGED = 2 };
typedef struct gb_steady_history {
    int32_t count, nonfinite, n_residuals, n_monitors;
    double res_ref[GB_CRITERION_MAX_RESIDUALS], res_last[GB_CRITERION_MAX_RESIDUALS];
    int32_t monitor_values[GB_CRITERION_MAX_MONITORS];   /* values in each monitor's window */
    double monitor_last[GB_CRITERION_MAX_MONITORS];
} gb_steady_history;
/* The parameters are o's residual_* and monitor_* (validate, Source/
 * SteadyCriterion.cpp:26-48: each violation names its key); the names label
 * the verdict's reasons; each monitor scale finite and > 0. */
gb_status gb_criterion_create(const gb_driver_opts* o, int32_t n_residuals, const char* const* residual_names,
                              int32_t n_monitors, const char* const* monitor_names, const double* monitor_scales,
                              gb_criterion** out);
gb_status gb_criterion_destroy(gb_criterion* c);
/* SteadyCriterion::add: one iteration's residuals and monitors. */
gb_status gb_criterion_add(gb_criterion* c, const double* residuals, const double* monitors);
/* SteadyCriterion::seed_reference (grid sequencing): before the first add. */
gb_status gb_criterion_seed_reference(gb_criterion* c, const double* ref);
/* SteadyCriterion::verdict: *status GB_NOT_STEADY, _STEADY or _DIVERGED;
 * reasons (may be NULL) receives why it is not steady, one per line. */
gb_status gb_criterion_verdict(const gb_criterion* c, int32_t* status, int32_t* residuals_met, int32_t* monitors_met,
                               char* reasons, int32_t reasons_cap);
gb_status gb_criterion_history(const gb_criterion* c, gb_steady_history* h);
/* Monitor m's window, oldest first: *n values (at most cap copied). */
gb_status gb_criterion_monitor_window(const gb_criterion* c, int32_t m, double* values, int32_t cap, int32_t* n);

/* steady.sequencing_* (gust::SequencingOptions, Source/Sequencing.H:87-95). */
typedef struct gb_sequencing_opts {
    int32_t enabled;                 /* steady.sequencing */
    double drop_orders;              /* steady.sequencing_drop_orders (2) */
    double monitor_tol;              /* steady.sequencing_monitor_tol (0: off) */
    int32_t hold;                    /* steady.sequencing_hold (0 | 1; 0) */
    int32_t cfl_previous;            /* steady.sequencing_cfl_start = previous (1) or cfl0 (0) */
} gb_sequencing_opts;
/* check_sequencing_options (Source/Sequencing.cpp:120-169) for a mesh of
 * nx x ny cells over hierarchy_levels levels; strict: the run's criterion. */
gb_status gb_sequencing_check(const gb_sequencing_opts* o, const gb_driver_opts* strict, int32_t nx, int32_t ny,
                              int32_t hierarchy_levels);
enum { GB_LOOSE_NONE = 0, GB_LOOSE_RESIDUALS = 1, GB_LOOSE_MONITORS = 2 };
/* loose_stop (Source/Sequencing.cpp:172-222) after the last iteration c
 * recorded: *branch GB_LOOSE_NONE, (a) _RESIDUALS or (b) _MONITORS; reason
 * (may be NULL) the branch's text. hold_iterations: the level's reference
 * hold (gb_driver_hold_iterations). */
gb_status gb_loose_stop(const gb_criterion* c, const gb_sequencing_opts* o, int32_t hold_iterations, int32_t* branch,
                        char* reason, int32_t reason_cap);

enum { GB_DRIVER_RUNNING = 0, GB_DRIVER_STEADY = 1, GB_DRIVER_DIVERGED = 2, GB_DRIVER_FAILED = 3 };

typedef struct gb_driver gb_driver;

/* The defaults (cfl0 1, cfl_max 8 with steady.sweep = lusgs else 10 (Source/
 * Driver.cpp:133-136), ser_exponent 1, ser_max_growth 2, residual_tol 5e-5,
 * residual_drop_orders 4, residual_ref_iterations 5, monitor_rel_tol 1e-3,
 * monitor_window 50). */
gb_status gb_driver_options_default(gb_driver_opts* o, int32_t line_sweep);
/* gust::Driver for one stage and state (allocates the local dtau). */
gb_status gb_driver_create(gb_simplec* s, const gb_state* q, const gb_driver_opts* o, gb_driver** out);
gb_status gb_driver_destroy(gb_driver* d);
/* Driver::step (Source/Driver.cpp:403-468): the local dtau at the current CFL,
 * one SIMPLEC iteration, the residuals and monitors (max_speed, mean_tke and,
 * with a surface-layer ground, mean_ustar; stage_monitor_specs, Source/
 * Simplec.cpp:365-371, scales gb_physics.scale_velocity, scale_tke and 0.1)
 * into the criterion, r_n after the reference hold, the next CFL (cfl0
 * during the hold, then the SER law). *verdict: GB_DRIVER_RUNNING, _STEADY
 * or _DIVERGED (a non-finite iteration, residual or monitor); info and cfl
 * (the CFL used) may be NULL. */
gb_status gb_driver_step(gb_driver* d, int32_t* verdict, gb_iter_info* info, double* cfl);
/* The driver's criterion (owned by the driver): history, verdict, loose stop. */
gb_status gb_driver_criterion(gb_driver* d, gb_criterion** c);
/* Driver::seed_reference, release_reference_hold and start_cfl (Source/
 * Driver.cpp:275-313), each only before the first step: the coarsest
 * level's references; no reference hold (needs a seed); the first CFL
 * (with the hold released; brought up to cfl0, at most cfl_max). */
gb_status gb_driver_seed_reference(gb_driver* d, const double* ref);
gb_status gb_driver_release_hold(gb_driver* d);
gb_status gb_driver_start_cfl(gb_driver* d, double cfl);
/* SimplecStage::confidence (Source/Simplec.cpp:411-445) on the residual of the
 * last iteration's start: the share of cells whose six residuals are within
 * thresholds[6] (the criterion's per equation, in the scaled units of the
 * norms) and the largest height above the ground of a cell that is not. */
gb_status gb_simplec_confidence(gb_simplec* s, const double* thresholds, double* share, double* height);
/* Driver::hold_iterations, the CFL of the next step and r_n of the last. */
gb_status gb_driver_status(const gb_driver* d, int32_t* hold_iterations, double* next_cfl, double* relative_residual);
/* Many drivers at once: each steps until its verdict is not RUNNING or it
 * has taken max_iterations steps, on `threads` host threads (<= 0: one per
 * driver), so that one driver's host synchronisations overlap the others'
 * kernels. verdicts[n] (GB_DRIVER_FAILED when a step returned an error) and
 * iterations[n] receive each driver's outcome. Drivers must not share a
 * context. */
gb_status gb_driver_run(gb_driver* const* drivers, int32_t n, int32_t max_iterations, int32_t threads,
                        int32_t* verdicts, int32_t* iterations);

#ifdef __cplusplus
}
#endif

#endif /* GUST_B200_H_ */
