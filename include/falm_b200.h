/*
 * falm_b200 -- C ABI of the B200 (sm_100a) implementation of FALM's LES step.
 *
 * Drop-in boundary for the reference's solver classes: FalmCFD, FalmEq,
 * FalmMV, Alm::AlmHandler and the application boundary routines.  Every
 * entry point cites the reference interface it replaces (paths relative to
 * the reference project ki2098/falm).
 *
 * Conventions
 *  - Fields are caller-owned DEVICE arrays in the reference's layout
 *    (src/matrix.h:20, src/util.h:74-76): column-major SoA over the box with
 *    guide cells, value(idx, col) = ptr[idx + col*N], idx = i + j*sx + k*sx*sy,
 *    N = sx*sy*sz.  Vector fields (u, uu, ff) have 3 columns.
 *  - Element type of every field pointer (void*) is the context precision:
 *    double for FALM_FP64, float for FALM_MIXED.  Inner products, norms,
 *    residual checks and returned scalars are double in both modes.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    Entry points that return a scalar on the host synchronise that stream;
 *    the others are asynchronous.
 *  - Every entry point returns a falm_status; nothing aborts the process.
 *  - Metrics (ja, kx, g of src/falm.h:383-404) are not passed per call: they
 *    are evaluated from the 1D control-volume tables given at falm_create,
 *    which is what the reference builds its 3D metric planes from.
 */
#ifndef FALM_B200_H
#define FALM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FALM_B200_ABI_VERSION 1

typedef enum {
    FALM_OK = 0,
    FALM_ERR_ARG = 1,        /* bad argument (null pointer, size, enum)                    */
    FALM_ERR_CUDA = 2,       /* CUDA runtime error (see falm_last_error)                   */
    FALM_ERR_NAN = 3,        /* non-finite value detected in a reduction                   */
    FALM_ERR_BREAKDOWN = 4,  /* BiCGStab |rho| < FLT_MIN (src/FalmEq.cpp:348)              */
    FALM_ERR_MAXIT = 5,      /* linear solver stopped at maxit without reaching tol        */
    FALM_ERR_TIMEOUT = 6,    /* a bounded device-side wait gave up                         */
    FALM_ERR_ALLOC = 7,      /* device allocation failed                                   */
    FALM_ERR_STATE = 8,      /* call order (e.g. solve before the operator was built)      */
    FALM_ERR_NOALM = 9,      /* ALM entry point called without falm_alm_init               */
    FALM_ERR_SIZE = 10       /* request larger than a fixed capacity (falm_mv_dot_static)  */
} falm_status;

typedef enum { FALM_FP64 = 0, FALM_MIXED = 1 } falm_precision;

/* src/FalmCFDDevCall.h (AdvectionSchemeType, SGSType) */
enum { FALM_ADV_UPWIND1 = 0, FALM_ADV_UPWIND3 = 1, FALM_ADV_QUICK = 2, FALM_ADV_UTOPIA = 3, FALM_ADV_KK = 4 };
enum { FALM_SGS_EMPTY = 0, FALM_SGS_SMAGORINSKY = 1, FALM_SGS_CSM = 2 };
/* src/FalmEqDevCall.h:143-149 (SolverType) */
enum { FALM_LS_EMPTY = 0, FALM_LS_JACOBI = 1, FALM_LS_SOR = 2, FALM_LS_PBICGSTAB = 4 };
/* boundary-condition sets of the application drivers */
enum { FALM_BC_CHANNEL = 0,  /* app/nedo, app/windtunnel: inlet, convective outlet, slip y+-, wall z-, slip z+ */
       FALM_BC_CAVITY  = 1 };/* app/lid3d: walls, lid y+ moving with (1,0,0), zero normal face flux     */

typedef struct falm_ctx falm_ctx;

/* Control-volume description (src/FalmIO.h:99-116, src/FalmMeshBase.h):
 * shape with guide cells and 1D centre/width tables, HOST pointers (copied). */
typedef struct {
    int sx, sy, sz;            /* pdm.shape incl. guide cells            */
    int gc;                    /* guide cells (src/typedef.h:41), 2      */
    const double *x, *y, *z;   /* cell centres, lengths sx, sy, sz       */
    const double *hx, *hy, *hz;/* cell widths,  lengths sx, sy, sz       */
} falm_grid;

/* Turbines and actuator points (src/alm/turbineHandler.h:13-104,
 * src/alm/apHandler.h:12-143).  HOST pointers, copied by falm_alm_init. */
typedef struct {
    int n_turbine, n_blade, n_ap_per_blade, n_attack;
    double radius, hub_radius, euler_eps;
    const double *base;        /* 3*n_turbine                                        */
    const double *hub;         /* 3*n_turbine, rotor centre in the turbine frame     */
    const double *tip_rate;    /* n_turbine                                          */
    const double *motion;      /* 3*n_turbine: amplitude [rad], angular freq, phase  */
    const int    *angle_type;  /* n_turbine: 0 none, 1 roll, 2 pitch, 3 yaw          */
    const double *ap_r, *ap_chord, *ap_twist;  /* apcount                           */
    const double *attack;      /* n_attack [deg]                                     */
    const double *cl, *cd;     /* apcount*n_attack, (ap, atk) at ap + atk*apcount    */
    double pitch;              /* collective pitch offset [deg] added to every twist */
} falm_alm_desc;

/* Fields of one step, caller-owned device arrays (FalmBasicVar, src/falm.h:16-43). */
typedef struct {
    void *u;      /* 3N velocity                                            */
    void *uu;     /* 3N contravariant face velocity                         */
    void *p;      /* N  pressure                                            */
    void *nut;    /* N  eddy viscosity                                      */
    void *ff;     /* 3N ALM body force, or NULL: the force is then evaluated
                     inside the pseudo-velocity kernel and never stored     */
} falm_fields;

typedef struct {
    int    it;          /* Poisson iterations this step (BiCGStab, summed over refinement passes) */
    double err;         /* final ||r||_2 / N_interior (src/FalmEq.cpp:403)                          */
    double divnorm;     /* sqrt(sum div^2) / N_interior (app/nedo/main.cpp:194-197,230)             */
    int    outer;       /* refinement passes (1 in FP64 mode)                                      */
    int    status;      /* falm_status of the linear solve                                          */
    double torque[8];   /* per turbine (src/alm/almDevCall.cu:362-370)                              */
    double thrust[8];
} falm_step_stats;

/* ---------------- context ---------------------------------------------------------------- */
/* FalmCore::computation_init (src/falm.h:342-431) minus IO; one GPU, no MPI. */
int falm_create(const falm_grid *grid, int precision, falm_ctx **out);
int falm_destroy(falm_ctx *ctx);
const char *falm_last_error(const falm_ctx *ctx);
int falm_abi_version(void);
/* number of this library's kernels launched since creation (for launch accounting) */
long long falm_kernel_launches(const falm_ctx *ctx);

/* ---------------- FalmCFD (src/FalmCFD.h:15-109, src/FalmCFDDevCall.h) --------------------- */
int falm_cfd_init(falm_ctx *ctx, double Re, int adv_scheme, int sgs_model, double Cs);
/* FalmCFD::FSPseudoU (src/FalmCFD.cpp:5-67): ua = un + dt(-adv(u,uu) + vis(u,nut) + ff) on the
   interior.  ua must not alias u (the reference's aliased call is a data race). ff may be NULL
   when falm_alm_init was called: the ALM force is then projected inside the kernel. */
int falm_cfd_pseudo_u(falm_ctx *ctx, const void *un, const void *u, const void *uu, void *ua,
                      const void *nut, const void *ff, double dt, double t, void *stream);
/* FalmCFD::UtoUU (src/FalmCFD.cpp:69-129) */
int falm_cfd_utouu(falm_ctx *ctx, const void *u, void *uu, void *stream);
/* FalmCFD::MACCalcPoissonRHS (src/FalmCFD.h:96-109) */
int falm_cfd_poisson_rhs(falm_ctx *ctx, const void *uu, void *rhs, double dt, double maxdiag, void *stream);
/* FalmCFD::ProjectP (src/FalmCFD.cpp:131-185); u may alias ua and uu may alias uua */
int falm_cfd_project_p(falm_ctx *ctx, void *u, const void *ua, void *uu, const void *uua,
                       const void *p, double dt, void *stream);
/* FalmCFD::SGS (src/FalmCFD.cpp:187-238) */
int falm_cfd_sgs(falm_ctx *ctx, const void *u, void *nut, void *stream);
/* FalmCFD::Divergence (src/FalmCFD.h:84-94) */
int falm_cfd_divergence(falm_ctx *ctx, const void *uu, void *div, void *stream);

/* ---------------- FalmEq (src/FalmEq.h:14-76) -------------------------------------------- */
/* FalmEq::init (src/FalmEq.h:23-25).  type: FALM_LS_PBICGSTAB, or the plain FALM_LS_JACOBI /
   FALM_LS_SOR solvers (relax is the SOR relaxation factor); pc_type (SOR or Jacobi) is used
   by PBiCGStab only, and a plain solver also accepts FALM_LS_EMPTY. */
int falm_eq_init(falm_ctx *ctx, int type, int maxit, double tol, double relax,
                 int pc_type, int pc_maxit, double pc_relax);
/* Poisson operator of the application drivers (app/nedo/main.cpp:25-100,
   app/lid3d/main.cpp:22-92) + FalmMV::MaxDiag + ScaleMatrix; kept as 1D
   coefficient tables.  Returns maxdiag. */
int falm_eq_poisson_operator(falm_ctx *ctx, int bc_kind, double *maxdiag_out);
/* Use an explicit caller-owned 7-column matrix (columns c,w,e,s,n,b,t,
   src/dev/FalmEqDevCall.cu:69-75) instead; NULL returns to the Poisson tables. */
int falm_eq_set_matrix(falm_ctx *ctx, const void *A);
/* FalmEq::Solve (src/FalmEq.h:56-64) -> Jacobi (src/FalmEq.cpp:80-127), SOR (:173-240; Black
   then Red half sweep, then the residual, per iteration) or PBiCGStab (:305-410).  For the plain
   solvers r holds the residual of the final iterate; both iterate in the storage type with
   FP64 residual norms.  For PBiCGStab in FALM_MIXED the
   iteration runs in FP32 storage with FP64 inner products and is wrapped in an FP64
   true-residual refinement loop.  it/err as FalmEq::it/err (src/FalmEqDevCall.h:27-30).
   r is work storage; on return it holds the last iteration's updated residual (as the
   reference's r), or the true residual when the refinement ran out of passes. */
int falm_eq_solve(falm_ctx *ctx, void *x, const void *b, void *r, void *stream, int *it_out, double *err_out);
/* FalmEq::Res (src/FalmEq.cpp:45-78) */
int falm_eq_res(falm_ctx *ctx, const void *x, const void *b, void *r, void *stream);
/* FalmEqDevCall::SORSweep (src/dev/FalmEqDevCall.cu:175-221), one colour */
int falm_eq_sor_sweep(falm_ctx *ctx, void *x, const void *b, double omega, int color, void *stream);

/* ---------------- FalmMV (src/MV.h:11-136) ------------------------------------------------ */
int falm_mv_mv(falm_ctx *ctx, const void *x, void *ax, void *stream);
int falm_mv_dot(falm_ctx *ctx, const void *a, const void *b, double *out, void *stream);
int falm_mv_normsq(falm_ctx *ctx, const void *a, int ncol, double *out, void *stream);
int falm_mv_maxdiag(falm_ctx *ctx, double *out);
int falm_mv_scale(falm_ctx *ctx, void *a, long long n, double scale, void *stream);
int falm_mv_axby(falm_ctx *ctx, double a, const void *x, double b, const void *y, void *result,
                 long long n, void *stream);

/* ---------------- boundary conditions (application drivers) -------------------------------- */
/* kind and inlet velocity (app/windtunnel/bcdevcall.cu:8-22 takes u_inlet) */
int falm_bc_init(falm_ctx *ctx, int kind, double u_inlet);
/* Seeded inflow: periodic perturbation box, HOST FP64 array 3 x nb x (sy-2gc) x (sz-2gc)
   (component-major, then x-plane, then j, then k), sampled at x = u_inlet*t, plane spacing dx.
   NULL removes it.  No reference counterpart (the reference has uniform inflow only). */
int falm_bc_set_inflow(falm_ctx *ctx, const double *box, int nb, double dx);
/* ubc (app/nedo/bc.h, app/lid3d/bc.h): velocity ghost cells.  uprev feeds the convective outlet. */
int falm_bc_ubc(falm_ctx *ctx, void *u, const void *uprev, double dt, double t, void *stream);
/* pbc: pressure ghost cells */
int falm_bc_pbc(falm_ctx *ctx, void *p, void *stream);
/* uubc (app/lid3d/bc.h): zero wall-normal face flux, cavity only (no-op for the channel) */
int falm_bc_uubc(falm_ctx *ctx, void *uu, void *stream);

/* ---------------- ALM (src/alm/alm.h:12-140) ----------------------------------------------- */
/* AlmHandler::init (src/alm/alm.h:20-57) after the AP tables were built */
int falm_alm_init(falm_ctx *ctx, const falm_alm_desc *desc);
/* BladeHandler::buildAP (src/alm/bladeHandler.h:16-104), host only: station polars row-major
   [station][attack]; outputs in the APFrame layout. */
int falm_alm_build_aps(int n_station, const double *st_r, const double *st_chord, const double *st_twist,
                       const double *st_cl, const double *st_cd, int n_attack, int apcount,
                       int n_ap_per_blade, double radius, double hub_radius,
                       double *ap_r, double *ap_chord, double *ap_twist, double *ap_cl, double *ap_cd);
/* change the collective pitch offset [deg] */
int falm_alm_set_pitch(falm_ctx *ctx, double pitch_deg);
/* AlmHandler::Alm (src/alm/alm.h:66-77): AP forces at time t from u, projected into ff
   (3N, interior written).  torque/thrust per turbine returned if non-NULL (syncs). */
int falm_alm_run(falm_ctx *ctx, const void *u, void *ff, double t, void *stream,
                 double *torque, double *thrust);
/* AP state after the last ALM evaluation (host FP64 arrays, any may be NULL) */
int falm_alm_get_aps(falm_ctx *ctx, double *xyz, double *force, double *torque, double *thrust);

/* ---------------- one fused time step ------------------------------------------------------ */
/* app/nedo/main.cpp:150-204 (channel) / app/lid3d/main.cpp:121-168 (cavity):
   ALM -> pseudo-velocity -> UtoUU [-> uubc] -> RHS -> Poisson -> pbc -> projection -> ubc ->
   SGS -> divergence norm, with the race-free pseudo-velocity convention.  t = it*dt. */
int falm_step(falm_ctx *ctx, const falm_fields *f, double dt, double t, void *stream, falm_step_stats *st);

/* Streamed inflow: the inlet velocity (u,v,w) of the NEXT velocity BC (falm_step or
   falm_bc_ubc) as a HOST FP64 array 3 x (sz-2gc) x (sy-2gc) (component, then k, then j
   fastest).  That call copies it to the device (a step recorded as a CUDA graph does so
   beside the phases before the BC), so the array must stay valid and unchanged until the
   call returns; pass pinned memory.  `stream` is not used.  Takes precedence over the
   inflow box for that one call.  No reference counterpart (the reference has uniform inflow
   only). */
int falm_bc_set_inlet_plane(falm_ctx *ctx, const double *plane, void *stream);

/* ---------------- FalmIO (src/FalmIO.h) and time averaging (src/falm.h:433-478) ----------- */
/* FalmSolver::TAvg (src/falm.h:433-444): avg = (1 - 1/count) avg + (1/count) f over the whole
   arrays (ncol columns of the context's grid, guide cells included), count = it - start + 1. */
int falm_tavg(falm_ctx *ctx, void *avg, const void *f, int ncol, long long count, void *stream);
/* FalmIO::writeVectorFile (src/FalmIO.h:69-97) as outputUVWP calls it (src/falm.h:446-475): the
   header imax, jmax, kmax, ncol, gc, step (8-byte unsigned each), time (double), dsize (8-byte),
   then the columns of the whole array (guide cells included, i fastest, then j, k), column after
   column.  The columns are those of `nfields` device fields of ncols[q] columns each, in order
   (the drivers' uvwp: u then p).  dsize is the context's storage size, or 8 with as_fp64 (an FP32
   context's values cast on the device).  The copies run on `stream` into one of two pinned
   staging buffers and a host thread of the context writes the file, so the call returns before
   the file exists (a third call waits for a free buffer); falm_io_wait waits for every queued
   file and returns the first write error since its last call. */
int falm_io_write_vector_file(falm_ctx *ctx, const char *path, const void *const *fields, const int *ncols, int nfields,
                              unsigned long long step, double time, int as_fp64, void *stream);
/* No reference counterpart (the reference writes these files and never reads them back): the
   inverse of falm_io_write_vector_file, for restarting a run from a snapshot.  Reads `path` into
   the DEVICE fields (ncols[q] columns each, in the file's column order), converting FP64 <-> FP32
   to the context's precision; the file's grid (sx, sy, sz, gc) and column count must be the
   context's.  step_out / time_out (optional) receive the header's step and time.  A truncated
   file, a mismatched header or data beyond the announced columns return FALM_ERR_ARG and leave
   the fields unchanged.  Synchronous. */
int falm_io_read_vector_file(falm_ctx *ctx, const char *path, void *const *fields, const int *ncols, int nfields,
                             unsigned long long *step_out, double *time_out, void *stream);
int falm_io_wait(falm_ctx *ctx);
/* FalmIO::writeIndexFile (src/FalmIO.h:25-67) for one rank: nlohmann::json's dump(2) of
   {dataType, global, guidePoint, outputSteps[{step, time, timeAvg}], ranks, variables}, byte for
   byte (the reference spells the float32 key "dateType"; this writes "dataType" for both).
   nx, ny, nz are interior sizes; tavg may be NULL; dsize 4 or 8. */
int falm_io_write_index_file(const char *path, int nx, int ny, int nz, int gc, const unsigned long long *steps,
                             const double *times, const int *tavg, int nsnap, int dsize);
/* FalmIO::writeControlVolumeFile (src/FalmIO.h:118-135) of the context's grid ("sx sy sz gc",
   then x hx, y hy, z hz per line as "\t%.15e\t%.15e") and FalmIO::readControlVolumeFile
   (:99-116): dims = {sx, sy, sz, gc}; with all six arrays NULL only dims is read. */
int falm_io_write_cv_file(falm_ctx *ctx, const char *path);
int falm_io_read_cv_file(const char *path, int dims[4], double *x, double *hx, double *y, double *hy, double *z, double *hz);
/* Mesher::build_mesh (src/mesher/mesher.hpp:12-260), host only: the control-volume file
   `outputfile` (gc guide cells) from the node coordinates in meshpath/{x,y,z}.txt (a count,
   then one value per line) with meshpath/mesh.json {"coordinatePoint": "node"}; cvcenter
   "cell" (the nodes are cell faces) or "innerNode" (the nodes are cell centres, one guide
   cell included on each side). */
int falm_mesh_build(const char *cvcenter, const char *meshpath, const char *outputfile, int gc);

/* ---------------- discrete adjoint of the step ---------------------------------------------- */
/* No reference counterpart.  Adjoint of falm_step (Upwind3/UTOPIA/KK advection, Smagorinsky or no
   SGS, channel or cavity, the ALM forcing, one slab), with the Poisson solve treated as exact (its
   adjoint is one solve with the transposed operator, started from an extrapolation of the previous
   calls', to a relative residual of 1e-5, or 1e-12 when the context's tolerance is below 1e-12; see
   falm_adjoint_set_tol).  The adjoint fields and the gradient are FP64 in every context.  In a
   FALM_MIXED context the states f0, f1 are the context's FP32 fields and the recomputed step is the
   mixed-precision step, while the transposed solve runs in FP64 (on FP64 solver vectors of the
   adjoint workspace); the operator must be falm_eq_poisson_operator's (FALM_ERR_ARG after
   falm_eq_set_matrix).  f0: the DEVICE state
   (u, uu, p, nut; ff unused) at the start of the step, left unchanged; t: that step's time (as given
   to falm_step); w_power: the weight of this step's rotor power (sum over turbines of torque x tip
   rate) in the objective.  au (3N), auu (3N), anut (N): DEVICE FP64 adjoint of the state after the step
   on entry, of the state before it on return.  grad: DEVICE array of 1 + 2*apcount doubles
   (collective pitch [deg], per-AP chord, per-AP twist [deg]) to which the step's gradient
   contributions are added.  f1: the DEVICE state after the step (only its u is read), or NULL:
   the step is then recomputed internally from f0 (the context's solver tolerance applies).
   With f1 given only the ALM is re-evaluated, so a driver that keeps the states of a segment
   pays one forward step less per adjoint step. */
int falm_step_adjoint(falm_ctx *ctx, const falm_fields *f0, const falm_fields *f1, double dt, double t,
                      double w_power, void *au, void *auu, void *anut, double *grad, void *stream);
/* No reference counterpart.  Relative residual (||r|| / ||b||) to which falm_step_adjoint solves
   its transposed Poisson system; 0 restores the default (1e-5, or 1e-12 when the context's
   tolerance is below 1e-12).  The gradient's error from an inexact transposed solve is of the
   order of this tolerance times the sensitivity carried by the pressure: on the 128x64x64
   rotor case over 200 steps, 1e-4 and 1e-5 leave the gradient within 1e-5 of central finite
   differences, as an exact solve does. */
int falm_adjoint_set_tol(falm_ctx *ctx, double rel_tol);

/* ---------------- allocation-free inner product --------------------------------------------- */
/* No reference counterpart.  The interior inner product of falm_mv_dot for callers that hold
   device fields but may not allocate (a coupled solver or in-situ monitor beside a simulation
   that has claimed the device memory, where creating a context could fail): no context, and
   nothing is allocated -- the partial sums, arrival counter and result live in a fixed 128 KiB
   device array inside the library, which every GPU that loads the library holds until exit.
   - One 256-thread block per 8 interior rows, (sy-2gc)*(sz-2gc) rows: grids with more than
     131072 interior rows return FALM_ERR_SIZE without touching the device; gc must be 1..64.
   - Every call clears the arrival counter on its stream before its kernel.
   - All calls on a device share the array, which keeps the last call's contents: two calls in
     flight at once (two streams or two host threads) race and give wrong results.
   - The first call on a device (and the first after that device's context was replaced, e.g.
     by cudaDeviceReset) performs the set-up: it takes the array's address with
     cudaGetSymbolAddress, which may load the library's device code; make it before any
     stream capture.
   - The blocks sum in another order than falm_mv_dot's, so the two results agree to rounding
     (relative 1e-12 in FP64), not bit for bit.
   precision FALM_FP64 (double fields) or FALM_MIXED (float fields); *out is a host double. */
int falm_mv_dot_static(int sx, int sy, int sz, int gc, int precision, const void *a, const void *b,
                       double *out, void *stream);

/* ---------------- RMCP rotor model (the reference's alternate forcing) ---------------------- */
/* Rmcp::RmcpAlm (src/rmcp/alm.h:13-96; TurbineHandler src/rmcp/turbineHandler.h:119-185,
   BladeHandler src/rmcp/bladeHandler.h:134-185): turbines with a fixed orientation whose rotating
   blades paint the cells they cover (kernel_SetALMFlag, src/rmcp/almDevCall.cu:13-65); every
   painted cell gets the blade-element force of its own velocity (kernel_ALM, :144-209).
   angle_type 0 none, 1 roll, 2 pitch, 3 yaw (one Euler angle, in radians); hub = (-overhang, 0,
   tower); blade_width / blade_thick: the blade strip's width about the blade axis and its
   thickness downstream of the rotor plane (the reference's BLADE_WIDTH and BLADE_THICK, 0.1,
   src/rmcp/almDevCall.cu:6-7); stations: r/R, chord/R, twist [deg] and the Cl/Cd rows
   (station-major, n_attack per station) over attack [deg].  Lengths in rotor radii, as the
   reference's tables require. */
typedef struct falm_rmcp_desc {
    int n_turbine, n_blade;
    double radius, hub_radius;
    double blade_width, blade_thick;
    const double *base, *hub, *angle;   /* 3 per turbine */
    const int *angle_type;
    const double *tip_rate;
    int n_station, n_attack;
    const double *st_r, *st_chord, *st_twist, *attack, *cl, *cd;
} falm_rmcp_desc;
/* RmcpAlm::init: the RMCP model becomes the step's forcing (replacing the ALM; falm_alm_init
   replaces it in turn).  falm_step then paints and forces the cells of each turbine's box into a
   force field of the context and reports per turbine the torque sum(r |f_t|) over its painted
   cells (the reference's CalcTorque formula, almDevCall.cu:368-411) and the thrust sum(|f_x|). */
int falm_rmcp_init(falm_ctx *ctx, const falm_rmcp_desc *d);
/* RmcpAlm::SetALMFlag + RmcpAlm::ALM at time t: the force of every cell of the turbines' boxes
   into ff (3 components, zero where not painted; cells outside the boxes are not written, keep
   them zero), the paint (0 or turbine + 1) of the box cells into the optional DEVICE int field
   flag, and per turbine torque and thrust (host arrays of n_turbine, optional). */
int falm_rmcp_run(falm_ctx *ctx, const void *u, void *ff, double t, void *stream, int *flag, double *torque, double *thrust);

/* ---------------- z-slab decomposition over several GPUs ------------------------------------ */
/* The reference decomposes the grid into per-rank boxes with a 6-face MPI halo exchange (CPM:
   partition src/CPMBase.h:36-112, exchange src/CPMComm.h:182-364, pack/unpack
   src/dev/CPMDevCall.cu:7-60; its drivers split x, app/nedo/main.cpp:105).  Here the grid is
   split into slabs of whole z planes, one per GPU, so every halo is a run of contiguous planes
   of each component (no packing), exchanged through a transport:
     exchange: send `bytes` from send_lo to the rank below (it receives them into its recv_hi)
               and from send_hi to the rank above (into its recv_lo), ordered on `stream`; NULL
               pointers where there is no neighbour.  On return, work queued on `stream` may
               read the received planes and overwrite the sent ones.
     allreduce: reduce n doubles in device memory in place over all ranks (op FALM_REDUCE_SUM or
               FALM_REDUCE_MAX), ordered on `stream`; every rank gets the same values.
   Both return a falm_status.  Two transports are built in (below); a caller may supply its own. */
typedef struct falm_transport {
    void *user;
    int (*exchange)(void *user, const void *send_lo, void *recv_lo, const void *send_hi, void *recv_hi,
                    size_t bytes, void *stream);
    int (*allreduce)(void *user, double *buf, int n, int op, void *stream);
} falm_transport;
enum { FALM_REDUCE_SUM = 0, FALM_REDUCE_MAX = 1 };

/* Make ctx one slab of a grid decomposed along z: the context was created with the slab's grid
   (its nz_local interior planes plus the guide planes, with the global grid's z and hz values
   there: across a slab interface the guide planes are the neighbour's interior planes).
   z_offset: global interior index of the slab's first plane; nz_global: interior planes of the
   whole grid; rank 0 holds the lowest slab.  Call right after falm_create, before
   falm_bc_set_inflow (whose box then covers the whole grid's inlet) and falm_eq_poisson_operator
   (a collective: every rank calls it; the operator keeps its coefficients across interfaces and
   maxdiag is the maximum over the slabs).  falm_step and falm_eq_solve then exchange the halos
   they need and reduce every inner product, norm and AP force over the slabs (BiCGStab solver;
   preconditioner half sweeps one at a time, each after an exchange of the iterate's halo);
   boundary conditions apply on physical faces only.  Every rank makes the same calls in the same
   order.  The other entry points act on the slab alone: exchange halos before them with
   falm_slab_halo.  The discrete adjoint and the plain Jacobi/SOR solvers are single-slab only. */
int falm_slab_init(falm_ctx *ctx, int rank, int nranks, int z_offset, int nz_global, const falm_transport *t);
/* exchange `depth` (1 or 2) guide planes of a field of ncomp components with the neighbours (CPM
   IExchange6Face + PostExchange6Face, src/CPMComm.h:182-325, for the z faces) */
int falm_slab_halo(falm_ctx *ctx, void *field, int ncomp, int depth, void *stream);

/* In-process transport: the ranks are contexts of one process, each driven by its own host
   thread (on one GPU or several).  Every exchange and reduction is a host rendezvous of the
   threads (limited to 120 s, then FALM_ERR_TIMEOUT on every rank) followed by device copies
   ordered by CUDA events; no kernel waits on another.  Reductions sum in rank order, so every
   rank gets bitwise the same values; at most 64 doubles per reduction. */
int falm_local_hub_create(int nranks, void **hub);
int falm_local_hub_transport(void *hub, int rank, falm_transport *out);
int falm_local_hub_destroy(void *hub);

/* NCCL transport (one process per GPU): libnccl.so.2 is loaded at run time (the copy already in
   the process, else the system's).  Rank 0 calls falm_nccl_unique_id and hands the 128 bytes to
   every rank (e.g. through torch.distributed); each rank then creates its communicator on its
   current device.  exchange = grouped ncclSend/ncclRecv, allreduce = ncclAllReduce (FP64). */
int falm_nccl_unique_id(unsigned char id[128]);
int falm_nccl_transport_create(const unsigned char id[128], int rank, int nranks, falm_transport *out);
int falm_nccl_transport_destroy(falm_transport *t);

/* ---------------- instrumentation ----------------------------------------------------------- */
/* Test hook for the bounded device waits (the reference only prints errors, src/error.h:20-26):
   the next falm_step on this context first runs one wait on a barrier that no copy completes,
   through the same bounded wait the plane-stream kernels use, limited to `cycles` clock64 cycles
   (1 .. 2e9).  That step then returns FALM_ERR_TIMEOUT after the rest of it has run; the device
   error word is cleared and the context stays usable.  One step only. */
int falm_debug_arm_wait_probe(falm_ctx *ctx, long long cycles);
/* Kernel classes timed with CUDA events when profiling is on (one event pair per launch). */
enum { FALM_K_ALM = 0, FALM_K_PSEUDO_U, FALM_K_UTOUU_RHS, FALM_K_RES, FALM_K_BICG_P, FALM_K_SOR, FALM_K_MV_DOT1,
       FALM_K_BICG_S, FALM_K_MV_DOT2, FALM_K_BICG_XR, FALM_K_PBC, FALM_K_PROJECT, FALM_K_UBC, FALM_K_SGS_DIV,
       FALM_K_OTHER, FALM_K_COUNT };
int falm_profile_enable(falm_ctx *ctx, int enable);
/* milliseconds and launch counts per class since the last reset (synchronises the device) */
int falm_profile_read(falm_ctx *ctx, double *ms, long long *launches, int nclass, int reset);

#ifdef __cplusplus
}
#endif
#endif
