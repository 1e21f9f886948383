/*
 * FALM LES step -- CPU oracle (test infrastructure only).
 *
 * A plain FP64 C++/OpenMP restatement of the reference (ki2098/falm) algorithm
 * for the LES time step.  It exists to check the CUDA product path and to be
 * timed as the CPU baseline; it is never linked into the product library.
 * Every function cites the reference file:line it restates.
 *
 * Parity: pinned against (1) the analytic known-answer material in the
 * reference's own test directory (test/dot.py, test/heat1d2.cpp,
 * test/coloridx.py) and (2) the reference's own CUDA step built from its
 * sources (oracle/Makefile -> oracle/_ref) and run on the same inputs.
 *
 * Layout (as the reference, src/matrix.h:20, src/util.h:74-76): every field is
 * column-major SoA over the ghost-padded box, value(idx, col) = ptr[idx + col*N],
 * idx = i + j*sx + k*sx*sy, N = sx*sy*sz.
 */
#ifndef FALM_ORACLE_H
#define FALM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* boundary-condition sets of the reference's application drivers */
enum { OR_BC_CHANNEL = 0,   /* app/nedo + app/windtunnel: inlet, convective outlet, slip y+-, no-slip z-, slip z+ */
       OR_BC_CAVITY  = 1 }; /* app/lid3d: walls, lid on y+ moving with u=(1,0,0)                                 */

/* advection schemes, src/FalmCFDDevCall.h (AdvectionSchemeType) */
enum { OR_ADV_UPWIND1 = 0, OR_ADV_UPWIND3 = 1, OR_ADV_QUICK = 2, OR_ADV_UTOPIA = 3, OR_ADV_KK = 4 };
enum { OR_SGS_EMPTY = 0, OR_SGS_SMAGORINSKY = 1, OR_SGS_CSM = 2 };
enum { OR_PC_NONE = 0, OR_PC_JACOBI = 1, OR_PC_SOR = 2 };

typedef struct {
    int n_turbine, n_blade, n_ap_per_blade, n_attack;
    double radius, hub_radius, euler_eps;
    const double *base;       /* 3*n_turbine, turbine base position                         */
    const double *hub;        /* 3*n_turbine, rotor centre in the turbine frame             */
    const double *tip_rate;   /* n_turbine                                                   */
    const double *motion;     /* 3*n_turbine: amplitude [rad], angular frequency, phase      */
    const int    *angle_type; /* n_turbine: 0 none, 1 roll, 2 pitch, 3 yaw                   */
    const double *ap_r, *ap_chord, *ap_twist;   /* apcount                                  */
    const double *attack;     /* n_attack [deg]                                              */
    const double *cl, *cd;    /* apcount*n_attack, element (ap, atk) at ap + atk*apcount     */
    double pitch;             /* collective pitch offset [deg] added to every twist (0 = reference) */
} or_alm;

typedef struct {
    int sx, sy, sz, gc;                       /* ghost-padded shape and guide-cell count */
    const double *x, *hx, *y, *hy, *z, *hz;   /* 1D cell centres / widths, length sx, sy, sz */
    double Re, Cs, dt;
    int adv, sgs;
    int ls_maxit; double ls_tol; int pc_type; int pc_maxit; double pc_relax;
    int bc;
    double u_inlet;
    /* optional seeded inflow: periodic box of perturbations (3 x nb x sy_int x sz_int),
       sampled at x = u_inlet * t with linear interpolation; NULL = uniform inflow */
    const double *inflow_box; int inflow_nb; double inflow_dx;
    int alm_on;
    or_alm alm;
} or_case;

/* RMCP rotor model (src/rmcp/turbineHandler.h:13-185, bladeHandler.h:11-134): turbines with
   a fixed orientation whose rotating blades paint the cells they cover */
typedef struct {
    int n_turbine, n_blade;
    double radius, hub_radius;
    double width, thick;      /* blade strip width and axial thickness (almDevCall.cu:6-7: 0.1) */
    const double *base;       /* 3*n_turbine                                                 */
    const double *hub;        /* 3*n_turbine: (-overhang, 0, tower)                          */
    const double *angle;      /* 3*n_turbine [rad], one non-zero entry at most               */
    const int    *angle_type; /* n_turbine: 0 none, 1 roll, 2 pitch, 3 yaw                   */
    const double *tip_rate;   /* n_turbine                                                   */
    int n_station, n_attack;
    const double *st_r, *st_chord, *st_twist;   /* n_station                                 */
    const double *attack;                        /* n_attack [deg]                            */
    const double *cl, *cd;    /* n_station*n_attack, element (station, atk) at station*n_attack + atk */
} or_rmcp;

typedef struct {
    int it; double err; double divnorm;   /* BiCGStab iterations, residual, sqrt(sum div^2)/N */
    double torque[8], thrust[8];          /* per turbine                                        */
} or_stats;

/* ---- metrics and assembly ------------------------------------------------ */
void oracle_metrics(const or_case *c, double *kx, double *g, double *ja);
double oracle_poisson_matrix(const or_case *c, const double *g, const double *ja, double *A);
/* ---- FalmCFD -------------------------------------------------------------- */
void oracle_pseudo_u(const or_case *c, const double *un, const double *u, const double *uu,
                     double *ua, const double *nut, const double *kx, const double *g,
                     const double *ja, const double *ff);
void oracle_utouu(const or_case *c, const double *u, double *uu, const double *kx, const double *ja);
void oracle_divergence(const or_case *c, const double *uu, double *div, const double *ja);
void oracle_poisson_rhs(const or_case *c, const double *uu, double *rhs, const double *ja, double maxdiag);
void oracle_project_p(const or_case *c, double *u, const double *ua, double *uu, const double *uua,
                      const double *p, const double *kx, const double *g);
void oracle_sgs(const or_case *c, const double *u, double *nut, const double *kx, const double *ja);
/* ---- FalmMV / FalmEq --------------------------------------------------------- */
void   oracle_mv(const or_case *c, const double *A, const double *x, double *ax);
double oracle_dot(const or_case *c, const double *a, const double *b);
double oracle_normsq(const or_case *c, const double *a, int ncol);
void   oracle_res(const or_case *c, const double *A, const double *x, const double *b, double *r);
void   oracle_sor_sweep(const or_case *c, const double *A, double *x, const double *b, double omega, int color);
void   oracle_pbicgstab(const or_case *c, const double *A, double *x, const double *b, double *r,
                        int *it_out, double *err_out);
/* plain Jacobi (ls_type 1) or red-black SOR (ls_type 2, relaxation `relax`) solver with
   c->ls_maxit and c->ls_tol */
void   oracle_plain_solve(const or_case *c, int ls_type, double relax, const double *A, double *x,
                          const double *b, double *r, int *it_out, double *err_out);
/* ---- boundary conditions (application drivers) ---------------------------------- */
void oracle_ubc(const or_case *c, double *u, const double *uprev, double t);
void oracle_pbc(const or_case *c, double *p);
void oracle_uubc(const or_case *c, double *uu);
/* ---- actuator line model -------------------------------------------------------- */
void oracle_build_aps(int n_station, const double *st_r, const double *st_chord, const double *st_twist,
                      const double *st_cl, const double *st_cd, int n_attack,
                      int apcount, int n_ap_per_blade, double radius, double hub_radius,
                      double *ap_r, double *ap_chord, double *ap_twist, double *ap_cl, double *ap_cd);
void oracle_alm(const or_case *c, const double *u, double *ff, double t,
                double *ap_xyz, double *ap_force, double *ap_torque, double *ap_thrust,
                double *turb_torque, double *turb_thrust);
/* ---- one full step (app/nedo/main.cpp:150-204 order, race-free pseudo-velocity) ----- */
/* RMCP forcing at time t: flag (0, or turbine + 1) and force ff of every interior cell from
   the cell-centre velocity u; torque[t] = sum of r x |tangential force| over the turbine's
   cells (the formula of the reference's CalcTorque for its other turbine description,
   almDevCall.cu:368-411), thrust[t] = sum of the axial force magnitudes (no counterpart) */
void oracle_rmcp(const or_case *c, const or_rmcp *r, const double *u, double *ff, int *flag, double t,
                 double *torque, double *thrust);
void oracle_step(const or_case *c, double *u, double *uu, double *p, double *nut, double *ff,
                 const double *kx, const double *g, const double *ja, const double *A, double maxdiag,
                 double t, or_stats *st);
int oracle_num_threads(void);

/* Discrete adjoint of oracle_step (no reference counterpart; FP64, exact
 * Poisson solve).  u0, uu0, nut0, p0: state at the start of the step; t: the
 * step's time; wP: weight of this step's rotor power sum_t tip_t torque_t in
 * the objective.  au, auu, anut: adjoint of the state after the step on
 * entry, of the state before it on return.  The gradients of the objective
 * with respect to the collective pitch [deg] and the per-AP chord and twist
 * [deg] are added into g_pitch, g_chord, g_twist.  AT: oracle_transpose_matrix(A).
 * Returns 1 for an unsupported scheme or SGS model. */
void oracle_transpose_matrix(const or_case *c, const double *A, double *AT);
int oracle_step_adjoint(const or_case *c, const double *u0, const double *uu0, const double *nut0, const double *p0,
                        const double *kx, const double *g, const double *ja, const double *A, const double *AT,
                        double maxdiag, double t, double wP, double *au, double *auu, double *anut,
                        double *g_pitch, double *g_chord, double *g_twist);

#ifdef __cplusplus
}
#endif
#endif
