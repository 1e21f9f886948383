// Internal declarations of the falm_b200 library (sm_100a).
//
// Data layout in HBM: the reference's column-major SoA over the ghost-padded
// box (value(idx, col) = ptr[idx + col*N], idx = i + j*sx + k*sx*sy).  Metrics
// are never stored as 3D planes: every kernel rebuilds ja = hx*hy*hz, kx = 1/h
// and g = ja*kx*kx from 1D tables (a few KB, L1-resident), which removes the
// seven metric planes the reference streams through every stencil.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "falm_b200.h"

namespace fb {

constexpr int kMaxTurbines = 8;
constexpr int kMaxFusedAp = 384;         // actuator points staged in shared memory
constexpr int kRowThreads = 256;          // threads per block of the row kernels
constexpr int kWarpsPerBlock = kRowThreads / 32;

// 1D metric tables of one precision (device pointers into one allocation)
template <typename T>
struct Metric {
    const T *x[3];    // cell centres
    const T *h[3];    // widths
    const T *k[3];    // 1/h  (kx, src/falm.h:395)
};

// Poisson operator as separable 1D tables (see poisson.cu for the derivation)
template <typename T>
struct PoissonTables {
    const T *cm[3];   // scaled coefficient towards the minus neighbour  (w, s, b)
    const T *cp[3];   // scaled coefficient towards the plus neighbour   (e, n, t)
    const T *um[3];   // unscaled minus coefficients (for the diagonal)
    const T *up[3];   // unscaled plus coefficients
    const T *dx0;     // (-e) - w, unscaled, per i: first two terms of the diagonal
    T scale;          // 1/maxdiag
    int koff;         // the grid's Geom::koff: red-black colour (i + j + k + koff) & 1
};

struct Geom {
    int sx, sy, sz, gc;
    long long n;      // sx*sy*sz
    int nx, ny, nz;   // interior sizes
    // z slab of a decomposed grid (falm_slab_init); one slab covers the grid otherwise
    int koff;         // global index of local plane 0 minus 0: the red-black colour is (i + j + k + koff) & 1
    int zphys;        // physical z faces: bit 0 the lower (k = gc - 1), bit 1 the upper; the others are slab interfaces
    int nzg;          // interior planes of the whole grid
    __host__ __device__ inline long long id(int i, int j, int k) const {
        return (long long)i + (long long)j * sx + (long long)k * sx * sy;
    }
};

// device-side solver scalars (one per context)
struct SolverScalars {
    double rho, rrho, alpha, beta, omega;
    double err, gsize, tol;
    double red[4];      // scratch reduction results
    int it, maxit, done, status;
    int first;          // 1 before the first BiCGStab iteration of a solve
    int kerr;           // bounded device-side wait gave up (FALM_ERR_TIMEOUT)
    int checked;        // the queued outer check of the true residual ran (mixed precision)
    int defer;          // slab mode: reduction kernels leave their local totals in red[] for a reduction
                        // over the slabs, and k_slab_derive derives the scalars from the reduced totals
    int it_total;       // a recorded step (CUDA graph): iterations of all passes
    int passes;         // a recorded step: passes run
};

struct AlmScalars {
    double torque[kMaxTurbines], thrust[kMaxTurbines];
    double bbox[6];     // xmin,xmax,ymin,ymax,zmin,zmax of the AP cloud (+cutoff)
};

// reduction workspace: per-block partials + arrival counter + results
struct RedWork {
    double *partials;     // capacity maxBlocks * 4
    unsigned int *counter;
    int maxBlocks;
};

// Force boxes of the fused ALM projection.  Box t is the index box of the
// interior cells within |hub_t| + max AP radius + cutoff (+1 cell) of turbine
// t's base, so it holds every cell that an AP of turbine t can reach.  The
// projected force of a box cell (the sum over ALL actuator points) is stored
// there once per ALM evaluation: 3 components with stride `total`.
struct BoxSet {
    int n;
    int lo[kMaxTurbines][3], ext[kMaxTurbines][3];
    long long off[kMaxTurbines];
    long long total;
};

struct AlmDev {
    BoxSet bs;
    void *fbox;            // 3 * bs.total values of the context precision
    int n_turbine, n_blade, n_ap_per_blade, n_attack, apcount;
    double radius, hub_radius, euler_eps, pitch, rcut2;
    const double *base, *hub, *tip_rate, *motion;
    const int *angle_type;
    const double *ap_r, *ap_chord, *ap_twist, *attack, *cl, *cd;
    double *ap_xyz, *ap_force, *ap_torque, *ap_thrust;
    AlmScalars *scal;
};

struct IoWriter;
struct RmcpDev;
}  // namespace fb

// host-side context
struct falm_ctx {
    int precision;
    fb::Geom geo;
    int device;
    // metrics
    void *metric_mem;                       // one allocation holding both precisions
    fb::Metric<double> m64;
    fb::Metric<float> m32;
    std::vector<double> *hx, *hy, *hz, *xc, *yc, *zc;  // host copies
    // CFD parameters
    double Re, Cs;
    int adv, sgs;
    // solver parameters
    int ls_type, maxit, pc_type, pc_maxit;
    double tol, relax, pc_relax;
    int max_outer;
    // Poisson operator
    int op_ready;
    int op_symmetric;                       // the table operator equals its transpose over the interior
    int bc_kind_op;
    double maxdiag;
    void *op_mem;
    fb::PoissonTables<double> pt64;
    fb::PoissonTables<float> pt32;
    const void *A_explicit;                 // caller-owned 7-column matrix or NULL
    // BC
    int bc_kind;
    double u_inlet;
    double *inflow_box;                     // device FP64
    int inflow_nb;
    double inflow_dx;
    // work vectors (element size = precision), allocated lazily
    size_t esize;
    void *work_mem;
    void *adj_mem;                          // discrete-adjoint workspace (allocated on first use)
    double adj_rel_tol;                     // relative residual of the adjoint's transposed Poisson solve (0: default)
    void *w_rr, *w_p, *w_q, *w_s, *w_pp, *w_ss, *w_t, *w_r, *w_rhs, *w_ua, *w_div, *w_xp;
    void *w_outlet;                         // 3 planes x 3 comps of the previous velocity at the outlet
    // reductions
    fb::RedWork red;
    fb::SolverScalars *scal;                // device
    fb::SolverScalars *scal_host;           // pinned
    // ALM
    int alm_on;
    void *alm_mem;
    fb::AlmDev alm;
    std::vector<double> *alm_host;          // host copy of tables
    fb::AlmScalars *alm_scal_host;          // pinned
    // bookkeeping
    long long launches;
    // per-class event timing (falm_profile_enable)
    int profiling;
    struct EvRec { int cls; cudaEvent_t a, b; };
    std::vector<EvRec> *ev_pending;
    std::vector<cudaEvent_t> *ev_pool;
    double prof_ms[FALM_K_COUNT];
    long long prof_n[FALM_K_COUNT];
    // streamed inlet plane
    double *inlet_plane;                    // device 3 x nz x ny
    int inlet_plane_valid;                  // the next velocity BC takes the streamed plane
    const double *inlet_host;               // its host array, copied by that BC (or by the recorded step's copy node)
    int inlet_pending;                      // inlet_host not yet copied
    int sm_count;
    int *kerr;                              // device error word of bounded waits (FALM_ERR_TIMEOUT)
    int no_tma;                             // force the row kernels (tests, fallback)
    int sor_v1;                             // blocked SOR kernel: 0 by size, 1 the 32 x 8 tile, 2 the 28 x 16 skewed one (tests)
    int pu_v1;                              // FP32 pseudo-velocity on the one-cell-per-thread kernel (tests)
    int check_sync;                         // synchronise after every launch (fault location)
    long long wait_probe_cycles;            // >0: the next falm_step first runs a wait that nothing completes (tests)
    // RMCP rotor model (falm_rmcp_init): the step's forcing instead of the ALM
    int rmcp_on;
    void *rmcp_mem;
    fb::RmcpDev *rmcp;                      // host copy of the device tables' descriptor
    void *w_ff;                             // 3N force field of the RMCP step (zero outside the boxes)
    double *rmcp_sums;                      // device: torque, thrust per turbine (2 x kMaxTurbines)
    double *rmcp_sums_host;                 // pinned
    // z slab of a decomposed grid (falm_slab_init)
    int slab_on, slab_rank, slab_nranks;
    falm_transport transport;               // halo exchange and reductions between the slabs
    std::string *last_error;
    fb::IoWriter *io;                       // snapshot writer (falm_io.cuh), created on first use
    // device-side BiCGStab loops (CUDA graphs), one per solve signature
    struct SolveGraph {
        const void *x, *b, *r, *w0, *A;
        int esize, pp_ready, prefix, per_iter;
        cudaGraph_t graph;
        cudaGraphExec_t exec;
    };
    std::vector<SolveGraph> *graphs;
    // whole steps recorded as CUDA graphs (small grids), one per set of fields and dt
    struct StepGraph {
        const void *u, *uu, *p, *nut, *ff;
        double dt;
        int inlet;                      // recorded with a streamed inlet plane
        cudaGraphNode_t inlet_node;     // its host-to-device copy (a root node; the source set per launch)
        long long fixed, per_iter;      // kernels outside the loops, kernels per iteration
        cudaGraph_t graph;
        cudaGraphExec_t exec;
    };
    std::vector<StepGraph> *step_graphs;
    double *t_dev;                          // the recorded step's time (device), from t_host
    double *t_host;                         // pinned
    int graph_mode;                         // 1 record steps and solver loops as CUDA graphs, 0 never (FALM_B200_GRAPH=0)
    cudaStream_t cap_stream;                // stream the graphs are captured on
    cudaStream_t side_stream;               // a recorded step's side branch (guide-shell copy, outlet save)
    cudaEvent_t side_fork, side_join;       // its fork from and join to the capture stream
};
