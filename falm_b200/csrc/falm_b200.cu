// falm_b200: host side of the C ABI (include/falm_b200.h).
//
// One context per GPU and grid.  The context owns the 1D metric tables, the
// Poisson operator tables, the solver work vectors (FalmEq::alloc,
// src/FalmEq.h:27-40), the device-side reduction workspace and the ALM
// tables; the caller owns the fields.  Every call is asynchronous on the given
// stream except those that return scalars on the host.
#include <vector>
#include <fstream>
#include <string>
#include <cstring>
#include <cstddef>
#include <cstdio>
#include <cmath>
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <map>
#include <climits>
#include <tuple>
#include <functional>
#include <condition_variable>
#include <chrono>
#include <dlfcn.h>
#include <nccl.h>
#include <nvtx3/nvToolsExt.h>
#include "falm_internal.cuh"
#include "common.cuh"
#include "cfd.cuh"
#include "poisson.cuh"
#include "alm_bc.cuh"
#include "stencil_tma.cuh"
#include "poisson_tma.cuh"
#include "plane3_tma.cuh"
#include "falm_io.cuh"
#include "sor_rb_tma.cuh"
#include "adjoint.cuh"
#include "rmcp.cuh"
#include <cudaTypedefs.h>

using namespace fb;

namespace {

inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

#include "launch.cuh"

#include "operator.cuh"

#include "solve.cuh"

#include "step.cuh"

#include "slab.cuh"

// run f with a value of the context's storage type (double or float)
template <typename F>
int dispatch(const falm_ctx *ctx, F &&f) {
    if (ctx->precision == FALM_FP64) return f(double(0));
    return f(float(0));
}

}  // namespace

extern "C" {

int falm_abi_version(void) { return FALM_B200_ABI_VERSION; }

const char *falm_last_error(const falm_ctx *ctx) { return ctx && ctx->last_error ? ctx->last_error->c_str() : "null context"; }

long long falm_kernel_launches(const falm_ctx *ctx) { return ctx ? ctx->launches : 0; }

int falm_create(const falm_grid *grid, int precision, falm_ctx **out) {
    if (!grid || !out || !grid->x || !grid->y || !grid->z || !grid->hx || !grid->hy || !grid->hz) return FALM_ERR_ARG;
    if (grid->gc < 2 || grid->sx < 2 * grid->gc + 1 || grid->sy < 2 * grid->gc + 1 || grid->sz < 2 * grid->gc + 1) return FALM_ERR_ARG;
    if (precision != FALM_FP64 && precision != FALM_MIXED) return FALM_ERR_ARG;
    *out = nullptr;
    falm_ctx *ctx = new falm_ctx();
    memset((void *)ctx, 0, sizeof(*ctx));
    ctx->last_error = new std::string();
    ctx->graphs = new std::vector<falm_ctx::SolveGraph>();
    ctx->step_graphs = new std::vector<falm_ctx::StepGraph>();
    {
        const char *gm = getenv("FALM_B200_GRAPH");
        ctx->graph_mode = (gm && gm[0] == '0') ? 0 : 1;
    }
    ctx->precision = precision;
    ctx->esize = precision == FALM_FP64 ? sizeof(double) : sizeof(float);
    Geom &g = ctx->geo;
    g.sx = grid->sx; g.sy = grid->sy; g.sz = grid->sz; g.gc = grid->gc;
    g.n = (long long)g.sx * g.sy * g.sz;
    g.nx = g.sx - 2 * g.gc; g.ny = g.sy - 2 * g.gc; g.nz = g.sz - 2 * g.gc;
    g.koff = 0; g.zphys = 3; g.nzg = g.nz;
    ctx->hx = new std::vector<double>(grid->hx, grid->hx + g.sx);
    ctx->hy = new std::vector<double>(grid->hy, grid->hy + g.sy);
    ctx->hz = new std::vector<double>(grid->hz, grid->hz + g.sz);
    ctx->xc = new std::vector<double>(grid->x, grid->x + g.sx);
    ctx->yc = new std::vector<double>(grid->y, grid->y + g.sy);
    ctx->zc = new std::vector<double>(grid->z, grid->z + g.sz);
    ctx->alm_host = new std::vector<double>();
    ctx->ev_pending = new std::vector<falm_ctx::EvRec>();
    ctx->ev_pool = new std::vector<cudaEvent_t>();
    ctx->Re = 1e4; ctx->Cs = 0.1; ctx->adv = FALM_ADV_UPWIND3; ctx->sgs = FALM_SGS_SMAGORINSKY;
    ctx->ls_type = FALM_LS_PBICGSTAB; ctx->maxit = 1000; ctx->tol = 1e-8; ctx->relax = 1.0;
    ctx->pc_type = FALM_LS_SOR; ctx->pc_maxit = 2; ctx->pc_relax = 1.2; ctx->max_outer = 5;
    ctx->bc_kind = FALM_BC_CHANNEL; ctx->u_inlet = 1.0;
    if (cudaGetDevice(&ctx->device) != cudaSuccess) { cudaGetLastError(); falm_destroy(ctx); return FALM_ERR_CUDA; }
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    if (ctx->sm_count <= 0) ctx->sm_count = 148;
    // metric tables: x, h, k for 3 axes in FP64 then FP32
    size_t tot = 3 * ((size_t)g.sx + g.sy + g.sz);
    std::vector<double> m(tot);
    std::vector<float> mf(tot);
    size_t off = 0, o_x[3], o_h[3], o_k[3];
    const std::vector<double> *xs[3] = {ctx->xc, ctx->yc, ctx->zc}, *hs[3] = {ctx->hx, ctx->hy, ctx->hz};
    const int s[3] = {g.sx, g.sy, g.sz};
    for (int d = 0; d < 3; d++) {
        o_x[d] = off; for (int q = 0; q < s[d]; q++) m[off + q] = (*xs[d])[q]; off += s[d];
        o_h[d] = off; for (int q = 0; q < s[d]; q++) m[off + q] = (*hs[d])[q]; off += s[d];
        o_k[d] = off; for (int q = 0; q < s[d]; q++) m[off + q] = 1.0 / (*hs[d])[q]; off += s[d];
    }
    for (size_t q = 0; q < tot; q++) mf[q] = (float)m[q];
    if (cudaMalloc(&ctx->metric_mem, tot * (sizeof(double) + sizeof(float))) != cudaSuccess) { cudaGetLastError(); falm_destroy(ctx); return FALM_ERR_ALLOC; }
    double *d64 = (double *)ctx->metric_mem;
    float *d32 = (float *)(d64 + tot);
    cudaMemcpy(d64, m.data(), tot * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d32, mf.data(), tot * sizeof(float), cudaMemcpyHostToDevice);
    for (int d = 0; d < 3; d++) {
        ctx->m64.x[d] = d64 + o_x[d]; ctx->m64.h[d] = d64 + o_h[d]; ctx->m64.k[d] = d64 + o_k[d];
        ctx->m32.x[d] = d32 + o_x[d]; ctx->m32.h[d] = d32 + o_h[d]; ctx->m32.k[d] = d32 + o_k[d];
    }
    // reduction workspace sized to the persistent grid
    ctx->red.maxBlocks = 1 << 16;   // partial sums of up to 65536 blocks per reduction
    if (cudaMalloc(&ctx->red.partials, sizeof(double) * 4 * ctx->red.maxBlocks) != cudaSuccess ||
        cudaMalloc(&ctx->red.counter, sizeof(unsigned int) * 4) != cudaSuccess ||
        cudaMalloc(&ctx->scal, sizeof(SolverScalars)) != cudaSuccess ||
        cudaMallocHost(&ctx->scal_host, sizeof(SolverScalars)) != cudaSuccess ||
        cudaMallocHost(&ctx->alm_scal_host, sizeof(AlmScalars)) != cudaSuccess) {
        cudaGetLastError();
        falm_destroy(ctx);
        return FALM_ERR_ALLOC;
    }
    cudaMemset(ctx->red.counter, 0, sizeof(unsigned int) * 4);
    ctx->kerr = (int *)(ctx->red.counter + 2);
    {
        const char *e = getenv("FALM_B200_NO_TMA");
        ctx->no_tma = (e && e[0] == '1') ? 1 : 0;
        const char *v = getenv("FALM_B200_SOR_V1");
        ctx->sor_v1 = (v && v[0] == '1') ? 1 : ((v && v[0] == '2') ? 2 : 0);
        const char *pv = getenv("FALM_B200_PU_V1");
        ctx->pu_v1 = (pv && pv[0] == '1') ? 1 : 0;
        const char *c = getenv("FALM_B200_CHECK");
        ctx->check_sync = (c && c[0] == '1') ? 1 : 0;
    }
    cudaMemset(ctx->scal, 0, sizeof(SolverScalars));
    memset(ctx->scal_host, 0, sizeof(SolverScalars));
    if (cudaDeviceSynchronize() != cudaSuccess) { cudaGetLastError(); falm_destroy(ctx); return FALM_ERR_CUDA; }
    *out = ctx;
    return FALM_OK;
}

int falm_destroy(falm_ctx *ctx) {
    if (!ctx) return FALM_ERR_ARG;
    delete ctx->io;   // writes the queued snapshots, then stops its thread
    graphs_clear(ctx);
    delete ctx->graphs;
    delete ctx->step_graphs;
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    if (ctx->side_fork) cudaEventDestroy(ctx->side_fork);
    if (ctx->side_join) cudaEventDestroy(ctx->side_join);
    cudaFree(ctx->t_dev);
    if (ctx->t_host) cudaFreeHost(ctx->t_host);
    cudaFree(ctx->metric_mem);
    cudaFree(ctx->op_mem);
    cudaFree(ctx->work_mem);
    cudaFree(ctx->adj_mem);
    cudaFree(ctx->rmcp_mem);
    cudaFree(ctx->w_ff);
    if (ctx->rmcp_sums_host) cudaFreeHost(ctx->rmcp_sums_host);
    delete ctx->rmcp;
    cudaFree(ctx->red.partials);
    cudaFree(ctx->red.counter);
    cudaFree(ctx->scal);
    cudaFree(ctx->inflow_box);
    cudaFree(ctx->alm_mem);
    cudaFree(ctx->alm.fbox);
    if (ctx->scal_host) cudaFreeHost(ctx->scal_host);
    if (ctx->alm_scal_host) cudaFreeHost(ctx->alm_scal_host);
    delete ctx->hx; delete ctx->hy; delete ctx->hz; delete ctx->xc; delete ctx->yc; delete ctx->zc;
    delete ctx->alm_host;
    if (ctx->ev_pending) {
        for (auto &r : *ctx->ev_pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        delete ctx->ev_pending;
    }
    if (ctx->ev_pool) {
        for (auto e : *ctx->ev_pool) cudaEventDestroy(e);
        delete ctx->ev_pool;
    }
    cudaFree(ctx->inlet_plane);
    delete ctx->last_error;
    delete ctx;
    return FALM_OK;
}

// ---------------------------------------------------------------- FalmCFD
int falm_cfd_init(falm_ctx *ctx, double Re, int adv, int sgs, double Cs) {
    if (ctx) graphs_clear(ctx);   // recorded steps take these settings as kernel arguments
    if (!ctx || !(Re > 0) || adv < 0 || adv > 4 || sgs < 0 || sgs > 2) return FALM_ERR_ARG;
    ctx->Re = Re; ctx->adv = adv; ctx->sgs = sgs; ctx->Cs = Cs;
    return FALM_OK;
}

int falm_cfd_pseudo_u(falm_ctx *ctx, const void *un, const void *u, const void *uu, void *ua, const void *nut,
                      const void *ff, double dt, double t, void *stream) {
    (void)t;
    if (!ctx || !un || !u || !uu || !ua || !nut) return FALM_ERR_ARG;
    if (ua == u || ua == un) return fail(ctx, FALM_ERR_ARG, "pseudo_u: ua aliases u (a data race in the reference's aliased call)");
    if (!ff && !ctx->alm_on) return fail(ctx, FALM_ERR_NOALM, "pseudo_u: ff is NULL and no ALM is configured");
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        return pseudo_u_t<T>(ctx, (const T *)un, (const T *)u, (const T *)uu, (T *)ua, (const T *)nut, (const T *)ff, dt, true, S(stream));
    });
}

int falm_cfd_utouu(falm_ctx *ctx, const void *u, void *uu, void *stream) {
    if (!ctx || !u || !uu) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = facemap(ctx->geo);
        P3_OR(FALM_K_UTOUU_RHS, S(stream), T, 1, 0, R, 1, FB_ARR(u), FB_ARR(3),
              (UtoUUBody<T, false, false>{ctx->geo, mview<T>(ctx), (T *)uu, (T *)nullptr, T(0)}),
              (k_utouu<T, false, false><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, mview<T>(ctx), (const T *)u,
                                                                                      (const T *)u, (T *)uu, (T *)nullptr, T(0))));
        return (int)FALM_OK;
    });
}

int falm_cfd_poisson_rhs(falm_ctx *ctx, const void *uu, void *rhs, double dt, double maxdiag, void *stream) {
    if (!ctx || !uu || !rhs || !(dt > 0) || !(maxdiag > 0)) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = interior(ctx->geo);
        LAUNCH(FALM_K_OTHER, S(stream), k_divergence<T><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, mview<T>(ctx), (const T *)uu, (T *)rhs,
                                                                          (T)(1.0 / (dt * maxdiag)), 1));
        return (int)FALM_OK;
    });
}

int falm_cfd_divergence(falm_ctx *ctx, const void *uu, void *div, void *stream) {
    if (!ctx || !uu || !div) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = interior(ctx->geo);
        LAUNCH(FALM_K_OTHER, S(stream), k_divergence<T><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, mview<T>(ctx), (const T *)uu, (T *)div, T(1), 0));
        return (int)FALM_OK;
    });
}

int falm_cfd_project_p(falm_ctx *ctx, void *u, const void *ua, void *uu, const void *uua, const void *p, double dt, void *stream) {
    if (!ctx || !u || !ua || !uu || !uua || !p) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = facemap(ctx->geo);
        P3_OR(FALM_K_PROJECT, S(stream), T, 1, 0, R, 1, FB_ARR(p), FB_ARR(1),
              (ProjectBody<T>{ctx->geo, mview<T>(ctx), (T *)u, (const T *)ua, (T *)uu, (const T *)uua, (T)dt}),
              (k_project<T><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, mview<T>(ctx), (T *)u, (const T *)ua, (T *)uu,
                                                                          (const T *)uua, (const T *)p, (T)dt)));
        return (int)FALM_OK;
    });
}

int falm_cfd_sgs(falm_ctx *ctx, const void *u, void *nut, void *stream) {
    if (!ctx || !u || !nut) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = interior(ctx->geo);
        // the second field is only read for the divergence, which is off here
        P3_OR(FALM_K_SGS_DIV, S(stream), T, 2, 1, R, 2, FB_ARR(u, u), FB_ARR(3, 3),
              (SgsDivBody<T>{ctx->geo, mview<T>(ctx), ctx->m64, (T *)nut, (T)ctx->Cs, ctx->sgs, (T *)nullptr, (double *)nullptr}),
              (k_sgs_div<T, false><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, mview<T>(ctx), ctx->m64, (const T *)u, (T *)nut,
                                                                                 (T)ctx->Cs, ctx->sgs, (const T *)nullptr, (T *)nullptr, ctx->red, nullptr)));
        return (int)FALM_OK;
    });
}

// ---------------------------------------------------------------- FalmEq
int falm_eq_init(falm_ctx *ctx, int type, int maxit, double tol, double relax, int pc_type, int pc_maxit, double pc_relax) {
    if (!ctx || maxit < 1 || !(tol >= 0)) return FALM_ERR_ARG;
    if (type != FALM_LS_PBICGSTAB && type != FALM_LS_SOR && type != FALM_LS_JACOBI)
        return fail(ctx, FALM_ERR_ARG, "eq_init: solver must be Jacobi (1), SOR (2) or PBiCGStab (4)");
    const bool plain = type != FALM_LS_PBICGSTAB;
    if (plain && pc_type == FALM_LS_EMPTY) {
        // a plain solver has no preconditioner; the adjoint's transposed solve
        // (always PBiCGStab) then uses the drivers' SOR x2, omega 1.2
        pc_type = FALM_LS_SOR; pc_maxit = 2; pc_relax = 1.2;
    }
    if (pc_type != FALM_LS_SOR && pc_type != FALM_LS_JACOBI) return fail(ctx, FALM_ERR_ARG, "eq_init: preconditioner must be SOR (2) or Jacobi (1)");
    if (pc_maxit < 1) return FALM_ERR_ARG;
    ctx->ls_type = type; ctx->maxit = maxit; ctx->tol = tol; ctx->relax = relax;
    ctx->pc_type = pc_type; ctx->pc_maxit = pc_maxit; ctx->pc_relax = pc_relax;
    graphs_clear(ctx);   // the preconditioner settings are kernel arguments of the recorded loops
    return FALM_OK;
}

int falm_eq_poisson_operator(falm_ctx *ctx, int bc_kind, double *maxdiag_out) {
    if (!ctx || (bc_kind != FALM_BC_CHANNEL && bc_kind != FALM_BC_CAVITY)) return FALM_ERR_ARG;
    graphs_clear(ctx);
    int rc = build_poisson(ctx, bc_kind);
    if (rc) return rc;
    if (maxdiag_out) *maxdiag_out = ctx->maxdiag;
    return FALM_OK;
}

int falm_eq_set_matrix(falm_ctx *ctx, const void *A) {
    if (!ctx) return FALM_ERR_ARG;
    graphs_clear(ctx);
    ctx->A_explicit = A;
    return FALM_OK;
}

int falm_eq_solve(falm_ctx *ctx, void *x, const void *b, void *r, void *stream, int *it_out, double *err_out) {
    if (!ctx || !x || !b || !r) return FALM_ERR_ARG;
    int rc = dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        if (ctx->slab_on) return slab_solve_t<T>(ctx, (T *)x, (const T *)b, (T *)r, S(stream), it_out, err_out, nullptr);
        return solve_t<T>(ctx, (T *)x, (const T *)b, (T *)r, S(stream), it_out, err_out, nullptr);
    });
    if (rc) return rc;
    int st = ctx->scal_host->status;
    return st == FALM_ERR_MAXIT || st == FALM_ERR_BREAKDOWN ? st : FALM_OK;
}

int falm_eq_res(falm_ctx *ctx, const void *x, const void *b, void *r, void *stream) {
    if (!ctx || !x || !b || !r) return FALM_ERR_ARG;
    if (!ctx->op_ready && !ctx->A_explicit) return fail(ctx, FALM_ERR_STATE, "res: no operator");
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = interior(ctx->geo);
        S7_OR(FALM_K_RES, S(stream), T, 2, (const T *)x, (ResBody<T>{op7<T>(ctx), (const T *)b, (T *)r, (T *)nullptr, (SolverScalars *)nullptr, 0}),
              (k_res<T><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, op7<T>(ctx), (const T *)x, (const T *)b, (T *)r,
                                                                       (T *)nullptr, ctx->red, nullptr, 0)));
        return (int)FALM_OK;
    });
}

int falm_eq_sor_sweep(falm_ctx *ctx, void *x, const void *b, double omega, int color, void *stream) {
    if (!ctx || !x || !b || (color != 0 && color != 1)) return FALM_ERR_ARG;
    if (!ctx->op_ready && !ctx->A_explicit) return fail(ctx, FALM_ERR_STATE, "sor: no operator");
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = interior(ctx->geo);
        S7_OR(FALM_K_SOR, S(stream), T, 0, (const T *)x, (SorBody<T>{op7<T>(ctx), (T *)x, (const T *)b, (T)omega, color, (const SolverScalars *)nullptr}),
              (k_sor<T><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, op7<T>(ctx), (T *)x, (const T *)b, (T)omega, color,
                                                                       (const SolverScalars *)nullptr)));
        return (int)FALM_OK;
    });
}

// ---------------------------------------------------------------- FalmMV
int falm_mv_mv(falm_ctx *ctx, const void *x, void *ax, void *stream) {
    if (!ctx || !x || !ax) return FALM_ERR_ARG;
    if (!ctx->op_ready && !ctx->A_explicit) return fail(ctx, FALM_ERR_STATE, "mv: no operator");
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = interior(ctx->geo);
        S7_OR(FALM_K_OTHER, S(stream), T, 0, (const T *)x, (MvBody<T>{op7<T>(ctx), (T *)ax}),
              (k_mv<T><<<row_grid(ctx, R), kRowThreads, 0, S(stream)>>>(ctx->geo, R, op7<T>(ctx), (const T *)x, (T *)ax)));
        return (int)FALM_OK;
    });
}

int falm_mv_dot(falm_ctx *ctx, const void *a, const void *b, double *out, void *stream) {
    if (!ctx || !a || !b || !out) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        return dot_t<T>(ctx, (const T *)a, (const T *)b, 1, out, S(stream));
    });
}

int falm_mv_normsq(falm_ctx *ctx, const void *a, int ncol, double *out, void *stream) {
    if (!ctx || !a || !out || ncol < 1) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        return dot_t<T>(ctx, (const T *)a, (const T *)nullptr, ncol, out, S(stream));
    });
}

int falm_mv_maxdiag(falm_ctx *ctx, double *out) {
    if (!ctx || !out) return FALM_ERR_ARG;
    if (!ctx->A_explicit) {
        if (!ctx->op_ready) return fail(ctx, FALM_ERR_STATE, "maxdiag: no operator");
        *out = ctx->maxdiag;
        return FALM_OK;
    }
    unsigned long long *d = nullptr, h = 0;
    CK(cudaMalloc(&d, sizeof(unsigned long long)));
    CK(cudaMemset(d, 0, sizeof(unsigned long long)));
    int rc = dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        const Region3 R = interior(ctx->geo);
        LAUNCH(FALM_K_OTHER, (cudaStream_t)0, k_absmax<T><<<row_grid(ctx, R), kRowThreads>>>(ctx->geo, R, (const T *)ctx->A_explicit, d));
        return (int)FALM_OK;
    });
    if (rc) { cudaFree(d); return rc; }
    CK(cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost));
    cudaFree(d);
    double v;
    memcpy(&v, &h, sizeof(v));
    *out = v;
    return FALM_OK;
}

int falm_mv_scale(falm_ctx *ctx, void *a, long long n, double scale, void *stream) {
    if (!ctx || !a || n < 0) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        LAUNCH(FALM_K_OTHER, (cudaStream_t)0, k_scale<T><<<ctx->sm_count * 4, 256, 0, S(stream)>>>((T *)a, n, (T)scale));
        return (int)FALM_OK;
    });
}

int falm_mv_axby(falm_ctx *ctx, double a, const void *x, double b, const void *y, void *result, long long n, void *stream) {
    if (!ctx || !x || !y || !result || n < 0) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        LAUNCH(FALM_K_OTHER, S(stream), k_axby<T><<<ctx->sm_count * 4, 256, 0, S(stream)>>>((T)a, (const T *)x, (T)b, (const T *)y, (T *)result, n));
        return (int)FALM_OK;
    });
}

// ---------------------------------------------------------------- FalmIO + TAvg
int falm_tavg(falm_ctx *ctx, void *avg, const void *f, int ncol, long long count, void *stream) {
    if (!ctx || !avg || !f || ncol < 1 || count < 1) return FALM_ERR_ARG;
    const double b = 1.0 / (double)count, a = 1.0 - b;
    return falm_mv_axby(ctx, a, avg, b, f, avg, (long long)ncol * ctx->geo.n, stream);
}

int falm_io_write_vector_file(falm_ctx *ctx, const char *path, const void *const *fields, const int *ncols, int nfields,
                              unsigned long long step, double time, int as_fp64, void *stream) {
    if (!ctx || !path || !fields || !ncols || nfields < 1) return FALM_ERR_ARG;
    long long cols = 0;
    for (int q = 0; q < nfields; q++) {
        if (!fields[q] || ncols[q] < 1) return FALM_ERR_ARG;
        cols += ncols[q];
    }
    const Geom &g = ctx->geo;
    const size_t n = (size_t)g.n, es = ctx->esize;
    const bool cast = as_fp64 && es == sizeof(float);
    const size_t ds = cast ? sizeof(double) : es, bytes = (size_t)cols * n * ds;
    if (!ctx->io) {
        ctx->io = new IoWriter();
        ctx->io->device = ctx->device;
        IoWriter *w = ctx->io;
        ctx->io->worker = std::thread([w] { w->run(); });
    }
    IoWriter &w = *ctx->io;
    int bi = -1;
    {
        std::unique_lock<std::mutex> lk(w.m);
        w.cv.wait(lk, [&] { return !w.bufs[0].in_use || !w.bufs[1].in_use; });
        bi = w.bufs[0].in_use ? 1 : 0;
        w.bufs[bi].in_use = true;
    }
    IoBuf &b = w.bufs[bi];
    auto release = [&](int rc, const char *msg) {
        { std::lock_guard<std::mutex> lk(w.m); b.in_use = false; }
        w.cv.notify_all();
        return fail(ctx, rc, msg);
    };
    if (b.cap < bytes) {
        if (b.host) cudaFreeHost(b.host);
        b.host = nullptr; b.cap = 0;
        if (cudaHostAlloc(&b.host, bytes, cudaHostAllocDefault) != cudaSuccess) { cudaGetLastError(); return release(FALM_ERR_ALLOC, "io: pinned staging buffer"); }
        b.cap = bytes;
    }
    if (cast && b.dcap < bytes) {
        if (b.dev) cudaFree(b.dev);
        b.dev = nullptr; b.dcap = 0;
        if (cudaMalloc(&b.dev, bytes) != cudaSuccess) { cudaGetLastError(); return release(FALM_ERR_ALLOC, "io: device staging buffer"); }
        b.dcap = bytes;
    }
    if (!b.ready && cudaEventCreateWithFlags(&b.ready, cudaEventDisableTiming) != cudaSuccess) return release(FALM_ERR_CUDA, "io: event");
    // the columns, field after field: the reference's uvwp layout (u's 3, then p's 1)
    cudaStream_t st = S(stream);
    size_t off = 0;
    for (int q = 0; q < nfields; q++) {
        const size_t len = (size_t)ncols[q] * n;
        if (cast) {
            LAUNCH(FALM_K_OTHER, st, k_cast_f64<<<ctx->sm_count * 4, 256, 0, st>>>((const float *)fields[q], (double *)b.dev + off, (long long)len));
        } else if (cudaMemcpyAsync((char *)b.host + off * ds, fields[q], len * ds, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
            return release(FALM_ERR_CUDA, "io: snapshot copy");
        }
        off += len;
    }
    if (cast && cudaMemcpyAsync(b.host, b.dev, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess) return release(FALM_ERR_CUDA, "io: snapshot copy");
    if (cudaEventRecord(b.ready, st) != cudaSuccess) return release(FALM_ERR_CUDA, "io: event record");
    IoJob job;
    job.path = path;
    job.head[0] = (uint64_t)g.sx; job.head[1] = (uint64_t)g.sy; job.head[2] = (uint64_t)g.sz;
    job.head[3] = (uint64_t)cols; job.head[4] = (uint64_t)g.gc; job.head[5] = (uint64_t)step;
    job.time = time;
    job.dsize = ds;
    job.bytes = bytes;
    job.buf = bi;
    {
        std::lock_guard<std::mutex> lk(w.m);
        w.jobs.push_back(job);
        w.pending++;
    }
    w.cv.notify_all();
    return FALM_OK;
}

int falm_io_read_vector_file(falm_ctx *ctx, const char *path, void *const *fields, const int *ncols, int nfields,
                             unsigned long long *step_out, double *time_out, void *stream) {
    if (!ctx || !path || !fields || !ncols || nfields < 1) return FALM_ERR_ARG;
    long long cols = 0;
    for (int q = 0; q < nfields; q++) {
        if (!fields[q] || ncols[q] < 1) return FALM_ERR_ARG;
        cols += ncols[q];
    }
    const Geom &g = ctx->geo;
    const size_t n = (size_t)g.n, es = ctx->esize;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(ctx, FALM_ERR_ARG, (std::string("io: cannot open ") + path).c_str());
    uint64_t head[6] = {0, 0, 0, 0, 0, 0}, dsize = 0;
    double time = 0;
    bool ok = fread(head, sizeof(uint64_t), 6, f) == 6 && fread(&time, sizeof(double), 1, f) == 1 &&
              fread(&dsize, sizeof(uint64_t), 1, f) == 1;
    if (!ok) { fclose(f); return fail(ctx, FALM_ERR_ARG, "io: truncated header"); }
    if (head[0] != (uint64_t)g.sx || head[1] != (uint64_t)g.sy || head[2] != (uint64_t)g.sz || head[3] != (uint64_t)cols ||
        head[4] != (uint64_t)g.gc || (dsize != 4 && dsize != 8)) {
        fclose(f);
        return fail(ctx, FALM_ERR_ARG, "io: the file's grid, column count or value size does not match");
    }
    const size_t count = (size_t)cols * n;
    std::vector<unsigned char> raw(count * dsize);
    ok = fread(raw.data(), 1, raw.size(), f) == raw.size();
    const bool extra = ok && fgetc(f) != EOF;
    fclose(f);
    if (!ok) return fail(ctx, FALM_ERR_ARG, "io: truncated data");
    if (extra) return fail(ctx, FALM_ERR_ARG, "io: data beyond the columns the header announces");
    // to the context's precision on the host (FP64 -> FP32 rounds to nearest)
    std::vector<unsigned char> conv;
    const unsigned char *src = raw.data();
    if (dsize != es) {
        conv.resize(count * es);
        if (es == sizeof(float))
            for (size_t q = 0; q < count; q++) ((float *)conv.data())[q] = (float)((const double *)raw.data())[q];
        else
            for (size_t q = 0; q < count; q++) ((double *)conv.data())[q] = (double)((const float *)raw.data())[q];
        src = conv.data();
    }
    cudaStream_t st = S(stream);
    size_t off = 0;
    for (int q = 0; q < nfields; q++) {
        const size_t len = (size_t)ncols[q] * n;
        CK(cudaMemcpyAsync(fields[q], src + off * es, len * es, cudaMemcpyHostToDevice, st));
        off += len;
    }
    CK(cudaStreamSynchronize(st));   // the host buffers go out of scope
    if (step_out) *step_out = head[5];
    if (time_out) *time_out = time;
    return FALM_OK;
}

int falm_io_wait(falm_ctx *ctx) {
    if (!ctx) return FALM_ERR_ARG;
    if (!ctx->io) return FALM_OK;
    IoWriter &w = *ctx->io;
    std::unique_lock<std::mutex> lk(w.m);
    w.cv.wait(lk, [&] { return w.pending == 0; });
    const int rc = w.error;
    const std::string msg = w.error_msg;
    w.error = 0;
    w.error_msg.clear();
    lk.unlock();
    return rc ? fail(ctx, rc, msg.c_str()) : FALM_OK;
}

int falm_io_write_index_file(const char *path, int nx, int ny, int nz, int gc, const unsigned long long *steps,
                             const double *times, const int *tavg, int nsnap, int dsize) {
    if (!path || nx < 1 || ny < 1 || nz < 1 || gc < 0 || nsnap < 0 || (nsnap > 0 && (!steps || !times))) return FALM_ERR_ARG;
    if (dsize != 4 && dsize != 8) return FALM_ERR_ARG;
    for (int q = 0; q < nsnap; q++)
        if (!std::isfinite(times[q])) return FALM_ERR_ARG;
    // nlohmann::json's dump(2) of the reference's index object: keys in
    // lexicographic order, two-space indent, every array element on a line of
    // its own, no newline at the end
    std::string o = "{\n";
    o += std::string("  \"dataType\": \"") + (dsize == 4 ? "float32" : "float64") + "\",\n";
    o += "  \"global\": [\n    " + std::to_string(nx) + ",\n    " + std::to_string(ny) + ",\n    " + std::to_string(nz) + "\n  ],\n";
    o += "  \"guidePoint\": " + std::to_string(gc) + ",\n";
    if (nsnap > 0) {
        o += "  \"outputSteps\": [\n";
        for (int q = 0; q < nsnap; q++) {
            o += "    {\n      \"step\": " + std::to_string(steps[q]) + ",\n      \"time\": " + json_double(times[q]);
            if (tavg && tavg[q]) o += ",\n      \"timeAvg\": 1";
            o += std::string("\n    }") + (q + 1 < nsnap ? "," : "") + "\n";
        }
        o += "  ],\n";
    }
    o += "  \"ranks\": [\n    {\n      \"offset\": [\n        0,\n        0,\n        0\n      ],\n      \"rank\": 0,\n";
    o += "      \"voxel\": [\n        " + std::to_string(nx) + ",\n        " + std::to_string(ny) + ",\n        " + std::to_string(nz) +
         "\n      ]\n    }\n  ],\n";
    o += "  \"variables\": [\n    \"u\",\n    \"v\",\n    \"w\",\n    \"p\"\n  ]\n}";
    FILE *f = fopen(path, "wb");
    if (!f) return FALM_ERR_ARG;
    const bool ok = fwrite(o.data(), 1, o.size(), f) == o.size();
    return (fclose(f) == 0 && ok) ? FALM_OK : FALM_ERR_ARG;
}

int falm_io_write_cv_file(falm_ctx *ctx, const char *path) {
    if (!ctx || !path || !ctx->xc || !ctx->hx) return FALM_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return fail(ctx, FALM_ERR_ARG, "io: cannot open the control-volume file");
    const Geom &g = ctx->geo;
    fprintf(f, "%d %d %d %d\n", g.sx, g.sy, g.sz, g.gc);
    const std::vector<double> *c[3] = {ctx->xc, ctx->yc, ctx->zc}, *h[3] = {ctx->hx, ctx->hy, ctx->hz};
    for (int d = 0; d < 3; d++)
        for (size_t q = 0; q < c[d]->size(); q++) fprintf(f, "\t%.15e\t%.15e\n", (*c[d])[q], (*h[d])[q]);
    return fclose(f) == 0 ? FALM_OK : fail(ctx, FALM_ERR_ARG, "io: control-volume write");
}

// Mesher::build_mesh (src/mesher/mesher.hpp:12-260): control volumes from node
// coordinates.  Each of meshpath/{x,y,z}.txt holds a count, then one
// coordinate per line; meshpath/mesh.json names them "node" points.
//  - "cell": the nodes are the cell faces.  A cell's width is the node
//    spacing and its centre the midpoint; gc guide cells are extrapolated
//    linearly (constant widths when an axis has fewer than 3 nodes).
//  - "innerNode": the nodes are the centres of the interior cells plus one
//    guide cell on each side.  Widths are half the distance between the two
//    neighbours, the end ones extrapolated.  The upper z guide widths repeat
//    the last one where the x and y ones extrapolate linearly, as the
//    reference computes them.
// Guide-cell centres step outwards by the mean of adjacent widths.
int falm_mesh_build(const char *cvcenter, const char *meshpath, const char *outputfile, int gc) {
    if (!cvcenter || !meshpath || !outputfile || gc < 1) return FALM_ERR_ARG;
    const std::string dir(meshpath);
    std::string kind;
    {
        FILE *f = fopen((dir + "/mesh.json").c_str(), "rb");
        if (!f) return FALM_ERR_ARG;
        std::string js;
        char buf[4096];
        size_t got;
        while ((got = fread(buf, 1, sizeof(buf), f)) > 0) js.append(buf, got);
        fclose(f);
        size_t p = js.find("\"coordinatePoint\"");
        if (p != std::string::npos) p = js.find(':', p);
        if (p != std::string::npos) p = js.find('"', p);
        const size_t q = p == std::string::npos ? p : js.find('"', p + 1);
        if (q == std::string::npos) return FALM_ERR_ARG;
        kind = js.substr(p + 1, q - p - 1);
    }
    const std::string mode(cvcenter);
    if (kind != "node" || (mode != "cell" && mode != "innerNode")) return FALM_ERR_ARG;
    auto read_nodes = [&](const char *name, std::vector<double> &v) -> bool {
        std::ifstream in(dir + "/" + name);
        std::string line;
        if (!std::getline(in, line)) return false;
        int n = 0;
        try { n = std::stoi(line); } catch (...) { return false; }
        if (n < 1) return false;
        v.resize(n);
        for (int q = 0; q < n; q++) {
            if (!std::getline(in, line)) return false;
            try { v[q] = std::stod(line); } catch (...) { return false; }
        }
        return true;
    };
    std::vector<double> nodes[3], c[3], h[3];
    const char *names[3] = {"x.txt", "y.txt", "z.txt"};
    for (int d = 0; d < 3; d++)
        if (!read_nodes(names[d], nodes[d])) return FALM_ERR_ARG;
    for (int d = 0; d < 3; d++) {
        const std::vector<double> &t = nodes[d];
        std::vector<double> &x = c[d], &w = h[d];
        const int n = (int)t.size();
        int m, g;
        if (mode == "innerNode") {
            g = gc - 1;
            m = n + 2 * g;
            if (m < 3) return FALM_ERR_ARG;
            x.assign(m, 0.0); w.assign(m, 0.0);
            for (int i = g; i < m - g; i++) x[i] = t[i - g];
            for (int i = g + 1; i < m - g - 1; i++) w[i] = 0.5 * (x[i + 1] - x[i - 1]);
            for (int i = g; i >= 0; i--) w[i] = 2 * w[i + 1] - w[i + 2];
            for (int i = m - g - 1; i < m; i++) w[i] = d < 2 ? 2 * w[i - 1] - w[i - 2] : w[i - 1];
        } else {
            g = gc;
            m = n - 1 + 2 * g;
            if (n < 2) return FALM_ERR_ARG;
            x.assign(m, 0.0); w.assign(m, 0.0);
            for (int i = g; i < m - g; i++) w[i] = t[i - g + 1] - t[i - g];
            for (int i = g - 1; i >= 0; i--) w[i] = n >= 3 ? 2 * w[i + 1] - w[i + 2] : w[i + 1];
            for (int i = m - g; i < m; i++) w[i] = n >= 3 ? 2 * w[i - 1] - w[i - 2] : w[i - 1];
            for (int i = g; i < m - g; i++) x[i] = t[i - g] + 0.5 * w[i];
        }
        for (int i = g - 1; i >= 0; i--) x[i] = x[i + 1] - 0.5 * (w[i] + w[i + 1]);
        for (int i = m - g; i < m; i++) x[i] = x[i - 1] + 0.5 * (w[i] + w[i - 1]);
    }
    FILE *f = fopen(outputfile, "w");
    if (!f) return FALM_ERR_ARG;
    fprintf(f, "%d %d %d %d\n", (int)c[0].size(), (int)c[1].size(), (int)c[2].size(), gc);
    for (int d = 0; d < 3; d++)
        for (size_t q = 0; q < c[d].size(); q++) fprintf(f, "\t%.15e\t%.15e\n", c[d][q], h[d][q]);
    return fclose(f) == 0 ? FALM_OK : FALM_ERR_ARG;
}

int falm_io_read_cv_file(const char *path, int dims[4], double *x, double *hx, double *y, double *hy, double *z, double *hz) {
    if (!path || !dims) return FALM_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return FALM_ERR_ARG;
    int d4[4];
    if (fscanf(f, "%d %d %d %d", &d4[0], &d4[1], &d4[2], &d4[3]) != 4 || d4[0] < 1 || d4[1] < 1 || d4[2] < 1 || d4[3] < 0) {
        fclose(f);
        return FALM_ERR_ARG;
    }
    for (int q = 0; q < 4; q++) dims[q] = d4[q];
    double *c[3] = {x, y, z}, *h[3] = {hx, hy, hz};
    int rc = FALM_OK;
    if (x && hx && y && hy && z && hz) {
        for (int d = 0; d < 3 && rc == FALM_OK; d++)
            for (int q = 0; q < d4[d]; q++)
                if (fscanf(f, "%lf %lf", &c[d][q], &h[d][q]) != 2) { rc = FALM_ERR_ARG; break; }
    }
    fclose(f);
    return rc;
}

// ---------------------------------------------------------------- boundary conditions
int falm_bc_init(falm_ctx *ctx, int kind, double u_inlet) {
    if (ctx) graphs_clear(ctx);   // recorded steps take these settings as kernel arguments
    if (!ctx || (kind != FALM_BC_CHANNEL && kind != FALM_BC_CAVITY)) return FALM_ERR_ARG;
    ctx->bc_kind = kind;
    ctx->u_inlet = u_inlet;
    return FALM_OK;
}

int falm_bc_set_inflow(falm_ctx *ctx, const double *box, int nb, double dx) {
    if (ctx) graphs_clear(ctx);   // recorded steps take these settings as kernel arguments
    if (!ctx) return FALM_ERR_ARG;
    if (ctx->inflow_box) { cudaFree(ctx->inflow_box); ctx->inflow_box = nullptr; }
    if (!box) return FALM_OK;
    if (nb < 2 || !(dx > 0)) return FALM_ERR_ARG;
    size_t n = 3ull * nb * ctx->geo.ny * ctx->geo.nzg;   // the whole grid's inlet (a slab reads its own planes)
    CK(cudaMalloc(&ctx->inflow_box, n * sizeof(double)));
    CK(cudaMemcpy(ctx->inflow_box, box, n * sizeof(double), cudaMemcpyHostToDevice));
    ctx->inflow_nb = nb;
    ctx->inflow_dx = dx;
    return FALM_OK;
}

int falm_bc_ubc(falm_ctx *ctx, void *u, const void *uprev, double dt, double t, void *stream) {
    if (!ctx || !u || !uprev) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        return ubc_t<T>(ctx, (T *)u, UPrev<T>{(const T *)uprev, 0}, dt, t, S(stream));
    });
}

int falm_bc_pbc(falm_ctx *ctx, void *p, void *stream) {
    if (!ctx || !p) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        LAUNCH(FALM_K_PBC, S(stream), k_pbc<T><<<dim3(face_blocks(ctx), 3), 256, 0, S(stream)>>>(ctx->geo, ctx->bc_kind, (T *)p));
        return (int)FALM_OK;
    });
}

int falm_bc_uubc(falm_ctx *ctx, void *uu, void *stream) {
    if (!ctx || !uu) return FALM_ERR_ARG;
    if (ctx->bc_kind != FALM_BC_CAVITY) return FALM_OK;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        LAUNCH(FALM_K_OTHER, S(stream), k_uubc<T><<<dim3(face_blocks(ctx), 3), 256, 0, S(stream)>>>(ctx->geo, (T *)uu));
        return (int)FALM_OK;
    });
}

// ---------------------------------------------------------------- ALM
int falm_alm_build_aps(int n_station, const double *st_r, const double *st_chord, const double *st_twist,
                       const double *st_cl, const double *st_cd, int n_attack, int apcount, int n_ap_per_blade,
                       double radius, double hub_radius, double *ap_r, double *ap_chord, double *ap_twist, double *ap_cl,
                       double *ap_cd) {
    if (n_station < 1 || !st_r || !st_chord || !st_twist || !st_cl || !st_cd || n_attack < 1 || apcount < 1 ||
        n_ap_per_blade < 1 || !ap_r || !ap_chord || !ap_twist || !ap_cl || !ap_cd)
        return FALM_ERR_ARG;
    // src/alm/bladeHandler.h:46-104: r = (k+1/2) dr + r_hub, linear interpolation in r/R between
    // stations (clamped at both ends) of chord, twist and every polar value
    const double dr = (radius - hub_radius) / n_ap_per_blade;
    for (int ap = 0; ap < apcount; ap++) {
        double apr = (ap % n_ap_per_blade + 0.5) * dr + hub_radius;
        int lo = 0;
        double w = 0.0;
        int mode = 2;
        if (apr < st_r[0]) mode = 0;
        else if (apr >= st_r[n_station - 1]) mode = 1;
        else {
            int i = 0;
            for (; i < n_station - 1; i++)
                if (st_r[i] <= apr && st_r[i + 1] > apr) { w = (apr - st_r[i]) / (st_r[i + 1] - st_r[i]); break; }
            lo = i;
        }
        auto interp = [&](const double *v, int stride, int col) {
            if (mode == 0) return v[col];
            if (mode == 1) return v[(long long)(n_station - 1) * stride + col];
            return (1. - w) * v[(long long)lo * stride + col] + w * v[(long long)(lo + 1) * stride + col];
        };
        ap_r[ap] = apr;
        ap_chord[ap] = interp(st_chord, 1, 0);
        ap_twist[ap] = interp(st_twist, 1, 0);
        for (int a = 0; a < n_attack; a++) {
            ap_cl[ap + (long long)a * apcount] = interp(st_cl, n_attack, a);
            ap_cd[ap + (long long)a * apcount] = interp(st_cd, n_attack, a);
        }
    }
    return FALM_OK;
}

int falm_alm_init(falm_ctx *ctx, const falm_alm_desc *d) {
    if (ctx) graphs_clear(ctx);   // recorded steps take these settings as kernel arguments
    if (!ctx || !d || d->n_turbine < 1 || d->n_turbine > kMaxTurbines || d->n_blade < 1 || d->n_ap_per_blade < 1 ||
        d->n_attack < 2 || !(d->euler_eps > 0) || !d->base || !d->hub || !d->tip_rate || !d->motion || !d->angle_type ||
        !d->ap_r || !d->ap_chord || !d->ap_twist || !d->attack || !d->cl || !d->cd)
        return FALM_ERR_ARG;
    const int nt = d->n_turbine, apc = d->n_turbine * d->n_blade * d->n_ap_per_blade, na = d->n_attack;
    // the projection kernels stage every actuator point in shared memory
    if (apc > kMaxFusedAp) return fail(ctx, FALM_ERR_ARG, "alm_init: more than 384 actuator points");
    // one allocation: doubles then ints
    size_t nd = 3 * nt + 3 * nt + nt + 3 * nt + 3 * apc + na + 2 * (size_t)apc * na + 3 * apc + 3 * apc + apc + apc;
    size_t bytes = nd * sizeof(double) + sizeof(AlmScalars) + nt * sizeof(int) + 512;
    if (ctx->alm_mem) { cudaFree(ctx->alm_mem); ctx->alm_mem = nullptr; }
    CK(cudaMalloc(&ctx->alm_mem, bytes));
    CK(cudaMemset(ctx->alm_mem, 0, bytes));
    double *p = (double *)ctx->alm_mem;
    auto put = [&](const double *src, size_t n) -> double * {
        double *dst = p;
        p += n;
        if (src) cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice);
        return dst;
    };
    ctx->rmcp_on = 0;
    AlmDev &a = ctx->alm;
    a.n_turbine = nt; a.n_blade = d->n_blade; a.n_ap_per_blade = d->n_ap_per_blade; a.n_attack = na; a.apcount = apc;
    a.radius = d->radius; a.hub_radius = d->hub_radius; a.euler_eps = d->euler_eps; a.pitch = d->pitch;
    a.rcut2 = 36.0 * d->euler_eps * d->euler_eps;
    a.base = put(d->base, 3 * nt); a.hub = put(d->hub, 3 * nt); a.tip_rate = put(d->tip_rate, nt); a.motion = put(d->motion, 3 * nt);
    a.ap_r = put(d->ap_r, apc); a.ap_chord = put(d->ap_chord, apc); a.ap_twist = put(d->ap_twist, apc);
    a.attack = put(d->attack, na); a.cl = put(d->cl, (size_t)apc * na); a.cd = put(d->cd, (size_t)apc * na);
    a.ap_xyz = put(nullptr, 3 * apc); a.ap_force = put(nullptr, 3 * apc); a.ap_torque = put(nullptr, apc); a.ap_thrust = put(nullptr, apc);
    char *q = (char *)p;
    q = (char *)(((uintptr_t)q + 255) & ~(uintptr_t)255);
    a.scal = (AlmScalars *)q;
    q += sizeof(AlmScalars);
    int *ip = (int *)q;
    CK(cudaMemcpy(ip, d->angle_type, nt * sizeof(int), cudaMemcpyHostToDevice));
    a.angle_type = ip;
    // force boxes: every AP of turbine t stays within |hub_t| + max r of its base
    // (the motions rotate about the base), so a cell that an AP can reach lies
    // within that distance + the cutoff of the base on every axis
    {
        BoxSet &bs = a.bs;
        memset(&bs, 0, sizeof(bs));
        const Geom &g = ctx->geo;
        const std::vector<double> *cs[3] = {ctx->xc, ctx->yc, ctx->zc};
        const int s3[3] = {g.sx, g.sy, g.sz};
        const int nappt = d->n_blade * d->n_ap_per_blade;
        const double rc = std::sqrt(a.rcut2);
        long long off = 0;
        for (int t = 0; t < nt; t++) {
            double rmax = 0.0;
            for (int q = t * nappt; q < (t + 1) * nappt; q++) rmax = std::max(rmax, std::fabs(d->ap_r[q]));
            const double *hb = d->hub + 3 * t;
            const double reach = std::sqrt(hb[0] * hb[0] + hb[1] * hb[1] + hb[2] * hb[2]) + rmax + rc;
            long long cells = 1;
            for (int ax = 0; ax < 3; ax++) {
                int lo = s3[ax], hi = -1;
                for (int q = g.gc; q < s3[ax] - g.gc; q++) {
                    const double c = (*cs[ax])[q], b = d->base[3 * t + ax];
                    if (c >= b - reach && c <= b + reach) { lo = std::min(lo, q); hi = std::max(hi, q); }
                }
                if (hi >= lo) { lo = std::max(g.gc, lo - 1); hi = std::min(s3[ax] - g.gc - 1, hi + 1); }
                bs.lo[t][ax] = hi >= lo ? lo : g.gc;
                bs.ext[t][ax] = hi >= lo ? hi - lo + 1 : 0;
                cells *= bs.ext[t][ax];
            }
            bs.off[t] = off;
            off += cells;
        }
        if (off > (long long)INT_MAX / 3) return fail(ctx, FALM_ERR_ARG, "alm_init: force boxes hold more than 2^31 / 3 cells");
        bs.n = nt;
        bs.total = off;
        if (a.fbox) { cudaFree(a.fbox); a.fbox = nullptr; }
        if (off > 0) CK(cudaMalloc(&a.fbox, 3 * (size_t)off * ctx->esize));
    }
    ctx->alm_on = 1;
    return FALM_OK;
}

int falm_alm_set_pitch(falm_ctx *ctx, double pitch_deg) {
    if (ctx) graphs_clear(ctx);   // recorded steps take these settings as kernel arguments
    if (!ctx) return FALM_ERR_ARG;
    if (!ctx->alm_on) return FALM_ERR_NOALM;
    ctx->alm.pitch = pitch_deg;
    return FALM_OK;
}

int falm_alm_run(falm_ctx *ctx, const void *u, void *ff, double t, void *stream, double *torque, double *thrust) {
    if (!ctx || !u) return FALM_ERR_ARG;
    if (!ctx->alm_on) return FALM_ERR_NOALM;
    int rc = dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        return alm_run_t<T>(ctx, (const T *)u, (T *)ff, t, S(stream));
    });
    if (rc) return rc;
    if (torque || thrust) {
        CK(cudaMemcpyAsync(ctx->alm_scal_host, ctx->alm.scal, sizeof(AlmScalars), cudaMemcpyDeviceToHost, S(stream)));
        CK(cudaStreamSynchronize(S(stream)));
        for (int q = 0; q < ctx->alm.n_turbine; q++) {
            if (torque) torque[q] = ctx->alm_scal_host->torque[q];
            if (thrust) thrust[q] = ctx->alm_scal_host->thrust[q];
        }
    }
    return FALM_OK;
}

int falm_alm_get_aps(falm_ctx *ctx, double *xyz, double *force, double *torque, double *thrust) {
    if (!ctx) return FALM_ERR_ARG;
    if (!ctx->alm_on) return FALM_ERR_NOALM;
    CK(cudaDeviceSynchronize());
    const size_t n = ctx->alm.apcount;
    if (xyz) CK(cudaMemcpy(xyz, ctx->alm.ap_xyz, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
    if (force) CK(cudaMemcpy(force, ctx->alm.ap_force, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
    if (torque) CK(cudaMemcpy(torque, ctx->alm.ap_torque, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (thrust) CK(cudaMemcpy(thrust, ctx->alm.ap_thrust, n * sizeof(double), cudaMemcpyDeviceToHost));
    return FALM_OK;
}

// ---------------------------------------------------------------- step
int falm_rmcp_init(falm_ctx *ctx, const falm_rmcp_desc *d) {
    if (ctx) graphs_clear(ctx);   // recorded steps take these settings as kernel arguments
    if (!ctx || !d || d->n_turbine < 1 || d->n_turbine > kMaxTurbines || d->n_blade < 1 || d->n_station < 1 || d->n_attack < 1 ||
        !(d->radius > 0) || !(d->blade_width > 0) || !(d->blade_thick > 0) || !d->base || !d->hub || !d->angle || !d->angle_type ||
        !d->tip_rate || !d->st_r || !d->st_chord || !d->st_twist || !d->attack || !d->cl || !d->cd)
        return FALM_ERR_ARG;
    const int nt = d->n_turbine, ns = d->n_station, na = d->n_attack;
    for (int q = 0; q < nt; q++)
        if (d->angle_type[q] < 0 || d->angle_type[q] > 3) return FALM_ERR_ARG;
    const size_t nd = 3 * nt + 3 * nt + 3 * nt + nt + 3 * (size_t)ns + na + 2 * (size_t)ns * na;
    const size_t bytes = nd * sizeof(double) + nt * sizeof(int) + 2 * kMaxTurbines * sizeof(double) + 512;
    if (ctx->rmcp_mem) { cudaFree(ctx->rmcp_mem); ctx->rmcp_mem = nullptr; }
    CK(cudaMalloc(&ctx->rmcp_mem, bytes));
    CK(cudaMemset(ctx->rmcp_mem, 0, bytes));
    if (!ctx->rmcp) ctx->rmcp = new RmcpDev();
    if (!ctx->rmcp_sums_host) CK(cudaMallocHost(&ctx->rmcp_sums_host, 2 * kMaxTurbines * sizeof(double)));
    double *p = (double *)ctx->rmcp_mem;
    auto put = [&](const double *src, size_t n) -> const double * {
        double *dst = p;
        p += n;
        cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice);
        return dst;
    };
    RmcpDev &a = *ctx->rmcp;
    a.n_turbine = nt; a.n_blade = d->n_blade; a.n_station = ns; a.n_attack = na;
    a.radius = d->radius; a.hub_radius = d->hub_radius; a.width = d->blade_width; a.thick = d->blade_thick;
    a.base = put(d->base, 3 * nt); a.hub = put(d->hub, 3 * nt); a.angle = put(d->angle, 3 * nt); a.tip_rate = put(d->tip_rate, nt);
    a.st_r = put(d->st_r, ns); a.st_chord = put(d->st_chord, ns); a.st_twist = put(d->st_twist, ns); a.attack = put(d->attack, na);
    a.cl = put(d->cl, (size_t)ns * na); a.cd = put(d->cd, (size_t)ns * na);
    ctx->rmcp_sums = p;
    p += 2 * kMaxTurbines;
    int *ip = (int *)p;
    CK(cudaMemcpy(ip, d->angle_type, nt * sizeof(int), cudaMemcpyHostToDevice));
    a.angle_type = ip;
    if (cudaGetLastError() != cudaSuccess) return fail(ctx, FALM_ERR_CUDA, "rmcp_init: table copy");
    // boxes: every painted point lies within |hub| + radius + thickness of its turbine's base
    {
        BoxSet &bs = a.bs;
        memset(&bs, 0, sizeof(bs));
        const Geom &g = ctx->geo;
        const std::vector<double> *cs[3] = {ctx->xc, ctx->yc, ctx->zc};
        const int s3[3] = {g.sx, g.sy, g.sz};
        long long off = 0;
        for (int t = 0; t < nt; t++) {
            const double *hb = d->hub + 3 * t;
            const double reach = std::sqrt(hb[0] * hb[0] + hb[1] * hb[1] + hb[2] * hb[2]) + d->radius + d->blade_thick;
            long long cells = 1;
            for (int ax = 0; ax < 3; ax++) {
                int lo = s3[ax], hi = -1;
                for (int q = g.gc; q < s3[ax] - g.gc; q++) {
                    const double c = (*cs[ax])[q], b = d->base[3 * t + ax];
                    if (c >= b - reach && c <= b + reach) { lo = std::min(lo, q); hi = std::max(hi, q); }
                }
                if (hi >= lo) { lo = std::max(g.gc, lo - 1); hi = std::min(s3[ax] - g.gc - 1, hi + 1); }
                bs.lo[t][ax] = hi >= lo ? lo : g.gc;
                bs.ext[t][ax] = hi >= lo ? hi - lo + 1 : 0;
                cells *= bs.ext[t][ax];
            }
            bs.off[t] = off;
            off += cells;
        }
        bs.n = nt;
        bs.total = off;
    }
    if (!ctx->w_ff) CK(cudaMalloc(&ctx->w_ff, 3 * (size_t)ctx->geo.n * ctx->esize));
    CK(cudaMemset(ctx->w_ff, 0, 3 * (size_t)ctx->geo.n * ctx->esize));
    ctx->rmcp_on = 1;
    ctx->alm_on = 0;
    return FALM_OK;
}

int falm_rmcp_run(falm_ctx *ctx, const void *u, void *ff, double t, void *stream, int *flag, double *torque, double *thrust) {
    if (!ctx || !u || !ff) return FALM_ERR_ARG;
    if (!ctx->rmcp_on) return fail(ctx, FALM_ERR_STATE, "rmcp_run: no RMCP model (falm_rmcp_init)");
    cudaStream_t st = S(stream);
    int rc = dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        return rmcp_run_t<T>(ctx, (const T *)u, (T *)ff, flag, t, st);
    });
    if (rc) return rc;
    if ((rc = slab_reduce(ctx, ctx->rmcp_sums, 2 * kMaxTurbines, FALM_REDUCE_SUM, st))) return rc;
    CK(cudaMemcpyAsync(ctx->rmcp_sums_host, ctx->rmcp_sums, 2 * kMaxTurbines * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int q = 0; q < ctx->rmcp->n_turbine; q++) {
        if (torque) torque[q] = ctx->rmcp_sums_host[q];
        if (thrust) thrust[q] = ctx->rmcp_sums_host[kMaxTurbines + q];
    }
    return FALM_OK;
}

int falm_step(falm_ctx *ctx, const falm_fields *f, double dt, double t, void *stream, falm_step_stats *st) {
    if (!ctx || !f || !f->u || !f->uu || !f->p || !f->nut || !(dt > 0)) return FALM_ERR_ARG;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        if (ctx->slab_on) return slab_step_t<T>(ctx, f, dt, t, S(stream), st);
        return step_t<T>(ctx, f, dt, t, S(stream), st);
    });
}

}  // extern "C"

extern "C" {

int falm_bc_set_inlet_plane(falm_ctx *ctx, const double *plane, void *stream) {
    (void)stream;   // the copy goes on the stream of the call that uses the plane
    if (!ctx || !plane) return FALM_ERR_ARG;
    const size_t n = 3ull * ctx->geo.ny * ctx->geo.nz;
    if (!ctx->inlet_plane) CK(cudaMalloc(&ctx->inlet_plane, n * sizeof(double)));
    ctx->inlet_host = plane;
    ctx->inlet_pending = 1;
    ctx->inlet_plane_valid = 1;
    return FALM_OK;
}

int falm_slab_init(falm_ctx *ctx, int rank, int nranks, int z_offset, int nz_global, const falm_transport *t) {
    if (!ctx || nranks < 1 || rank < 0 || rank >= nranks || !t || !t->exchange || !t->allreduce) return FALM_ERR_ARG;
    Geom &g = ctx->geo;
    if (z_offset < 0 || nz_global < g.nz || z_offset + g.nz > nz_global || g.nz < g.gc) return FALM_ERR_ARG;
    if (ctx->op_ready || ctx->inflow_box || ctx->work_mem) return fail(ctx, FALM_ERR_STATE, "slab_init: call it right after falm_create");
    if (rank == 0 && z_offset != 0) return FALM_ERR_ARG;
    if (rank == nranks - 1 && z_offset + g.nz != nz_global) return FALM_ERR_ARG;
    g.koff = z_offset;
    g.nzg = nz_global;
    g.zphys = (rank == 0 ? 1 : 0) | (rank == nranks - 1 ? 2 : 0);
    ctx->slab_on = 1;
    ctx->slab_rank = rank;
    ctx->slab_nranks = nranks;
    ctx->transport = *t;
    return FALM_OK;
}

int falm_slab_halo(falm_ctx *ctx, void *field, int ncomp, int depth, void *stream) {
    if (!ctx || !field || ncomp < 1 || depth < 1) return FALM_ERR_ARG;
    if (!ctx->slab_on) return FALM_OK;
    return dispatch(ctx, [&](auto z) {
        using T = decltype(z);
        return slab_halo<T>(ctx, (T *)field, ncomp, depth, S(stream));
    });
}

int falm_local_hub_create(int nranks, void **hub) {
    if (nranks < 1 || !hub) return FALM_ERR_ARG;
    LocalHub *h = new LocalHub();
    h->n = nranks;
    h->r.resize(nranks);
    for (int q = 0; q < nranks; q++) h->users.push_back(new HubUser{h, q});
    *hub = h;
    return FALM_OK;
}

int falm_local_hub_transport(void *hub, int rank, falm_transport *out) {
    LocalHub *h = (LocalHub *)hub;
    if (!h || !out || rank < 0 || rank >= h->n) return FALM_ERR_ARG;
    out->user = h->users[rank];
    out->exchange = hub_exchange;
    out->allreduce = hub_allreduce;
    return FALM_OK;
}

int falm_local_hub_destroy(void *hub) {
    LocalHub *h = (LocalHub *)hub;
    if (!h) return FALM_ERR_ARG;
    for (auto &r : h->r) {
        if (r.ready) cudaEventDestroy(r.ready);
        if (r.done) cudaEventDestroy(r.done);
        if (r.scratch) cudaFree(r.scratch);
    }
    for (void *u : h->users) delete (HubUser *)u;
    delete h;
    return FALM_OK;
}

int falm_nccl_unique_id(unsigned char id[128]) {
    const NcclApi *a = nccl_api();
    if (!id) return FALM_ERR_ARG;
    if (!a) return FALM_ERR_STATE;
    static_assert(sizeof(ncclUniqueId) == 128, "ncclUniqueId is 128 bytes");
    ncclUniqueId u;
    if (a->get_unique_id(&u) != ncclSuccess) return FALM_ERR_CUDA;
    memcpy(id, &u, 128);
    return FALM_OK;
}

int falm_nccl_transport_create(const unsigned char id[128], int rank, int nranks, falm_transport *out) {
    const NcclApi *a = nccl_api();
    if (!id || !out || nranks < 1 || rank < 0 || rank >= nranks) return FALM_ERR_ARG;
    if (!a) return FALM_ERR_STATE;
    ncclUniqueId u;
    memcpy(&u, id, 128);
    NcclUser *nu = new NcclUser{nullptr, rank, nranks};
    if (a->comm_init_rank(&nu->comm, nranks, u, rank) != ncclSuccess) { delete nu; return FALM_ERR_CUDA; }
    out->user = nu;
    out->exchange = nccl_exchange;
    out->allreduce = nccl_allreduce;
    return FALM_OK;
}

int falm_nccl_transport_destroy(falm_transport *t) {
    const NcclApi *a = nccl_api();
    if (!t || !t->user || t->exchange != nccl_exchange) return FALM_ERR_ARG;
    NcclUser *nu = (NcclUser *)t->user;
    if (a && nu->comm) a->comm_destroy(nu->comm);
    delete nu;
    t->user = nullptr;
    return FALM_OK;
}

int falm_debug_arm_wait_probe(falm_ctx *ctx, long long cycles) {
    if (!ctx || cycles <= 0 || cycles > kWaitCycles) return FALM_ERR_ARG;
    ctx->wait_probe_cycles = cycles;
    return FALM_OK;
}

int falm_profile_enable(falm_ctx *ctx, int enable) {
    if (!ctx) return FALM_ERR_ARG;
    ctx->profiling = enable ? 1 : 0;
    return FALM_OK;
}

int falm_profile_read(falm_ctx *ctx, double *ms, long long *launches, int nclass, int reset) {
    if (!ctx || nclass < 0) return FALM_ERR_ARG;
    CK(cudaDeviceSynchronize());
    for (auto &r : *ctx->ev_pending) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
            ctx->prof_ms[r.cls] += t;
            ctx->prof_n[r.cls] += 1;
        }
        cudaGetLastError();
        ctx->ev_pool->push_back(r.a);
        ctx->ev_pool->push_back(r.b);
    }
    ctx->ev_pending->clear();
    for (int c = 0; c < nclass && c < FALM_K_COUNT; c++) {
        if (ms) ms[c] = ctx->prof_ms[c];
        if (launches) launches[c] = ctx->prof_n[c];
    }
    if (reset)
        for (int c = 0; c < FALM_K_COUNT; c++) { ctx->prof_ms[c] = 0; ctx->prof_n[c] = 0; }
    return FALM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free inner product
// falm_mv_dot_static: the interior inner product of k_dot for callers that hold
// device fields but may not allocate.  A coupled solver or an in-situ monitor
// running beside a simulation that has claimed the device memory is such a
// caller: creating a context (metric tables, reduction workspace, pinned
// scalars) could fail there, or fragment the other code's memory pool.
// Everything the reduction needs lives in one fixed device array, so the call
// allocates nothing:
//   [0, 8*kStaticDotBlocks)   per-block partial sums (written before use)
//   counter at kCounterOff    arrival counter; cleared on the stream at the
//                             start of every call (an earlier call that failed
//                             part way may have left it non-zero)
//   result at kResultOff      the total, copied back to the host
// The array is shared by all calls on a device and keeps the last call's
// contents: two calls in flight at once (two streams, two host threads) race.
namespace {
constexpr int kStaticDotBlocks = 16384;                                   // 8 rows per block: 131072 rows
constexpr size_t kCounterOff = (size_t)kStaticDotBlocks * sizeof(double);
constexpr size_t kResultOff = kCounterOff + 64;
constexpr size_t kStaticDotBytes = kResultOff + 64;                       // 131200 bytes
constexpr int kMaxStaticDevices = 64;
constexpr int kMaxStaticGc = 64;

// the set-up of a device: the array's address in the device context it was
// taken in (a context torn down by cudaDeviceReset is replaced by one with a
// new id, whose module copy may sit at another address)
struct StaticScratch {
    unsigned long long ctx_id;
    unsigned char *ptr;
};
std::mutex g_static_mu;
StaticScratch g_static[kMaxStaticDevices];

typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);

// the unique id of the calling thread's current context (0 when none is current)
unsigned long long current_ctx_id() {
    static PfnCtxGetCurrent get_cur = nullptr;
    static PfnCtxGetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_cur = (PfnCtxGetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_id = (PfnCtxGetId)f;
        cudaGetLastError();
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}
}  // namespace

static __device__ __align__(256) unsigned char g_dot_scratch[kStaticDotBytes];

namespace {
// once per device (and again if that device's context was replaced), with the
// device current: the array's address, taken by cudaGetSymbolAddress
int static_scratch(unsigned char **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return FALM_ERR_CUDA; }
    if (dev < 0 || dev >= kMaxStaticDevices) return FALM_ERR_ARG;
    unsigned long long id = current_ctx_id();
    if (!id) {   // no context current yet on this thread: make the device's primary context current
        if (cudaSetDevice(dev) != cudaSuccess) { cudaGetLastError(); return FALM_ERR_CUDA; }
        id = current_ctx_id();
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    StaticScratch &e = g_static[dev];
    if (!e.ptr || e.ctx_id != id || !id) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_dot_scratch) != cudaSuccess || !p) { cudaGetLastError(); return FALM_ERR_CUDA; }
        e.ptr = (unsigned char *)p;
        e.ctx_id = id;
    }
    *out = e.ptr;
    return FALM_OK;
}
}  // namespace

extern "C" int falm_mv_dot_static(int sx, int sy, int sz, int gc, int precision, const void *a, const void *b, double *out,
                                  void *stream) {
    if (!a || !b || !out || gc < 1 || gc > kMaxStaticGc || sx < 2 * gc + 1 || sy < 2 * gc + 1 || sz < 2 * gc + 1 ||
        (precision != FALM_FP64 && precision != FALM_MIXED))
        return FALM_ERR_ARG;
    const long long rows = (long long)(sy - 2 * gc) * (sz - 2 * gc);
    const long long blocks = (rows + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > kStaticDotBlocks) return FALM_ERR_SIZE;   // more interior rows than the fixed partial-sum array holds
    unsigned char *p = nullptr;
    int rc = static_scratch(&p);
    if (rc) return rc;
    Geom g;
    g.sx = sx; g.sy = sy; g.sz = sz; g.gc = gc;
    g.n = (long long)sx * sy * sz;
    g.nx = sx - 2 * gc; g.ny = sy - 2 * gc; g.nz = sz - 2 * gc;
    g.koff = 0; g.zphys = 3; g.nzg = g.nz;
    const Region3 R = interior(g);
    RedWork rw{(double *)p, (unsigned int *)(p + kCounterOff), kStaticDotBlocks};
    double *res = (double *)(p + kResultOff);
    cudaStream_t st = S(stream);
    if (cudaMemsetAsync(p + kCounterOff, 0, sizeof(unsigned int), st) != cudaSuccess) { cudaGetLastError(); return FALM_ERR_CUDA; }
    if (precision == FALM_FP64)
        k_dot<double><<<(int)blocks, kRowThreads, 0, st>>>(g, R, (const double *)a, (const double *)b, 1, rw, res);
    else
        k_dot<float><<<(int)blocks, kRowThreads, 0, st>>>(g, R, (const float *)a, (const float *)b, 1, rw, res);
    if (cudaGetLastError() != cudaSuccess) return FALM_ERR_CUDA;
    if (cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return FALM_ERR_CUDA;
    }
    return FALM_OK;
}

// ---------------------------------------------------------------- discrete adjoint of the step
namespace {

struct AdjWork {
    double *uc, *uuc, *pc, *nutc, *au0, *auu0, *anut0, *aua, *auu1, *aff, *ap, *arhs, *r, *AT, *aF, *arhs1;
    double *v64;  // mixed contexts: the eight FP64 vectors of the transposed BiCGStab solve
};

// initial guess of the transposed solve: linear extrapolation from the two
// previous (normalised) solutions, y <- 2 y - y_prev, y_prev <- old y
__global__ void k_adj_extrapolate(double *y, double *yprev, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const double a = y[q];
        y[q] = 2 * a - yprev[q];
        yprev[q] = a;
    }
}

__global__ void k_adj_zero_interior(Geom g, double *a) {
    ADJ_FOR_BOX(g.gc, g.sx - g.gc, g.gc, g.sy - g.gc, g.gc, g.sz - g.gc, i, j, k) { a[g.id(i, j, k)] = 0; }
}

int adj_work(falm_ctx *ctx, AdjWork *w) {
    const size_t n = (size_t)ctx->geo.n;
    const size_t apc = ctx->alm_on ? (size_t)ctx->alm.apcount : 0;
    const size_t v64n = ctx->precision == FALM_FP64 ? 1 : 8 * ((n + 31) / 32 * 32);
    const size_t counts[17] = {3 * n, 3 * n, n, n, 3 * n, 3 * n, n, 3 * n, 3 * n, 3 * n, n, n, n, 7 * n, 3 * apc + 1, n, v64n};
    size_t bytes = 0;
    for (int q = 0; q < 17; q++) bytes += (counts[q] * sizeof(double) + 255) / 256 * 256;
    if (!ctx->adj_mem) {
        if (cudaMalloc(&ctx->adj_mem, bytes) != cudaSuccess) { cudaGetLastError(); ctx->adj_mem = nullptr; return fail(ctx, FALM_ERR_ALLOC, "step_adjoint: workspace"); }
        if (cudaMemset(ctx->adj_mem, 0, bytes) != cudaSuccess) { cudaGetLastError(); return fail(ctx, FALM_ERR_CUDA, "step_adjoint: workspace"); }
    }
    char *p = (char *)ctx->adj_mem;
    double **dst[16] = {&w->uc, &w->uuc, &w->pc, &w->nutc, &w->au0, &w->auu0, &w->anut0, &w->aua, &w->auu1, &w->aff, &w->ap,
                        &w->arhs, &w->r, &w->AT, &w->aF, &w->arhs1};
    for (int q = 0; q < 16; q++) { *dst[q] = (double *)p; p += (counts[q] * sizeof(double) + 255) / 256 * 256; }
    w->v64 = (double *)p;
    return FALM_OK;
}

// The transposed Poisson solve of the adjoint, A^T y = b with |b| = 1 (b = w.ap),
// y in w.arhs (FP64; on entry the extrapolated guess), to |b - A^T y| <= rel,
// by the context's PBiCGStab in FP64.  A mixed-precision context runs it on
// FP64 copies of its solver vectors (swapped in for the call) and its FP64
// operator tables: FP32 BiCGStab cannot be used here, since on the nearly
// singular operator of a long channel (one Dirichlet face) the transposed
// solves take hundreds of iterations, over which the FP32 recursion breaks
// down (non-finite scalars at 512x128x128 where FP64 converges in ~300
// iterations), and FP32 storage of y would bound its residual near
// 2 eps_32 / lambda_min, a few 1e-2 for smooth solutions 1024 cells long.
template <typename T>
int adj_transposed_solve(falm_ctx *ctx, AdjWork &w, double rel, cudaStream_t st) {
    const Geom &g = ctx->geo;
    int it = 0, outer = 0;
    double err = 0;
    ctx->tol = rel / ((double)g.nx * g.ny * g.nz);
    if constexpr (sizeof(T) == 8) {
        return solve_t<double>(ctx, w.arhs, w.ap, w.r, st, &it, &err, &outer);
    } else {
        void **vec[8] = {&ctx->w_rr, &ctx->w_p, &ctx->w_q, &ctx->w_s, &ctx->w_pp, &ctx->w_ss, &ctx->w_t, &ctx->w_xp};
        void *saved[8];
        const size_t stride = (size_t)(g.n + 31) / 32 * 32;
        for (int q = 0; q < 8; q++) { saved[q] = *vec[q]; *vec[q] = w.v64 + q * stride; }
        const int outer_saved = ctx->max_outer;
        ctx->max_outer = 1;   // y is FP64: no outer checks of an FP32 iterate
        const int rc = solve_t<double>(ctx, w.arhs, w.ap, w.r, st, &it, &err, &outer);
        ctx->max_outer = outer_saved;
        for (int q = 0; q < 8; q++) *vec[q] = saved[q];
        return rc;
    }
}

}  // namespace

extern "C" int falm_adjoint_set_tol(falm_ctx *ctx, double rel_tol) {
    if (!ctx || !(rel_tol >= 0) || rel_tol >= 1) return FALM_ERR_ARG;
    ctx->adj_rel_tol = rel_tol;
    return FALM_OK;
}

namespace {

// falm_step_adjoint for a context of storage type T (the forward state f0, f1)
template <typename T>
int step_adjoint_t(falm_ctx *ctx, const falm_fields *f0, const falm_fields *f1, double dt, double t, double w_power,
                   void *au, void *auu, void *anut, double *grad, cudaStream_t st) {
    NvtxRange range("falm_step_adjoint");
    int rc = ensure_work(ctx);
    if (rc) return rc;
    AdjWork w;
    if ((rc = adj_work(ctx, &w))) return rc;
    const Geom &g = ctx->geo;
    const size_t n = (size_t)g.n, nb = n * sizeof(double), nt = n * sizeof(T);
    const T *un;
    if (f1 && f1->u) {
        // the state after the step is given: only the ALM state of the step is needed again
        un = (const T *)f1->u;
        if (ctx->alm_on && (rc = alm_run_t<T>(ctx, (const T *)f0->u, nullptr, t, st))) return rc;
    } else {
        // forward recomputation of the step on copies of the state
        T *uc = (T *)w.uc, *uuc = (T *)w.uuc, *pc = (T *)w.pc, *nutc = (T *)w.nutc;
        CK(cudaMemcpyAsync(uc, f0->u, 3 * nt, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(uuc, f0->uu, 3 * nt, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(pc, f0->p, nt, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(nutc, f0->nut, nt, cudaMemcpyDeviceToDevice, st));
        falm_fields fc{uc, uuc, pc, nutc, nullptr};
        falm_step_stats sst;
        if ((rc = step_t<T>(ctx, &fc, dt, t, st, &sst))) return rc;
        un = uc;
    }
    // reverse sweep
    for (double *z : {w.au0, w.auu0, w.aua, w.auu1, w.aff}) CK(cudaMemsetAsync(z, 0, 3 * nb, st));
    // arhs and arhs1 keep the previous two calls' transposed-Poisson solutions: the
    // initial guess of this call's solve extrapolates them
    CK(cudaMemsetAsync(w.ap, 0, nb, st));
    CK(cudaMemcpyAsync(w.anut0, anut, nb, cudaMemcpyDeviceToDevice, st));
    const int grid = ctx->sm_count * 8;
    const MetricView<double> mv = mview<double>(ctx);
    double *pu = (double *)au, *puu = (double *)auu, *pnut = (double *)anut;
    if (ctx->sgs == FALM_SGS_SMAGORINSKY) {
        LAUNCH(FALM_K_OTHER, st, k_adj_zero_interior<<<grid, 256, 0, st>>>(g, w.anut0));
        LAUNCH(FALM_K_OTHER, st, k_adj_sgs<T><<<grid, 256, 0, st>>>(g, mv, un, pnut, pu, ctx->Cs));
    }
    LAUNCH(FALM_K_OTHER, st, k_adj_ubc<<<dim3(64, 3), 256, 0, st>>>(g, ctx->bc_kind, pu, w.au0, ctx->m64.x[0], dt));
    LAUNCH(FALM_K_OTHER, st, k_adj_carry_edges<<<grid, 256, 0, st>>>(g, pu, w.au0, 3));
    LAUNCH(FALM_K_OTHER, st, k_adj_project<<<grid, 256, 0, st>>>(g, mv, pu, puu, w.aua, w.auu1, w.auu0, w.ap, dt));
    LAUNCH(FALM_K_OTHER, st, k_adj_pbc<<<dim3(64, 3), 256, 0, st>>>(g, ctx->bc_kind, w.ap));
    LAUNCH(FALM_K_OTHER, st, k_adj_zero_ghosts<<<grid, 256, 0, st>>>(g, w.ap));
    // transposed Poisson solve, warm-started; a symmetric table operator is its
    // own transpose, otherwise the transpose is built as an explicit FP64
    // 7-column matrix
    const bool use_tables = !ctx->A_explicit && ctx->op_symmetric;
    if (!use_tables) LAUNCH(FALM_K_OTHER, st, k_adj_transpose_op<<<grid, 256, 0, st>>>(g, op7<double>(ctx), w.AT));
    // the right-hand side is normalised to unit norm (the solver's breakdown test
    // |rho| < FLT_MIN is absolute) and the solution is kept normalised as the next guess
    double apn = 0.0;
    if ((rc = dot_t<double>(ctx, w.ap, w.ap, 1, &apn, st))) return rc;
    apn = sqrt(apn);
    if (apn > 0) {
        LAUNCH(FALM_K_OTHER, st, k_scale<double><<<grid, 256, 0, st>>>(w.ap, (long long)n, 1.0 / apn));
        const void *a_saved = ctx->A_explicit;
        const double tol_saved = ctx->tol;
        const int ls_saved = ctx->ls_type;
        ctx->ls_type = FALM_LS_PBICGSTAB;   // whatever solver the forward step uses
        if (!use_tables) ctx->A_explicit = w.AT;
        LAUNCH(FALM_K_OTHER, st, k_adj_extrapolate<<<grid, 256, 0, st>>>(w.arhs, w.arhs1, (long long)n));
        // relative residual ctx->adj_rel_tol (falm_adjoint_set_tol); by default 1e-5
        // (1e-12 when the context's tolerance is below 1e-12)
        const double rel = ctx->adj_rel_tol > 0 ? ctx->adj_rel_tol : (tol_saved < 1e-12 ? 1e-12 : 1e-5);
        rc = adj_transposed_solve<T>(ctx, w, rel, st);
        ctx->A_explicit = a_saved;
        ctx->tol = tol_saved;
        ctx->ls_type = ls_saved;
        if (rc) return rc;
    }
    const double scale = apn / (dt * ctx->maxdiag);   // arhs holds the solution for the normalised right-hand side
    if (apn > 0) LAUNCH(FALM_K_OTHER, st, k_adj_rhs<<<grid, 256, 0, st>>>(g, mv, w.arhs, w.auu1, scale));
    if (ctx->bc_kind == FALM_BC_CAVITY) LAUNCH(FALM_K_OTHER, st, k_adj_uubc<<<grid, 256, 0, st>>>(g, w.auu1));
    LAUNCH(FALM_K_OTHER, st, k_adj_utouu<<<grid, 256, 0, st>>>(g, mv, w.auu1, w.aua));
    LAUNCH(FALM_K_OTHER, st, k_adj_carry_ghosts<<<grid, 256, 0, st>>>(g, w.aua, w.au0));
    const double alpha = ctx->adv == FALM_ADV_UTOPIA ? 1. / 12. : (ctx->adv == FALM_ADV_KK ? 1. / 4. : 1. / 24.);
    LAUNCH(FALM_K_OTHER, st, k_adj_pseudo_u<T><<<grid, 256, 0, st>>>(g, mv, (const T *)f0->u, (const T *)f0->uu, (const T *)f0->nut,
                                                                     w.aua, w.au0, w.auu0, w.anut0, w.aff, 1.0 / ctx->Re, dt, alpha));
    if (ctx->alm_on) {
        const int apc = ctx->alm.apcount;
        LAUNCH(FALM_K_ALM, st, k_adj_alm_project<<<apc, 256, 0, st>>>(g, ctx->alm, ctx->m64.x[0], ctx->m64.x[1], ctx->m64.x[2], w.aff, w.aF));
        LAUNCH(FALM_K_ALM, st, k_adj_alm_ap<T><<<(apc + 127) / 128, 128, 0, st>>>(g, ctx->alm, ctx->m64.x[0], ctx->m64.x[1], ctx->m64.x[2],
                                                                                 (const T *)f0->u, t, w.aF, w_power, w.au0, grad));
    }
    CK(cudaMemcpyAsync(pu, w.au0, 3 * nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(puu, w.auu0, 3 * nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(pnut, w.anut0, nb, cudaMemcpyDeviceToDevice, st));
    return FALM_OK;
}

}  // namespace

extern "C" int falm_step_adjoint(falm_ctx *ctx, const falm_fields *f0, const falm_fields *f1, double dt, double t, double w_power,
                                 void *au, void *auu, void *anut, double *grad, void *stream) {
    if (!ctx || !f0 || !f0->u || !f0->uu || !f0->p || !f0->nut || !au || !auu || !anut || !grad || !(dt > 0)) return FALM_ERR_ARG;
    if (ctx->slab_on && ctx->slab_nranks > 1) return fail(ctx, FALM_ERR_ARG, "step_adjoint: a grid of one slab only");
    if (ctx->rmcp_on) return fail(ctx, FALM_ERR_ARG, "step_adjoint: the ALM forcing only (not the RMCP model)");
    if (ctx->adv != FALM_ADV_UPWIND3 && ctx->adv != FALM_ADV_UTOPIA && ctx->adv != FALM_ADV_KK)
        return fail(ctx, FALM_ERR_ARG, "step_adjoint: the 4th-order advection schemes (Upwind3, UTOPIA, KK) only");
    if (ctx->sgs != FALM_SGS_EMPTY && ctx->sgs != FALM_SGS_SMAGORINSKY) return fail(ctx, FALM_ERR_ARG, "step_adjoint: Smagorinsky or no SGS model only");
    cudaStream_t st = S(stream);
    if (ctx->precision == FALM_FP64) return step_adjoint_t<double>(ctx, f0, f1, dt, t, w_power, au, auu, anut, grad, st);
    if (ctx->A_explicit)
        return fail(ctx, FALM_ERR_ARG, "step_adjoint: mixed precision needs the operator of falm_eq_poisson_operator (not a caller's matrix)");
    return step_adjoint_t<float>(ctx, f0, f1, dt, t, w_power, au, auu, anut, grad, st);
}
