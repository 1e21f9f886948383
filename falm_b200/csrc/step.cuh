// The step (app/nedo/main.cpp:150-204): forcing, pseudo-velocity, face
// velocity + right-hand side, the solve, projection and boundary conditions,
// SGS + divergence; host-driven or recorded as a CUDA graph.
// Included by falm_b200.cu inside its anonymous namespace (after the headers
// it includes and the code before this point); not a standalone header.
#pragma once

AlmFuse alm_fuse(const falm_ctx *ctx) {
    AlmFuse af;
    memset(&af, 0, sizeof(af));
    if (!ctx->alm_on || ctx->alm.apcount > kMaxFusedAp) return af;
    af.apcount = ctx->alm.apcount;
    af.xyz = ctx->alm.ap_xyz;
    af.force = ctx->alm.ap_force;
    af.scal = ctx->alm.scal;
    af.eps = ctx->alm.euler_eps;
    double sq = std::sqrt(M_PI) * af.eps;
    af.eta = 1. / (sq * sq * sq);
    af.rcut2 = ctx->alm.rcut2;
    af.bs = ctx->alm.bs;
    af.fbox = ctx->alm.fbox;
    return af;
}

template <typename T> struct PUConf;
template <> struct PUConf<double> { static constexpr int NS = 4; };
template <> struct PUConf<float> { static constexpr int NS = 6; };

template <typename T>
int pseudo_u_t(falm_ctx *ctx, const T *un, const T *u, const T *uu, T *ua, const T *nut, const T *ff, double dt, bool fuse, cudaStream_t st) {
    const Region3 R = interior(ctx->geo);
    AlmFuse af;
    memset(&af, 0, sizeof(af));
    if (!ff && fuse) af = alm_fuse(ctx);
    const Geom &g = ctx->geo;
    constexpr int NS = PUConf<T>::NS;
    using L = PUTile<T, NS>;
    CUtensorMap mu, muu, mnut;
    if (!ctx->no_tma && make_map(ctx, &mu, u, 3, L::BX, L::BY) && make_map(ctx, &muu, uu, 3, L::BX, L::BY) &&
        make_map(ctx, &mnut, nut, 1, L::BX, L::BY)) {
        // FP32 with a 4th-order scheme and an even interior width: the x-pair kernel
        if constexpr (sizeof(T) == 4) {
            if (!ctx->pu_v1 && (g.nx & 1) == 0 &&
                (ctx->adv == FALM_ADV_UPWIND3 || ctx->adv == FALM_ADV_UTOPIA || ctx->adv == FALM_ADV_KK)) {
                // a ring of 4 planes (49 KB) and at most 128 registers: 4 CTAs per SM
                constexpr int NS2 = 4;
                using L = PUTile<T, NS2>;
                auto k2 = k_pseudo_u_tma2<NS2, FALM_ADV_UPWIND3>;
                if (ctx->adv == FALM_ADV_UTOPIA) k2 = k_pseudo_u_tma2<NS2, FALM_ADV_UTOPIA>;
                if (ctx->adv == FALM_ADV_KK) k2 = k_pseudo_u_tma2<NS2, FALM_ADV_KK>;
                const int bx = (g.nx + L::TX - 1) / L::TX, by = (g.ny + L::TY - 1) / L::TY;
                const int kc = chunk_len(ctx, (long long)bx * by, g.nz, resident_per_sm(k2, 128, L::SMEM), 64, 4);
                cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
                dim3 grid(bx, by, (g.nz + kc - 1) / kc);
                LAUNCH(FALM_K_PSEUDO_U, st, k2<<<grid, 128, L::SMEM, st>>>(g, kc, mview<T>(ctx), mu, muu, mnut, un, un == u ? 1 : 0, ua, ff, af,
                                                                         (T)(1.0 / ctx->Re), (T)dt, ctx->kerr));
                return FALM_OK;
            }
        }
        auto kern = k_pseudo_u_tma<T, NS, FALM_ADV_KK>;
        switch (ctx->adv) {
            case FALM_ADV_UPWIND1: kern = k_pseudo_u_tma<T, NS, FALM_ADV_UPWIND1>; break;
            case FALM_ADV_UPWIND3: kern = k_pseudo_u_tma<T, NS, FALM_ADV_UPWIND3>; break;
            case FALM_ADV_QUICK: kern = k_pseudo_u_tma<T, NS, FALM_ADV_QUICK>; break;
            case FALM_ADV_UTOPIA: kern = k_pseudo_u_tma<T, NS, FALM_ADV_UTOPIA>; break;
            default: break;
        }
        const int bx = (g.nx + L::TX - 1) / L::TX, by = (g.ny + L::TY - 1) / L::TY;
        const int kc = chunk_len(ctx, (long long)bx * by, g.nz, resident_per_sm(kern, 256, L::SMEM), 64, 4);
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
        dim3 grid(bx, by, (g.nz + kc - 1) / kc);
        LAUNCH(FALM_K_PSEUDO_U, st, kern<<<grid, 256, L::SMEM, st>>>(g, kc, mview<T>(ctx), mu, muu, mnut, un, un == u ? 1 : 0, ua, ff, af,
                                                                    (T)(1.0 / ctx->Re), (T)dt, ctx->kerr));
        return FALM_OK;
    }
    LAUNCH(FALM_K_PSEUDO_U, st, k_pseudo_u<T><<<row_grid(ctx, R), kRowThreads, 0, st>>>(ctx->geo, R, mview<T>(ctx), un, u, uu, ua, nut, ff, af,
                                                            (T)(1.0 / ctx->Re), (T)dt, ctx->adv));
    return FALM_OK;
}

template <typename T>
int alm_run_t(falm_ctx *ctx, const T *u, T *ff, double t, cudaStream_t st, const double *t_dev = nullptr) {
    // stage the coordinate tables in shared memory when they fit in 96 KB
    const int csm = (ctx->geo.sx + ctx->geo.sy + ctx->geo.sz) * (int)sizeof(double);
    const int stage = csm <= 96 * 1024 ? 1 : 0;
    if (stage && csm > 32 * 1024) cudaFuncSetAttribute(k_alm_force<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
    LAUNCH(FALM_K_ALM, st, k_alm_force<T><<<1, 256, stage ? csm : 0, st>>>(ctx->geo, ctx->alm, ctx->m64.x[0], ctx->m64.x[1], ctx->m64.x[2], u, t, stage,
                                                                            t_dev));
    if (ff) {
        const Region3 R = interior(ctx->geo);
        LAUNCH(FALM_K_ALM, st, k_alm_project<T><<<row_grid(ctx, R), kRowThreads, 0, st>>>(ctx->geo, R, mview<T>(ctx), ctx->alm, ff));
    } else if (ctx->alm.bs.total > 0) {
        // force boxes for the fused projection of the plane-streaming pseudo-velocity kernel
        const long long blocks = std::min<long long>((ctx->alm.bs.total + 255) / 256, (long long)ctx->sm_count * 8);
        LAUNCH(FALM_K_ALM, st, k_alm_box<T><<<(int)blocks, 256, 0, st>>>(ctx->alm, ctx->m64.x[0], ctx->m64.x[1], ctx->m64.x[2]));
    }
    return FALM_OK;
}

template <typename T>
int ubc_t(falm_ctx *ctx, T *u, UPrev<T> up, double dt, double t, cudaStream_t st, const double *t_dev = nullptr) {
    // a streamed inlet plane: its copy, unless a recorded step's copy node makes it
    if (ctx->inlet_plane_valid && ctx->inlet_pending && !t_dev) {
        CK(cudaMemcpyAsync(ctx->inlet_plane, ctx->inlet_host, 3ull * ctx->geo.ny * ctx->geo.nz * sizeof(double), cudaMemcpyHostToDevice, st));
        ctx->inlet_pending = 0;
    }
    Inflow inf{ctx->inflow_box, ctx->inflow_nb, ctx->inflow_dx, ctx->inlet_plane_valid ? ctx->inlet_plane : nullptr};
    ctx->inlet_plane_valid = 0;
    dim3 grid(face_blocks(ctx), 3);
    LAUNCH(FALM_K_UBC, st, k_ubc<T><<<grid, 256, 0, st>>>(ctx->geo, ctx->bc_kind, u, up, ctx->m64.x[0], dt, t, ctx->u_inlet, inf, t_dev));
    return FALM_OK;
}

// the RMCP forcing into ff over the turbines' boxes; torque and thrust sums
// into ctx->rmcp_sums (device)
template <typename T>
int rmcp_run_t(falm_ctx *ctx, const T *u, T *ff, int *flag, double t, cudaStream_t st, const double *t_dev = nullptr) {
    const RmcpDev &a = *ctx->rmcp;
    const long long blocks = std::max(1LL, std::min<long long>((a.bs.total + 255) / 256, (long long)ctx->sm_count * 8));
    // 2 x kMaxTurbines values per block: a quarter of the workspace's blocks
    const RedWork rw{ctx->red.partials, ctx->red.counter, ctx->red.maxBlocks / 4};
    LAUNCH(FALM_K_ALM, st, k_rmcp<T><<<(int)blocks, 256, 0, st>>>(ctx->geo, a, ctx->m64.x[0], ctx->m64.x[1], ctx->m64.x[2], u, ff, flag, t, rw,
                                                                 ctx->rmcp_sums, t_dev));
    return FALM_OK;
}

// A wait on an mbarrier that nothing ever completes, through the same bounded
// wait the plane-stream kernels use: it gives up after `cycles` clock64 cycles
// and records FALM_ERR_TIMEOUT in the device error word.  No copy is issued,
// so nothing is left in flight when the block returns.
__global__ void k_wait_probe(int *err, long long cycles) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait_cycles(&bar, 0, err, cycles);
    __syncthreads();
}

// The phases of the step before and after the Poisson solve, shared by the
// host-driven step and the recorded one: t_dev is the recorded step's time in
// device memory (NULL: the host passes t), phase the NVTX phases (or NULL).
template <typename T>
int step_pre_t(falm_ctx *ctx, const falm_fields *f, double dt, double t, cudaStream_t st, const double *t_dev, bool *fused_res_out,
               NvtxPhases *phase) {
    int rc;
    const Geom &g = ctx->geo;
    T *u = (T *)f->u, *uu = (T *)f->uu, *p = (T *)f->p, *nut = (T *)f->nut, *ff = (T *)f->ff;
    T *ua = (T *)ctx->w_ua, *rhs = (T *)ctx->w_rhs;
    const bool chan = ctx->bc_kind == FALM_BC_CHANNEL;
    bool fused_res = false;
    // recording: the guide-shell copy (u -> ua) and, in a channel, the saved
    // outlet velocity (u -> w_outlet, read by the velocity BC after the
    // projection) depend only on the step's input velocity, so they run on a
    // side branch beside the forcing and the pseudo-velocity, which write
    // neither; the branch joins before the face-velocity pass reads ua
    const bool side = t_dev && ctx->side_stream;
    if (side) {
        const cudaStream_t ss = ctx->side_stream;
        CK(cudaEventRecord(ctx->side_fork, st));
        CK(cudaStreamWaitEvent(ss, ctx->side_fork, 0));
        LAUNCH(FALM_K_OTHER, ss, k_copy_shell<T><<<ctx->sm_count * 8, 256, 0, ss>>>(g, u, ua));
        if (chan) { LAUNCH(FALM_K_OTHER, ss, k_save_outlet<T><<<std::min(ctx->sm_count * 4, (3 * g.sy * g.sz + 255) / 256), 256, 0, ss>>>(g, u, (T *)ctx->w_outlet)); }
        CK(cudaEventRecord(ctx->side_join, ss));
    }
    // 1. ALM (src/alm/alm.h:66-77) at the previous velocity, or the RMCP model
    if (phase) phase->next("forcing");
    if (ctx->alm_on) {
        if ((rc = alm_run_t<T>(ctx, u, ff, t, st, t_dev))) return rc;
    } else if (ctx->rmcp_on) {
        ff = (T *)ctx->w_ff;
        if ((rc = rmcp_run_t<T>(ctx, u, ff, nullptr, t, st, t_dev))) return rc;
    }
    // 2. pseudo-velocity into ua (ALM force projected in-kernel when ff == NULL)
    if (phase) phase->next("pseudo_velocity");
    if ((rc = pseudo_u_t<T>(ctx, u, u, uu, ua, nut, ff, dt, ctx->alm_on != 0, st))) return rc;
    // 3. face velocity + [uubc] + RHS in one pass
    if (phase) phase->next("face_velocity_rhs");
    {
        const Region3 R = facemap(g);
        T scale = (T)(1.0 / (dt * ctx->maxdiag));
        // the guide layer of ua takes the previous velocity (the reference's aliased u)
        if (side) CK(cudaStreamWaitEvent(st, ctx->side_join, 0));
        else LAUNCH(FALM_K_OTHER, st, k_copy_shell<T><<<ctx->sm_count * 8, 256, 0, st>>>(g, u, ua));
        // the plane stream also computes the solve's first residual (rr) and
        // first preconditioner sweep (pp) from the pressure p, the initial guess
        fused_res = false;
        if (!ctx->A_explicit && ctx->ls_type == FALM_LS_PBICGSTAB && (ctx->pc_type == FALM_LS_SOR || ctx->pc_type == FALM_LS_JACOBI)) {
            if ((rc = ensure_work(ctx))) return rc;
            if (t_dev) {   // recording: the solver start as a kernel (the mixed pass limit included)
                const int pass_its = ctx->precision == FALM_MIXED ? std::min(ctx->maxit, kMixedPassIts) : ctx->maxit;
                LAUNCH(FALM_K_OTHER, st, k_solver_init<<<1, 1, 0, st>>>(ctx->scal, (double)g.nx * g.ny * g.nzg, ctx->tol, pass_its));
            } else if ((rc = solver_init(ctx, st))) {
                return rc;
            }
            T *ppt = pc_first_in_xp<T>(ctx) ? (T *)ctx->w_xp : (T *)ctx->w_pp;
            const void *const fp[2] = {ua, p};
            const int nc[2] = {3, 1};
            int s3;
            if (chan)
                s3 = p3_launch<T, 2, 2>(ctx, FALM_K_UTOUU_RHS, st, R, 1, fp, nc,
                                        UtoUUResBody<T, false>{UtoUUBody<T, true, false>{g, mview<T>(ctx), uu, rhs, scale}, mview<T>(ctx),
                                                               op7<T>(ctx), (T *)ctx->w_rr, ppt, ctx->pc_type, (T)ctx->pc_relax, ctx->scal});
            else
                s3 = p3_launch<T, 2, 2>(ctx, FALM_K_UTOUU_RHS, st, R, 1, fp, nc,
                                        UtoUUResBody<T, true>{UtoUUBody<T, true, true>{g, mview<T>(ctx), uu, rhs, scale}, mview<T>(ctx),
                                                              op7<T>(ctx), (T *)ctx->w_rr, ppt, ctx->pc_type, (T)ctx->pc_relax, ctx->scal});
            if (s3 < 0) return -s3;
            fused_res = s3 == 1;
        }
        if (!fused_res) {
            if (chan)
                P3_OR(FALM_K_UTOUU_RHS, st, T, 1, 0, R, 1, FB_ARR(ua), FB_ARR(3), (UtoUUBody<T, true, false>{g, mview<T>(ctx), uu, rhs, scale}),
                      (k_utouu<T, true, false><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), ua, u, uu, rhs, scale)));
            else
                P3_OR(FALM_K_UTOUU_RHS, st, T, 1, 0, R, 1, FB_ARR(ua), FB_ARR(3), (UtoUUBody<T, true, true>{g, mview<T>(ctx), uu, rhs, scale}),
                      (k_utouu<T, true, true><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), ua, u, uu, rhs, scale)));
        }
    }
    *fused_res_out = fused_res;
    return FALM_OK;
}

template <typename T>
int step_post_t(falm_ctx *ctx, const falm_fields *f, double dt, double t, cudaStream_t st, const double *t_dev, NvtxPhases *phase) {
    int rc;
    const Geom &g = ctx->geo;
    T *u = (T *)f->u, *uu = (T *)f->uu, *p = (T *)f->p, *nut = (T *)f->nut;
    T *ua = (T *)ctx->w_ua;
    const bool chan = ctx->bc_kind == FALM_BC_CHANNEL;
    // 5. pbc
    if (phase) phase->next("projection_bcs");
    LAUNCH(FALM_K_PBC, st, k_pbc<T><<<dim3(face_blocks(ctx), 3), 256, 0, st>>>(g, ctx->bc_kind, p));
    // 6. keep the previous velocity at the outlet planes (a recorded step did it
    // on its side branch), then project
    if (chan && !(t_dev && ctx->side_stream)) { LAUNCH(FALM_K_OTHER, st, k_save_outlet<T><<<std::min(ctx->sm_count * 4, (3 * g.sy * g.sz + 255) / 256), 256, 0, st>>>(g, u, (T *)ctx->w_outlet)); }
    {
        const Region3 R = facemap(g);
        P3_OR(FALM_K_PROJECT, st, T, 1, 0, R, 1, FB_ARR(p), FB_ARR(1), (ProjectBody<T>{g, mview<T>(ctx), u, ua, uu, uu, (T)dt}),
              (k_project<T><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), u, ua, uu, uu, p, (T)dt)));
    }
    // 7. ubc
    if ((rc = ubc_t<T>(ctx, u, UPrev<T>{(const T *)ctx->w_outlet, 1}, dt, t, st, t_dev))) return rc;
    // 8. SGS + divergence norm
    if (phase) phase->next("sgs_divergence");
    {
        const Region3 R = interior(g);
        P3_OR(FALM_K_SGS_DIV, st, T, 2, 1, R, 2, FB_ARR(u, uu), FB_ARR(3, 3),
              (SgsDivBody<T>{g, mview<T>(ctx), ctx->m64, nut, (T)ctx->Cs, ctx->sgs, (T *)nullptr, &ctx->scal->red[3]}),
              (k_sgs_div<T, true><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), ctx->m64, u, nut, (T)ctx->Cs, ctx->sgs, uu,
                                                                            nullptr, ctx->red, &ctx->scal->red[3])));
    }
    return FALM_OK;
}

// the step's results into the pinned host copies
int step_stats_copy(falm_ctx *ctx, cudaStream_t st) {
    CK(cudaMemcpyAsync(ctx->scal_host, ctx->scal, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
    if (ctx->alm_on) CK(cudaMemcpyAsync(ctx->alm_scal_host, ctx->alm.scal, sizeof(AlmScalars), cudaMemcpyDeviceToHost, st));
    if (ctx->rmcp_on) CK(cudaMemcpyAsync(ctx->rmcp_sums_host, ctx->rmcp_sums, 2 * kMaxTurbines * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&ctx->scal_host->kerr, ctx->kerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    return FALM_OK;
}

// after the step's synchronisation: the device error word, then the statistics
int step_finish(falm_ctx *ctx, cudaStream_t st, falm_step_stats *out, int it, double err, int outer, int solve_status) {
    const Geom &g = ctx->geo;
    if (ctx->scal_host->kerr) {
        cudaMemsetAsync(ctx->kerr, 0, sizeof(int), st);
        std::string m = "step: device error word " + std::to_string(ctx->scal_host->kerr) +
                        (ctx->scal_host->kerr >= 300 ? " (a staged stencil neighbourhood failed its self-check)"
                         : ctx->scal_host->kerr >= 200 ? " (a TMA load request failed its self-check)" : " (a bounded wait gave up)");
        *ctx->last_error = m;
        return ctx->scal_host->kerr >= 200 ? FALM_ERR_ARG : FALM_ERR_TIMEOUT;
    }
    if (out) {
        memset(out, 0, sizeof(*out));
        out->it = it;
        out->err = err;
        out->outer = outer;
        out->status = solve_status;
        out->divnorm = std::sqrt(ctx->scal_host->red[3]) / ((double)g.nx * g.ny * g.nz);
        if (ctx->alm_on)
            for (int q = 0; q < ctx->alm.n_turbine && q < kMaxTurbines; q++) {
                out->torque[q] = ctx->alm_scal_host->torque[q];
                out->thrust[q] = ctx->alm_scal_host->thrust[q];
            }
        if (ctx->rmcp_on)
            for (int q = 0; q < ctx->rmcp->n_turbine && q < kMaxTurbines; q++) {
                out->torque[q] = ctx->rmcp_sums_host[q];
                out->thrust[q] = ctx->rmcp_sums_host[kMaxTurbines + q];
            }
    }
    return FALM_OK;
}

// Whole steps as CUDA graphs (see use_graph): the phases before the solve, the solve with its
// loops on the device (solve_t's recording), the phases after it and the
// copies of the results, recorded once per set of fields and dt; the time goes
// in through device memory, written by the graph's first node from a pinned
// host value; a streamed inlet plane (falm_bc_set_inlet_plane, copied into
// the context's fixed plane buffer before the step) makes a recording of its
// own.  Not for z slabs, the plain solvers or an explicit matrix.
template <typename T>
bool step_graph_ok(const falm_ctx *ctx) {
    return use_graph(ctx) && !ctx->slab_on && ctx->wait_probe_cycles == 0 && ctx->op_ready &&
           !ctx->A_explicit && ctx->ls_type == FALM_LS_PBICGSTAB && (ctx->pc_type == FALM_LS_SOR || ctx->pc_type == FALM_LS_JACOBI);
}

template <typename T>
int step_graph_t(falm_ctx *ctx, const falm_fields *f, double dt, double t, cudaStream_t st, falm_step_stats *out) {
    falm_ctx::StepGraph *sg = nullptr;
    const int inlet = ctx->inlet_plane_valid ? 1 : 0;
    for (auto &e : *ctx->step_graphs)
        if (e.u == f->u && e.uu == f->uu && e.p == f->p && e.nut == f->nut && e.ff == f->ff && e.dt == dt && e.inlet == inlet) sg = &e;
    if (!sg) {
        if (!ctx->cap_stream) CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
        if (!ctx->side_stream) {
            CK(cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&ctx->side_fork, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->side_join, cudaEventDisableTiming));
        }
        if (!ctx->t_dev) {
            CK(cudaMalloc(&ctx->t_dev, sizeof(double)));
            CK(cudaHostAlloc(&ctx->t_host, sizeof(double), cudaHostAllocDefault));
        }
        const cudaStream_t cs = ctx->cap_stream;
        cudaGraph_t gr = nullptr;
        CK(cudaGraphCreate(&gr, 0));
        SolveRec rec;
        rec.graph = gr;
        bool fused = false;
        const long long l0 = ctx->launches;
        int rc = capture_into(ctx, gr, rec.deps, [&]() -> int {
            CK(cudaMemcpyAsync(ctx->t_dev, ctx->t_host, sizeof(double), cudaMemcpyHostToDevice, cs));
            return step_pre_t<T>(ctx, f, dt, t, cs, ctx->t_dev, &fused, nullptr);
        });
        const long long n_pre = ctx->launches - l0;
        ctx->launches = l0;
        int it = 0, outer = 0;
        double err = 0;
        if (!rc) rc = solve_t<T>(ctx, (T *)f->p, (const T *)ctx->w_rhs, (T *)ctx->w_r, st, &it, &err, &outer, fused, &rec);
        // a streamed inlet plane: its copy as a root node that runs beside the
        // phases before the velocity BC (its source is set at every launch)
        cudaGraphNode_t inlet_node = nullptr;
        if (!rc && inlet) {
            if (cudaGraphAddMemcpyNode1D(&inlet_node, gr, nullptr, 0, ctx->inlet_plane, ctx->inlet_host,
                                         3ull * ctx->geo.ny * ctx->geo.nz * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
                cudaGetLastError();
                rc = fail(ctx, FALM_ERR_CUDA, "step graph: inlet copy node");
            } else {
                rec.deps.push_back(inlet_node);
            }
        }
        if (!rc) rc = capture_into(ctx, gr, rec.deps, [&]() -> int {
            int q = step_post_t<T>(ctx, f, dt, t, cs, ctx->t_dev, nullptr);
            if (!q) q = step_stats_copy(ctx, cs);
            return q;
        });
        const long long n_post = ctx->launches - l0;
        ctx->launches = l0;
        cudaGraphExec_t ex = nullptr;
        if (!rc && cudaGraphInstantiate(&ex, gr, 0) != cudaSuccess) rc = fail(ctx, FALM_ERR_CUDA, "step graph: instantiate");
        cudaGetLastError();
        if (rc) {
            cudaGraphDestroy(gr);
            return rc;
        }
        if (ctx->step_graphs->size() >= kMaxRecordings) {   // many sets of fields: drop the oldest recording
            cudaGraphExecDestroy(ctx->step_graphs->front().exec);
            cudaGraphDestroy(ctx->step_graphs->front().graph);
            ctx->step_graphs->erase(ctx->step_graphs->begin());
        }
        ctx->step_graphs->push_back(falm_ctx::StepGraph{f->u, f->uu, f->p, f->nut, f->ff, dt, inlet, inlet_node, n_pre + rec.fixed + n_post,
                                                        rec.per_iter, gr, ex});
        sg = &ctx->step_graphs->back();
    }
    *ctx->t_host = t;
    if (inlet)
        CK(cudaGraphExecMemcpyNodeSetParams1D(sg->exec, sg->inlet_node, ctx->inlet_plane, ctx->inlet_host,
                                              3ull * ctx->geo.ny * ctx->geo.nz * sizeof(double), cudaMemcpyHostToDevice));
    ctx->inlet_plane_valid = 0;   // the streamed plane serves one step
    ctx->inlet_pending = 0;
    CK(cudaGraphLaunch(sg->exec, st));
    CK(cudaStreamSynchronize(st));
    const SolverScalars &sh = *ctx->scal_host;
    ctx->launches += sg->fixed + sg->per_iter * std::max(0, sh.it_total);
    if (sh.status == FALM_ERR_NAN) return fail(ctx, FALM_ERR_NAN, "solve: non-finite scalar");
    return step_finish(ctx, st, out, sh.it_total, sh.err, std::max(1, sh.passes), sh.status);
}

template <typename T>
int step_t(falm_ctx *ctx, const falm_fields *f, double dt, double t, cudaStream_t st, falm_step_stats *out) {
    NvtxRange whole("falm_step");
    NvtxPhases phase;
    int rc = ensure_work(ctx);
    if (rc) return rc;
    if (ctx->wait_probe_cycles > 0) {   // armed by falm_debug_arm_wait_probe: one step only
        const long long cycles = ctx->wait_probe_cycles;
        ctx->wait_probe_cycles = 0;
        LAUNCH(FALM_K_OTHER, st, k_wait_probe<<<1, 32, 0, st>>>(ctx->kerr, cycles));
    }
    if (!ctx->op_ready) {
        if ((rc = build_poisson(ctx, ctx->bc_kind))) return rc;
    }
    if (step_graph_ok<T>(ctx)) return step_graph_t<T>(ctx, f, dt, t, st, out);
    bool fused_res = false;
    if ((rc = step_pre_t<T>(ctx, f, dt, t, st, nullptr, &fused_res, &phase))) return rc;
    // 4. Poisson
    phase.next("poisson");
    int it = 0, outer = 1;
    double err = 0;
    rc = solve_t<T>(ctx, (T *)f->p, (const T *)ctx->w_rhs, (T *)ctx->w_r, st, &it, &err, &outer, fused_res);
    const int solve_status = ctx->scal_host->status;
    if (rc) return rc;
    if ((rc = step_post_t<T>(ctx, f, dt, t, st, nullptr, &phase))) return rc;
    if ((rc = step_stats_copy(ctx, st))) return rc;
    CK(cudaStreamSynchronize(st));
    return step_finish(ctx, st, out, it, err, outer, solve_status);
}
