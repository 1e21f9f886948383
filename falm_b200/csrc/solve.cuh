// The solvers of FalmEq::Solve on the device: the plain Jacobi/SOR loops,
// PBiCGStab with its host-driven and recorded (CUDA graph) forms, and the
// inner product of the host API.
// Included by falm_b200.cu inside its anonymous namespace (after the headers
// it includes and the code before this point); not a standalone header.
#pragma once

// ---------------------------------------------------------------- solver driver
// solver scalars at the start of a solve
int solver_init(falm_ctx *ctx, cudaStream_t st) {
    const Geom &g = ctx->geo;
    SolverScalars init;
    memset(&init, 0, sizeof(init));
    init.gsize = (double)g.nx * g.ny * g.nzg;   // interior cells of the whole grid (of all slabs)
    init.tol = ctx->tol;
    init.maxit = ctx->maxit;
    CK(cudaMemcpyAsync(ctx->scal, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    return FALM_OK;
}

// The plain solvers of FalmEq::Solve (src/FalmEq.h:56-64): Jacobi
// (src/FalmEq.cpp:80-127) and red-black SOR (:173-240, the Black half sweep then
// the Red one, with the solver's relaxation factor).  Each iteration ends with
// the residual r = b - A x and the loop test (k_res_plain).  Iterations are
// queued in batches of 1, 2, 4, 8, 8, ... between host checks of the stop
// flag, and every kernel of an iteration queued after the stop returns at once.
// Jacobi alternates between x and the work vector xp instead of copying x to
// xp each iteration: after one copy of x (ghosts included) the ghost cells of
// both agree, iteration n reads {x, xp}[n % 2] and writes the other, and an odd
// final count copies the result back into x.
template <typename T>
int plain_solve_t(falm_ctx *ctx, T *x, const T *b, T *r, cudaStream_t st, int *it_out, double *err_out, int *outer_out) {
    int rc = solver_init(ctx, st);
    if (rc) return rc;
    const Geom &g = ctx->geo;
    const Region3 R = interior(g);
    const int grid = row_grid(ctx, R);
    const Op7<T> op = op7<T>(ctx);
    SolverScalars *sc = ctx->scal;
    T *xp = (T *)ctx->w_xp;
    const bool jac = ctx->ls_type == FALM_LS_JACOBI;
    const T w = (T)ctx->relax;
    if (jac) CK(cudaMemcpyAsync(xp, x, (size_t)g.n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    int batch = 1, queued = 0;
    for (int n = 0;; n++) {
        T *dst = x;
        if (jac) {
            const T *src = (n & 1) ? xp : x;
            dst = (n & 1) ? x : xp;
            LAUNCH(FALM_K_SOR, st, k_jacobi<T><<<grid, kRowThreads, 0, st>>>(g, R, op, dst, src, b, sc));
        } else {
            for (int color = 0; color < 2; color++)
                S7_OR(FALM_K_SOR, st, T, 0, x, (SorBody<T>{op, x, b, w, color, sc}),
                      (k_sor<T><<<grid, kRowThreads, 0, st>>>(g, R, op, x, b, w, color, sc)));
        }
        LAUNCH(FALM_K_RES, st, k_res_plain<T><<<grid, kRowThreads, 0, st>>>(g, R, op, dst, b, r, ctx->red, sc));
        if (++queued < batch) continue;
        CK(cudaMemcpyAsync(ctx->scal_host, sc, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (ctx->scal_host->done) break;
        queued = 0;
        batch = std::min(2 * batch, 8);
    }
    const int it = ctx->scal_host->it;
    if (jac && (it & 1)) CK(cudaMemcpyAsync(x, xp, (size_t)g.n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    if (it_out) *it_out = it;
    if (err_out) *err_out = ctx->scal_host->err;
    if (outer_out) *outer_out = 1;
    return ctx->scal_host->status == FALM_ERR_NAN ? fail(ctx, FALM_ERR_NAN, "solve: non-finite residual") : FALM_OK;
}

// ---------------------------------------------------------------- device-side BiCGStab loop
// A pass's iterations as one CUDA graph: iterations 0 and 1 of the pass, then
// a conditional while node whose body is one later iteration; the last kernel
// of the prefix and of the body sets the loop condition from the solver's done
// flag (convergence, maxit, breakdown or a non-finite scalar), so the loop ends
// on the device within maxit iterations.  Graphs are kept per solve signature
// (vectors, element type, whether the first preconditioner sweep is ready) and
// dropped when the solver settings or the operator change.  Used by default
// (FALM_B200_GRAPH=0 turns it off), never while profiling or checking launches
// one by one: the unconditional iteration 1 and the condition kernels cost
// less than the host round trips they replace, even at 1-2 iterations per
// step on the 512x256x256 grid.
constexpr int kMixedPassIts = 50;   // FP32 BiCGStab iterations between FP64 true-residual checks
constexpr size_t kMaxRecordings = 16;   // recorded solves (and steps) kept per context

bool use_graph(const falm_ctx *ctx) {
    return !(ctx->profiling || ctx->check_sync || ctx->graph_mode == 0);
}

__global__ void k_graph_continue(const SolverScalars *sc, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, sc->done ? 0u : 1u);
}

// drop every recorded loop and step (the settings they were recorded with changed)
void graphs_clear(falm_ctx *ctx) {
    if (ctx->graphs) {
        for (auto &e : *ctx->graphs) {
            cudaGraphExecDestroy(e.exec);
            cudaGraphDestroy(e.graph);
        }
        ctx->graphs->clear();
    }
    if (ctx->step_graphs) {
        for (auto &e : *ctx->step_graphs) {
            cudaGraphExecDestroy(e.exec);
            cudaGraphDestroy(e.graph);
        }
        ctx->step_graphs->clear();
    }
}

// ---- recording on the device: the solver control the host loop does otherwise
// the scalars of a solve's start (solver_init on the device)
__global__ void k_solver_init(SolverScalars *sc, double gsize, double tol, int maxit) {
    SolverScalars z;
    memset(&z, 0, sizeof(z));
    z.gsize = gsize;
    z.tol = tol;
    z.maxit = maxit;
    *sc = z;
}
// a pass has ended: its iterations into the totals
__global__ void k_pass_end(SolverScalars *sc) {
    sc->it_total += sc->it;
    sc->passes += 1;
}
// a new pass: iteration count zero, the pass's limit
__global__ void k_pass_reset(SolverScalars *sc, int maxit) {
    sc->it = 0;
    sc->maxit = maxit;
}
// after the FP64 check of a mixed pass: another pass while the true residual
// misses the tolerance and passes remain (a breakdown's status is cleared: the
// pass restarts from the true residual); non-finite data ends the solve (done)
__global__ void k_outer_cond(SolverScalars *sc, cudaGraphConditionalHandle h, int max_passes) {
    const bool more = !sc->done && sc->passes < max_passes;
    if (more) sc->status = FALM_OK;
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

// the recording stream's current leaf nodes after fn's launches on it, which go
// into `graph` after `deps` (deps becomes the new leaves)
int capture_into(falm_ctx *ctx, cudaGraph_t graph, std::vector<cudaGraphNode_t> &deps, const std::function<int()> &fn) {
    const cudaStream_t cs = ctx->cap_stream;
    if (cudaStreamBeginCaptureToGraph(cs, graph, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                      cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, FALM_ERR_CUDA, "graph: begin capture");
    }
    int rc = fn();
    cudaStreamCaptureStatus stt;
    const cudaGraphNode_t *d = nullptr;
    size_t nd = 0;
    std::vector<cudaGraphNode_t> leaves;
    if (cudaStreamGetCaptureInfo(cs, &stt, nullptr, nullptr, &d, &nd) == cudaSuccess && d) leaves.assign(d, d + nd);
    cudaGraph_t got = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cs, &got);
    cudaGetLastError();
    if (!rc && (e != cudaSuccess || got != graph)) rc = fail(ctx, FALM_ERR_CUDA, "graph: end capture");
    if (!rc && !leaves.empty()) deps = leaves;
    return rc;
}

// a conditional while node after deps (deps becomes the node); its body graph in *body
int add_while(falm_ctx *ctx, cudaGraph_t graph, std::vector<cudaGraphNode_t> &deps, cudaGraphConditionalHandle h, cudaGraph_t *body) {
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};   // every other byte zero
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, graph, deps.empty() ? nullptr : deps.data(), deps.size(), &cp) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, FALM_ERR_CUDA, "graph: while node");
    }
    deps.assign(1, node);
    *body = cp.conditional.phGraph_out[0];
    return FALM_OK;
}

// a solve recorded into a graph after deps (see solve_t); counts the kernels
// recorded outside and inside the iteration loops
struct SolveRec {
    cudaGraph_t graph;
    std::vector<cudaGraphNode_t> deps;
    long long fixed = 0, per_iter = 0;
};

// the graph of a pass (built on first use: emit(itp) launches iteration itp's
// kernels on `ist`, which points at the capture stream meanwhile); prefix and
// per_iter: kernel launches of iterations 0-1 and of one later iteration
int solve_graph(falm_ctx *ctx, const void *x, const void *b, const void *r, int esize, int pp_ready,
                const std::function<int(int)> &emit, cudaStream_t &ist, cudaGraphExec_t *out, int *prefix, int *per_iter) {
    for (auto &e : *ctx->graphs)
        if (e.x == x && e.b == b && e.r == r && e.w0 == ctx->w_rr && e.A == ctx->A_explicit && e.esize == esize && e.pp_ready == pp_ready) {
            *out = e.exec; *prefix = e.prefix; *per_iter = e.per_iter;
            return FALM_OK;
        }
    if (!ctx->cap_stream) CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
    cudaGraph_t gr = nullptr;
    CK(cudaGraphCreate(&gr, 0));
    cudaGraphConditionalHandle h;
    cudaGraphExec_t ex = nullptr;
    const cudaStream_t saved = ist;
    ist = ctx->cap_stream;
    // capture iterations first..last and the condition kernel into `into`
    auto capture = [&](cudaGraph_t into, int first, int last, int *count) -> int {
        if (cudaStreamBeginCaptureToGraph(ist, into, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
            return fail(ctx, FALM_ERR_CUDA, "solve graph: capture");
        const long long l0 = ctx->launches;
        int crc = FALM_OK;
        for (int itp = first; itp <= last && !crc; itp++) crc = emit(itp);
        if (!crc) {
            k_graph_continue<<<1, 1, 0, ist>>>(ctx->scal, h);
            if (cudaGetLastError() != cudaSuccess) crc = fail(ctx, FALM_ERR_CUDA, "solve graph: condition kernel");
        }
        *count = (int)(ctx->launches - l0);
        ctx->launches = l0;
        cudaGraph_t got = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ist, &got);
        if (!crc && (e != cudaSuccess || got != into)) crc = fail(ctx, FALM_ERR_CUDA, "solve graph: end of capture");
        cudaGetLastError();
        return crc;
    };
    int rc = FALM_OK, np = 0, nb = 0;
    if (cudaGraphConditionalHandleCreate(&h, gr, 1, cudaGraphCondAssignDefault) != cudaSuccess) rc = fail(ctx, FALM_ERR_CUDA, "solve graph: handle");
    if (!rc) rc = capture(gr, 0, 1, &np);
    if (!rc) {
        // the loop follows the prefix's last node(s)
        size_t nn = 0, ne = 0;
        cudaGraphGetNodes(gr, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (nn) cudaGraphGetNodes(gr, nodes.data(), &nn);
        cudaGraphGetEdges(gr, nullptr, nullptr, &ne);
        std::vector<cudaGraphNode_t> from(ne), to(ne);
        if (ne) cudaGraphGetEdges(gr, from.data(), to.data(), &ne);
        std::vector<cudaGraphNode_t> leaves;
        for (auto nd : nodes)
            if (std::find(from.begin(), from.end(), nd) == from.end()) leaves.push_back(nd);
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};   // every other byte zero
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        if (cudaGraphAddNode(&cn, gr, leaves.data(), leaves.size(), &cp) != cudaSuccess) rc = fail(ctx, FALM_ERR_CUDA, "solve graph: loop node");
        else rc = capture(cp.conditional.phGraph_out[0], 2, 2, &nb);
    }
    if (!rc && cudaGraphInstantiate(&ex, gr, 0) != cudaSuccess) rc = fail(ctx, FALM_ERR_CUDA, "solve graph: instantiate");
    ist = saved;
    cudaGetLastError();
    if (rc) {
        if (ex) cudaGraphExecDestroy(ex);
        cudaGraphDestroy(gr);
        return rc;
    }
    if (ctx->graphs->size() >= kMaxRecordings) {   // a caller cycling through many vectors: drop the oldest
        cudaGraphExecDestroy(ctx->graphs->front().exec);
        cudaGraphDestroy(ctx->graphs->front().graph);
        ctx->graphs->erase(ctx->graphs->begin());
    }
    ctx->graphs->push_back(falm_ctx::SolveGraph{x, b, r, ctx->w_rr, ctx->A_explicit, esize, pp_ready, np, nb, gr, ex});
    *out = ex; *prefix = np; *per_iter = nb;
    return FALM_OK;
}

template <typename T>
int solve_t(falm_ctx *ctx, T *x, const T *b, T *r, cudaStream_t st, int *it_out, double *err_out, int *outer_out,
            bool first_res_done = false, SolveRec *rec = nullptr) {
    NvtxRange range("falm_solve");
    int rc = ensure_work(ctx);
    if (rc) return rc;
    if (!ctx->op_ready && !ctx->A_explicit) return fail(ctx, FALM_ERR_STATE, "solve: no operator (call falm_eq_poisson_operator or falm_eq_set_matrix)");
    if (ctx->ls_type == FALM_LS_JACOBI || ctx->ls_type == FALM_LS_SOR) {
        if (first_res_done || rec) return fail(ctx, FALM_ERR_STATE, "solve: a BiCGStab start was prepared for a plain solver");
        return plain_solve_t<T>(ctx, x, b, r, st, it_out, err_out, outer_out);
    }
    if (ctx->ls_type != FALM_LS_PBICGSTAB) return fail(ctx, FALM_ERR_ARG, "solve: unknown linear solver type");
    const Geom &g = ctx->geo;
    const Region3 R = interior(g);
    const int grid = row_grid(ctx, R);
    const int grid_p = row_grid_wave(ctx, R, k_bicg_p<T>), grid_s = row_grid_wave(ctx, R, k_bicg_s<T>);
    const int grid_xr = row_grid_wave(ctx, R, k_bicg_xr<T>);
    const Op7<T> op = op7<T>(ctx);
    T *rr = (T *)ctx->w_rr, *p = (T *)ctx->w_p, *q = (T *)ctx->w_q, *s = (T *)ctx->w_s, *pp = (T *)ctx->w_pp;
    T *ss = (T *)ctx->w_ss, *t = (T *)ctx->w_t, *xp = (T *)ctx->w_xp;
    // first_res_done: the caller initialised the scalars (solver_init) and a
    // kernel of its own already computed the first pass's residual into rr with
    // the first preconditioner sweep into pp (the step's face-velocity kernel)
    if (!first_res_done && !rec && (rc = solver_init(ctx, st))) return rc;
    const T pcw = (T)ctx->pc_relax;
    const int pct = ctx->pc_type, m = ctx->pc_maxit;
    SolverScalars *sc = ctx->scal;
    int total_it = 0, outer = 0;
    const bool mixed = ctx->precision == FALM_MIXED;
    // Mixed precision: a pass runs at most kMixedPassIts FP32 iterations before
    // the FP64 true residual replaces the recursive one (a check, then a new
    // pass from it), and as many passes as maxit needs: over longer FP32
    // recursions BiCGStab diverged on the nearly singular operator of a long
    // channel (unit-norm right-hand sides at 512x128x128).
    const int pass_its = mixed ? std::min(ctx->maxit, kMixedPassIts) : ctx->maxit;
    const int max_outer = mixed ? std::max(ctx->max_outer, (ctx->maxit + kMixedPassIts - 1) / kMixedPassIts) : 1;
    // the stream of the iteration kernels: st, or the capture stream while a
    // device-side loop (CUDA graph) is recorded
    cudaStream_t ist = st;
    const bool first_xp = pc_first_in_xp<T>(ctx);
    auto first_target = [&](T *z) -> T * { return first_xp ? xp : z; };
    // launch the remaining sweeps of one preconditioner application z ~ A^-1 v
    // (the first, pointwise sweep wrote first_target(z)); the temporally blocked
    // sweeps run out of place, alternating between xp and z
    auto precondition_rest = [&](T *z, const T *v) -> int {
        if (pct == FALM_LS_SOR) {
            int hs = 1;
            T *src = first_target(z);
            while (hs < 2 * m) {                       // up to 3 half sweeps per pass over HBM
                const int H = std::min(3, 2 * m - hs);
                T *dst = src == z ? xp : z;
                const int lr = sor_rb_launch<T>(ctx, ist, H, src, v, dst, pcw, hs & 1, sc);
                if (lr < 0) return -lr;
                if (lr == 0) break;
                src = dst;
                hs += H;
            }
            // a pass declined after all (pc_first_in_xp checks the same conditions)
            if (src != z) CK(cudaMemcpyAsync(z, src, (size_t)g.n * sizeof(T), cudaMemcpyDeviceToDevice, ist));
            for (; hs < 2 * m; hs++) {                // red, then (black, red) x (m-1)
                const int color = hs & 1;
                S7_OR(FALM_K_SOR, ist, T, 0, z, (SorBody<T>{op, z, v, pcw, color, sc}),
                      (k_sor<T><<<grid, kRowThreads, 0, ist>>>(g, R, op, z, v, pcw, color, sc)));
            }
        } else if (pct == FALM_LS_JACOBI) {
            // sweeps 2..m ping-pong between xp and z; the first sweep wrote to
            // the buffer that makes the last one land in z
            T *bufs[2] = {z, xp};
            for (int it = 2; it <= m; it++) {
                T *dst = bufs[(m - it) & 1], *src = bufs[(m - it + 1) & 1];
                LAUNCH(FALM_K_SOR, ist, k_jacobi<T><<<grid, kRowThreads, 0, ist>>>(g, R, op, dst, src, v, sc));
            }
        }
        return FALM_OK;
    };
    // a pass's residual also gives the first iteration's first preconditioner
    // sweep (pp_ready: the stream kernel stored it, so k_bicg_p is skipped)
    bool pp_ready = first_res_done;
    auto res_pass = [&](int check) -> int {
        int s7;
        if (check) {
            s7 = s7_launch<T, 1>(ctx, FALM_K_RES, ist, x, ResBody<T, true>{op, b, nullptr, nullptr, sc, 1});
        } else {
            ResBody<T> body{op, b, nullptr, rr, sc, 0};
            body.pp = first_target(pp); body.pc_type = pct; body.pc_omega = pcw;
            s7 = s7_launch<T, 2>(ctx, FALM_K_RES, ist, x, body);
        }
        if (s7 < 0) return -s7;
        if (s7 == 0) LAUNCH(FALM_K_RES, ist, (k_res<T><<<grid, kRowThreads, 0, ist>>>(g, R, op, x, b, r, rr, ctx->red, sc, check)));
        pp_ready = !check && s7 == 1;
        return FALM_OK;
    };
    // a new pass: iteration count zero, the pass's iteration limit
    static_assert(offsetof(SolverScalars, maxit) == offsetof(SolverScalars, it) + sizeof(int), "it, maxit adjacent");
    auto zero_it = [&]() -> int {
        const int itmax[2] = {0, pass_its};   // SolverScalars::it, ::maxit
        CK(cudaMemcpyAsync(&sc->it, itmax, sizeof(itmax), cudaMemcpyHostToDevice, st));
        return FALM_OK;
    };
    // the kernels of iteration itp of the pass (2 stands for every later
    // one): r equals rr until the first k_bicg_xr, and the first
    // iteration's p equals r, so it reads rr in their place
    auto emit_iter = [&](int itp) -> int {
        const T *rin = itp == 0 ? rr : r;
        T *pout = itp == 0 ? nullptr : p;
        const T *pin = itp == 1 ? rr : p, *pv = itp == 0 ? rr : p;
        int erc;
        if (!(itp == 0 && pp_ready))
            LAUNCH(FALM_K_BICG_P, ist, k_bicg_p<T><<<grid_p, kRowThreads, 0, ist>>>(g, R, op, pout, pin, q, rin, first_target(pp), pct, pcw, sc));
        if ((erc = precondition_rest(pp, pv))) return erc;
        S7_OR(FALM_K_MV_DOT1, ist, T, 1, pp, (MvDot1Body<T>{op, q, rr, sc}),
              (k_mv_dot1<T><<<grid, kRowThreads, 0, ist>>>(g, R, op, pp, q, rr, ctx->red, sc)));
        LAUNCH(FALM_K_BICG_S, ist, k_bicg_s<T><<<grid_s, kRowThreads, 0, ist>>>(g, R, op, s, q, rin, first_target(ss), pct, pcw, sc));
        if ((erc = precondition_rest(ss, s))) return erc;
        S7_OR(FALM_K_MV_DOT2, ist, T, 2, ss, (MvDot2Body<T>{op, t, s, sc}),
              (k_mv_dot2<T><<<grid, kRowThreads, 0, ist>>>(g, R, op, ss, t, s, ctx->red, sc)));
        LAUNCH(FALM_K_BICG_XR, ist, k_bicg_xr<T><<<grid_xr, kRowThreads, 0, ist>>>(g, R, x, pp, ss, r, s, t, rr, ctx->red, sc));
        return FALM_OK;
    };
    if (rec) {
        // The whole solve recorded into rec->graph after rec->deps, with no
        // host decision: pass 0 (solver start and first residual unless the
        // caller recorded them), and in mixed precision a while node of FP64
        // checks and further passes; a pass is iterations 0 and 1 and a while
        // node of later iterations, its condition the done flag.
        ist = ctx->cap_stream;
        const long long l_start = ctx->launches;
        long long fixed = 0, per_iter = 0;
        auto cap = [&](cudaGraph_t gr, std::vector<cudaGraphNode_t> &deps, long long *cnt, const std::function<int()> &fn) -> int {
            const long long l0 = ctx->launches;
            const int crc = capture_into(ctx, gr, deps, fn);
            *cnt += ctx->launches - l0;
            ctx->launches = l0;
            return crc;
        };
        auto cond = [&](cudaGraphConditionalHandle h) -> int {
            k_graph_continue<<<1, 1, 0, ist>>>(sc, h);
            return cudaGetLastError() == cudaSuccess ? FALM_OK : fail(ctx, FALM_ERR_CUDA, "graph: condition kernel");
        };
        auto rec_pass = [&](cudaGraph_t gr, std::vector<cudaGraphNode_t> &deps) -> int {
            cudaGraphConditionalHandle h;
            if (cudaGraphConditionalHandleCreate(&h, gr, 1, cudaGraphCondAssignDefault) != cudaSuccess)
                return fail(ctx, FALM_ERR_CUDA, "graph: handle");
            int e = cap(gr, deps, &fixed, [&]() -> int {
                int q2 = emit_iter(0);
                if (!q2) q2 = emit_iter(1);
                if (!q2) q2 = cond(h);
                return q2;
            });
            cudaGraph_t body = nullptr;
            if (!e) e = add_while(ctx, gr, deps, h, &body);
            std::vector<cudaGraphNode_t> bd;
            long long pi = 0;
            if (!e) e = cap(body, bd, &pi, [&]() -> int {
                int q2 = emit_iter(2);
                if (!q2) q2 = cond(h);
                return q2;
            });
            per_iter = pi;
            if (!e) e = cap(gr, deps, &fixed, [&]() -> int {
                LAUNCH(FALM_K_OTHER, ist, k_pass_end<<<1, 1, 0, ist>>>(sc));
                return FALM_OK;
            });
            return e;
        };
        int e = FALM_OK;
        if (!first_res_done)
            e = cap(rec->graph, rec->deps, &fixed, [&]() -> int {
                LAUNCH(FALM_K_OTHER, ist, k_solver_init<<<1, 1, 0, ist>>>(sc, (double)g.nx * g.ny * g.nzg, ctx->tol, pass_its));
                return res_pass(0);
            });
        if (!e) e = rec_pass(rec->graph, rec->deps);
        if (!e && mixed && max_outer > 1) {
            cudaGraphConditionalHandle ho;
            if (cudaGraphConditionalHandleCreate(&ho, rec->graph, 0, cudaGraphCondAssignDefault) != cudaSuccess)
                e = fail(ctx, FALM_ERR_CUDA, "graph: handle");
            auto check = [&]() -> int {
                int q2 = res_pass(1);
                if (!q2) LAUNCH(FALM_K_OTHER, ist, k_outer_cond<<<1, 1, 0, ist>>>(sc, ho, max_outer));
                return q2;
            };
            if (!e) e = cap(rec->graph, rec->deps, &fixed, check);
            cudaGraph_t ob = nullptr;
            if (!e) e = add_while(ctx, rec->graph, rec->deps, ho, &ob);
            std::vector<cudaGraphNode_t> od;
            if (!e) e = cap(ob, od, &fixed, [&]() -> int {
                LAUNCH(FALM_K_OTHER, ist, k_pass_reset<<<1, 1, 0, ist>>>(sc, pass_its));
                return res_pass(0);
            });
            if (!e) e = rec_pass(ob, od);
            if (!e) e = cap(ob, od, &fixed, check);
        }
        ist = st;
        ctx->launches = l_start;
        rec->fixed += fixed;
        rec->per_iter = per_iter;
        return e;
    }
    if (mixed && pass_its != ctx->maxit)
        CK(cudaMemcpyAsync(&sc->maxit, &pass_its, sizeof(int), cudaMemcpyHostToDevice, st));
    // In mixed precision each pass but the last is followed by a check of the
    // true residual in FP64 (stop when it meets the tolerance; the check stores
    // nothing). The check is queued behind the pass's iterations and runs only
    // once the pass has stopped, so one host synchronisation serves both; where
    // the stream kernel is not available it runs at the start of the next pass.
    // A pass stores its residual in rr only: r equals rr until the pass's first
    // k_bicg_xr, which writes r, and the iteration reads rr before.
    // a device-side loop (CUDA graph) runs a pass's iterations without host
    // checks in between; the FP64 check of a mixed-precision pass then follows
    // it as a kernel of its own
    const bool graph = use_graph(ctx);
    bool explicit_check = graph, pass_queued = first_res_done;
    int passes = 0;   // passes run (a pass whose success an explicit check finds ends the loop at the next outer step)
    bool restart_check = false;   // the previous pass broke down: check the true residual before restarting
    for (outer = 0; outer < max_outer; outer++) {
        if (outer > 0 && (explicit_check || restart_check)) {
            restart_check = false;
            if ((rc = res_pass(1))) return rc;
            CK(cudaMemcpyAsync(ctx->scal_host, sc, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (ctx->scal_host->done) break;
        }
        if (!pass_queued) {
            if ((rc = res_pass(0))) return rc;
            if (outer > 0 && (rc = zero_it())) return rc;
        }
        pass_queued = false;
        const bool want_check = mixed && outer + 1 < max_outer && !explicit_check;
        bool checked = false;
        if (graph) {
            // the whole pass on the device: one graph launch, one host read
            cudaGraphExec_t ge = nullptr;
            int prefix = 0, per_iter = 0;
            if ((rc = solve_graph(ctx, x, b, r, (int)sizeof(T), pp_ready ? 1 : 0, emit_iter, ist, &ge, &prefix, &per_iter))) return rc;
            CK(cudaGraphLaunch(ge, st));
            CK(cudaMemcpyAsync(ctx->scal_host, sc, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            ctx->launches += prefix + (long long)per_iter * std::max(0, ctx->scal_host->it - 2);
        }
        // otherwise iterations are queued in batches of 1, 2, 4, 8, 8, ... between
        // host checks of the convergence flag; every kernel of an iteration
        // queued after convergence returns at once
        int batch = 1, queued = 0;
        for (int itp = 0; !graph; itp++) {
            if ((rc = emit_iter(itp))) return rc;
            if (++queued < batch) continue;
            if (want_check && !explicit_check) {
                ResBody<T, true> cb{op, b, nullptr, nullptr, sc, 1};
                cb.queued_check = 1;
                const int s7 = s7_launch<T, 1>(ctx, FALM_K_RES, st, x, cb);
                if (s7 < 0) return -s7;
                if (s7 == 0) explicit_check = true;
            }
            CK(cudaMemcpyAsync(ctx->scal_host, sc, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (want_check && !explicit_check && ctx->scal_host->checked) { checked = true; break; }
            if (ctx->scal_host->done) break;
            queued = 0;
            batch = std::min(2 * batch, 8);
        }
        total_it += ctx->scal_host->it;
        passes++;
        if (ctx->scal_host->status == FALM_ERR_NAN) {
            // In mixed precision a non-finite alpha or omega of the FP32
            // recursion (a breakdown: the kernels after it skipped, so x is the
            // last iterate) restarts a pass from the FP64 true residual while
            // passes remain; non-finite data ends the solve.
            if (!mixed || outer + 1 >= max_outer) break;
            static const int ok = FALM_OK;
            CK(cudaMemcpyAsync(&sc->status, &ok, sizeof(int), cudaMemcpyHostToDevice, st));
            restart_check = true;
            continue;
        }
        if (checked) {
            if (ctx->scal_host->done) break;   // the true residual meets the tolerance
            if ((rc = res_pass(0))) return rc;
            if ((rc = zero_it())) return rc;
            pass_queued = true;
        }
    }
    if (mixed && outer >= max_outer) {
        // report the true residual of the final iterate
        LAUNCH(FALM_K_RES, st, k_res<T><<<grid, kRowThreads, 0, st>>>(g, R, op, x, b, r, nullptr, ctx->red, nullptr, 0));
    } else if (std::min(outer, max_outer - 1) == 0 && ctx->scal_host->it == 0) {
        // no iteration followed the first residual, which went to rr only
        LAUNCH(FALM_K_RES, st, k_res<T><<<grid, kRowThreads, 0, st>>>(g, R, op, x, b, r, nullptr, ctx->red, nullptr, 0));
    }
    if (it_out) *it_out = total_it;
    if (err_out) *err_out = ctx->scal_host->err;
    if (outer_out) *outer_out = std::max(1, passes);
    return ctx->scal_host->status == FALM_ERR_NAN ? fail(ctx, FALM_ERR_NAN, "solve: non-finite scalar") : FALM_OK;
}

template <typename T>
int dot_t(falm_ctx *ctx, const T *a, const T *b, int ncol, double *out, cudaStream_t st) {
    const Region3 R = interior(ctx->geo);
    LAUNCH(FALM_K_OTHER, st, k_dot<T><<<row_grid(ctx, R), kRowThreads, 0, st>>>(ctx->geo, R, a, b, ncol, ctx->red, &ctx->scal->red[0]));
    CK(cudaMemcpyAsync(ctx->scal_host, ctx->scal, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *out = ctx->scal_host->red[0];
    return FALM_OK;
}
