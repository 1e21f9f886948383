// Z-slab decomposition of the step over several GPUs: the transports (an
// in-process hub and NCCL), halo exchanges, the slab-reduced BiCGStab solve
// and the slab step.  Included by falm_b200.cu inside its anonymous namespace,
// after step_t.
//
// The reference decomposes the grid into per-rank boxes exchanged over MPI
// (src/CPMBase.h:36-112, src/CPMComm.h:182-364).  Here a slab is a run of whole
// z planes of the reference's layout, so a halo of a component is `depth`
// contiguous planes: no pack or unpack kernels, one transfer per component and
// direction.  What crosses the interfaces, per step:
//   start       u (2 planes: the 4th-order advection), nut (1)
//   ALM         the per-point force, torque and thrust, summed over the slabs
//               (each point is evaluated by the slab that owns its lower
//               interpolation plane)
//   face vel.   the pseudo-velocity ua (1 plane)
//   solve       the iterate before the first residual; pp and ss before each
//               preconditioner half sweep after the first and before each
//               matrix-vector product (1 plane); the totals of every inner
//               product and norm
//   projection  p (1 plane)
//   SGS         u (1 plane); the divergence norm's total
// (the reference exchanges the same fields at the same points:
// src/FalmCFD.cpp:27-45, 87-99, 149-154, 205-217, src/FalmEq.cpp).
#pragma once
// (falm_b200.cu includes <condition_variable>, <chrono>, <dlfcn.h> and <nccl.h>
// at file scope for this part)

// ---------------------------------------------------------------- in-process hub
struct LocalHub {
    static constexpr int kMaxVals = 64;
    static constexpr double kTimeoutS = 120.0;
    struct Rank {
        long long count = 0;          // operations issued by this rank
        long long seq = -1;           // the posted operation
        long long done_seq = -1;      // the operation whose copies this rank has queued
        int kind = 0;                 // 1 exchange, 2 reduction
        const void *send_lo = nullptr, *send_hi = nullptr;
        void *recv_lo = nullptr, *recv_hi = nullptr;
        size_t bytes = 0;
        double *buf = nullptr;
        int nval = 0, op = 0;
        cudaEvent_t ready = nullptr, done = nullptr;
        double *scratch = nullptr;    // nranks x kMaxVals doubles on the rank's device
        int device = -1;
    };
    int n = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::vector<Rank> r;
    std::vector<void *> users;
    bool failed = false;
};

struct HubUser {
    LocalHub *hub;
    int rank;
};

// reduce n values of each rank's copy, in rank order (every rank gets bitwise the same result)
__global__ void k_hub_reduce(const double *scratch, int nranks, int n, int op, double *buf) {
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        double v = scratch[q];
        for (int k = 1; k < nranks; k++) {
            const double w = scratch[(long long)k * LocalHub::kMaxVals + q];
            v = op == FALM_REDUCE_MAX ? fmax(v, w) : v + w;
        }
        buf[q] = v;
    }
}

int hub_prepare(LocalHub::Rank &me, int nranks) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return FALM_ERR_CUDA; }
    if (me.ready && me.device == dev) return FALM_OK;
    if (me.ready) return FALM_ERR_STATE;   // a rank stays on one device
    if (cudaEventCreateWithFlags(&me.ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&me.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&me.scratch, sizeof(double) * LocalHub::kMaxVals * nranks) != cudaSuccess) {
        cudaGetLastError();
        return FALM_ERR_CUDA;
    }
    me.device = dev;
    return FALM_OK;
}

// wait on the hub's condition until pred holds (or the hub failed, or time ran out)
template <class P>
bool hub_wait(LocalHub *h, std::unique_lock<std::mutex> &lk, P pred) {
    const bool ok = h->cv.wait_for(lk, std::chrono::duration<double>(LocalHub::kTimeoutS), [&] { return h->failed || pred(); });
    if (!ok) h->failed = true;
    if (h->failed) h->cv.notify_all();
    return ok && !h->failed;
}

// the rendezvous of one operation: post it, wait until the partners posted the
// same one (partners: the z neighbours of an exchange, every rank of a
// reduction), run `copy` (queues this rank's device copies), then wait until
// the partners have queued theirs and order this rank's stream after them, so
// that no rank overwrites a buffer another still reads
template <class Post, class Copy>
int hub_op(HubUser *u, int kind, cudaStream_t st, Post post, Copy copy) {
    LocalHub *h = u->hub;
    const int r = u->rank, n = h->n;
    LocalHub::Rank &me = h->r[r];
    int rc = hub_prepare(me, n);
    if (rc) return rc;
    if (cudaEventRecord(me.ready, st) != cudaSuccess) { cudaGetLastError(); return FALM_ERR_CUDA; }
    auto partner = [&](int q) { return kind == 2 ? q != r : (q == r - 1 || q == r + 1); };
    long long seq;
    {
        std::unique_lock<std::mutex> lk(h->mu);
        seq = me.count++;
        me.kind = kind;
        post(me);
        me.seq = seq;
        h->cv.notify_all();
        if (!hub_wait(h, lk, [&] {
                for (int q = 0; q < n; q++)
                    if (partner(q) && h->r[q].seq != seq) return false;
                return true;
            }))
            return FALM_ERR_TIMEOUT;
        for (int q = 0; q < n; q++)
            if (partner(q) && h->r[q].kind != kind) { h->failed = true; h->cv.notify_all(); return FALM_ERR_STATE; }
    }
    rc = copy(h, me);
    if (cudaEventRecord(me.done, st) != cudaSuccess) { cudaGetLastError(); rc = FALM_ERR_CUDA; }
    {
        std::unique_lock<std::mutex> lk(h->mu);
        if (rc) { h->failed = true; h->cv.notify_all(); return rc; }
        me.done_seq = seq;
        h->cv.notify_all();
        if (!hub_wait(h, lk, [&] {
                for (int q = 0; q < n; q++)
                    if (partner(q) && h->r[q].done_seq < seq) return false;
                return true;
            }))
            return FALM_ERR_TIMEOUT;
    }
    for (int q = 0; q < n; q++)
        if (partner(q) && cudaStreamWaitEvent(st, h->r[q].done, 0) != cudaSuccess) { cudaGetLastError(); return FALM_ERR_CUDA; }
    return FALM_OK;
}

int hub_exchange(void *user, const void *send_lo, void *recv_lo, const void *send_hi, void *recv_hi, size_t bytes, void *stream) {
    HubUser *u = (HubUser *)user;
    cudaStream_t st = (cudaStream_t)stream;
    const int r = u->rank, n = u->hub->n;
    if ((r > 0) != (send_lo && recv_lo) || (r < n - 1) != (send_hi && recv_hi)) return FALM_ERR_ARG;
    return hub_op(
        u, 1, st,
        [&](LocalHub::Rank &me) {
            me.send_lo = send_lo; me.recv_lo = recv_lo; me.send_hi = send_hi; me.recv_hi = recv_hi; me.bytes = bytes;
        },
        [&](LocalHub *h, LocalHub::Rank &me) -> int {
            // the lower neighbour's top planes into recv_lo, the upper one's bottom planes into recv_hi
            for (int side = 0; side < 2; side++) {
                const int q = side == 0 ? r - 1 : r + 1;
                if (q < 0 || q >= n) continue;
                const LocalHub::Rank &o = h->r[q];
                if (o.bytes != bytes) return FALM_ERR_STATE;
                void *dst = side == 0 ? me.recv_lo : me.recv_hi;
                const void *src = side == 0 ? o.send_hi : o.send_lo;
                if (cudaStreamWaitEvent(st, o.ready, 0) != cudaSuccess ||
                    cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st) != cudaSuccess) {
                    cudaGetLastError();
                    return FALM_ERR_CUDA;
                }
            }
            return FALM_OK;
        });
}

int hub_allreduce(void *user, double *buf, int nval, int op, void *stream) {
    HubUser *u = (HubUser *)user;
    cudaStream_t st = (cudaStream_t)stream;
    if (nval < 1 || nval > LocalHub::kMaxVals || !buf || (op != FALM_REDUCE_SUM && op != FALM_REDUCE_MAX)) return FALM_ERR_ARG;
    const int n = u->hub->n;
    int rc = hub_op(
        u, 2, st, [&](LocalHub::Rank &me) { me.buf = buf; me.nval = nval; me.op = op; },
        [&](LocalHub *h, LocalHub::Rank &me) -> int {
            // every rank's values into this rank's scratch, in rank order
            for (int q = 0; q < n; q++) {
                const LocalHub::Rank &o = h->r[q];
                if (o.nval != nval || o.op != op) return FALM_ERR_STATE;
                if ((q != u->rank && cudaStreamWaitEvent(st, o.ready, 0) != cudaSuccess) ||
                    cudaMemcpyAsync(me.scratch + (size_t)q * LocalHub::kMaxVals, o.buf, sizeof(double) * nval, cudaMemcpyDefault,
                                    st) != cudaSuccess) {
                    cudaGetLastError();
                    return FALM_ERR_CUDA;
                }
            }
            return FALM_OK;
        });
    if (rc) return rc;
    // every rank has copied every buffer: reduce into this rank's own
    k_hub_reduce<<<1, 64, 0, st>>>(u->hub->r[u->rank].scratch, n, nval, op, buf);
    return cudaGetLastError() == cudaSuccess ? FALM_OK : FALM_ERR_CUDA;
}

// ---------------------------------------------------------------- NCCL transport
struct NcclApi {
    void *lib = nullptr;
    ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t) = nullptr;
};

const NcclApi *nccl_api() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        // the copy the process has loaded already (torch's), else the system's
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        NcclApi a;
        a.lib = h;
        a.get_unique_id = (decltype(a.get_unique_id))dlsym(h, "ncclGetUniqueId");
        a.comm_init_rank = (decltype(a.comm_init_rank))dlsym(h, "ncclCommInitRank");
        a.comm_destroy = (decltype(a.comm_destroy))dlsym(h, "ncclCommDestroy");
        a.send = (decltype(a.send))dlsym(h, "ncclSend");
        a.recv = (decltype(a.recv))dlsym(h, "ncclRecv");
        a.group_start = (decltype(a.group_start))dlsym(h, "ncclGroupStart");
        a.group_end = (decltype(a.group_end))dlsym(h, "ncclGroupEnd");
        a.all_reduce = (decltype(a.all_reduce))dlsym(h, "ncclAllReduce");
        if (a.get_unique_id && a.comm_init_rank && a.comm_destroy && a.send && a.recv && a.group_start && a.group_end && a.all_reduce)
            api = a;
    });
    return api.lib ? &api : nullptr;
}

struct NcclUser {
    ncclComm_t comm;
    int rank, n;
};

int nccl_exchange(void *user, const void *send_lo, void *recv_lo, const void *send_hi, void *recv_hi, size_t bytes, void *stream) {
    const NcclApi *a = nccl_api();
    NcclUser *u = (NcclUser *)user;
    if (!a || !u) return FALM_ERR_STATE;
    if ((u->rank > 0) != (send_lo && recv_lo) || (u->rank < u->n - 1) != (send_hi && recv_hi)) return FALM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    ncclResult_t e = a->group_start();
    if (e == ncclSuccess && send_lo) e = a->send(send_lo, bytes, ncclInt8, u->rank - 1, u->comm, st);
    if (e == ncclSuccess && recv_lo) e = a->recv(recv_lo, bytes, ncclInt8, u->rank - 1, u->comm, st);
    if (e == ncclSuccess && send_hi) e = a->send(send_hi, bytes, ncclInt8, u->rank + 1, u->comm, st);
    if (e == ncclSuccess && recv_hi) e = a->recv(recv_hi, bytes, ncclInt8, u->rank + 1, u->comm, st);
    const ncclResult_t e2 = a->group_end();
    return (e == ncclSuccess && e2 == ncclSuccess) ? FALM_OK : FALM_ERR_CUDA;
}

int nccl_allreduce(void *user, double *buf, int nval, int op, void *stream) {
    const NcclApi *a = nccl_api();
    NcclUser *u = (NcclUser *)user;
    if (!a || !u) return FALM_ERR_STATE;
    if (nval < 1 || !buf || (op != FALM_REDUCE_SUM && op != FALM_REDUCE_MAX)) return FALM_ERR_ARG;
    return a->all_reduce(buf, buf, (size_t)nval, ncclFloat64, op == FALM_REDUCE_MAX ? ncclMax : ncclSum, u->comm,
                         (cudaStream_t)stream) == ncclSuccess
               ? FALM_OK
               : FALM_ERR_CUDA;
}

// ---------------------------------------------------------------- slab helpers
// exchange `depth` guide planes of each of the ncomp components of f with the z neighbours
template <typename T>
int slab_halo(falm_ctx *ctx, T *f, int ncomp, int depth, cudaStream_t st) {
    if (!ctx->slab_on || ctx->slab_nranks == 1) return FALM_OK;
    const Geom &g = ctx->geo;
    if (depth < 1 || depth > g.gc || g.nz < depth) return fail(ctx, FALM_ERR_ARG, "slab halo: depth");
    const size_t sxy = (size_t)g.sx * g.sy, bytes = sxy * depth * sizeof(T);
    const bool lo = ctx->slab_rank > 0, hi = ctx->slab_rank < ctx->slab_nranks - 1;
    for (int c = 0; c < ncomp; c++) {
        T *b = f + (size_t)c * g.n;
        const int rc = ctx->transport.exchange(ctx->transport.user, lo ? b + g.gc * sxy : nullptr, lo ? b + (g.gc - depth) * sxy : nullptr,
                                               hi ? b + (g.sz - g.gc - depth) * sxy : nullptr, hi ? b + (g.sz - g.gc) * sxy : nullptr,
                                               bytes, st);
        if (rc) return fail(ctx, rc, "slab halo: transport exchange");
    }
    return FALM_OK;
}

int slab_reduce(falm_ctx *ctx, double *buf, int n, int op, cudaStream_t st) {
    if (!ctx->slab_on || ctx->slab_nranks == 1) return FALM_OK;
    const int rc = ctx->transport.allreduce(ctx->transport.user, buf, n, op, st);
    return rc ? fail(ctx, rc, "slab reduction: transport allreduce") : FALM_OK;
}

// the reduced totals in red[0..n) of a deferred reduction kernel, then the scalars of `stage`
int slab_derive(falm_ctx *ctx, int n, int stage, cudaStream_t st) {
    int rc = slab_reduce(ctx, ctx->scal->red, n, FALM_REDUCE_SUM, st);
    if (rc) return rc;
    LAUNCH(FALM_K_OTHER, st, k_slab_derive<<<1, 1, 0, st>>>(ctx->scal, stage));
    return FALM_OK;
}

// The BiCGStab solve of a slab (src/FalmEq.cpp:305-410) on the 7-point plane
// streams (row kernels where a grid is not streamable):
// every reduction kernel leaves its slab's totals in red[] (SolverScalars::
// defer), the totals are summed over the slabs and k_slab_derive derives the
// scalars; each preconditioner half sweep after the first (pointwise, from
// zero) follows an exchange of the iterate's halo, and each matrix-vector
// product an exchange of its operand's.  Mixed precision: passes with an FP64
// check of the true residual between them, as in the one-slab solve.
template <typename T>
int slab_solve_t(falm_ctx *ctx, T *x, const T *b, T *r, cudaStream_t st, int *it_out, double *err_out, int *outer_out) {
    int rc = ensure_work(ctx);
    if (rc) return rc;
    if (!ctx->op_ready) return fail(ctx, FALM_ERR_STATE, "slab solve: no operator (call falm_eq_poisson_operator)");
    if (ctx->A_explicit) return fail(ctx, FALM_ERR_STATE, "slab solve: the table operator only");
    if (ctx->ls_type != FALM_LS_PBICGSTAB) return fail(ctx, FALM_ERR_ARG, "slab solve: PBiCGStab only");
    if ((rc = solver_init(ctx, st))) return rc;
    static const int one = 1;
    CK(cudaMemcpyAsync(&ctx->scal->defer, &one, sizeof(int), cudaMemcpyHostToDevice, st));
    const Geom &g = ctx->geo;
    const Region3 R = interior(g);
    const int grid = row_grid(ctx, R);
    const Op7<T> op = op7<T>(ctx);
    T *rr = (T *)ctx->w_rr, *p = (T *)ctx->w_p, *q = (T *)ctx->w_q, *s = (T *)ctx->w_s, *pp = (T *)ctx->w_pp;
    T *ss = (T *)ctx->w_ss, *t = (T *)ctx->w_t, *xp = (T *)ctx->w_xp;
    const T pcw = (T)ctx->pc_relax;
    const int pct = ctx->pc_type, m = ctx->pc_maxit;
    SolverScalars *sc = ctx->scal;
    const bool mixed = ctx->precision == FALM_MIXED;
    const int max_outer = mixed ? ctx->max_outer : 1;
    // the preconditioner after its pointwise first sweep (in k_bicg_p / k_bicg_s)
    auto precondition_rest = [&](T *z, const T *v) -> int {
        if (pct == FALM_LS_SOR) {
            for (int hs = 1; hs < 2 * m; hs++) {            // red, then (black, red) x (m - 1)
                int rc2 = slab_halo<T>(ctx, z, 1, 1, st);
                if (rc2) return rc2;
                S7_OR(FALM_K_SOR, st, T, 0, z, (SorBody<T>{op, z, v, pcw, hs & 1, sc}),
                      (k_sor<T><<<grid, kRowThreads, 0, st>>>(g, R, op, z, v, pcw, hs & 1, sc)));
            }
        } else if (pct == FALM_LS_JACOBI) {
            // the first sweep wrote to the buffer that makes the last one land in z
            T *bufs[2] = {z, xp};
            for (int it = 2; it <= m; it++) {
                T *dst = bufs[(m - it) & 1], *src = bufs[(m - it + 1) & 1];
                int rc2 = slab_halo<T>(ctx, src, 1, 1, st);
                if (rc2) return rc2;
                LAUNCH(FALM_K_SOR, st, k_jacobi<T><<<grid, kRowThreads, 0, st>>>(g, R, op, dst, src, v, sc));
            }
        }
        return FALM_OK;
    };
    auto first_target = [&](T *z) -> T * { return (pct == FALM_LS_JACOBI && ((m - 1) & 1)) ? xp : z; };
    static const int zero = 0;
    int total_it = 0, outer = 0;
    for (outer = 0; outer < max_outer; outer++) {
        // a pass starts from the residual (after the first pass: a check of the true residual)
        if ((rc = slab_halo<T>(ctx, x, 1, 1, st))) return rc;
        {
            const ResBody<T> body{op, b, r, rr, sc, outer > 0 ? 1 : 0};   // r, rr and the totals (deferred)
            S7_OR(FALM_K_RES, st, T, 2, x, body, (k_res<T><<<grid, kRowThreads, 0, st>>>(g, R, op, x, b, r, rr, ctx->red, sc, outer > 0)));
        }
        if ((rc = slab_derive(ctx, 2, outer > 0 ? 1 : 0, st))) return rc;
        CK(cudaMemcpyAsync(&sc->it, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->scal_host, sc, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (ctx->scal_host->done) break;
        int batch = 1, queued = 0;
        for (;;) {
            LAUNCH(FALM_K_BICG_P, st, k_bicg_p<T><<<grid, kRowThreads, 0, st>>>(g, R, op, p, p, q, r, first_target(pp), pct, pcw, sc));
            if ((rc = precondition_rest(pp, p))) return rc;
            if ((rc = slab_halo<T>(ctx, pp, 1, 1, st))) return rc;
            S7_OR(FALM_K_MV_DOT1, st, T, 1, pp, (MvDot1Body<T>{op, q, rr, sc}),
                  (k_mv_dot1<T><<<grid, kRowThreads, 0, st>>>(g, R, op, pp, q, rr, ctx->red, sc)));
            if ((rc = slab_derive(ctx, 1, 2, st))) return rc;
            LAUNCH(FALM_K_BICG_S, st, k_bicg_s<T><<<grid, kRowThreads, 0, st>>>(g, R, op, s, q, r, first_target(ss), pct, pcw, sc));
            if ((rc = precondition_rest(ss, s))) return rc;
            if ((rc = slab_halo<T>(ctx, ss, 1, 1, st))) return rc;
            S7_OR(FALM_K_MV_DOT2, st, T, 2, ss, (MvDot2Body<T>{op, t, s, sc}),
                  (k_mv_dot2<T><<<grid, kRowThreads, 0, st>>>(g, R, op, ss, t, s, ctx->red, sc)));
            if ((rc = slab_derive(ctx, 2, 3, st))) return rc;
            LAUNCH(FALM_K_BICG_XR, st, k_bicg_xr<T><<<grid, kRowThreads, 0, st>>>(g, R, x, pp, ss, r, s, t, rr, ctx->red, sc));
            if ((rc = slab_derive(ctx, 2, 4, st))) return rc;
            if (++queued < batch) continue;
            CK(cudaMemcpyAsync(ctx->scal_host, sc, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (ctx->scal_host->done) break;
            queued = 0;
            batch = std::min(2 * batch, 8);
        }
        total_it += ctx->scal_host->it;
        if (ctx->scal_host->status == FALM_ERR_NAN || !mixed) break;
    }
    CK(cudaMemcpyAsync(&ctx->scal->defer, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
    if (it_out) *it_out = total_it;
    if (err_out) *err_out = ctx->scal_host->err;
    if (outer_out) *outer_out = std::min(outer + 1, max_outer);
    return ctx->scal_host->status == FALM_ERR_NAN ? fail(ctx, FALM_ERR_NAN, "solve: non-finite scalar") : FALM_OK;
}

// the ALM of a slab: each point evaluated by the slab that owns it, then the
// per-point force, torque and thrust summed over the slabs, the turbine sums
// and the force boxes of the slab's cells
template <typename T>
int slab_alm_t(falm_ctx *ctx, const T *u, double t, cudaStream_t st) {
    const int csm = (ctx->geo.sx + ctx->geo.sy + ctx->geo.sz) * (int)sizeof(double);
    const int stage = csm <= 96 * 1024 ? 1 : 0;
    if (stage && csm > 32 * 1024) cudaFuncSetAttribute(k_alm_force<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
    LAUNCH(FALM_K_ALM, st, k_alm_force<T><<<1, 256, stage ? csm : 0, st>>>(ctx->geo, ctx->alm, ctx->m64.x[0], ctx->m64.x[1], ctx->m64.x[2], u, t, stage,
                                                                            nullptr));
    const int apc = ctx->alm.apcount;
    int rc;
    for (int q = 0; q < 3 * apc; q += LocalHub::kMaxVals)
        if ((rc = slab_reduce(ctx, ctx->alm.ap_force + q, std::min(LocalHub::kMaxVals, 3 * apc - q), FALM_REDUCE_SUM, st))) return rc;
    for (double *a : {ctx->alm.ap_torque, ctx->alm.ap_thrust})
        for (int q = 0; q < apc; q += LocalHub::kMaxVals)
            if ((rc = slab_reduce(ctx, a + q, std::min(LocalHub::kMaxVals, apc - q), FALM_REDUCE_SUM, st))) return rc;
    LAUNCH(FALM_K_ALM, st, k_alm_turbine_sums<<<1, 32, 0, st>>>(ctx->alm));
    if (ctx->alm.bs.total > 0) {
        const long long blocks = std::min<long long>((ctx->alm.bs.total + 255) / 256, (long long)ctx->sm_count * 8);
        LAUNCH(FALM_K_ALM, st, k_alm_box<T><<<(int)blocks, 256, 0, st>>>(ctx->alm, ctx->m64.x[0], ctx->m64.x[1], ctx->m64.x[2]));
    }
    return FALM_OK;
}

// One step of a slab (the order of step_t, app/nedo/main.cpp:150-204), with
// the exchanges and reductions listed at the top of this file.  The face
// velocity, right-hand side and first residual run as separate passes here.
template <typename T>
int slab_step_t(falm_ctx *ctx, const falm_fields *f, double dt, double t, cudaStream_t st, falm_step_stats *out) {
    NvtxRange range("falm_step_slab");
    int rc = ensure_work(ctx);
    if (rc) return rc;
    if (!ctx->op_ready) return fail(ctx, FALM_ERR_STATE, "slab step: build the operator first (falm_eq_poisson_operator, a collective)");
    const Geom &g = ctx->geo;
    T *u = (T *)f->u, *uu = (T *)f->uu, *p = (T *)f->p, *nut = (T *)f->nut, *ff = (T *)f->ff;
    T *ua = (T *)ctx->w_ua, *rhs = (T *)ctx->w_rhs, *r = (T *)ctx->w_r;
    const bool chan = ctx->bc_kind == FALM_BC_CHANNEL;
    // 0. halos of the state
    if ((rc = slab_halo<T>(ctx, u, 3, 2, st)) || (rc = slab_halo<T>(ctx, nut, 1, 1, st))) return rc;
    // 1. ALM at the previous velocity, or the RMCP model (cells of the slab; sums over the slabs)
    if (ctx->alm_on) {
        if ((rc = slab_alm_t<T>(ctx, u, t, st))) return rc;
        if (ff) {
            const Region3 R = interior(g);
            LAUNCH(FALM_K_ALM, st, k_alm_project<T><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), ctx->alm, ff));
        }
    } else if (ctx->rmcp_on) {
        ff = (T *)ctx->w_ff;
        if ((rc = rmcp_run_t<T>(ctx, u, ff, nullptr, t, st))) return rc;
        if ((rc = slab_reduce(ctx, ctx->rmcp_sums, 2 * kMaxTurbines, FALM_REDUCE_SUM, st))) return rc;
    }
    // 2. pseudo-velocity; its guide layer takes the previous velocity, across
    //    the slab interfaces the neighbours' pseudo-velocity
    if ((rc = pseudo_u_t<T>(ctx, u, u, uu, ua, nut, ff, dt, ctx->alm_on != 0 && !ff, st))) return rc;
    LAUNCH(FALM_K_OTHER, st, k_copy_shell<T><<<ctx->sm_count * 8, 256, 0, st>>>(g, u, ua));
    if ((rc = slab_halo<T>(ctx, ua, 3, 1, st))) return rc;
    // 3. face velocity [+ uubc] + RHS
    {
        const Region3 R = facemap(g);
        const T scale = (T)(1.0 / (dt * ctx->maxdiag));
        if (chan)
            P3_OR(FALM_K_UTOUU_RHS, st, T, 1, 0, R, 1, FB_ARR(ua), FB_ARR(3), (UtoUUBody<T, true, false>{g, mview<T>(ctx), uu, rhs, scale}),
                  (k_utouu<T, true, false><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), ua, u, uu, rhs, scale)));
        else
            P3_OR(FALM_K_UTOUU_RHS, st, T, 1, 0, R, 1, FB_ARR(ua), FB_ARR(3), (UtoUUBody<T, true, true>{g, mview<T>(ctx), uu, rhs, scale}),
                  (k_utouu<T, true, true><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), ua, u, uu, rhs, scale)));
    }
    // 4. Poisson
    int it = 0, outer = 1;
    double err = 0;
    rc = slab_solve_t<T>(ctx, p, rhs, r, st, &it, &err, &outer);
    const int solve_status = ctx->scal_host->status;
    if (rc) return rc;
    // 5. pbc on the physical faces, the pressure's halo
    LAUNCH(FALM_K_PBC, st, k_pbc<T><<<dim3(face_blocks(ctx), 3), 256, 0, st>>>(g, ctx->bc_kind, p));
    if ((rc = slab_halo<T>(ctx, p, 1, 1, st))) return rc;
    // 6. previous velocity at the outlet, projection
    if (chan) { LAUNCH(FALM_K_OTHER, st, k_save_outlet<T><<<std::min(ctx->sm_count * 4, (3 * g.sy * g.sz + 255) / 256), 256, 0, st>>>(g, u, (T *)ctx->w_outlet)); }
    {
        const Region3 R = facemap(g);
        P3_OR(FALM_K_PROJECT, st, T, 1, 0, R, 1, FB_ARR(p), FB_ARR(1), (ProjectBody<T>{g, mview<T>(ctx), u, ua, uu, uu, (T)dt}),
              (k_project<T><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), u, ua, uu, uu, p, (T)dt)));
    }
    // 7. ubc on the physical faces, the velocity's halo
    if ((rc = ubc_t<T>(ctx, u, UPrev<T>{(const T *)ctx->w_outlet, 1}, dt, t, st))) return rc;
    if ((rc = slab_halo<T>(ctx, u, 3, 1, st))) return rc;
    // 8. SGS + the divergence norm's total over the slabs
    {
        const Region3 R = interior(g);
        P3_OR(FALM_K_SGS_DIV, st, T, 2, 1, R, 2, FB_ARR(u, uu), FB_ARR(3, 3),
              (SgsDivBody<T>{g, mview<T>(ctx), ctx->m64, nut, (T)ctx->Cs, ctx->sgs, (T *)nullptr, &ctx->scal->red[3]}),
              (k_sgs_div<T, true><<<row_grid(ctx, R), kRowThreads, 0, st>>>(g, R, mview<T>(ctx), ctx->m64, u, nut, (T)ctx->Cs, ctx->sgs, uu,
                                                                            nullptr, ctx->red, &ctx->scal->red[3])));
    }
    if ((rc = slab_reduce(ctx, &ctx->scal->red[3], 1, FALM_REDUCE_SUM, st))) return rc;
    CK(cudaMemcpyAsync(ctx->scal_host, ctx->scal, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st));
    if (ctx->alm_on) CK(cudaMemcpyAsync(ctx->alm_scal_host, ctx->alm.scal, sizeof(AlmScalars), cudaMemcpyDeviceToHost, st));
    if (ctx->rmcp_on) CK(cudaMemcpyAsync(ctx->rmcp_sums_host, ctx->rmcp_sums, 2 * kMaxTurbines * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&ctx->scal_host->kerr, ctx->kerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ctx->scal_host->kerr) {
        cudaMemsetAsync(ctx->kerr, 0, sizeof(int), st);
        *ctx->last_error = "slab step: device error word " + std::to_string(ctx->scal_host->kerr);
        return ctx->scal_host->kerr >= 200 ? FALM_ERR_ARG : FALM_ERR_TIMEOUT;
    }
    if (out) {
        memset(out, 0, sizeof(*out));
        out->it = it;
        out->err = err;
        out->outer = outer;
        out->status = solve_status;
        out->divnorm = std::sqrt(ctx->scal_host->red[3]) / ((double)g.nx * g.ny * g.nzg);
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
