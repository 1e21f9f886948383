// Host plumbing of the launches: status and error text, the launch wrapper with
// per-class event timing, occupancy and z-chunk choice, row grids, the context's
// work vectors, TMA tensor maps and the launchers of the plane-stream kernels
// (7-point, blocked red-black SOR, multi-field) with their row-kernel fallbacks.
// Included by falm_b200.cu inside its anonymous namespace (after the headers
// it includes and the code before this point); not a standalone header.
#pragma once

int fail(falm_ctx *c, int code, const char *msg) {
    if (c && c->last_error) *c->last_error = msg;
    return code;
}

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t _e = (call);                                                           \
        if (_e != cudaSuccess) {                                                           \
            if (ctx && ctx->last_error) *ctx->last_error = std::string(#call ": ") + cudaGetErrorString(_e); \
            return (int)FALM_ERR_CUDA;                                                     \
        }                                                                                  \
    } while (0)

#define LAUNCHED()                                                                         \
    do {                                                                                   \
        ctx->launches++;                                                                   \
        cudaError_t _e = cudaGetLastError();                                               \
        if (_e != cudaSuccess) {                                                           \
            *ctx->last_error = std::string("launch: ") + cudaGetErrorString(_e);           \
            return (int)FALM_ERR_CUDA;                                                     \
        }                                                                                  \
    } while (0)

cudaEvent_t ev_get(falm_ctx *ctx) {
    if (!ctx->ev_pool->empty()) {
        cudaEvent_t e = ctx->ev_pool->back();
        ctx->ev_pool->pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// launch one kernel of class `cls`; with profiling on, bracket it with an event pair
template <typename F>
int launch_k(falm_ctx *ctx, int cls, cudaStream_t st, F &&f) {
    cudaEvent_t a = nullptr;
    if (ctx->profiling) {
        a = ev_get(ctx);
        cudaEventRecord(a, st);
    }
    f();
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && ctx->check_sync) e = cudaStreamSynchronize(st);   // FALM_B200_CHECK=1: locate faults
    if (e != cudaSuccess) {
        *ctx->last_error = std::string("launch of kernel class ") + std::to_string(cls) + ": " + cudaGetErrorString(e);
        return FALM_ERR_CUDA;
    }
    if (ctx->check_sync) {   // and the device error word of the kernels' self-checks
        int w = 0;
        if (cudaMemcpy(&w, ctx->kerr, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && w) {
            cudaMemset(ctx->kerr, 0, sizeof(int));
            *ctx->last_error = std::string("kernel class ") + std::to_string(cls) + ": device error word " + std::to_string(w);
            return w >= 200 ? FALM_ERR_ARG : FALM_ERR_TIMEOUT;
        }
    }
    if (ctx->profiling) {
        cudaEvent_t b = ev_get(ctx);
        cudaEventRecord(b, st);
        ctx->ev_pending->push_back(falm_ctx::EvRec{cls, a, b});
    }
    return FALM_OK;
}

#define LAUNCH(CLS, ST, ...)                                                                 \
    do {                                                                                     \
        int _lrc = launch_k(ctx, (CLS), (ST), [&] { __VA_ARGS__; });                         \
        if (_lrc) return _lrc;                                                               \
    } while (0)

// NVTX ranges (a profiler or tracer attached through NVTX shows them; without
// one they cost a few ns): one range per call and one per phase of the step
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
struct NvtxPhases {   // consecutive ranges: next() closes the open one
    bool open = false;
    void next(const char *name) {
        if (open) nvtxRangePop();
        nvtxRangePushA(name);
        open = true;
    }
    ~NvtxPhases() { if (open) nvtxRangePop(); }
};

// resident CTAs per SM of a kernel at a launch shape, looked up once per
// kernel and shape
template <typename K>
int resident_per_sm(K kernel, int threads, int smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void *, int, int>, int> known;
    const auto key = std::make_tuple((const void *)kernel, threads, smem);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = known.find(key);
        if (it != known.end()) return it->second;
    }
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        n = 1;
    }
    std::lock_guard<std::mutex> lk(mu);
    known[key] = n;
    return n;
}

// z planes per CTA of a plane-streaming kernel: the chunk length kc in
// [8, cap] that minimises the modelled time ceil(CTAs / resident slots) *
// (kc + halo + 2): the CTAs run in waves of SMs x per_sm, and a CTA's time
// grows with its planes (the halo planes included) plus a start-up of about
// two planes.  Ties keep the longer chunk.
int chunk_len(const falm_ctx *ctx, long long blocks_xy, int nz, int per_sm, int cap, int halo) {
    const long long slots = (long long)ctx->sm_count * std::max(1, per_sm);
    const int lo = std::min(8, nz), hi = std::max(lo, std::min(cap, nz));
    int best = hi;
    long long best_t = -1;
    for (int kc = hi; kc >= lo; kc--) {
        const long long ctas = blocks_xy * ((nz + kc - 1) / kc);
        const long long t = ((ctas + slots - 1) / slots) * (kc + halo + 2);
        if (best_t < 0 || t < best_t) { best_t = t; best = kc; }
    }
    return std::max(1, best);
}

// blocks along x of a face-pair kernel (blockIdx.y = pair): the largest face's
// cells at one per thread, at most four blocks per SM
int face_blocks(const falm_ctx *ctx) {
    const Geom &g = ctx->geo;
    const long long mx = std::max({(long long)g.ny * g.nz, (long long)g.nx * g.nz, (long long)g.nx * g.ny});
    return (int)std::max(1LL, std::min((mx + 255) / 256, (long long)ctx->sm_count * 4));
}

int row_grid(const falm_ctx *ctx, const Region3 &R) {
    long long rows = R.nrows();
    long long need = (rows + kWarpsPerBlock - 1) / kWarpsPerBlock;
    long long cap = (long long)ctx->sm_count * 8;
    return (int)std::max(1LL, std::min(need, cap));
}

// one wave of a row kernel: as many blocks as are resident at once on all SMs
// (the kernel's occupancy, looked up once per kernel), at most one warp per row
template <typename K>
int row_grid_wave(const falm_ctx *ctx, const Region3 &R, K kernel) {
    static std::mutex mu;
    static std::unordered_map<const void *, int> per_sm_of;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = per_sm_of.find((const void *)kernel);
        if (it != per_sm_of.end()) per_sm = it->second;
    }
    if (per_sm <= 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kRowThreads, 0) != cudaSuccess || per_sm <= 0) {
            cudaGetLastError();
            return row_grid(ctx, R);
        }
        std::lock_guard<std::mutex> lk(mu);
        per_sm_of[(const void *)kernel] = per_sm;
    }
    const long long need = ((long long)R.nrows() + kWarpsPerBlock - 1) / kWarpsPerBlock;
    return (int)std::max(1LL, std::min(need, (long long)ctx->sm_count * per_sm));
}

template <typename T> MetricView<T> mview(const falm_ctx *ctx);
template <> MetricView<double> mview<double>(const falm_ctx *ctx) { return MetricView<double>{ctx->m64}; }
template <> MetricView<float> mview<float>(const falm_ctx *ctx) { return MetricView<float>{ctx->m32}; }

template <typename T> Op7<T> op7(const falm_ctx *ctx);
template <> Op7<double> op7<double>(const falm_ctx *ctx) { return Op7<double>{ctx->pt64, (const double *)ctx->A_explicit, ctx->geo.n}; }
template <> Op7<float> op7<float>(const falm_ctx *ctx) { return Op7<float>{ctx->pt32, (const float *)ctx->A_explicit, ctx->geo.n}; }

int ensure_work(falm_ctx *ctx) {
    if (ctx->work_mem) return FALM_OK;
    const size_t n = (size_t)ctx->geo.n, e = ctx->esize;
    const int nvec = 12;   // rr p q s pp ss t r rhs div xp + ua(3)
    size_t outlet = 9ull * ctx->geo.sy * ctx->geo.sz;
    size_t bytes = ((size_t)(nvec + 2) * n + outlet) * e + 256 * 16;
    void *mem = nullptr;
    if (cudaMalloc(&mem, bytes) != cudaSuccess) { cudaGetLastError(); return fail(ctx, FALM_ERR_ALLOC, "work vectors: cudaMalloc failed"); }
    if (cudaMemset(mem, 0, bytes) != cudaSuccess) return fail(ctx, FALM_ERR_CUDA, "work vectors: cudaMemset failed");
    char *p = (char *)mem;
    auto take = [&](size_t count) { void *r = p; p += ((count * e + 255) / 256) * 256; return r; };
    ctx->w_rr = take(n); ctx->w_p = take(n); ctx->w_q = take(n); ctx->w_s = take(n);
    ctx->w_pp = take(n); ctx->w_ss = take(n); ctx->w_t = take(n); ctx->w_r = take(n);
    ctx->w_rhs = take(n); ctx->w_div = take(n); ctx->w_xp = take(n);
    ctx->w_ua = take(3 * n);
    ctx->w_outlet = take(outlet);
    ctx->work_mem = mem;
    return FALM_OK;
}

// ---------------------------------------------------------------- TMA tensor maps
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

bool tma_encode_available() {
    static int state = -1;
    if (state < 0) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        state = (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
                 q == cudaDriverEntryPointSuccess && fn)
                    ? 1 : 0;
        cudaGetLastError();
        g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    return state == 1;
}

// 4D map (x, y, z, component) of a field in the reference layout with a
// (bx, by, 1, ncomp) box.  TMA needs a 16 B aligned base and row pitch; the
// caller falls back to the row kernels otherwise.
template <typename T>
bool make_map(const falm_ctx *ctx, CUtensorMap *m, const T *base, int ncomp, int bx, int by) {
    const Geom &g = ctx->geo;
    const size_t e = sizeof(T);   // the field's own type (a mixed context also runs FP64 vectors)
    // every box lies inside the tensor: x and y at least one box long (the
    // kernels clamp the box origins), x rows a whole number of 16-byte units
    // (the kernels' box x origins are 16-byte aligned for gc = 2)
    if (!tma_encode_available() || ((uintptr_t)base & 15) || ((g.sx * e) & 15) || g.sx < bx || g.sy < by || g.gc != 2) return false;
    cuuint64_t dims[4] = {(cuuint64_t)g.sx, (cuuint64_t)g.sy, (cuuint64_t)g.sz, (cuuint64_t)ncomp};
    cuuint64_t strides[3] = {(cuuint64_t)(g.sx * e), (cuuint64_t)(g.sx * (size_t)g.sy * e), (cuuint64_t)(g.n * e)};
    cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)ncomp};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = g_encode(m, e == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base,
                          dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 7-point scalar stencil over the interior through the TMA plane stream;
// returns 1 when launched, 0 when the operand is not TMA-eligible (the caller
// then uses its row kernel), <0 on a launch error.
template <typename T, int NV, class Body>
int s7_launch(falm_ctx *ctx, int cls, cudaStream_t st, const T *x, const Body &body) {
    CUtensorMap m;
    if (ctx->no_tma || !make_map(ctx, &m, x, 1, S7Tile<T>::BX, S7Tile<T>::BY)) return 0;
    const Geom &g = ctx->geo;
    const int bx = (g.nx + S7Tile<T>::TX - 1) / S7Tile<T>::TX, by = (g.ny + S7Tile<T>::TY - 1) / S7Tile<T>::TY;
    const int kc = chunk_len(ctx, (long long)bx * by, g.nz, resident_per_sm(k_s7_tma<T, NV, Body>, 256, s7_smem<T>()), 64, 2);
    dim3 grid(bx, by, (g.nz + kc - 1) / kc);
    if ((long long)grid.x * grid.y * grid.z > ctx->red.maxBlocks) return 0;
    if (s7_smem<T>() > 48 * 1024) cudaFuncSetAttribute(k_s7_tma<T, NV, Body>, cudaFuncAttributeMaxDynamicSharedMemorySize, s7_smem<T>());
    int rc = launch_k(ctx, cls, st, [&] {
        k_s7_tma<T, NV, Body><<<grid, 256, s7_smem<T>(), st>>>(g, kc, m, body, ctx->red, ctx->kerr);
    });
    return rc ? -rc : 1;
}

#define S7_OR(CLS, ST, T_, NV_, X_, BODY_, ROWLAUNCH)                                     \
    do {                                                                                   \
        int _s7 = s7_launch<T_, NV_>(ctx, (CLS), (ST), (X_), BODY_);                       \
        if (_s7 < 0) return -_s7;                                                          \
        if (_s7 == 0) LAUNCH((CLS), (ST), ROWLAUNCH);                                      \
    } while (0)

// H consecutive red-black half sweeps (first colour c1) in one pass, x_in -> x_out;
// 1 launched, 0 not eligible, <0 launch error
template <typename T, int H>
int sor_rb_launch_h(falm_ctx *ctx, cudaStream_t st, const T *xin, const T *b, T *xout, T omega, int c1, const SolverScalars *sc) {
    using L = RBTile<T, H>;
    if (ctx->no_tma || ctx->A_explicit) return 0;
    CUtensorMap mx, mb;
    if (!make_map(ctx, &mx, xin, 1, L::BX, L::BY) || !make_map(ctx, &mb, b, 1, L::BX, L::BY)) return 0;
    const Geom &g = ctx->geo;
    const int bx = (g.nx + L::TX - 1) / L::TX, by = (g.ny + L::TY - 1) / L::TY;
    const int kc = chunk_len(ctx, (long long)bx * by, g.nz, resident_per_sm(k_sor_rb_tma<T, H>, 256, L::SMEM), 64, 2 * H);
    dim3 grid(bx, by, (g.nz + kc - 1) / kc);
    cudaFuncSetAttribute(k_sor_rb_tma<T, H>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
    const PoissonTables<T> tb = op7<T>(ctx).t;
    int rc = launch_k(ctx, FALM_K_SOR, st, [&] {
        k_sor_rb_tma<T, H><<<grid, 256, L::SMEM, st>>>(g, kc, mx, mb, tb, xout, omega, c1, sc, ctx->kerr);
    });
    return rc ? -rc : 1;
}

// three half sweeps on the 28 x 16 tile (skewed wavefront); 1 launched, 0 not eligible, <0 launch error
template <typename T>
int sor_rb2_launch(falm_ctx *ctx, cudaStream_t st, const T *xin, const T *b, T *xout, T omega, int c1, const SolverScalars *sc) {
    using L = RB2Tile<T>;
    if (ctx->no_tma || ctx->A_explicit) return 0;
    CUtensorMap mx, mb;
    if (!make_map(ctx, &mx, xin, 1, L::BX, L::BY) || !make_map(ctx, &mb, b, 1, L::BXB, L::BYB)) return 0;
    const Geom &g = ctx->geo;
    const int bx = (g.nx + L::TX - 1) / L::TX, by = (g.ny + L::TY - 1) / L::TY;
    // a CTA runs kc + 3H iterations and stages at most ZMAX planes of z coefficients
    const int kc = chunk_len(ctx, (long long)bx * by, g.nz, resident_per_sm(k_sor_rb2_tma<T>, L::NT, L::SMEM),
                             std::min(64, L::ZMAX - 2 * L::H), 3 * L::H);
    dim3 grid(bx, by, (g.nz + kc - 1) / kc);
    cudaFuncSetAttribute(k_sor_rb2_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
    const PoissonTables<T> tb = op7<T>(ctx).t;
    int rc = launch_k(ctx, FALM_K_SOR, st, [&] {
        k_sor_rb2_tma<T><<<grid, L::NT, L::SMEM, st>>>(g, kc, mx, mb, tb, xout, omega, c1, sc, ctx->kerr);
    });
    return rc ? -rc : 1;
}

// whether three half sweeps run on the 28 x 16 skewed kernel rather than the
// 32 x 8 one: always in FP32; in FP64 (2 CTAs per SM instead of 3) once every
// CTA slot marches at least 128 planes, where its single barrier per plane
// outweighs its longer pipeline fill (512x256x256: 0.725 -> 0.631 ms per pass;
// 256x128x128, 35 planes per slot: 0.076 -> 0.083 ms)
template <typename T>
bool sor_skewed(const falm_ctx *ctx) {
    if (ctx->sor_v1) return ctx->sor_v1 == 2;
    if (sizeof(T) == 4) return true;
    using L = RB2Tile<T>;
    const Geom &g = ctx->geo;
    const long long tiles = (long long)((g.nx + L::TX - 1) / L::TX) * ((g.ny + L::TY - 1) / L::TY);
    return tiles * g.nz >= 128LL * ctx->sm_count * L::MINB;
}

template <typename T>
int sor_rb_launch(falm_ctx *ctx, cudaStream_t st, int H, const T *xin, const T *b, T *xout, T omega, int c1, const SolverScalars *sc) {
    // the blocked kernels take the colour parity of local plane indices: a grid
    // whose planes are offset by koff flips the first colour instead
    c1 ^= ctx->geo.koff & 1;
    if (H == 3 && sor_skewed<T>(ctx)) {
        const int r = sor_rb2_launch<T>(ctx, st, xin, b, xout, omega, c1, sc);
        if (r != 0) return r;
    }
    if (H == 1) return sor_rb_launch_h<T, 1>(ctx, st, xin, b, xout, omega, c1, sc);
    if (H == 2) return sor_rb_launch_h<T, 2>(ctx, st, xin, b, xout, omega, c1, sc);
    return sor_rb_launch_h<T, 3>(ctx, st, xin, b, xout, omega, c1, sc);
}

// the conditions of make_map for a context vector (256-byte aligned) of element size e
bool map_ok(const falm_ctx *ctx, size_t e, int bx, int by) {
    const Geom &g = ctx->geo;
    return tma_encode_available() && ((g.sx * e) & 15) == 0 && g.sx >= bx && g.sy >= by && g.gc == 2;
}

// whether sor_rb_launch runs an H-half-sweep blocked pass on the context's vectors
// (1) or declines (0), decided without a launch
template <typename T>
bool sor_pass_ok(const falm_ctx *ctx, int H) {
    if (ctx->no_tma || ctx->A_explicit) return false;
    const size_t e = sizeof(T);
    using L2 = RB2Tile<T>;
    if (H == 3 && sor_skewed<T>(ctx) && map_ok(ctx, e, L2::BX, L2::BY) && map_ok(ctx, e, L2::BXB, L2::BYB)) return true;
    if (H == 1) return map_ok(ctx, e, RBTile<T, 1>::BX, RBTile<T, 1>::BY);
    if (H == 2) return map_ok(ctx, e, RBTile<T, 2>::BX, RBTile<T, 2>::BY);
    return map_ok(ctx, e, RBTile<T, 3>::BX, RBTile<T, 3>::BY);
}

// Whether the preconditioner's pointwise first sweep writes the work vector xp
// rather than its target z: the sweeps after it that run out of place (Jacobi
// sweeps 2..m; blocked SOR passes) alternate between xp and z, so an odd
// number of them starts from xp and the last one lands in z.  The buffers of
// an application are then the same at every iteration.
template <typename T>
bool pc_first_in_xp(const falm_ctx *ctx) {
    const int m = ctx->pc_maxit;
    if (ctx->pc_type == FALM_LS_JACOBI) return ((m - 1) & 1) != 0;
    if (ctx->pc_type != FALM_LS_SOR) return false;
    int passes = 0;
    for (int hs = 1; hs < 2 * m;) {
        const int H = std::min(3, 2 * m - hs);
        if (!sor_pass_ok<T>(ctx, H)) break;
        passes++;
        hs += H;
    }
    return (passes & 1) != 0;
}

// ring depth of the multi-field plane stream: keep >= 2 planes in flight and
// at least two CTAs per SM
template <typename T, int NF> struct P3Conf { static constexpr int NS = NF > 1 ? 4 : 6; };
// a body's own slot count (Body::kSlots, FP32 only): a deeper ring for a body
// whose register use already limits the CTAs per SM, so shared memory is free
template <typename T, int NF, class Body, class = void> struct P3NS { static constexpr int v = P3Conf<T, NF>::NS; };
template <typename T, int NF, class Body> struct P3NS<T, NF, Body, std::void_t<decltype(Body::kSlots)>> {
    static constexpr int v = sizeof(T) == 4 ? Body::kSlots : P3Conf<T, NF>::NS;
};

// multi-field radius-1 plane stream over region R (see plane3_tma.cuh);
// 1 launched, 0 not eligible (row-kernel fallback), <0 launch error
template <typename T, int NF, int NV, class Body>
int p3_launch(falm_ctx *ctx, int cls, cudaStream_t st, const Region3 &R, int org, const void *const (&ptr)[NF],
              const int (&ncomp)[NF], const Body &body) {
    if (ctx->no_tma) return 0;
    using L = P3Layout<T, NF, P3Rows<T, Body>::v>;
    constexpr int NS = P3NS<T, NF, Body>::v;
    MapSet<NF> maps;
    int slot = 0;
    for (int f = 0; f < NF; f++) {
        if (!make_map(ctx, &maps.m[f], (const T *)ptr[f], ncomp[f], L::BX, L::BY)) return 0;
        maps.ncomp[f] = ncomp[f];
        slot += ncomp[f] * L::FB;
    }
    // the kernel lays the slot out from the body's component counts
    if (slot != (Body::NC0 + Body::NC1) * L::FB) return -fail(ctx, FALM_ERR_ARG, "plane stream: field components do not match the body");
    const int smem = NS * slot + 256;
    const int bx = (R.i1 - R.i0 + L::TX - 1) / L::TX, by = (R.j1 - R.j0 + L::TY - 1) / L::TY;
    auto kern = k_plane3_tma<T, NF, NS, NV, Body>;
    const int kc = chunk_len(ctx, (long long)bx * by, R.k1 - R.k0, resident_per_sm(kern, 256, smem), 64, 2);
    dim3 grid(bx, by, (R.k1 - R.k0 + kc - 1) / kc);
    if ((long long)grid.x * grid.y * grid.z > ctx->red.maxBlocks) return 0;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int rc = launch_k(ctx, cls, st, [&] { kern<<<grid, 256, smem, st>>>(ctx->geo, R, org, kc, maps, body, ctx->red, ctx->kerr); });
    return rc ? -rc : 1;
}

#define P3_OR(CLS, ST, T_, NF_, NV_, R_, ORG_, PTRS_, NCOMP_, BODY_, ROWLAUNCH)            \
    do {                                                                                   \
        const void *const _pp[NF_] = PTRS_;                                                \
        const int _nc[NF_] = NCOMP_;                                                       \
        int _p3 = p3_launch<T_, NF_, NV_>(ctx, (CLS), (ST), (R_), (ORG_), _pp, _nc, BODY_);\
        if (_p3 < 0) return -_p3;                                                          \
        if (_p3 == 0) LAUNCH((CLS), (ST), ROWLAUNCH);                                      \
    } while (0)
#define FB_ARR(...) {__VA_ARGS__}
