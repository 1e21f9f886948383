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

// three FP32 half sweeps on the 28 x 16 tile; 1 launched, 0 not eligible, <0 launch error
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

template <typename T>
int sor_rb_launch(falm_ctx *ctx, cudaStream_t st, int H, const T *xin, const T *b, T *xout, T omega, int c1, const SolverScalars *sc) {
    // the blocked kernels take the colour parity of local plane indices: a grid
    // whose planes are offset by koff flips the first colour instead
    c1 ^= ctx->geo.koff & 1;
    if constexpr (sizeof(T) == 4) {
        if (H == 3 && !ctx->sor_v1) {
            const int r = sor_rb2_launch<T>(ctx, st, xin, b, xout, omega, c1, sc);
            if (r != 0) return r;
        }
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
    if constexpr (sizeof(T) == 4) {
        using L2 = RB2Tile<T>;
        if (H == 3 && !ctx->sor_v1 && map_ok(ctx, e, L2::BX, L2::BY) && map_ok(ctx, e, L2::BXB, L2::BYB)) return true;
    }
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

// multi-field radius-1 plane stream over region R (see plane3_tma.cuh);
// 1 launched, 0 not eligible (row-kernel fallback), <0 launch error
template <typename T, int NF, int NV, class Body>
int p3_launch(falm_ctx *ctx, int cls, cudaStream_t st, const Region3 &R, int org, const void *const (&ptr)[NF],
              const int (&ncomp)[NF], const Body &body) {
    if (ctx->no_tma) return 0;
    using L = P3Layout<T, NF>;
    constexpr int NS = P3Conf<T, NF>::NS;
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

// Build the separable Poisson tables.  For a Cartesian control volume
//   0.5*(g_d(c) + g_d(c+e_d))/ja(c)  with g_d = ja*kx_d^2
// depends on the index along d only; the table entry is evaluated with the
// reference's arithmetic (src/falm.h:394-400, app/nedo/main.cpp:43-83) at the
// cell (i, gc, gc) (resp. (gc, j, gc), (gc, gc, k)).  A dropped (Neumann)
// coefficient is stored as 0.
int build_poisson(falm_ctx *ctx, int kind) {
    const Geom &g = ctx->geo;
    const std::vector<double> *h[3] = {ctx->hx, ctx->hy, ctx->hz};
    const int s[3] = {g.sx, g.sy, g.sz};
    std::vector<double> up[3], um[3];
    double maxdiag = 0.0;
    auto gmet = [&](int d, int i, int j, int k) {
        double vol = (*h[0])[i] * (*h[1])[j] * (*h[2])[k];
        int id = d == 0 ? i : (d == 1 ? j : k);
        double kd = 1.0 / (*h[d])[id];
        return vol * kd * kd;
    };
    for (int d = 0; d < 3; d++) {
        up[d].assign(s[d], 0.0);
        um[d].assign(s[d], 0.0);
        for (int q = g.gc; q < s[d] - g.gc; q++) {
            int c[3] = {g.gc, g.gc, g.gc};
            c[d] = q;
            int cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
            cp[d] += 1; cm[d] -= 1;
            double jac = (*h[0])[c[0]] * (*h[1])[c[1]] * (*h[2])[c[2]];
            double gc0 = gmet(d, c[0], c[1], c[2]);
            double coef_p = 0.5 * (gc0 + gmet(d, cp[0], cp[1], cp[2])) / jac;
            double coef_m = 0.5 * (gc0 + gmet(d, cm[0], cm[1], cm[2])) / jac;
            // app/nedo/main.cpp:55 keeps the x+ coefficient (p = 0 guide cell); every other
            // physical face is Neumann (:60-83, app/lid3d/main.cpp:52-80); a slab interface
            // keeps its coefficients (the neighbour's plane lies beyond it)
            int plus_limit = (d == 0 && kind == FALM_BC_CHANNEL) ? s[d] - g.gc : s[d] - g.gc - 1;
            if (d == 2 && !(g.zphys & 2)) plus_limit = s[d] - g.gc;
            if (q < plus_limit) up[d][q] = coef_p;
            if (q > g.gc || (d == 2 && !(g.zphys & 1))) um[d][q] = coef_m;
        }
    }
    // maxdiag over the interior: |ac| is separable as well, but take the
    // exact maximum of the reference's accumulation order
    for (int k = g.gc; k < g.sz - g.gc; k++)
        for (int j = g.gc; j < g.sy - g.gc; j++)
            for (int i = g.gc; i < g.sx - g.gc; i++) {
                double ac = ((((-up[0][i]) - um[0][i]) - up[1][j]) - um[1][j] - up[2][k]) - um[2][k];
                maxdiag = std::max(maxdiag, std::fabs(ac));
            }
    if (ctx->slab_on && ctx->slab_nranks > 1) {
        // the maximum over the slabs (a collective: every rank builds its operator)
        double *d = nullptr;
        if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) { cudaGetLastError(); return fail(ctx, FALM_ERR_ALLOC, "poisson: maxdiag"); }
        int rc = cudaMemcpy(d, &maxdiag, sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess ? FALM_OK : FALM_ERR_CUDA;
        if (!rc) rc = ctx->transport.allreduce(ctx->transport.user, d, 1, FALM_REDUCE_MAX, nullptr);
        if (!rc && (cudaMemcpy(&maxdiag, d, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)) rc = FALM_ERR_CUDA;
        cudaFree(d);
        if (rc) { cudaGetLastError(); return fail(ctx, rc, "poisson: maxdiag over the slabs"); }
    }
    double scale = 1.0 / maxdiag;
    // layout: for each d: cm, cp, um, up (s[d] each), then dx0 (sx)
    size_t tot = 0;
    for (int d = 0; d < 3; d++) tot += 4 * (size_t)s[d];
    tot += g.sx;
    std::vector<double> h64(tot);
    std::vector<float> h32(tot);
    size_t off = 0;
    size_t o_cm[3], o_cp[3], o_um[3], o_up[3], o_dx0;
    for (int d = 0; d < 3; d++) {
        o_cm[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = um[d][q] * scale; off += s[d];
        o_cp[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = up[d][q] * scale; off += s[d];
        o_um[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = um[d][q]; off += s[d];
        o_up[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = up[d][q]; off += s[d];
    }
    o_dx0 = off;
    for (int q = 0; q < g.sx; q++) h64[off + q] = (-up[0][q]) - um[0][q];
    off += g.sx;
    for (size_t q = 0; q < tot; q++) h32[q] = (float)h64[q];
    if (ctx->op_mem) { cudaFree(ctx->op_mem); ctx->op_mem = nullptr; }
    void *mem = nullptr;
    if (cudaMalloc(&mem, tot * (sizeof(double) + sizeof(float))) != cudaSuccess) { cudaGetLastError(); return fail(ctx, FALM_ERR_ALLOC, "poisson tables"); }
    double *d64 = (double *)mem;
    float *d32 = (float *)(d64 + tot);
    if (cudaMemcpy(d64, h64.data(), tot * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d32, h32.data(), tot * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(ctx, FALM_ERR_CUDA, "poisson tables copy");
    ctx->op_mem = mem;
    for (int d = 0; d < 3; d++) {
        ctx->pt64.cm[d] = d64 + o_cm[d]; ctx->pt64.cp[d] = d64 + o_cp[d]; ctx->pt64.um[d] = d64 + o_um[d]; ctx->pt64.up[d] = d64 + o_up[d];
        ctx->pt32.cm[d] = d32 + o_cm[d]; ctx->pt32.cp[d] = d32 + o_cp[d]; ctx->pt32.um[d] = d32 + o_um[d]; ctx->pt32.up[d] = d32 + o_up[d];
    }
    ctx->pt64.dx0 = d64 + o_dx0; ctx->pt32.dx0 = d32 + o_dx0;
    ctx->pt64.scale = scale; ctx->pt32.scale = (float)scale;
    ctx->pt64.koff = ctx->pt32.koff = g.koff;
    ctx->maxdiag = maxdiag;
    ctx->op_ready = 1;
    ctx->bc_kind_op = kind;
    // the coefficient of cell q towards q+1 equals that of q+1 towards q on every
    // axis (uniform spacing): the operator is symmetric over the interior
    ctx->op_symmetric = 1;
    for (int d = 0; d < 3; d++)
        for (int q = g.gc; q + 1 < s[d] - g.gc; q++)
            if (std::fabs(up[d][q] - um[d][q + 1]) > 1e-13 * std::fabs(up[d][q])) ctx->op_symmetric = 0;
    return FALM_OK;
}

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
// dropped when the solver settings or the operator change.  Used where launch
// and host-synchronisation latency dominate: grids of at most kGraphCells
// interior cells (FALM_B200_GRAPH=1 / 0 forces it on / off), never while
// profiling or checking launches one by one.
constexpr long long kGraphCells = 1ll << 22;
constexpr int kMixedPassIts = 50;   // FP32 BiCGStab iterations between FP64 true-residual checks

bool use_graph(const falm_ctx *ctx) {
    if (ctx->profiling || ctx->check_sync || ctx->graph_mode == 0) return false;
    return ctx->graph_mode == 1 || (long long)ctx->geo.nx * ctx->geo.ny * ctx->geo.nz <= kGraphCells;
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
        LAUNCH(FALM_K_OTHER, st, k_copy_shell<T><<<ctx->sm_count * 8, 256, 0, st>>>(g, u, ua));
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
    // 6. keep the previous velocity at the outlet planes, then project
    if (chan) { LAUNCH(FALM_K_OTHER, st, k_save_outlet<T><<<std::min(ctx->sm_count * 4, (3 * g.sy * g.sz + 255) / 256), 256, 0, st>>>(g, u, (T *)ctx->w_outlet)); }
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

// Whole steps as CUDA graphs (grids where launch and synchronisation latency
// dominate, see use_graph): the phases before the solve, the solve with its
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
        ctx->step_graphs->push_back(falm_ctx::StepGraph{f->u, f->uu, f->p, f->nut, f->ff, dt, inlet, n_pre + rec.fixed + n_post, rec.per_iter,
                                                        gr, ex});
        sg = &ctx->step_graphs->back();
    }
    *ctx->t_host = t;
    ctx->inlet_plane_valid = 0;   // the streamed plane serves one step
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
        ctx->graph_mode = (gm && gm[0] == '0') ? 0 : ((gm && gm[0] == '1') ? 1 : -1);
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
        ctx->sor_v1 = (v && v[0] == '1') ? 1 : 0;
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
    if (!ctx || !plane) return FALM_ERR_ARG;
    const size_t n = 3ull * ctx->geo.ny * ctx->geo.nz;
    if (!ctx->inlet_plane) CK(cudaMalloc(&ctx->inlet_plane, n * sizeof(double)));
    CK(cudaMemcpyAsync(ctx->inlet_plane, plane, n * sizeof(double), cudaMemcpyHostToDevice, S(stream)));
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
