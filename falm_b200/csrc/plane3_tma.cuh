// Generic 2.5D TMA plane stream for radius-1 stencils over several fields
// (face velocity + RHS, projection, SGS + divergence).
//
// Each field f (ncomp_f components) is streamed as (36 x 10 x 1 x ncomp_f)
// boxes; a slot holds every field of one z plane and the ring keeps planes
// k-1, k, k+1 resident while k+2.. are in flight.  Tiles are 32 x 8 columns;
// the box starts one column/row before the tile (`org` = 1) or two columns
// before it (`org` = 2), whichever keeps the x coordinate 16-byte aligned for
// the tile origin the kernel uses:
//   interior kernels: tile i0 = gc + 32 bx, box x = i0 - 2  (org 2)
//   face-map kernels: tile i0 = gc - 1 + 32 bx, box x = i0 - 1  (org 1)
// (both start at 32 bx for gc = 2).
#pragma once
#include <type_traits>
#include "common.cuh"
#include "poisson.cuh"
#include "tma.cuh"

namespace fb {

template <int NF>
struct alignas(64) MapSet {
    CUtensorMap m[NF];
    int ncomp[NF];
};

template <typename T, int NF, int RY_ = 2>
struct P3Layout {
    static constexpr int RY = RY_;   // rows per thread: thread (tx, ty) computes rows ty (, ty + 8)
    static constexpr int TX = 32, TY = 8 * RY, BX = 36, BY = TY + 2, PE = BX * BY;
    static constexpr int FB = (PE * (int)sizeof(T) + 127) / 128 * 128;   // one component plane
};

// view of the resident planes for the body
template <typename T, int NF, int RY_ = 2>
struct P3View {
    const T *pl[3];   // slot base of planes k-1, k, k+1
    int foff[NF];     // byte offset of field f inside a slot
    int o;            // own element offset inside a component plane
    __device__ __forceinline__ T at(int f, int d, int dz, int dx = 0, int dy = 0) const {
        const T *base = (const T *)((const unsigned char *)pl[dz + 1] + foff[f]);
        return base[d * P3Layout<T, NF, RY_>::PE + o + dy * P3Layout<T, NF, RY_>::BX + dx];
    }
};

// metric factors of the 3 x 3 columns around (i, j) and of planes k-1..k+1, with
// MetricView's association (ja = (hx*hy)*hz, g_d = (ja*k_d)*k_d); offsets -1, 0, +1
template <typename T>
struct ColMet {
    T hx[3], kx[3], hy[3], ky[3], hz[3], kz[3];
    __device__ __forceinline__ T ja(int dx, int dy, int dz) const { return (hx[1 + dx] * hy[1 + dy]) * hz[1 + dz]; }
    __device__ __forceinline__ T k(int d, int dx, int dy, int dz) const { return d == 0 ? kx[1 + dx] : (d == 1 ? ky[1 + dy] : kz[1 + dz]); }
    __device__ __forceinline__ T g(int d, int dx, int dy, int dz) const {
        const T kk = k(d, dx, dy, dz);
        return (ja(dx, dy, dz) * kk) * kk;
    }
};

// pointwise operands (or per-column / per-plane state) of a body that has none
struct NoPW {};

// resident CTAs per SM asked of the register allocator: 4 in FP32 (at most 64
// registers), 2 in FP64, or the body's own kMinBlocks
template <typename T, class Body, class = void> struct P3MinB { static constexpr int v = sizeof(T) == 4 ? 4 : 2; };
template <typename T, class Body> struct P3MinB<T, Body, std::void_t<decltype(Body::kMinBlocks)>> {
    static constexpr int v = sizeof(T) == 4 ? Body::kMinBlocks : 2;
};
template <typename T, class Body> constexpr int p3_minb() { return P3MinB<T, Body>::v; }

// rows per thread: 2, or in FP64 the body's own kRows64 (one row halves the
// ring of a six-component stream, which otherwise admits one CTA per SM)
template <typename T, class Body, class = void> struct P3Rows { static constexpr int v = 2; };
template <typename T, class Body> struct P3Rows<T, Body, std::void_t<decltype(Body::kRows64)>> {
    static constexpr int v = sizeof(T) == 8 ? Body::kRows64 : 2;
};

// Body: bool skip() const; MetricView<T> mv; type PW (the cell's pointwise
//       operands) and PW pw_load(i, j, k, cc) const; types CS, ZS (state of a
//       column and of a plane) with CS col_state(i, j) const, ZS plane_state(k)
//       const, evaluated once per thread and row, and once per plane;
//       void cell(i, j, k, cc, const P3View&, const ColMet&, const PW&, const CS&,
//       const ZS&, acc); void finish(tot)
// The pointwise operands of a plane are loaded before the wait for the plane
// ahead, for every row of the thread, so their latency overlaps the wait.
template <typename T, int NF, int NS, int NV, class Body>
__global__ void __launch_bounds__(256, (p3_minb<T, Body>())) k_plane3_tma(Geom g, Region3 R, int org, int kc, const __grid_constant__ MapSet<NF> maps,
                                                  Body body, RedWork rw, int *err) {
    using L = P3Layout<T, NF, P3Rows<T, Body>::v>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    // slot layout from the body's component counts (compile-time offsets)
    constexpr int FOFF1 = Body::NC0 * L::FB, SLOTB = (Body::NC0 + Body::NC1) * L::FB;
    constexpr uint32_t TXB = (Body::NC0 + Body::NC1) * L::PE * sizeof(T);
    static_assert(NF == 1 ? Body::NC1 == 0 : Body::NC1 > 0, "component counts match the fields");
    uint64_t *bar = (uint64_t *)(smem + NS * SLOTB);
    if (body.skip()) return;
    constexpr int RY = L::RY;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i0 = R.i0 + blockIdx.x * L::TX, j0 = R.j0 + blockIdx.y * L::TY;
    const int k0 = R.k0 + blockIdx.z * kc, k1 = min(k0 + kc, R.k1);
    const int i = i0 + tx;
    const int P0 = k0 - 1, nplanes = (k1 + 1) - P0;
    P3View<T, NF, L::RY> v;
    v.foff[0] = 0;
    if (NF > 1) v.foff[NF - 1] = FOFF1;
    const int xb = box_origin(i0 - org, L::BX, g.sx, 16 / (int)sizeof(T)), yb = box_origin(j0 - 1, L::BY, g.sy, 1);
    const int ox = min(i, R.i1 - 1) - xb;
    int jr[RY], orr[RY];
    bool act[RY];
#pragma unroll
    for (int r = 0; r < RY; r++) {
        jr[r] = j0 + ty + 8 * r;
        act[r] = i < R.i1 && jr[r] < R.j1;
        const int oy = min(jr[r], R.j1 - 1) - yb;
        orr[r] = oy * L::BX + ox;
        // self-check: the radius-1 neighbourhood of a computed cell lies inside the staged box
        if (act[r] && (ox < 1 || ox > L::BX - 2 || oy < 1 || oy > L::BY - 2)) { atomicExch(err, 300 + 3); act[r] = false; }
    }
    double acc[NV > 0 ? NV : 1];
#pragma unroll
    for (int d = 0; d < (NV > 0 ? NV : 1); d++) acc[d] = 0.0;
    // column metric factors (x shared by the rows, y per row); z rolled per plane below
    ColMet<T> cm[RY];
    typename Body::CS cst[RY];
#pragma unroll
    for (int r = 0; r < RY; r++) cst[r] = body.col_state(min(i, R.i1 - 1), min(jr[r], R.j1 - 1));
    const MetricView<T> &mv = body.mv;
    {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int ic = min(max(i - 1 + q, 0), g.sx - 1);
            const T hxv = ldg(mv.m.h[0] + ic), kxv = ldg(mv.m.k[0] + ic);
#pragma unroll
            for (int r = 0; r < RY; r++) {
                const int jc = min(max(jr[r] - 1 + q, 0), g.sy - 1);
                cm[r].hx[q] = hxv; cm[r].kx[q] = kxv;
                cm[r].hy[q] = ldg(mv.m.h[1] + jc); cm[r].ky[q] = ldg(mv.m.k[1] + jc);
            }
        }
    }
    // plane q into slot s = q % NS (the caller passes s, a constant in the march)
    auto issue = [&](int q, int s) {
        uint64_t *b = bar + s;
        unsigned char *dst = smem + s * SLOTB;
        bool ok = true;
#pragma unroll
        for (int f = 0; f < NF; f++) ok = ok && tma_ok(dst + (f ? FOFF1 : 0), xb, yb, P0 + q, (int)sizeof(T), g.sx, g.sy, g.sz);
        if (!ok) {
            tma_reject(b, err, 3);
            return;
        }
        mbar_expect_tx(b, TXB);
#pragma unroll
        for (int f = 0; f < NF; f++) tma_load_4d(dst + (f ? FOFF1 : 0), &maps.m[f], xb, yb, P0 + q, 0, b);
    };
    // warp 0 polls the barriers; the block barrier that follows makes the
    // landed planes visible to every thread
    auto wait_s = [&](int s, int parity) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + s, parity, err); };
    if (threadIdx.x == 0) {
#pragma unroll
        for (int f = 0; f < NF; f++) prefetch_tmap(&maps.m[f]);
        for (int s = 0; s < NS; s++) mbar_init(bar + s, 1);
        mbar_fence_init();
    }
    __syncthreads();
    int issued = min(NS, nplanes), waited = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < issued; q++) issue(q, q % NS);
    // every plane is waited for exactly once, before its first read: planes 0
    // and 1 here, plane q+1 at iteration q
    bool fail = !wait_s(0, 0);
    fail = !wait_s(1 % NS, 1 / NS) || fail;
    waited = 2;
    if (__syncthreads_or(fail)) goto drain;
    {
        const long long sxy = (long long)g.sx * g.sy;
        long long ccr[RY];
#pragma unroll
        for (int r = 0; r < RY; r++) ccr[r] = g.id(i, jr[r], P0 + 1);
        // z metric factors of planes k-1, k, k+1 (rolled)
        T hz0 = ldg(mv.m.h[2] + max(P0, 0)), kz0 = ldg(mv.m.k[2] + max(P0, 0));
        T hz1 = ldg(mv.m.h[2] + P0 + 1), kz1 = ldg(mv.m.k[2] + P0 + 1);
        // pointwise operands, loaded one plane ahead of their use
        typename Body::PW pwv[RY], pwn[RY];
#pragma unroll
        for (int r = 0; r < RY; r++)
            if (act[r]) pwv[r] = body.pw_load(i, jr[r], P0 + 1, ccr[r]);
        // the march, unrolled over the slots: plane q = q0 + u is in slot u
        int ph = 0;   // (q0 / NS) & 1
        for (int q0 = 0; q0 < nplanes - 1; q0 += NS, ph ^= 1) {
#pragma unroll
            for (int u = 0; u < NS; u++) {
                const int q = q0 + u;
                if (q < 1) continue;
                if (q >= nplanes - 1) break;
                const int k = P0 + q;
                const bool ahead = q + 1 < nplanes - 1;
#pragma unroll
                for (int r = 0; r < RY; r++)
                    if (act[r] && ahead) pwn[r] = body.pw_load(i, jr[r], k + 1, ccr[r] + sxy);
                const int kn = min(k + 1, g.sz - 1);
                const T hz2 = ldg(mv.m.h[2] + kn), kz2 = ldg(mv.m.k[2] + kn);
                fail = !wait_s((u + 1) % NS, (u + 1 < NS) ? ph : ph ^ 1);
                waited = q + 2;
                if (__syncthreads_or(fail)) goto drain;
                // plane q-2 is no longer needed: refill its slot
                if (q >= 2 && q - 2 + NS < nplanes) {
                    if (threadIdx.x == 0) { fence_proxy_async(); issue(q - 2 + NS, (u + NS - 2) % NS); }
                    issued = q - 2 + NS + 1;
                }
                const typename Body::ZS zst = body.plane_state(k);
                v.pl[0] = (const T *)(smem + ((u + NS - 1) % NS) * SLOTB);
                v.pl[1] = (const T *)(smem + u * SLOTB);
                v.pl[2] = (const T *)(smem + ((u + 1) % NS) * SLOTB);
#pragma unroll
                for (int r = 0; r < RY; r++) {
                    if (act[r]) {
                        v.o = orr[r];
                        cm[r].hz[0] = hz0; cm[r].hz[1] = hz1; cm[r].hz[2] = hz2;
                        cm[r].kz[0] = kz0; cm[r].kz[1] = kz1; cm[r].kz[2] = kz2;
                        body.cell(i, jr[r], k, ccr[r], v, cm[r], pwv[r], cst[r], zst, acc);
                    }
                    ccr[r] += sxy;
                    pwv[r] = pwn[r];
                }
                hz0 = hz1; hz1 = hz2; kz0 = kz1; kz1 = kz2;
            }
        }
    }
    goto reduce;
drain:
    for (int q = waited; q < issued; q++) wait_s(q % NS, (q / NS) & 1);
reduce:
    if (NV > 0) {
        double tot[NV > 0 ? NV : 1];
        if (grid_sum<(NV > 0 ? NV : 1)>(acc, rw, tot) && threadIdx.x == 0) body.finish(tot);
    }
}

}  // namespace fb

namespace fb {

// ---------------------------------------------------------------- face velocity + RHS body
// UtoCU + InterpolateCU (src/dev/FalmCFDDevCall.cu:303-349) on the face map,
// [uubc, app/lid3d/bcdev.cu:251-322,] and the scaled divergence at interior
// cells (src/FalmCFD.h:96-109).  Field 0: the velocity to interpolate (3 comps),
// whose guide cells must hold the previous velocity.
template <typename T, bool RHS, bool CAVITY>
struct UtoUUBody {
    Geom g;
    MetricView<T> mv;
    T *uu, *rhs;
    T scale;
    static constexpr int NC0 = 3, NC1 = 0;   // field: the velocity to interpolate
    using PW = NoPW;
    using CS = NoPW;
    using ZS = NoPW;
    __device__ bool skip() const { return false; }
    __device__ PW pw_load(int, int, int, long long) const { return PW{}; }
    __device__ CS col_state(int, int) const { return CS{}; }
    __device__ ZS plane_state(int) const { return ZS{}; }
    __device__ __forceinline__ T ucv(const P3View<T, 1> &v, const ColMet<T> &cm, int d, int dx, int dy, int dz) const {
        return cm.ja(dx, dy, dz) * cm.k(d, dx, dy, dz) * v.at(0, d, dz, dx, dy);
    }
    __device__ __forceinline__ bool zero_face(int d, int i, int j, int k) const {
        if (!CAVITY) return false;
        const bool jin = j >= g.gc && j < g.sy - g.gc, kin = k >= g.gc && k < g.sz - g.gc, iin = i >= g.gc && i < g.sx - g.gc;
        if (d == 0) return (i == g.gc - 1 || i == g.sx - g.gc - 1) && jin && kin;
        if (d == 1) return (j == g.gc - 1 || j == g.sy - g.gc - 1) && iin && kin;
        return ((k == g.gc - 1 && (g.zphys & 1)) || (k == g.sz - g.gc - 1 && (g.zphys & 2))) && iin && jin;   // not at slab interfaces
    }
    // face d of cell (i+dx, j+dy, k+dz) (the face towards +d)
    __device__ __forceinline__ T face(const P3View<T, 1> &v, const ColMet<T> &cm, int d, int i, int j, int k, int dx, int dy,
                                      int dz) const {
        if (zero_face(d, i + dx, j + dy, k + dz)) return T(0);
        T a = ucv(v, cm, d, dx, dy, dz);
        T b = ucv(v, cm, d, dx + (d == 0), dy + (d == 1), dz + (d == 2));
        return T(0.5) * (a + b);
    }
    __device__ void cell(int i, int j, int k, long long c, const P3View<T, 1> &v, const ColMet<T> &cm, const PW &, const CS &,
                         const ZS &, double (&)[1]) const {
        const T UE = face(v, cm, 0, i, j, k, 0, 0, 0), VN = face(v, cm, 1, i, j, k, 0, 0, 0), WT = face(v, cm, 2, i, j, k, 0, 0, 0);
        uu[c] = UE; uu[c + g.n] = VN; uu[c + 2 * g.n] = WT;
        if (RHS && i >= g.gc && j >= g.gc && k >= g.gc) {
            const T UW = face(v, cm, 0, i, j, k, -1, 0, 0), VS = face(v, cm, 1, i, j, k, 0, -1, 0), WB = face(v, cm, 2, i, j, k, 0, 0, -1);
            // 1/ja as the product of the inverse widths
            T div = (UE - UW + VN - VS + WT - WB) * ((cm.kx[1] * cm.ky[1]) * cm.kz[1]);
            rhs[c] = div * scale;
        }
    }
    __device__ void finish(const double (&)[1]) const {}
};

// ---------------------------------------------------------------- projection body
// ProjectPGrid + ProjectPFace (src/dev/FalmCFDDevCall.cu:351-407) on the face
// map; field 0: the pressure (1 comp).  u may alias ua, uu may alias uua.
template <typename T>
struct ProjectBody {
    Geom g;
    MetricView<T> mv;
    T *u;
    const T *ua;
    T *uu;
    const T *uua;
    T dt;
    static constexpr int NC0 = 1, NC1 = 0;   // field: the pressure
    static constexpr int kMinBlocks = 3;     // FP32: room for the pointwise operands loaded a plane ahead
    // face velocity (f) and cell velocity (a, interior cells only) before the correction
    struct PW { T f0, f1, f2, a0, a1, a2; };
    using CS = NoPW;
    using ZS = NoPW;
    __device__ bool skip() const { return false; }
    __device__ CS col_state(int, int) const { return CS{}; }
    __device__ ZS plane_state(int) const { return ZS{}; }
    __device__ PW pw_load(int i, int j, int k, long long cc) const {
        const long long N = g.n;
        PW w;
        w.f0 = uua[cc]; w.f1 = uua[cc + N]; w.f2 = uua[cc + 2 * N];
        w.a0 = w.a1 = w.a2 = T(0);
        if (i >= g.gc && j >= g.gc && k >= g.gc) { w.a0 = ua[cc]; w.a1 = ua[cc + N]; w.a2 = ua[cc + 2 * N]; }
        return w;
    }
    __device__ void cell(int i, int j, int k, long long cc, const P3View<T, 1> &v, const ColMet<T> &cm, const PW &w, const CS &,
                         const ZS &, double (&)[1]) const {
        const long long N = g.n;
        const T pcc = v.at(0, 0, 0), pe = v.at(0, 0, 0, 1, 0), pn = v.at(0, 0, 0, 0, 1), pt = v.at(0, 0, 1);
        const T dpx = T(0.5) * (cm.g(0, 0, 0, 0) + cm.g(0, 1, 0, 0)) * (pe - pcc);
        const T dpy = T(0.5) * (cm.g(1, 0, 0, 0) + cm.g(1, 0, 1, 0)) * (pn - pcc);
        const T dpz = T(0.5) * (cm.g(2, 0, 0, 0) + cm.g(2, 0, 0, 1)) * (pt - pcc);
        const T f0 = w.f0, f1 = w.f1, f2 = w.f2;
        const bool in = i >= g.gc && j >= g.gc && k >= g.gc;
        T a0 = 0, a1 = 0, a2 = 0, gx = 0, gy = 0, gz = 0;
        if (in) {
            a0 = w.a0; a1 = w.a1; a2 = w.a2;
            gx = T(0.5) * cm.kx[1] * (pe - v.at(0, 0, 0, -1, 0));
            gy = T(0.5) * cm.ky[1] * (pn - v.at(0, 0, 0, 0, -1));
            gz = T(0.5) * cm.kz[1] * (pt - v.at(0, 0, -1));
        }
        uu[cc] = f0 - dt * dpx; uu[cc + N] = f1 - dt * dpy; uu[cc + 2 * N] = f2 - dt * dpz;
        if (in) { u[cc] = a0 - dt * gx; u[cc + N] = a1 - dt * gy; u[cc + 2 * N] = a2 - dt * gz; }
    }
    __device__ void finish(const double (&)[1]) const {}
};

// ---------------------------------------------------------------- face velocity + RHS + first residual
// UtoUUBody (RHS) fused with the residual that starts the Poisson solve (the
// pass residual of ResBody): r = rhs - A p in FP64 at interior cells, stored
// to rr with the first preconditioner sweep into pp, and the norms reduced
// into the solver scalars.  Fields: 0 the velocity to interpolate (3 comps),
// 1 the pressure (the solve's initial guess).
template <typename T, bool CAVITY>
struct UtoUUResBody {
    UtoUUBody<T, true, CAVITY> uub;
    MetricView<T> mv;
    Op7<T> op;
    T *rr, *pp;
    int pc_type;
    T pc_omega;
    SolverScalars *sc;
    static constexpr int NC0 = 3, NC1 = 1;
    static constexpr int kMinBlocks = 2;   // FP32: at most 128 registers (fewer spills than 3 CTAs per SM)
    static constexpr int kSlots = 6;       // FP32: 2 CTAs per SM leave room for 6 planes (3 in flight)
    using PW = NoPW;
    using CS = typename Op7<T>::Col;
    using ZS = typename Op7<T>::ZPl;
    __device__ bool skip() const { return false; }
    __device__ PW pw_load(int, int, int, long long) const { return PW{}; }
    __device__ CS col_state(int i, int j) const { return op.column(i, j); }
    __device__ ZS plane_state(int k) const { return op.zplane(k); }
    __device__ void cell(int i, int j, int k, long long c, const P3View<T, 2> &v, const ColMet<T> &cm, const PW &, const CS &cs,
                         const ZS &zs, double (&acc)[2]) const {
        const Geom &g = uub.g;
        // the face velocity and, at interior cells, the RHS (UtoUUBody's expressions)
        P3View<T, 1> v1;
        v1.pl[0] = v.pl[0]; v1.pl[1] = v.pl[1]; v1.pl[2] = v.pl[2];
        v1.foff[0] = v.foff[0];
        v1.o = v.o;
        const T UE = uub.face(v1, cm, 0, i, j, k, 0, 0, 0), VN = uub.face(v1, cm, 1, i, j, k, 0, 0, 0), WT = uub.face(v1, cm, 2, i, j, k, 0, 0, 0);
        uub.uu[c] = UE; uub.uu[c + g.n] = VN; uub.uu[c + 2 * g.n] = WT;
        if (i >= g.gc && j >= g.gc && k >= g.gc) {
            const T UW = uub.face(v1, cm, 0, i, j, k, -1, 0, 0), VS = uub.face(v1, cm, 1, i, j, k, 0, -1, 0),
                    WB = uub.face(v1, cm, 2, i, j, k, 0, 0, -1);
            const T div = (UE - UW + VN - VS + WT - WB) * ((cm.kx[1] * cm.ky[1]) * cm.kz[1]);
            const T bv = div * uub.scale;
            uub.rhs[c] = bv;
            // r = b - A p in FP64, the 7-point products accumulated in ResBody's order
            const T ac = op.ac_col(cs, zs);
            double ax = (double)ac * (double)v.at(1, 0, 0);
            ax = fma((double)cs.ae, (double)v.at(1, 0, 0, 1, 0), ax);
            ax = fma((double)cs.aw, (double)v.at(1, 0, 0, -1, 0), ax);
            ax = fma((double)cs.an, (double)v.at(1, 0, 0, 0, 1), ax);
            ax = fma((double)cs.as, (double)v.at(1, 0, 0, 0, -1), ax);
            ax = fma((double)zs.at, (double)v.at(1, 0, 1), ax);
            ax = fma((double)zs.ab, (double)v.at(1, 0, -1), ax);
            const double rv = (double)bv - ax;
            const T rt = (T)rv;
            rr[c] = rt;
            pp[c] = pc_first<T>(pc_type, i, j, k + op.t.koff, rt, ac, pc_omega);
            acc[0] += rv * rv;
            acc[1] += (double)rt * (double)rt;
        }
    }
    __device__ void finish(const double (&tot)[2]) const {
        // ResBody::finish of a pass residual
        const double err = sqrt(tot[0]) / sc->gsize;
        sc->err = err;
        sc->rho = tot[1];
        sc->rrho = 1.0; sc->alpha = 0.0; sc->omega = 1.0; sc->beta = 0.0;
        sc->first = 1;
        sc->done = 0;
        sc->checked = 0;
        if (!isfinite(err)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
        else if (fabs(tot[1]) < FLT_MIN) {
            sc->err = tot[1];
            sc->done = 1;
            sc->status = (err <= sc->tol) ? FALM_OK : FALM_ERR_BREAKDOWN;
        }
    }
};

// ---------------------------------------------------------------- SGS + divergence body
// Smagorinsky / CSM (src/dev/FalmCFDDevCall.cu:409-555) and the FP64
// divergence norm (:557-581 + app/nedo/main.cpp:194-197).  Fields: 0 u (3), 1 uu (3).
template <typename T>
struct SgsDivBody {
    Geom g;
    MetricView<T> mv;
    Metric<double> m64;
    T *nut;
    T Cs;
    int sgs;
    T *div_out;
    double *divsum;
    static constexpr int NC0 = 3, NC1 = 3;   // fields: the cell velocity, the face velocity
    static constexpr int kRows64 = 1;        // FP64: a 63 KB ring (2 CTAs per SM) instead of 126 KB
    using PW = NoPW;
    // filter width (cube root of the volume, as cbrt(hx) cbrt(hy) cbrt(hz)) and
    // the FP64 inverse widths, split into column and plane factors
    struct CS { T cbxy; double kxy; };
    struct ZS { T cbz; double kz; };
    __device__ bool skip() const { return false; }
    __device__ PW pw_load(int, int, int, long long) const { return PW{}; }
    __device__ CS col_state(int i, int j) const {
        return CS{cbrt(ldg(mv.m.h[0] + i)) * cbrt(ldg(mv.m.h[1] + j)), ldg(m64.k[0] + i) * ldg(m64.k[1] + j)};
    }
    __device__ ZS plane_state(int k) const { return ZS{cbrt(ldg(mv.m.h[2] + k)), ldg(m64.k[2] + k)}; }
    template <int RYV>
    __device__ void cell(int i, int j, int k, long long cc, const P3View<T, 2, RYV> &v, const ColMet<T> &cm, const PW &, const CS &cs,
                         const ZS &zs, double (&acc)[1]) const {
        if (sgs != FALM_SGS_EMPTY) {
            const T kxx = cm.kx[1], kxy = cm.ky[1], kxz = cm.kz[1];
            T dd[3][3];
#pragma unroll
            for (int m = 0; m < 3; m++) {
                dd[m][0] = T(0.5) * kxx * (v.at(0, m, 0, 1, 0) - v.at(0, m, 0, -1, 0));
                dd[m][1] = T(0.5) * kxy * (v.at(0, m, 0, 0, 1) - v.at(0, m, 0, 0, -1));
                dd[m][2] = T(0.5) * kxz * (v.at(0, m, 1) - v.at(0, m, -1));
            }
            const T dux = dd[0][0], duy = dd[0][1], duz = dd[0][2];
            const T dvx = dd[1][0], dvy = dd[1][1], dvz = dd[1][2];
            const T dwx = dd[2][0], dwy = dd[2][1], dwz = dd[2][2];
            T d1 = T(2) * (dux * dux), d2 = T(2) * (dvy * dvy), d3 = T(2) * (dwz * dwz);
            T d4 = (duy + dvx) * (duy + dvx), d5 = (dvz + dwy) * (dvz + dwy), d6 = (duz + dwx) * (duz + dwx);
            T Du = sqrt(d1 + d2 + d3 + d4 + d5 + d6);
            T De = cs.cbxy * zs.cbz;
            if (sgs == FALM_SGS_SMAGORINSKY) {
                T lc = Cs * De;
                nut[cc] = (lc * lc) * Du;
            } else {
                T e = dux * dux + duy * duy + duz * duz;
                e += dvx * dvx + dvy * dvy + dvz * dvz;
                e += dwx * dwx + dwy * dwy + dwz * dwz;
                e *= T(0.5);
                T q = dux * dux + duy * dvx + duz * dwx;
                q += dvx * duy + dvy * dvy + dvz * dwy;
                q += dwx * duz + dwy * dvz + dwz * dwz;
                q *= T(-0.5);
                T fcs = (q + copysign(T(1e-9), q)) / (e + copysign(T(1e-9), e));
                T CCsm = sqrt(fcs * fcs * fcs) * (T(1) - fcs) / T(22.0);
                nut[cc] = CCsm * (De * De) * Du;
            }
        }
        if (divsum) {
            double UE = to_d(v.at(1, 0, 0)), UW = to_d(v.at(1, 0, 0, -1, 0)), VN = to_d(v.at(1, 1, 0)), VS = to_d(v.at(1, 1, 0, 0, -1));
            double WT = to_d(v.at(1, 2, 0)), WB = to_d(v.at(1, 2, -1));
            // 1/ja as the product of the three FP64 inverse widths (one rounding
            // step per factor instead of a division)
            const double ija = cs.kxy * zs.kz;
            double dv = (UE - UW + VN - VS + WT - WB) * ija;
            if (div_out) div_out[cc] = (T)dv;
            acc[0] += dv * dv;
        }
    }
    __device__ void finish(const double (&tot)[1]) const {
        if (divsum) *divsum = tot[0];
    }
};

// ---------------------------------------------------------------- guide shell copy
// copy the first guide layer (cells of [gc-1, s-gc] outside the interior) of
// src into dst: the pseudo-velocity buffer then carries the previous
// velocity's guide values, as the reference's aliased u does.
template <typename T>
__global__ void k_copy_shell(Geom g, const T *__restrict__ src, T *__restrict__ dst) {
    // the shell of the a x b x c box (interior + one guide layer), enumerated
    // directly: the k = 0, c-1 planes, then the j = 0, b-1 rows, then the
    // i = 0, a-1 columns of the remaining (b-2) x (c-2) cells
    const int a = g.sx - 2 * g.gc + 2, b = g.sy - 2 * g.gc + 2, c = g.sz - 2 * g.gc + 2;
    const int ab = a * b, ac = a * (c - 2), bc = (b - 2) * (c - 2);
    const int tot = 2 * (ab + ac + bc);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) {
        int i, j, k, r = q;
        if (r < 2 * ab) {
            k = r < ab ? 0 : c - 1; r = r < ab ? r : r - ab;
            i = r % a; j = r / a;
        } else if ((r -= 2 * ab) < 2 * ac) {
            j = r < ac ? 0 : b - 1; r = r < ac ? r : r - ac;
            i = r % a; k = 1 + r / a;
        } else {
            r -= 2 * ac;
            i = r < bc ? 0 : a - 1; r = r < bc ? r : r - bc;
            j = 1 + r % (b - 2); k = 1 + r / (b - 2);
        }
        const long long id = g.id(i + g.gc - 1, j + g.gc - 1, k + g.gc - 1);
        dst[id] = src[id]; dst[id + g.n] = src[id + g.n]; dst[id + 2 * g.n] = src[id + 2 * g.n];
    }
}

}  // namespace fb
