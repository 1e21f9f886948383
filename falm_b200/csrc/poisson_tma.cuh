// 2.5D TMA versions of the 7-point Poisson kernels (residual, red-black SOR
// half sweep, operator application fused with the BiCGStab inner products).
//
// The stencil operand streams through a ring of shared-memory slots, one
// (36 x 10) TMA box per z plane: the 32 x 8 tile, one halo row on each y side
// and two halo columns on each x side (the box starts at i0-2 so that its x
// coordinate is 16-byte aligned).  The column's value at k-1 is kept in a
// register, k+1 comes from the next slot.  Pointwise operands (right-hand
// side, shadow residual, ...) are read with ordinary coalesced loads.
#pragma once
#include "poisson.cuh"
#include "tma.cuh"

namespace fb {

template <typename T>
struct S7Tile {
    static constexpr int RY = 2;   // rows per thread: thread (tx, ty) computes rows ty, ty + 8, ...
    static constexpr int TX = 32, TY = 8 * RY, BX = 36, BY = TY + 2, PE = BX * BY;
    static constexpr int SLOT = (PE * (int)sizeof(T) + 127) / 128 * 128;
};

template <typename T> struct S7Conf;
template <> struct S7Conf<double> { static constexpr int NS = 6; };
template <> struct S7Conf<float> { static constexpr int NS = 8; };

// resident CTAs per SM asked of the register allocator: 4 for FP32 arithmetic
// on an FP32 field (at most 64 registers), fewer where the body works in FP64
template <typename T, class Body>
constexpr int s7_minb() { return (sizeof(T) == 4 && sizeof(typename Body::V) == 4) ? 4 : (sizeof(T) == 4 ? 3 : 2); }

template <typename T>
constexpr int s7_smem() { return S7Conf<T>::NS * S7Tile<T>::SLOT + 128 + 128; }

// Body: type V (the stencil's arithmetic type: T, or double for an FP64
//       residual of an FP32 field); bool skip() const; const T *pw() const
//       (pointwise operand, or null); const Op7<T> &op_() const;
//       void cell(i, j, k, cc, a, xc, xe, xw, xn, xs, xt, xb, pv, acc); void finish(tot)
// The kernel hoists the x/y part of the operator out of the z march, loads the
// z part once per plane for all rows of a thread, and passes the cell's
// coefficients a (Coef7<V>) and neighbours in V: the column coefficients are
// converted once per column, the -1 neighbour is carried from the previous
// plane already converted.
// The pointwise operand of the next plane is loaded one iteration ahead (pv),
// so its latency overlaps the current plane's wait and arithmetic.
template <typename T, int NV, class Body>
__global__ void __launch_bounds__(256, (s7_minb<T, Body>())) k_s7_tma(Geom g, int kc, const __grid_constant__ CUtensorMap mx, Body body,
                                              RedWork rw, int *err) {
    using L = S7Tile<T>;
    using V = typename Body::V;
    constexpr int NS = S7Conf<T>::NS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t *bar = (uint64_t *)(smem + NS * L::SLOT);
    if (body.skip()) return;
    constexpr int RY = L::RY;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i0 = g.gc + blockIdx.x * L::TX, j0 = g.gc + blockIdx.y * L::TY;
    const int k0 = g.gc + blockIdx.z * kc, k1 = min(k0 + kc, g.sz - g.gc);
    const int i = i0 + tx;
    const int P0 = k0 - 1, nplanes = (k1 + 1) - P0;   // planes k0-1 .. k1
    const int xb = box_origin(i0 - 2, L::BX, g.sx, 16 / (int)sizeof(T)), yb = box_origin(j0 - 1, L::BY, g.sy, 1);
    const int ox = min(i, g.sx - g.gc - 1) - xb;
    int jr[RY], orr[RY];
    bool act[RY];
#pragma unroll
    for (int r = 0; r < RY; r++) {
        jr[r] = j0 + ty + 8 * r;
        act[r] = i < g.sx - g.gc && jr[r] < g.sy - g.gc;
        const int oy = min(jr[r], g.sy - g.gc - 1) - yb;
        orr[r] = oy * L::BX + ox;
        // self-check: the radius-1 neighbourhood of a computed cell lies inside the staged box
        if (act[r] && (ox < 1 || ox > L::BX - 2 || oy < 1 || oy > L::BY - 2)) { atomicExch(err, 300 + 2); act[r] = false; }
    }
    double acc[NV > 0 ? NV : 1];
#pragma unroll
    for (int d = 0; d < (NV > 0 ? NV : 1); d++) acc[d] = 0.0;
    auto slot = [&](int q) { return (const T *)(smem + (q % NS) * L::SLOT); };
    auto issue = [&](int q) {
        uint64_t *b = bar + (q % NS);
        unsigned char *dst = smem + (q % NS) * L::SLOT;
        if (tma_ok(dst, xb, yb, P0 + q, (int)sizeof(T), g.sx, g.sy, g.sz)) {
            mbar_expect_tx(b, L::PE * sizeof(T));
            tma_load_4d(dst, &mx, xb, yb, P0 + q, 0, b);
        } else {
            tma_reject(b, err, 2);
        }
    };
    // warp 0 polls the barriers; the block barrier that follows makes the
    // landed planes visible to every thread
    auto wait_q = [&](int q) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + (q % NS), (q / NS) & 1, err); };
    if (threadIdx.x == 0) {
        prefetch_tmap(&mx);
        for (int s = 0; s < NS; s++) mbar_init(bar + s, 1);
        mbar_fence_init();
    }
    __syncthreads();
    int issued = min(NS, nplanes), waited = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < issued; q++) issue(q);
    // every plane is waited for exactly once, before its first read: planes 0
    // and 1 here, plane q+1 at iteration q
    bool fail = !wait_q(0);
    fail = !wait_q(1) || fail;
    waited = 2;
    const T *pw = body.pw();
    const long long sxy = (long long)g.sx * g.sy;
    const Op7<T> &op = body.op_();
    long long ccr[RY];
    T pv[RY];
    V xm[RY];
    typename Op7<T>::Col col[RY];
    V cwv[RY], cev[RY], csv[RY], cnv[RY];
#pragma unroll
    for (int r = 0; r < RY; r++) {
        ccr[r] = g.id(i, jr[r], P0 + 1);   // cell of the first computed plane
        pv[r] = (pw && act[r]) ? pw[ccr[r]] : T(0);
        col[r] = op.column(min(i, g.sx - g.gc - 1), min(jr[r], g.sy - g.gc - 1));
        cwv[r] = (V)col[r].aw; cev[r] = (V)col[r].ae; csv[r] = (V)col[r].as; cnv[r] = (V)col[r].an;
    }
    if (__syncthreads_or(fail)) goto drain;
#pragma unroll
    for (int r = 0; r < RY; r++) xm[r] = (V)slot(0)[orr[r]];
    for (int q = 1; q < nplanes - 1; q++) {
        T pn[RY];
#pragma unroll
        for (int r = 0; r < RY; r++) pn[r] = (pw && act[r] && q + 1 < nplanes - 1) ? pw[ccr[r] + sxy] : T(0);
        fail = !wait_q(q + 1);
        waited = q + 2;
        if (__syncthreads_or(fail)) goto drain;
        if (q - 1 + NS < nplanes) {   // plane q-1 is no longer read (its values are in xm): refill its slot
            if (threadIdx.x == 0) { fence_proxy_async(); issue(q - 1 + NS); }
            issued = q - 1 + NS + 1;
        }
        const T *X0 = slot(q), *X1 = slot(q + 1);
        const int k = P0 + q;
        const typename Op7<T>::ZPl zp = op.zplane(k);
        const V abv = (V)zp.ab, atv = (V)zp.at;
#pragma unroll
        for (int r = 0; r < RY; r++) {
            const int o = orr[r];
            const V xc = (V)X0[o];
            if (act[r]) {
                Coef7<V> a;
                if (op.A) {
                    const Coef7<T> e = op.at_col(col[r], k, ccr[r]);
                    a = Coef7<V>{(V)e.ac, (V)e.aw, (V)e.ae, (V)e.as, (V)e.an, (V)e.ab, (V)e.at};
                } else {
                    a = Coef7<V>{(V)op.ac_col(col[r], zp), cwv[r], cev[r], csv[r], cnv[r], abv, atv};
                }
                body.cell(i, jr[r], k, ccr[r], a, xc, (V)X0[o + 1], (V)X0[o - 1], (V)X0[o + L::BX], (V)X0[o - L::BX], (V)X1[o], xm[r],
                          pv[r], acc);
            }
            xm[r] = xc;
            pv[r] = pn[r];
            ccr[r] += sxy;
        }
    }
    goto reduce;
drain:
    for (int q = waited; q < issued; q++) wait_q(q);
reduce:
    if (NV > 0) {
        double tot[NV > 0 ? NV : 1];
        if (grid_sum<(NV > 0 ? NV : 1)>(acc, rw, tot) && threadIdx.x == 0) body.finish(tot);
    }
}

// ---------------------------------------------------------------- bodies
template <typename T>
__device__ __forceinline__ T dot7(T ac, T ae, T aw, T an, T as, T at, T ab, T xc, T xe, T xw, T xn, T xs, T xt, T xb) {
    return ac * xc + ae * xe + aw * xw + an * xn + as * xs + at * xt + ab * xb;
}

// red-black SOR half sweep (src/dev/FalmEqDevCall.cu:175-211), in place
template <typename T>
struct SorBody {
    using V = T;
    Op7<T> op;
    T *x;
    const T *b;
    T omega;
    int color;
    const SolverScalars *sc;
    __device__ bool skip() const { return sc && sc->done; }
    __device__ const T *pw() const { return b; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell(int i, int j, int k, long long c, const Coef7<T> &a, T xc, T xe, T xw, T xn, T xs, T xt, T xb, T bv,
                         double (&)[1]) const {
        if (((i + j + k) & 1) != color) return;
        T cc = (bv - dot7(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb)) / a.ac;
        x[c] = xc + omega * cc;
    }
    __device__ void finish(const double (&)[1]) const {}
};

// ax = A x (src/dev/MVDevCall.cu:152-183)
template <typename T>
struct MvBody {
    using V = T;
    Op7<T> op;
    T *ax;
    __device__ bool skip() const { return false; }
    __device__ const T *pw() const { return nullptr; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell(int i, int j, int k, long long c, const Coef7<T> &a, T xc, T xe, T xw, T xn, T xs, T xt, T xb, T,
                         double (&)[1]) const {
        ax[c] = dot7(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb);
    }
    __device__ void finish(const double (&)[1]) const {}
};

// q = A pp and alpha = rho / (rr . q)
template <typename T>
struct MvDot1Body {
    using V = T;
    Op7<T> op;
    T *q;
    const T *rr;
    SolverScalars *sc;
    __device__ bool skip() const { return sc->done; }
    __device__ const T *pw() const { return rr; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell(int i, int j, int k, long long c, const Coef7<T> &a, T xc, T xe, T xw, T xn, T xs, T xt, T xb, T rrv,
                         double (&acc)[1]) const {
        T qv = dot7(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb);
        q[c] = qv;
        acc[0] += to_d(rrv) * to_d(qv);
    }
    __device__ void finish(const double (&tot)[1]) const {
        double alpha = sc->rho / tot[0];
        sc->alpha = alpha;
        if (!isfinite(alpha)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
    }
};

// t = A ss and omega = (t.s)/(t.t)
template <typename T>
struct MvDot2Body {
    using V = T;
    Op7<T> op;
    T *t;
    const T *s;
    SolverScalars *sc;
    __device__ bool skip() const { return sc->done; }
    __device__ const T *pw() const { return s; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell(int i, int j, int k, long long c, const Coef7<T> &a, T xc, T xe, T xw, T xn, T xs, T xt, T xb, T sv,
                         double (&acc)[2]) const {
        T tv = dot7(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb);
        t[c] = tv;
        double td = to_d(tv);
        acc[0] += td * to_d(sv);
        acc[1] += td * td;
    }
    __device__ void finish(const double (&tot)[2]) const {
        double omega = tot[0] / tot[1];
        sc->omega = omega;
        if (!isfinite(omega)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
    }
};

// r = b - A x (FP64 arithmetic), rr = r, solver start (see k_res)
template <typename T>
struct ResBody {
    using V = double;
    Op7<T> op;
    const T *b;
    T *r, *rr;
    SolverScalars *sc;
    int check_tol;
    __device__ bool skip() const { return false; }
    __device__ const T *pw() const { return b; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell(int i, int j, int k, long long c, const Coef7<double> &a, double xc, double xe, double xw, double xn,
                         double xs, double xt, double xb, T bv, double (&acc)[2]) const {
        double rv = to_d(bv) - dot7<double>(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb);
        T rt = (T)rv;
        if (r) r[c] = rt;
        if (rr) rr[c] = rt;
        acc[0] += rv * rv;
        acc[1] += to_d(rt) * to_d(rt);
    }
    __device__ void finish(const double (&tot)[2]) const {
        if (!sc) return;
        double err = sqrt(tot[0]) / sc->gsize;
        sc->err = err;
        sc->rho = tot[1];
        sc->rrho = 1.0; sc->alpha = 0.0; sc->omega = 1.0; sc->beta = 0.0;
        sc->first = 1;
        sc->done = 0;
        if (!isfinite(err)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
        else if (check_tol && err <= sc->tol) { sc->done = 1; sc->status = FALM_OK; }
        else if (fabs(tot[1]) < FLT_MIN) {
            sc->err = tot[1];
            sc->done = 1;
            sc->status = (err <= sc->tol) ? FALM_OK : FALM_ERR_BREAKDOWN;
        }
    }
};

}  // namespace fb
