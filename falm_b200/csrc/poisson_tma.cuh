// 2.5D TMA versions of the 7-point Poisson kernels (residual, red-black SOR
// half sweep, operator application fused with the BiCGStab inner products).
//
// The stencil operand streams through a ring of shared-memory slots, one
// (68 x 18) TMA box per z plane: the 64 x 16 tile, one halo row on each y side
// and two halo columns on each x side (the box starts at i0-2 so that its x
// coordinate is 16-byte aligned).  Each thread owns two adjacent cells (x, x+1)
// in each of two rows: the pair's values are one 64-bit (FP32) shared or
// global access, and FP32 arithmetic runs on the packed pipe.  The column's
// value at k-1 is kept in registers, k+1 comes from the next slot.  Pointwise
// operands (right-hand side, shadow residual, ...) are read with ordinary
// coalesced pair loads.  A field is streamed only when its row pitch is a
// multiple of 16 bytes, so the interior width is even and every pair is
// either inside the interior or outside it.
#pragma once
#include "poisson.cuh"
#include "pair.cuh"
#include "tma.cuh"

namespace fb {

template <typename T>
struct S7Tile {
    static constexpr int RY = 2;   // rows per thread: thread (tx, ty) computes rows ty, ty + 8
    static constexpr int TX = 64, TY = 8 * RY, BX = TX + 4, BY = TY + 2, PE = BX * BY;
    static constexpr int SLOT = (PE * (int)sizeof(T) + 127) / 128 * 128;
};

template <typename T> struct S7Conf;
template <> struct S7Conf<double> { static constexpr int NS = 6; };
template <> struct S7Conf<float> { static constexpr int NS = 8; };

// resident CTAs per SM asked of the register allocator: 3 for FP32 arithmetic
// on an FP32 field (at most 85 registers) and for the store-free FP64 residual
// check, 2 where the body works in FP64 and stores
template <typename T, class Body>
constexpr int s7_minb() { return (sizeof(T) == 4 && (sizeof(typename Body::V) == 4 || Body::kLean)) ? 3 : 2; }

template <typename T>
constexpr int s7_smem() { return S7Conf<T>::NS * S7Tile<T>::SLOT + 128 + 128; }

// Body: type V (the stencil's arithmetic type: T, or double for an FP64
//       residual of an FP32 field); bool skip() const; const T *pw() const
//       (pointwise operand, or null); const Op7<T> &op_() const;
//       void cell2(i, j, k, cc, a, xc, xe, xw, xn, xs, xt, xb, pv, acc): the
//       cells (i, j, k) and (i+1, j, k), with coefficient and value pairs;
//       void finish(tot)
// The kernel hoists the x/y part of the operator out of the z march, loads the
// z part once per plane for all rows of a thread, converts the column
// coefficients once, and carries the -1 neighbour pair from the previous plane.
// The pointwise operand of the next plane is loaded one iteration ahead (pv),
// so its latency overlaps the current plane's wait and arithmetic.
template <typename T, int NV, class Body>
__global__ void __launch_bounds__(256, (s7_minb<T, Body>())) k_s7_tma(Geom g, int kc, const __grid_constant__ CUtensorMap mx, Body body,
                                              RedWork rw, int *err) {
    using L = S7Tile<T>;
    using V = typename Body::V;
    using T2 = P2<T>;
    using V2 = P2<V>;
    constexpr int NS = S7Conf<T>::NS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t *bar = (uint64_t *)(smem + NS * L::SLOT);
    if (body.skip()) return;
    constexpr int RY = L::RY;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i0 = g.gc + blockIdx.x * L::TX, j0 = g.gc + blockIdx.y * L::TY;
    const int k0 = g.gc + blockIdx.z * kc, k1 = min(k0 + kc, g.sz - g.gc);
    const int i = i0 + 2 * tx;                              // the pair's first cell
    const int ihi = g.sx - g.gc, jhi = g.sy - g.gc;
    const int P0 = k0 - 1, nplanes = (k1 + 1) - P0;   // planes k0-1 .. k1
    const int xb = box_origin(i0 - 2, L::BX, g.sx, 16 / (int)sizeof(T)), yb = box_origin(j0 - 1, L::BY, g.sy, 1);
    const int ic = min(i, ihi - 2);                         // clamped pair (inactive threads read a staged pair)
    const int ox = ic - xb;
    int jr[RY], orr[RY];
    bool act[RY];
#pragma unroll
    for (int r = 0; r < RY; r++) {
        jr[r] = j0 + ty + 8 * r;
        act[r] = i < ihi && jr[r] < jhi;
        const int oy = min(jr[r], jhi - 1) - yb;
        orr[r] = oy * L::BX + ox;
        // self-check: the radius-1 neighbourhood of a computed pair lies inside the staged box, pair-aligned
        if (act[r] && (ox < 1 || ox + 2 > L::BX - 1 || oy < 1 || oy > L::BY - 2 || (orr[r] & 1))) {
            atomicExch(err, 300 + 2);
            act[r] = false;
        }
    }
    double acc[NV > 0 ? NV : 1];
#pragma unroll
    for (int d = 0; d < (NV > 0 ? NV : 1); d++) acc[d] = 0.0;
    auto slot = [&](int s) { return (const T *)(smem + s * L::SLOT); };
    // plane q into slot s = q % NS (the caller passes s, a constant in the march)
    auto issue = [&](int q, int s) {
        uint64_t *b = bar + s;
        unsigned char *dst = smem + s * L::SLOT;
        if (tma_ok(dst, xb, yb, P0 + q, (int)sizeof(T), g.sx, g.sy, g.sz)) {
            mbar_expect_tx(b, L::PE * sizeof(T));
            tma_load_4d(dst, &mx, xb, yb, P0 + q, 0, b);
        } else {
            tma_reject(b, err, 2);
        }
    };
    // warp 0 polls the barriers; the block barrier that follows makes the
    // landed planes visible to every thread
    auto wait_s = [&](int s, int parity) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + s, parity, err); };
    if (threadIdx.x == 0) {
        prefetch_tmap(&mx);
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
    fail = !wait_s(1, 0) || fail;
    waited = 2;
    const T *pw = body.pw();
    const long long sxy = (long long)g.sx * g.sy;
    const Op7<T> &op = body.op_();
    long long ccr[RY];
    T2 pv[RY];
    V2 xm[RY];
    bool pwr[RY];
    // x coefficients of the pair (both rows), y ones and the diagonal's x/y part per row
    V2 cw, ce;
    V2 csv[RY], cnv[RY];
    T2 dxy[RY];
    typename Op7<T>::Col col0[RY], col1[RY];
#pragma unroll
    for (int r = 0; r < RY; r++) {
        ccr[r] = g.id(i, jr[r], P0 + 1);   // cell of the first computed plane
        pwr[r] = pw && act[r];
        pv[r] = pwr[r] ? ld2(pw + ccr[r]) : mk2(T(0), T(0));
        const int jc = min(jr[r], jhi - 1);
        col0[r] = op.column(ic, jc);
        col1[r] = op.column(ic + 1, jc);
        csv[r] = mk2((V)col0[r].as, (V)col0[r].as);
        cnv[r] = mk2((V)col0[r].an, (V)col0[r].an);
        dxy[r] = mk2(col0[r].dxy, col1[r].dxy);
    }
    cw = mk2((V)col0[0].aw, (V)col1[0].aw);
    ce = mk2((V)col0[0].ae, (V)col1[0].ae);
    if (__syncthreads_or(fail)) goto drain;
#pragma unroll
    for (int r = 0; r < RY; r++) xm[r] = cvt2<V, T>(ld2(slot(0) + orr[r]));
    // the march, unrolled over the slots: plane q = q0 + u is in slot u
    for (int q0 = 0, ph = 0; q0 < nplanes - 1; q0 += NS, ph ^= 1) {
#pragma unroll
      for (int u = 0; u < NS; u++) {
        const int q = q0 + u;
        if (q < 1) continue;
        if (q >= nplanes - 1) break;
        T2 pn[RY];
#pragma unroll
        for (int r = 0; r < RY; r++) pn[r] = (pwr[r] && q + 1 < nplanes - 1) ? ld2(pw + ccr[r] + sxy) : mk2(T(0), T(0));
        fail = !wait_s((u + 1) % NS, (u + 1 < NS) ? ph : ph ^ 1);
        waited = q + 2;
        if (__syncthreads_or(fail)) goto drain;
        if (q - 1 + NS < nplanes) {   // plane q-1 is no longer read (its values are in xm): refill its slot
            if (threadIdx.x == 0) { fence_proxy_async(); issue(q - 1 + NS, (u + NS - 1) % NS); }
            issued = q - 1 + NS + 1;
        }
        const T *X0 = slot(u), *X1 = slot((u + 1) % NS);
        const int k = P0 + q;
        const typename Op7<T>::ZPl zp = op.zplane(k);
        const V2 abv = mk2((V)zp.ab, (V)zp.ab), atv = mk2((V)zp.at, (V)zp.at);
        const T2 zpp = mk2(zp.zp, zp.zp), zmm = mk2(zp.zm, zp.zm), scl = mk2(op.t.scale, op.t.scale);
#pragma unroll
        for (int r = 0; r < RY; r++) {
            const int o = orr[r];
            const T2 c2 = ld2(X0 + o);
            const V2 xc = cvt2<V, T>(c2);
            if (act[r]) {
                Coef7<V2> a;
                if (op.A) {
                    const Coef7<T> e0 = op.at_col(col0[r], k, ccr[r]), e1 = op.at_col(col1[r], k, ccr[r] + 1);
                    a = Coef7<V2>{mk2((V)e0.ac, (V)e1.ac), mk2((V)e0.aw, (V)e1.aw), mk2((V)e0.ae, (V)e1.ae), mk2((V)e0.as, (V)e1.as),
                                  mk2((V)e0.an, (V)e1.an), mk2((V)e0.ab, (V)e1.ab), mk2((V)e0.at, (V)e1.at)};
                } else {
                    // ((dxy - up_z) - um_z) * scale, as Op7::at_col
                    const T2 ac = mul2(sub2(sub2(dxy[r], zpp), zmm), scl);
                    a = Coef7<V2>{cvt2<V, T>(ac), cw, ce, csv[r], cnv[r], abv, atv};
                }
                const V xw0 = (V)X0[o - 1], xe1 = (V)X0[o + 2];
                body.cell2(i, jr[r], k, ccr[r], a, xc, mk2(xc.y, xe1), mk2(xw0, xc.x), cvt2<V, T>(ld2(X0 + o + L::BX)),
                           cvt2<V, T>(ld2(X0 + o - L::BX)), cvt2<V, T>(ld2(X1 + o)), xm[r], pv[r], acc);
            }
            xm[r] = xc;
            pv[r] = pn[r];
            ccr[r] += sxy;
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

// ---------------------------------------------------------------- bodies
// red-black SOR half sweep (src/dev/FalmEqDevCall.cu:175-211), in place: the
// pair's cell of this colour, with the scalar operations of the row kernel
template <typename T>
struct SorBody {
    using V = T;
    static constexpr bool kLean = false;
    Op7<T> op;
    T *x;
    const T *b;
    T omega;
    int color;
    const SolverScalars *sc;
    __device__ bool skip() const { return sc && sc->done; }
    __device__ const T *pw() const { return b; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell2(int i, int j, int k, long long c, const Coef7<P2<T>> &a, P2<T> xc, P2<T> xe, P2<T> xw, P2<T> xn, P2<T> xs,
                          P2<T> xt, P2<T> xb, P2<T> bv, double (&)[1]) const {
        const int e = (color ^ (i + j + k + op.t.koff)) & 1;
        auto L = [e](P2<T> v) { return e ? v.y : v.x; };
        const T ac = L(a.ac), xcc = L(xc);
        const T r7 = ac * xcc + L(a.ae) * L(xe) + L(a.aw) * L(xw) + L(a.an) * L(xn) + L(a.as) * L(xs) + L(a.at) * L(xt) + L(a.ab) * L(xb);
        x[c + e] = xcc + omega * ((L(bv) - r7) / ac);
    }
    __device__ void finish(const double (&)[1]) const {}
};

// ax = A x (src/dev/MVDevCall.cu:152-183)
template <typename T>
struct MvBody {
    using V = T;
    static constexpr bool kLean = false;
    Op7<T> op;
    T *ax;
    __device__ bool skip() const { return false; }
    __device__ const T *pw() const { return nullptr; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell2(int i, int j, int k, long long c, const Coef7<P2<T>> &a, P2<T> xc, P2<T> xe, P2<T> xw, P2<T> xn, P2<T> xs,
                          P2<T> xt, P2<T> xb, P2<T>, double (&)[1]) const {
        st2(ax + c, dot7p(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb));
    }
    __device__ void finish(const double (&)[1]) const {}
};

// q = A pp and alpha = rho / (rr . q)
template <typename T>
struct MvDot1Body {
    using V = T;
    static constexpr bool kLean = false;
    Op7<T> op;
    T *q;
    const T *rr;
    SolverScalars *sc;
    __device__ bool skip() const { return sc->done; }
    __device__ const T *pw() const { return rr; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell2(int i, int j, int k, long long c, const Coef7<P2<T>> &a, P2<T> xc, P2<T> xe, P2<T> xw, P2<T> xn, P2<T> xs,
                          P2<T> xt, P2<T> xb, P2<T> rrv, double (&acc)[1]) const {
        const P2<T> qv = dot7p(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb);
        st2(q + c, qv);
        acc[0] += to_d(rrv.x) * to_d(qv.x);
        acc[0] += to_d(rrv.y) * to_d(qv.y);
    }
    __device__ void finish(const double (&tot)[1]) const {
        if (sc->defer) sc->red[0] = tot[0];
        else derive_alpha(sc, tot);
    }
};

// t = A ss and omega = (t.s)/(t.t)
template <typename T>
struct MvDot2Body {
    using V = T;
    static constexpr bool kLean = false;
    Op7<T> op;
    T *t;
    const T *s;
    SolverScalars *sc;
    __device__ bool skip() const { return sc->done; }
    __device__ const T *pw() const { return s; }
    __device__ const Op7<T> &op_() const { return op; }
    __device__ void cell2(int i, int j, int k, long long c, const Coef7<P2<T>> &a, P2<T> xc, P2<T> xe, P2<T> xw, P2<T> xn, P2<T> xs,
                          P2<T> xt, P2<T> xb, P2<T> sv, double (&acc)[2]) const {
        const P2<T> tv = dot7p(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb);
        st2(t + c, tv);
        const double t0 = to_d(tv.x), t1 = to_d(tv.y);
        acc[0] += t0 * to_d(sv.x);
        acc[0] += t1 * to_d(sv.y);
        acc[1] += t0 * t0;
        acc[1] += t1 * t1;
    }
    __device__ void finish(const double (&tot)[2]) const {
        if (sc->defer) { sc->red[0] = tot[0]; sc->red[1] = tot[1]; }
        else derive_omega(sc, tot);
    }
};

// r = b - A x (FP64 arithmetic), rr = r, solver start (see k_res); with pp,
// also the pointwise first preconditioner sweep from zero of the new r (what
// k_bicg_p computes in a pass's first iteration, where p = r).  CHECK: the
// outer check of the true residual, which stores nothing.
template <typename T, bool CHECK = false>
struct ResBody {
    using V = double;
    static constexpr bool kLean = CHECK;
    Op7<T> op;
    const T *b;
    T *r, *rr;
    SolverScalars *sc;
    int check_tol;
    T *pp = nullptr;
    int pc_type = 0;
    T pc_omega = T(0);
    // a check queued behind a pass's iterations: it runs only once the pass has
    // stopped without a non-finite scalar, and records that it ran
    int queued_check = 0;
    __device__ bool skip() const { return queued_check && !(sc->done && sc->status != FALM_ERR_NAN && !sc->checked); }
    __device__ const T *pw() const { return b; }
    __device__ const Op7<T> &op_() const { return op; }
    static constexpr int NV = CHECK ? 1 : 2;   // the check reduces only the norm
    __device__ void cell2(int i, int j, int k, long long c, const Coef7<double2> &a, double2 xc, double2 xe, double2 xw, double2 xn,
                          double2 xs, double2 xt, double2 xb, P2<T> bv, double (&acc)[NV]) const {
        const double2 ax = dot7p(a.ac, a.ae, a.aw, a.an, a.as, a.at, a.ab, xc, xe, xw, xn, xs, xt, xb);
        const double r0 = to_d(bv.x) - ax.x, r1 = to_d(bv.y) - ax.y;
        const P2<T> rt = mk2((T)r0, (T)r1);
        if (!CHECK && r) st2(r + c, rt);
        if (!CHECK && rr) st2(rr + c, rt);
        if (!CHECK && pp) st2(pp + c, mk2(pc_first<T>(pc_type, i, j, k + op.t.koff, rt.x, (T)a.ac.x, pc_omega),
                                pc_first<T>(pc_type, i + 1, j, k + op.t.koff, rt.y, (T)a.ac.y, pc_omega)));
        acc[0] += r0 * r0;
        acc[0] += r1 * r1;
        if constexpr (!CHECK) {
            acc[NV - 1] += to_d(rt.x) * to_d(rt.x);
            acc[NV - 1] += to_d(rt.y) * to_d(rt.y);
        }
    }
    __device__ void finish(const double (&tot)[NV]) const {
        if (!sc) return;
        if (sc->defer) {   // slab mode: the totals, summed over the slabs before derive_res
            sc->red[0] = tot[0];
            sc->red[1] = tot[NV - 1];
            return;
        }
        double err = sqrt(tot[0]) / sc->gsize;
        sc->err = err;
        // a check that passes ends the solve; one that fails is followed by a
        // pass residual, which sets the iteration's scalars
        const double rho = tot[NV - 1];
        sc->rho = rho;
        sc->rrho = 1.0; sc->alpha = 0.0; sc->omega = 1.0; sc->beta = 0.0;
        sc->first = 1;
        sc->done = 0;
        sc->checked = queued_check;
        if (!isfinite(err)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
        else if (check_tol && err <= sc->tol) { sc->done = 1; sc->status = FALM_OK; }
        else if (!CHECK && fabs(rho) < FLT_MIN) {
            sc->err = rho;
            sc->done = 1;
            sc->status = (err <= sc->tol) ? FALM_OK : FALM_ERR_BREAKDOWN;
        }
    }
};

}  // namespace fb
