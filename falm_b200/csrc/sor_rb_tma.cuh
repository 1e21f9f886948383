// Temporally blocked red-black SOR: H consecutive half sweeps (colours c1,
// c1^1, ...) of FalmEqDevCall::SORSweep (src/dev/FalmEqDevCall.cu:175-211) in
// one pass over HBM, out of place (x_in -> x_out).
//
// A CTA owns a 32 x 8 tile of columns and a chunk of z planes.  Half sweep h
// must be evaluated on the tile plus a ring of H-h cells (in x, y and z) for
// the last one to be exact on the tile, so every plane of x_in and b is staged
// as one (tile + halo) TMA box.  The z march is a wavefront: when raw plane q
// has landed, half sweep 1 updates plane q-1, half sweep 2 plane q-2, ...,
// half sweep H plane q-H, each in place in shared memory and only on its own
// colour (which reads only the other colour, so in-place is exact), then the
// tile of plane q-H is final and is written to x_out.  Reads come from x_in
// only, so neighbouring CTAs never see a partially updated field.
//
// Each thread owns one horizontal pair of cells (x0, x0+1) of the widest
// ring: exactly one cell of the pair has a given colour on a given plane, so
// the thread updates that one in every half sweep whose ring holds it, with
// the pair's x/y operator coefficients kept in registers.
#pragma once
#include <type_traits>
#include "pair.cuh"
#include "poisson.cuh"
#include "tma.cuh"

namespace fb {

// one red-black SOR update of cell c from its six neighbours, with the fused
// multiply-adds spelled out so that every blocked kernel rounds the same way:
// x_c + omega (b_c - (ac x_c + ae x_e + aw x_w + an x_n + as x_s + at x_t + ab x_b)) / ac
template <typename T>
__device__ __forceinline__ T sor_point(T ac, T ae, T aw, T an, T as, T at, T ab, T xc, T xe, T xw, T xn, T xs, T xt, T xb, T bc,
                                       T omega) {
    T r7 = ac * xc;
    r7 = fma(ae, xe, r7);
    r7 = fma(aw, xw, r7);
    r7 = fma(an, xn, r7);
    r7 = fma(as, xs, r7);
    r7 = fma(at, xt, r7);
    r7 = fma(ab, xb, r7);
    return fma(omega, sor_div(bc - r7, ac), xc);
}

template <typename T, int H>
struct RBTile {
    static constexpr int TX = 32, TY = 8;
    static constexpr int R = H - 1;                                  // widest ring (half sweep 1)
    static constexpr int PX = (TX + 2 * R) / 2, PY = TY + 2 * R;     // pairs per row, rows
    // x halo of the box: >= H, and box origin i0 - HX = 32 bx + 2 - HX on a
    // 16-byte boundary for gc = 2
    static constexpr int HX = (H <= 2) ? 2 : (sizeof(T) == 4 ? 6 : 4);
    static constexpr int BX = TX + 2 * HX, BY = TY + 2 * H, PE = BX * BY;
    static constexpr int PB = (PE * (int)sizeof(T) + 127) / 128 * 128;   // one field plane
    static constexpr int SLOT = 2 * PB;                                   // x plane, then b plane
    // H+2 resident planes + look-ahead; a power of two keeps the slot index a mask
    static constexpr int NS = 8;
    static constexpr int SMEM = NS * SLOT + 128 + 128;
    static_assert(PX * PY <= 256, "one pair per thread");
};

template <typename T, int H>
__global__ void __launch_bounds__(256) k_sor_rb_tma(Geom g, int kc, const __grid_constant__ CUtensorMap mx,
                                                   const __grid_constant__ CUtensorMap mb, PoissonTables<T> tb, T *__restrict__ xout,
                                                   T omega, int c1, const SolverScalars *sc, int *err) {
    using L = RBTile<T, H>;
    constexpr unsigned NS = L::NS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t *bar = (uint64_t *)(smem + NS * L::SLOT);
    if (sc && sc->done) return;
    const int i0 = g.gc + blockIdx.x * L::TX, j0 = g.gc + blockIdx.y * L::TY;
    const int k0 = g.gc + blockIdx.z * kc, k1 = min(k0 + kc, g.sz - g.gc);
    const int P0 = k0 - H, nplanes = (k1 + H) - P0;
    const int xb = max(0, box_origin(i0 - L::HX, L::BX, g.sx, 16 / (int)sizeof(T)));
    const int yb = max(0, box_origin(j0 - H, L::BY, g.sy, 1));
    const int ilo = g.gc, ihi = g.sx - g.gc, jlo = g.gc, jhi = g.sy - g.gc, klo = g.gc, khi = g.sz - g.gc;
    // this thread's pair (x0, x0+1) in row y of the widest ring
    const int t = threadIdx.x;
    const bool owner = t < L::PX * L::PY;
    const int x0 = i0 - L::R + 2 * (t % L::PX), y = j0 - L::R + t / L::PX;
    // cell e (0: x0, 1: x0+1) takes part in half sweep h when it lies in ring
    // H-h of the tile and inside the interior: bit h-1 of live[e]
    unsigned live0 = 0u, live1 = 0u;
#pragma unroll
    for (int h = 1; h <= H; h++) {
        const int ring = H - h;
        const bool yin = owner && y >= j0 - ring && y < j0 + L::TY + ring && y >= jlo && y < jhi;
        const bool in0 = yin && x0 >= i0 - ring && x0 < i0 + L::TX + ring && x0 >= ilo && x0 < ihi;
        const bool in1 = yin && x0 + 1 >= i0 - ring && x0 + 1 < i0 + L::TX + ring && x0 + 1 >= ilo && x0 + 1 < ihi;
        live0 |= (in0 ? 1u : 0u) << (h - 1);
        live1 |= (in1 ? 1u : 0u) << (h - 1);
    }
    // x/y operator coefficients of both cells (same association as Op7::get)
    T aw0, aw1, ae0, ae1, dxy0, dxy1, as, an;
    {
        const int yc = min(max(y, 0), g.sy - 1);
        const int xc0 = min(max(x0, 0), g.sx - 1), xc1 = min(max(x0 + 1, 0), g.sx - 1);
        as = ldg(tb.cm[1] + yc); an = ldg(tb.cp[1] + yc);
        const T up1 = ldg(tb.up[1] + yc), um1 = ldg(tb.um[1] + yc);
        aw0 = ldg(tb.cm[0] + xc0); ae0 = ldg(tb.cp[0] + xc0); dxy0 = (ldg(tb.dx0 + xc0) - up1) - um1;
        aw1 = ldg(tb.cm[0] + xc1); ae1 = ldg(tb.cp[0] + xc1); dxy1 = (ldg(tb.dx0 + xc1) - up1) - um1;
    }
    const int o0 = (y - yb) * L::BX + (x0 - xb);   // used only for live cells, which lie inside the box
    auto slot = [&](int q) { return smem + ((unsigned)q % NS) * L::SLOT; };
    // planes outside the tensor (z < 0 or z >= sz) are never read: complete their barrier without a copy
    auto issue = [&](int q) {
        uint64_t *b = bar + ((unsigned)q % NS);
        const int z = P0 + q;
        if (z < 0 || z >= g.sz) { mbar_arrive(b); return; }
        unsigned char *s = slot(q);
        if (tma_ok(s, xb, yb, z, (int)sizeof(T), g.sx, g.sy, g.sz) && tma_ok(s + L::PB, xb, yb, z, (int)sizeof(T), g.sx, g.sy, g.sz)) {
            mbar_expect_tx(b, 2 * L::PE * sizeof(T));
            tma_load_4d(s, &mx, xb, yb, z, 0, b);
            tma_load_4d(s + L::PB, &mb, xb, yb, z, 0, b);
        } else {
            tma_reject(b, err, 4);
        }
    };
    // warp 0 polls the barriers; the block barrier that follows makes the
    // landed planes visible to every thread
    auto wait_q = [&](int q) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + ((unsigned)q % NS), ((unsigned)q / NS) & 1, err); };
    if (threadIdx.x == 0) {
        prefetch_tmap(&mx); prefetch_tmap(&mb);
        for (unsigned s = 0; s < NS; s++) mbar_init(bar + s, 1);
        mbar_fence_init();
    }
    __syncthreads();
    int issued = min((int)NS, nplanes), waited = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < issued; q++) issue(q);
    // write-out: thread t copies cell (i0 + t % 32, j0 + t / 32) of the tile
    const int wx = i0 + (t & (L::TX - 1)), wy = j0 + t / L::TX;
    const bool writer = t < L::TX * L::TY && wx < ihi && wy < jhi;
    const int wo = (wy - yb) * L::BX + (wx - xb);
    const long long sxy = (long long)g.sx * g.sy;
    T *wp = xout + (long long)wx + (long long)wy * g.sx + (long long)k0 * sxy;   // advanced one plane per write-out
    // registers rolled along the march: slot base of planes q, q-1, ..., q-H-1
    // and the z operator tables (cm, cp, up, um) of planes q-1, ..., q-H
    unsigned char *sl[H + 2];
    T zab[H], zat[H], zup[H], zum[H];
#pragma unroll
    for (int m = 0; m < H + 2; m++) sl[m] = slot(-1 - m);
#pragma unroll
    for (int h = 0; h < H; h++) { zab[h] = zat[h] = zup[h] = zum[h] = T(0); }
    for (int q = 0; q < nplanes; q++) {
#pragma unroll
        for (int m = H + 1; m > 0; m--) sl[m] = sl[m - 1];
        sl[0] = slot(q);
#pragma unroll
        for (int h = H - 1; h > 0; h--) { zab[h] = zab[h - 1]; zat[h] = zat[h - 1]; zup[h] = zup[h - 1]; zum[h] = zum[h - 1]; }
        {
            const int kz = min(max(P0 + q - 1, 0), g.sz - 1);
            zab[0] = ldg(tb.cm[2] + kz); zat[0] = ldg(tb.cp[2] + kz); zup[0] = ldg(tb.up[2] + kz); zum[0] = ldg(tb.um[2] + kz);
        }
        bool fail = !wait_q(q);
        waited = q + 1;
        if (__syncthreads_or(fail)) goto drain;
        // half sweeps 1..H on planes q-1 .. q-H (wavefront, ascending h)
#pragma unroll
        for (int h = 1; h <= H; h++) {
            const int p = q - h, kp = P0 + p, ring = H - h;
            if (p >= 1 && kp >= max(klo, k0 - ring) && kp < min(khi, k1 + ring)) {
                const int color = (c1 + h - 1) & 1;
                const int e = (color ^ (x0 + y + kp)) & 1;          // the pair's cell of this colour
                if ((((e ? live1 : live0) >> (h - 1)) & 1u) != 0u) {
                    T *X0 = (T *)sl[h];
                    const T *Xm = (const T *)sl[h + 1], *Xp = (const T *)sl[h - 1];
                    const T *B0 = (const T *)(sl[h] + L::PB);
                    const T ab = zab[h - 1], at = zat[h - 1];
                    const T ac = (((e ? dxy1 : dxy0) - zup[h - 1]) - zum[h - 1]) * tb.scale;
                    const int o = o0 + e;
                    X0[o] = sor_point(ac, e ? ae1 : ae0, e ? aw1 : aw0, an, as, at, ab, X0[o], X0[o + 1], X0[o - 1], X0[o + L::BX],
                                      X0[o - L::BX], Xp[o], Xm[o], B0[o], omega);
                }
            }
            __syncthreads();
        }
        // the tile of plane q-H is final
        {
            const int kp = P0 + q - H;
            if (kp >= k0 && kp < k1) {
                if (writer) *wp = ((const T *)sl[H])[wo];
                wp += sxy;
            }
        }
        // plane q-H-1 was last read by half sweep H above and by the previous
        // iteration's write-out, both behind a barrier: refill its slot
        {
            const int qn = q - H - 1 + (int)NS;
            if (q - H - 1 >= 0 && qn < nplanes) {
                if (threadIdx.x == 0) { fence_proxy_async(); issue(qn); }
                issued = qn + 1;
            }
        }
    }
    return;
drain:
    for (int q = waited; q < issued; q++) wait_q(q);
}

}  // namespace fb

namespace fb {

// Three half sweeps per pass on a 28 x 16 tile, skewed wavefront (FP32 with
// packed pair arithmetic; FP64 with the two lanes as scalar operations).
//
// Half sweep h of plane p runs at iteration q = p + 2h - 1 (planes q-1, q-3 and
// q-5 at iteration q).  Half sweep h reads the other colour of planes p-1, p,
// p+1, which half sweep h-1 finished at iterations q-3, q-2 and q-1 and which
// half sweep h+1 changes only from iteration q+1 on; so the three half sweeps
// of an iteration touch disjoint data and run without barriers between them,
// and one block barrier per iteration (after the new plane has landed) keeps
// every warp within one iteration of the others.  Plane p is final after
// iteration p+5 and written out at iteration p+6; the ring holds planes q-6..q
// plus NS-7 planes in flight.
//
// Work layout:
//  * 160 threads; thread t owns pair column m = t % 16 (cells x0 = i0-2+2m and
//    x0+1) in rows rw and rw+10 of the widest ring (rw = t / 16), so a half
//    warp covers one row and the two halves of a warp cover adjacent rows.
//    Same-colour cells of adjacent rows sit on opposite bank parities (the box
//    pitch is even), so every shared access of a half sweep is one wavefront.
//  * the two rows of a thread have the same parity, hence the same colour
//    offset e: both updates run as one pair (in FP32 through the packed pipe,
//    fma/add/mul.f32x2), each lane rounding exactly as the scalar sor_point()
//    does.
//  * the right-hand side is staged as its own (32 x 20) box covering just the
//    cells a half sweep updates; the chunk's z coefficients are staged once.
//  * the march is unrolled over the NS slots, so slot addresses are constants.
template <typename T>
struct RB2Tile {
    static constexpr int H = 3, R = H - 1;
    static constexpr int TX = 28, TY = 16;
    static constexpr int AL = 16 / (int)sizeof(T);                       // TMA x alignment (elements)
    static constexpr int HX = H + ((2 - H) % AL + AL) % AL;              // i0 - HX on the alignment for gc = 2
    static constexpr int BX = (HX + TX + H + AL - 1) / AL * AL, BY = TY + 2 * H, PE = BX * BY;
    static constexpr int BXB = 32, BYB = TY + 2 * R, PEB = BXB * BYB;    // right-hand side box from i0 - 2
    static constexpr int PBX = (PE * (int)sizeof(T) + 127) / 128 * 128, PBB = (PEB * (int)sizeof(T) + 127) / 128 * 128;
    static constexpr int SLOT = PBX + PBB;
    static constexpr int NS = 9;                                          // 7 resident planes + 2 in flight
    static constexpr int ZMAX = 72;                                       // z coefficient planes staged (kc <= ZMAX - 2H)
    static constexpr int PX = 16, PY = TY + 2 * R, HALF = PY / 2;        // pairs per row, rows, rows per set
    static constexpr int NT = PX * HALF;                                  // threads
    static constexpr int SMEM = NS * SLOT + ZMAX * 4 * (int)sizeof(T) + 128 + 128;
    static constexpr int MINB = sizeof(T) == 4 ? 4 : 2;                   // resident CTAs per SM (shared memory)
    static_assert(PY % 4 == 0, "the two rows of a thread have the same parity");
    static_assert(R <= 2 && TX + R <= 2 * PX - 2, "the pair columns (x from i0 - 2) cover the widest ring");
};

// the per-plane z coefficients of the chunk, staged once: ab, at, -up, -um
template <typename T> struct alignas(4 * sizeof(T)) ZCoef { T ab, at, nup, num; };

// sor_div on both lanes
__device__ __forceinline__ float2 sor_div2(float2 d, float2 ac) { return mul2(d, mk2(rcp_approx(ac.x), rcp_approx(ac.y))); }
__device__ __forceinline__ double2 sor_div2(double2 d, double2 ac) { return mk2(sor_div(d.x, ac.x), sor_div(d.y, ac.y)); }

// the two same-colour updates of a thread (lane s: row set s), lane by lane
// the operations of sor_point()
template <typename V2>
__device__ __forceinline__ V2 sor_point2(V2 ac, V2 ae, V2 aw, V2 an, V2 as, V2 at, V2 ab, V2 xc, V2 xe, V2 xw, V2 xn, V2 xs, V2 xt, V2 xb,
                                         V2 bc, V2 omega) {
    using S = decltype(ac.x);
    V2 r7 = mul2(ac, xc);
    r7 = fma2(ae, xe, r7);
    r7 = fma2(aw, xw, r7);
    r7 = fma2(an, xn, r7);
    r7 = fma2(as, xs, r7);
    r7 = fma2(at, xt, r7);
    r7 = fma2(ab, xb, r7);
    const V2 d = fma2(r7, mk2(S(-1), S(-1)), bc);                        // bc - r7, one rounding
    return fma2(omega, sor_div2(d, ac), xc);
}

template <typename T>
__global__ void __launch_bounds__(RB2Tile<T>::NT, RB2Tile<T>::MINB) k_sor_rb2_tma(Geom g, int kc, const __grid_constant__ CUtensorMap mx,
                                                                 const __grid_constant__ CUtensorMap mb, PoissonTables<T> tb,
                                                                 T *__restrict__ xout, T omega, int c1, const SolverScalars *sc,
                                                                 int *err) {
    using V2 = P2<T>;
    using L = RB2Tile<T>;
    constexpr int H = L::H;
    constexpr int NS = L::NS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    ZCoef<T> *ztab = (ZCoef<T> *)(smem + NS * L::SLOT);                  // per staged plane: ab, at, -up, -um
    uint64_t *bar = (uint64_t *)(smem + NS * L::SLOT + L::ZMAX * 4 * sizeof(T));
    if (sc && sc->done) return;
    const int i0 = g.gc + blockIdx.x * L::TX, j0 = g.gc + blockIdx.y * L::TY;
    const int k0 = g.gc + blockIdx.z * kc, k1 = min(k0 + kc, g.sz - g.gc);
    const int P0 = k0 - H, nplanes = (k1 + H) - P0;
    if (nplanes > L::ZMAX) { if (threadIdx.x == 0) atomicExch(err, 300 + 6); return; }
    const int xb = max(0, box_origin(i0 - L::HX, L::BX, g.sx, L::AL));
    const int yb = max(0, box_origin(j0 - H, L::BY, g.sy, 1));
    const int xbb = max(0, box_origin(i0 - 2, L::BXB, g.sx, L::AL));
    const int ybb = max(0, box_origin(j0 - L::R, L::BYB, g.sy, 1));
    const int ilo = g.gc, ihi = g.sx - g.gc, jlo = g.gc, jhi = g.sy - g.gc, klo = g.gc, khi = g.sz - g.gc;
    const int t = threadIdx.x;
    const int x0 = i0 - 2 + 2 * (t % L::PX);
    const int yr[2] = {j0 - L::R + t / L::PX, j0 - L::R + t / L::PX + L::HALF};
    // live bits: bit 3*(2s+e) + h-1 when cell e of set s takes part in half sweep h
    // (inside ring H-h of the tile and inside the interior), after a check that
    // its radius-1 neighbourhood lies in the staged boxes
    unsigned live = 0u;
#pragma unroll
    for (int s = 0; s < 2; s++) {
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int x = x0 + e, y = yr[s];
            unsigned bits = 0u;
#pragma unroll
            for (int h = 1; h <= H; h++) {
                const int ring = H - h;
                const bool in = y >= j0 - ring && y < j0 + L::TY + ring && y >= jlo && y < jhi && x >= i0 - ring &&
                                x < i0 + L::TX + ring && x >= ilo && x < ihi;
                bits |= (in ? 1u : 0u) << (h - 1);
            }
            if (bits && (x - 1 < xb || x + 1 >= xb + L::BX || y - 1 < yb || y + 1 >= yb + L::BY || x < xbb ||
                         x >= xbb + L::BXB || y < ybb || y >= ybb + L::BYB)) {
                atomicExch(err, 300 + 5);
                bits = 0u;
            }
            live |= bits << (3 * (2 * s + e));
        }
    }
    // coefficients as lane pairs: x ones (cell e, both lanes alike), y ones per
    // row set, dxy per (set, e); same association as Op7::get
    V2 aw2[2], ae2[2], an2, as2, dxy2[2];
    {
        const int xc0 = min(max(x0, 0), g.sx - 1), xc1 = min(max(x0 + 1, 0), g.sx - 1);
        const T aw0 = ldg(tb.cm[0] + xc0), ae0 = ldg(tb.cp[0] + xc0), aw1 = ldg(tb.cm[0] + xc1), ae1 = ldg(tb.cp[0] + xc1);
        aw2[0] = mk2(aw0, aw0); aw2[1] = mk2(aw1, aw1); ae2[0] = mk2(ae0, ae0); ae2[1] = mk2(ae1, ae1);
        const T d0 = ldg(tb.dx0 + xc0), d1 = ldg(tb.dx0 + xc1);
        T as_[2], an_[2], dd[2][2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int yc = min(max(yr[s], 0), g.sy - 1);
            as_[s] = ldg(tb.cm[1] + yc); an_[s] = ldg(tb.cp[1] + yc);
            const T up1 = ldg(tb.up[1] + yc), um1 = ldg(tb.um[1] + yc);
            dd[s][0] = (d0 - up1) - um1;
            dd[s][1] = (d1 - up1) - um1;
        }
        as2 = mk2(as_[0], as_[1]); an2 = mk2(an_[0], an_[1]);
        dxy2[0] = mk2(dd[0][0], dd[1][0]); dxy2[1] = mk2(dd[0][1], dd[1][1]);
    }
    // element offsets of cell x0 of each row set in the x box and the
    // right-hand side box, clamped into the boxes (exact for live cells; a
    // lane whose cell is not live computes on some staged cell and stores nothing)
    int ox[2], ob[2];
    {
        const int xcl = min(max(x0, xb + 1), xb + L::BX - 3), xbl = min(max(x0, xbb), xbb + L::BXB - 2);
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int ycl = min(max(yr[s], yb + 1), yb + L::BY - 2), ybl = min(max(yr[s], ybb), ybb + L::BYB - 1);
            ox[s] = (ycl - yb) * L::BX + (xcl - xb);
            ob[s] = (ybl - ybb) * L::BXB + (xbl - xbb);
        }
    }
    const int par0 = (x0 + yr[0]) & 1;
    // plane q into slot s = q % NS (the caller passes s)
    auto issue = [&](int q, int s) {
        uint64_t *b = bar + s;
        const int z = P0 + q;
        if (z < 0 || z >= g.sz) { mbar_arrive(b); return; }
        unsigned char *d = smem + s * L::SLOT;
        if (tma_ok(d, xb, yb, z, (int)sizeof(T), g.sx, g.sy, g.sz) && tma_ok(d + L::PBX, xbb, ybb, z, (int)sizeof(T), g.sx, g.sy, g.sz)) {
            mbar_expect_tx(b, (L::PE + L::PEB) * sizeof(T));
            tma_load_4d(d, &mx, xb, yb, z, 0, b);
            tma_load_4d(d + L::PBX, &mb, xbb, ybb, z, 0, b);
        } else {
            tma_reject(b, err, 5);
        }
    };
    auto wait_s = [&](int s, int parity) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + s, parity, err); };
    if (threadIdx.x == 0) {
        prefetch_tmap(&mx); prefetch_tmap(&mb);
        for (int s = 0; s < NS; s++) mbar_init(bar + s, 1);
        mbar_fence_init();
    }
    // the chunk's z coefficients
    for (int q = threadIdx.x; q < nplanes; q += blockDim.x) {
        const int kz = min(max(P0 + q, 0), g.sz - 1);
        ztab[q] = ZCoef<T>{ldg(tb.cm[2] + kz), ldg(tb.cp[2] + kz), -ldg(tb.up[2] + kz), -ldg(tb.um[2] + kz)};
    }
    __syncthreads();
    int issued = min(NS, nplanes), waited = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < issued; q++) issue(q, q % NS);
    const long long sxy = (long long)g.sx * g.sy;
    // write-out: this thread's cell pairs w = t and t + NT of the tile (14 pairs
    // per row): offsets in the x box and in a plane of x_out, -1 when outside
    constexpr int NW = ((L::TX / 2) * L::TY + L::NT - 1) / L::NT;
    int wso[NW], wgo[NW];
    bool wpair[NW];
#pragma unroll
    for (int n = 0; n < NW; n++) {
        const int w = t + n * L::NT;
        const int wx = i0 + 2 * (w % (L::TX / 2)), wy = j0 + w / (L::TX / 2);
        const bool ok = w < (L::TX / 2) * L::TY && wx < ihi && wy < jhi;
        wso[n] = ok ? (wy - yb) * L::BX + (wx - xb) : -1;
        wgo[n] = wy * g.sx + wx;
        wpair[n] = wx + 1 < ihi;
    }
    const V2 sc2 = mk2(tb.scale, tb.scale), om2 = mk2(omega, omega);
    const int nit = nplanes + H;   // the last tile plane, nplanes - H - 1, is written out at iteration nplanes + H - 1
    for (int q0 = 0, ph = 0; q0 < nit; q0 += NS, ph ^= 1) {
#pragma unroll
        for (int u = 0; u < NS; u++) {
            const int q = q0 + u;
            if (q >= nit) break;
            // slot of plane q - m (a constant once unrolled)
            auto sl = [&](int m) { return smem + ((u - m + 2 * NS) % NS) * L::SLOT; };
            bool fail = false;
            if (q < nplanes) {
                fail = !wait_s(u, ph);
                waited = q + 1;
            }
            if (__syncthreads_or(fail)) goto drain;
            // plane q - 2H is final (its last half sweep ran at iteration q - 1): write it out
            {
                const int kp = P0 + q - 2 * H;
                if (kp >= k0 && kp < k1) {
                    const T *Xf = (const T *)sl(2 * H);
                    T *plane = xout + (long long)kp * sxy;
#pragma unroll
                    for (int n = 0; n < NW; n++) {
                        if (wso[n] >= 0) {
                            if (wpair[n]) *reinterpret_cast<V2 *>(plane + wgo[n]) = *reinterpret_cast<const V2 *>(Xf + wso[n]);
                            else plane[wgo[n]] = Xf[wso[n]];
                        }
                    }
                }
            }
            // the slot of plane q - 2H - 1 was last read in iteration q - 1: refill it
            {
                const int qn = q - 2 * H - 1 + NS;
                if (q - 2 * H - 1 >= 0 && qn < nplanes) {
                    if (threadIdx.x == 0) { fence_proxy_async(); issue(qn, (u + NS - 2 * H - 1) % NS); }
                    issued = qn + 1;
                }
            }
            // half sweeps h = 1..H on planes q - (2h - 1), no barrier between them
#pragma unroll
            for (int h = 1; h <= H; h++) {
                const int p = q - (2 * h - 1), kp = P0 + p, ring = H - h;
                if (p >= 1 && p + 1 < nplanes && kp >= max(klo, k0 - ring) && kp < min(khi, k1 + ring)) {
                    const int color = (c1 + h - 1) & 1;
                    const int e = (color ^ par0 ^ kp) & 1;   // the pairs' cell of this colour (both row sets)
                    const unsigned l0 = (live >> (3 * e + h - 1)) & 1u, l1 = (live >> (3 * (2 + e) + h - 1)) & 1u;
                    if (l0 | l1) {
                        T *X0 = (T *)sl(2 * h - 1);
                        const T *Xm = (const T *)sl(2 * h), *Xp = (const T *)sl(2 * h - 2);
                        const T *B0 = (const T *)(sl(2 * h - 1) + L::PBX);
                        const ZCoef<T> z = ztab[p];
                        const int o0 = ox[0] + e, o1 = ox[1] + e;
                        const V2 ac = mul2(add2(add2(e ? dxy2[1] : dxy2[0], mk2(z.nup, z.nup)), mk2(z.num, z.num)), sc2);
                        const V2 r = sor_point2(ac, e ? ae2[1] : ae2[0], e ? aw2[1] : aw2[0], an2, as2, mk2(z.at, z.at), mk2(z.ab, z.ab), mk2(X0[o0], X0[o1]),
                                                mk2(X0[o0 + 1], X0[o1 + 1]), mk2(X0[o0 - 1], X0[o1 - 1]),
                                                mk2(X0[o0 + L::BX], X0[o1 + L::BX]), mk2(X0[o0 - L::BX], X0[o1 - L::BX]),
                                                mk2(Xp[o0], Xp[o1]), mk2(Xm[o0], Xm[o1]), mk2(B0[ob[0] + e], B0[ob[1] + e]), om2);
                        if (l0) X0[o0] = r.x;
                        if (l1) X0[o1] = r.y;
                    }
                }
            }
        }
    }
    return;
drain:
    for (int q = waited; q < issued; q++) wait_s(q % NS, (q / NS) & 1);
}

}  // namespace fb
