// 2.5D pseudo-velocity kernel with TMA plane streaming.
//
// A CTA owns a 32 x 8 tile of (i, j) columns and a chunk of z planes.  For
// every plane it needs the tile plus a halo of 2 of u (3 components), uu (3)
// and nut: one TMA box (36 x 12 x 1 x ncomp) per field and plane lands in a
// ring of NS shared-memory slots (plane q in slot q % NS, guarded by mbarrier
// q % NS with phase parity (q / NS) & 1).  x/y neighbours come from the slot
// of the current plane, the +1/+2 z neighbours from the two slots ahead, and
// the -1/-2 z neighbours from registers (the column's own values of the two
// previous planes).  Every HBM byte of the inputs is read once per CTA; the
// halo columns are re-read by the neighbouring CTAs, mostly from L2.
#pragma once
#include "cfd.cuh"
#include "pair.cuh"
#include "tma.cuh"

namespace fb {

// axis4r (one axis of the 4th-order schemes) with its operations spelled out,
// on one lane or on a lane pair (two axes of a component); each lane rounds as
// the scalar version
template <typename T>
__device__ __forceinline__ T axis4e(T ucc, T up1, T up2, T um1, T um2, T Ua, T JP, T JM, T c) {
    T dl = fma(T(27), up1, -up2);
    dl = fma(T(-27), ucc, dl) + um1;
    T dr = fma(T(27), ucc, -up1);
    dr = fma(T(-27), um1, dr) + um2;
    T d4 = fma(T(-4), up1, up2);
    d4 = fma(T(6), ucc, d4);
    d4 = fma(T(-4), um1, d4) + um2;
    T r = JP * dl;
    r = fma(JM, dr, r) * c;
    return fma(Ua, d4, r);
}
template <typename T2>
__device__ __forceinline__ T2 axis4p(T2 ucc, T2 up1, T2 up2, T2 um1, T2 um2, T2 Ua, T2 JP, T2 JM, T2 c) {
    using S = decltype(ucc.x);
    const T2 k27 = mk2(S(27), S(27)), m27 = mk2(S(-27), S(-27)), m4 = mk2(S(-4), S(-4)), k6 = mk2(S(6), S(6));
    T2 dl = fma2(k27, up1, mk2(-up2.x, -up2.y));
    dl = add2(fma2(m27, ucc, dl), um1);
    T2 dr = fma2(k27, ucc, mk2(-up1.x, -up1.y));
    dr = add2(fma2(m27, um1, dr), um2);
    T2 d4 = fma2(m4, up1, up2);
    d4 = fma2(k6, ucc, d4);
    d4 = add2(fma2(m4, um1, d4), um2);
    T2 r = mul2(JP, dl);
    r = mul2(fma2(JM, dr, r), c);
    return fma2(Ua, d4, r);
}

__host__ __device__ constexpr int round128(int b) { return (b + 127) / 128 * 128; }

template <typename T, int NS_>
struct PUTile {
    static constexpr int TX = 32, TY = 8, BX = TX + 4, BY = TY + 4, PE = BX * BY;
    static constexpr int U_BYTES = round128(3 * PE * (int)sizeof(T));
    static constexpr int N_BYTES = round128(PE * (int)sizeof(T));
    static constexpr int SLOT = 2 * U_BYTES + N_BYTES;
    static constexpr int NS = NS_;
    static constexpr int SMEM = NS * SLOT + 128;
    static constexpr uint32_t TX_BYTES = 7 * PE * sizeof(T);
};

// race-free FSPseudoU (src/dev/FalmCFDDevCall.cu:10-301), same expressions as
// k_pseudo_u; one instantiation per advection scheme ADV (FALM_ADV_*), so the
// three components' arithmetic is straight-line code
template <typename T, int NS, int ADV>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 2 : 3) k_pseudo_u_tma(Geom g, int kc, MetricView<T> mv,
    const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap muu,
    const __grid_constant__ CUtensorMap mnut, const T *__restrict__ un, int un_is_u, T *__restrict__ ua,
    const T *__restrict__ ff, AlmFuse af, T ReI, T dt, int *err) {
    constexpr int adv = ADV;
    using L = PUTile<T, NS>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = (uint64_t *)(smem + NS * L::SLOT);
    const long long N = g.n;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i0 = g.gc + blockIdx.x * L::TX, j0 = g.gc + blockIdx.y * L::TY;
    const int k0 = g.gc + blockIdx.z * kc, k1 = min(k0 + kc, g.sz - g.gc);
    const int i = i0 + tx, j = j0 + ty;
    bool active = i < g.sx - g.gc && j < g.sy - g.gc;
    const int P0 = k0 - 2, nplanes = (k1 + 2) - P0;
    // slots of planes q, q+1, q+2 and the barrier parity of plane q+2, rolled
    // along the march from q = 2 (NS need not be a power of two)
    int s0 = 2 % NS, s1 = 3 % NS, s2 = 4 % NS, ph2 = (4 / NS) & 1;
    // box origin (tile minus the halo of 2), kept inside the tensor when it is wide enough
    const int xb = box_origin(i0 - 2, L::BX, g.sx, 16 / (int)sizeof(T)), yb = box_origin(j0 - 2, L::BY, g.sy, 1);
    const int ox = min(i, g.sx - g.gc - 1) - xb, oy = min(j, g.sy - g.gc - 1) - yb;
    const int o = oy * L::BX + ox;
    // self-check: the radius-2 neighbourhood of a computed cell lies inside the staged box
    if (active && (ox < 2 || ox > L::BX - 3 || oy < 2 || oy > L::BY - 3)) { atomicExch(err, 300 + 1); active = false; }
    auto slot = [&](int q) { return smem + (q % NS) * L::SLOT; };
    auto issue = [&](int q) {
        unsigned char *s = slot(q);
        uint64_t *b = bar + (q % NS);
        const int e = (int)sizeof(T);
        if (tma_ok(s, xb, yb, P0 + q, e, g.sx, g.sy, g.sz) && tma_ok(s + L::U_BYTES, xb, yb, P0 + q, e, g.sx, g.sy, g.sz) &&
            tma_ok(s + 2 * L::U_BYTES, xb, yb, P0 + q, e, g.sx, g.sy, g.sz)) {
            mbar_expect_tx(b, L::TX_BYTES);
            tma_load_4d(s, &mu, xb, yb, P0 + q, 0, b);
            tma_load_4d(s + L::U_BYTES, &muu, xb, yb, P0 + q, 0, b);
            tma_load_4d(s + 2 * L::U_BYTES, &mnut, xb, yb, P0 + q, 0, b);
        } else {
            tma_reject(b, err, 1);
        }
    };
    // column constants (x, y metric factors and the ALM distance in x/y) and the
    // rolling z metric of planes k-1, k (k+1 is loaded per plane)
    const int ic = min(i, g.sx - g.gc - 1), jc = min(j, g.sy - g.gc - 1);
    const T hxc = ldg(mv.m.h[0] + ic), hyc = ldg(mv.m.h[1] + jc);
    const T Pc = hxc * hyc, Pe = ldg(mv.m.h[0] + ic + 1) * hyc, Pw = ldg(mv.m.h[0] + ic - 1) * hyc;
    const T Pn = hxc * ldg(mv.m.h[1] + jc + 1), Ps = hxc * ldg(mv.m.h[1] + jc - 1);
    const T kxc = ldg(mv.m.k[0] + ic), kxe = ldg(mv.m.k[0] + ic + 1), kxw = ldg(mv.m.k[0] + ic - 1);
    const T kyc = ldg(mv.m.k[1] + jc), kyn = ldg(mv.m.k[1] + jc + 1), kys = ldg(mv.m.k[1] + jc - 1);
    T hzb = ldg(mv.m.h[2] + P0 + 1), hzk = ldg(mv.m.h[2] + P0 + 2), kzb = ldg(mv.m.k[2] + P0 + 1), kzk = ldg(mv.m.k[2] + P0 + 2);
    // The face factors g_d(c) + g_d(c+-e_d) of the diffusion, g_d = ja k_d^2 and
    // ja = hx hy hz, separate: an x/y face's is hz times a column constant, a z
    // face's is hx hy times a plane constant (the reference's values up to
    // rounding); 1/ja is the product of the inverse widths.
    const T kxc2 = kxc * kxc, kyc2 = kyc * kyc;
    const T Axe = Pc * kxc2 + Pe * (kxe * kxe), Axw = Pc * kxc2 + Pw * (kxw * kxw);
    const T Ayn = Pc * kyc2 + Pn * (kyn * kyn), Ays = Pc * kyc2 + Ps * (kys * kys);
    const T kxy = kxc * kyc;
    // force boxes whose x/y extent holds this column (bit t for box t)
    unsigned colmask = 0;
    if (!ff && af.apcount > 0) {
#pragma unroll
        for (int t = 0; t < kMaxTurbines; t++)
            if (t < af.bs.n && (unsigned)(ic - af.bs.lo[t][0]) < (unsigned)af.bs.ext[t][0] &&
                (unsigned)(jc - af.bs.lo[t][1]) < (unsigned)af.bs.ext[t][1])
                colmask |= 1u << t;
    }
    int issued = 0, waited = 0;
    if (threadIdx.x == 0) {
        prefetch_tmap(&mu); prefetch_tmap(&muu); prefetch_tmap(&mnut);
        for (int s = 0; s < NS; s++) mbar_init(bar + s, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const int first = min(NS, nplanes);
    if (threadIdx.x == 0)
        for (int q = 0; q < first; q++) issue(q);
    issued = first;
    // warp 0 polls the barriers; the block barrier that follows makes the
    // landed planes visible to every thread
    auto wait_q = [&](int q) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + (q % NS), (q / NS) & 1, err); };
    // every plane is waited for exactly once, before its first read: planes
    // 0..3 here (iteration q = 2 reads q, q+1, q+2), plane q+2 at iteration q
    bool fail = !wait_q(0);
    fail = !wait_q(1) || fail;
    fail = !wait_q(2) || fail;
    fail = !wait_q(3) || fail;
    waited = 4;
    T um2[3], um1[3], nutm1, uu2m1;
    if (__syncthreads_or(fail)) goto drain;
    {
        const T *U0 = (const T *)slot(0), *U1 = (const T *)slot(1);
        const T *UU1 = (const T *)(slot(1) + L::U_BYTES), *N1 = (const T *)(slot(1) + 2 * L::U_BYTES);
#pragma unroll
        for (int d = 0; d < 3; d++) { um2[d] = U0[d * L::PE + o]; um1[d] = U1[d * L::PE + o]; }
        nutm1 = N1[o];
        uu2m1 = UU1[2 * L::PE + o];
    }
    // planes 0 and 1 now live in registers: refill their slots with planes NS
    // and NS+1 (iteration q waits for plane q+2, which must already be in flight)
    __syncthreads();
    {
        const int upto = min(NS + 1, nplanes - 1);
        if (upto >= issued) {
            if (threadIdx.x == 0) {
                fence_proxy_async();
                for (int pl = issued; pl <= upto; pl++) issue(pl);
            }
            issued = upto + 1;
        }
    }
    for (int q = 2; q < nplanes - 2; q++) {
        // planes q (= k), q+1, q+2 must be resident; q+2 is the new one
        fail = !(threadIdx.x >= 32 || mbar_wait(bar + s2, ph2, err));
        waited = q + 3;
        if (__syncthreads_or(fail)) goto drain;
        {   // planes up to q-1 are no longer read (held in registers): refill their slots
            const int upto = min(q - 1 + NS, nplanes - 1);
            if (upto >= issued) {
                if (threadIdx.x == 0) {
                    fence_proxy_async();
                    for (int pl = issued; pl <= upto; pl++) issue(pl);
                }
                issued = upto + 1;
            }
        }
        const int k = P0 + q;
        unsigned char *const sp0 = smem + s0 * L::SLOT, *const sp1 = smem + s1 * L::SLOT, *const sp2 = smem + s2 * L::SLOT;
        const T *U0 = (const T *)sp0, *UU0 = (const T *)(sp0 + L::U_BYTES), *N0 = (const T *)(sp0 + 2 * L::U_BYTES);
        const T *U1 = (const T *)sp1, *N1 = (const T *)(sp1 + 2 * L::U_BYTES);
        const T *U2 = (const T *)sp2;
        const T hzt = ldg(mv.m.h[2] + k + 1), kzt = ldg(mv.m.k[2] + k + 1);
        if (active) {
            const long long cc = g.id(i, j, k);
            const T hzkz2 = hzk * (kzk * kzk);
            const T Bzt = hzkz2 + hzt * (kzt * kzt), Bzb = hzkz2 + hzb * (kzb * kzb);
            // the scheme's divisions by the Jacobian become multiplications by 1/ja
            const T ij = kxy * kzk;
            const T UE = UU0[o], UW = UU0[o - 1], VN = UU0[L::PE + o], VS = UU0[L::PE + o - L::BX];
            const T WT = UU0[2 * L::PE + o], WB = uu2m1;
            const T nutcc = N0[o];
            // diffusion coefficients of the six faces, shared by the three components
            // (src/FalmCFDScheme.h:167-191)
            const T ce = (hzk * Axe) * (ReI + T(0.5) * (nutcc + N0[o + 1]));
            const T cw = (hzk * Axw) * (ReI + T(0.5) * (nutcc + N0[o - 1]));
            const T cn = (hzk * Ayn) * (ReI + T(0.5) * (nutcc + N0[o + L::BX]));
            const T cs = (hzk * Ays) * (ReI + T(0.5) * (nutcc + N0[o - L::BX]));
            const T ct = (Pc * Bzt) * (ReI + T(0.5) * (nutcc + N1[o]));
            const T cb = (Pc * Bzb) * (ReI + T(0.5) * (nutcc + nutm1));
            const T vscale = T(0.5) * ij;
            T fvec[3] = {0, 0, 0};
            if (ff) {
                fvec[0] = ff[cc]; fvec[1] = ff[cc + N]; fvec[2] = ff[cc + 2 * N];
            } else if (colmask) {
                // the first force box holding the cell has the full sum over all APs
                const T *fbx = (const T *)af.fbox;
#pragma unroll
                for (int t = 0; t < kMaxTurbines; t++) {
                    const int lk = k - af.bs.lo[t][2];
                    if (((colmask >> t) & 1u) && (unsigned)lk < (unsigned)af.bs.ext[t][2]) {
                        const long long qb = af.bs.off[t] + (i - af.bs.lo[t][0]) +
                                             (long long)af.bs.ext[t][0] * ((j - af.bs.lo[t][1]) + (long long)af.bs.ext[t][1] * lk);
                        fvec[0] = fbx[qb]; fvec[1] = fbx[qb + af.bs.total]; fvec[2] = fbx[qb + 2 * af.bs.total];
                        break;
                    }
                }
            }
            // advection: |U| k_d weights of the 4th-order dissipation (times alpha),
            // and the common factor of the two 4th-order fluxes, 1/(2*24*ja)
            const T alpha = adv == FALM_ADV_UTOPIA ? T(1. / 12.) : (adv == FALM_ADV_KK ? T(1. / 4.) : T(1. / 24.));
            const T Ua = fabs(U0[o] * kxc) * alpha, Va = fabs(U0[L::PE + o] * kyc) * alpha, Wa = fabs(U0[2 * L::PE + o] * kzk) * alpha;
            const T c4 = T(0.5 / 24.) * ij;
            // the x and y axes of a component run as one lane pair
            using T2 = P2<T>;
            const T2 JP2 = mk2(UE, VN), JM2 = mk2(UW, VS), UA2 = mk2(Ua, Va), C42 = mk2(c4, c4);
            const T2 CP2 = mk2(ce, cn), CM2 = mk2(cw, cs);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const T *Ud = U0 + d * L::PE;
                const T ucc = Ud[o];
                const T ue1 = Ud[o + 1], uw1 = Ud[o - 1], un1 = Ud[o + L::BX], us1 = Ud[o - L::BX];
                const T ut1 = U1[d * L::PE + o], ub1 = um1[d];
                const T2 cc2 = mk2(ucc, ucc), p1 = mk2(ue1, un1), m1 = mk2(uw1, us1);
                T adv_v;
                if constexpr (adv == FALM_ADV_UPWIND1) {
                    adv_v = T(0);
                    adv_v += upwind_flux1(ucc, ue1, UE);
                    adv_v -= upwind_flux1(uw1, ucc, UW);
                    adv_v += upwind_flux1(ucc, un1, VN);
                    adv_v -= upwind_flux1(us1, ucc, VS);
                    adv_v += upwind_flux1(ucc, ut1, WT);
                    adv_v -= upwind_flux1(ub1, ucc, WB);
                    adv_v *= ij;
                } else {
                    const T ue2 = Ud[o + 2], uw2 = Ud[o - 2], un2 = Ud[o + 2 * L::BX], us2 = Ud[o - 2 * L::BX];
                    const T ut2 = U2[d * L::PE + o], ub2 = um2[d];
                    if constexpr (adv == FALM_ADV_QUICK) {
                        adv_v = T(0.);
                        axis_quick(adv_v, ucc, ue1, ue2, uw1, uw2, UE, UW);
                        axis_quick(adv_v, ucc, un1, un2, us1, us2, VN, VS);
                        axis_quick(adv_v, ucc, ut1, ut2, ub1, ub2, WT, WB);
                        adv_v *= T(1. / 16.) * ij;
                    } else {
                        const T2 axy = axis4p(cc2, p1, mk2(ue2, un2), m1, mk2(uw2, us2), UA2, JP2, JM2, C42);
                        adv_v = axy.x + axy.y;
                        adv_v += axis4e(ucc, ut1, ut2, ub1, ub2, Wa, WT, WB, c4);
                    }
                }
                // diffusion: the (e, n) and (w, s) face terms as lane pairs
                const T2 dxy = sub2(mul2(CP2, sub2(p1, cc2)), mul2(CM2, sub2(cc2, m1)));
                T vis = (dxy.x + dxy.y) + (ct * (ut1 - ucc) - cb * (ucc - ub1));
                vis *= vscale;
                const T unv = un_is_u ? ucc : un[cc + d * N];
                ua[cc + d * N] = unv + dt * (-adv_v + vis + fvec[d]);
            }
        }
        hzb = hzk; hzk = hzt; kzb = kzk; kzk = kzt;
        // the column's own values of plane k become the -1 neighbours of the next plane
#pragma unroll
        for (int d = 0; d < 3; d++) { um2[d] = um1[d]; um1[d] = U0[d * L::PE + o]; }
        nutm1 = N0[o];
        uu2m1 = UU0[2 * L::PE + o];
        s0 = s1; s1 = s2;
        if (++s2 == NS) { s2 = 0; ph2 ^= 1; }
    }
    return;
drain:
    // a wait gave up: let this CTA's own copies land (bounded) before leaving
    for (int q = waited; q < issued; q++) wait_q(q);
}

// ---------------------------------------------------------------- x-pair version (FP32)
// The same update with each thread owning two x-adjacent cells (i, i+1) of one
// row: 128 threads on the 32 x 8 tile.  Every axis of every component runs on
// the packed FP32 pipe with the two cells as the lanes, a row's values come in
// 64-bit pair loads (the x neighbours i-2 .. i+3 in three of them), and the
// per-plane work of a thread (wait, addressing, z metric) is shared by two
// cells.  Each lane evaluates the operations of the one-cell kernel in the same
// order.  For the 4th-order schemes (Upwind3, UTOPIA, KK) and an even interior
// width, where every pair lies inside the interior or outside it.
template <int NS, int ADV>
__global__ void __launch_bounds__(128, 4) k_pseudo_u_tma2(Geom g, int kc, MetricView<float> mv,
    const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap muu,
    const __grid_constant__ CUtensorMap mnut, const float *__restrict__ un, int un_is_u, float *__restrict__ ua,
    const float *__restrict__ ff, AlmFuse af, float ReI, float dt, int *err) {
    using T = float;
    using T2 = float2;
    using L = PUTile<T, NS>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = (uint64_t *)(smem + NS * L::SLOT);
    const long long N = g.n;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int i0 = g.gc + blockIdx.x * L::TX, j0 = g.gc + blockIdx.y * L::TY;
    const int k0 = g.gc + blockIdx.z * kc, k1 = min(k0 + kc, g.sz - g.gc);
    const int ihi = g.sx - g.gc, jhi = g.sy - g.gc;
    const int i = i0 + 2 * tx, j = j0 + ty;                 // the pair's first cell
    bool active = i < ihi && j < jhi;
    const int P0 = k0 - 2, nplanes = (k1 + 2) - P0;
    int s0 = 2 % NS, s1 = 3 % NS, s2 = 4 % NS, ph2 = (4 / NS) & 1;
    const int xb = box_origin(i0 - 2, L::BX, g.sx, 4), yb = box_origin(j0 - 2, L::BY, g.sy, 1);
    const int ic = min(i, ihi - 2), jc = min(j, jhi - 1);   // inactive threads read a staged pair
    const int ox = ic - xb, oy = jc - yb;
    // self-check: the radius-2 neighbourhood of the pair lies inside the staged box, pair-aligned
    const bool inbox = ox >= 2 && ox + 3 <= L::BX - 1 && oy >= 2 && oy <= L::BY - 3 && ((oy * L::BX + ox) & 1) == 0;
    if (!inbox) {
        if (active) atomicExch(err, 300 + 7);
        active = false;
    }
    const int o = inbox ? oy * L::BX + ox : 2 * L::BX + 2;
    auto slot = [&](int q) { return smem + (q % NS) * L::SLOT; };
    auto issue = [&](int q) {
        unsigned char *sp = slot(q);
        uint64_t *b = bar + (q % NS);
        if (tma_ok(sp, xb, yb, P0 + q, 4, g.sx, g.sy, g.sz) && tma_ok(sp + L::U_BYTES, xb, yb, P0 + q, 4, g.sx, g.sy, g.sz) &&
            tma_ok(sp + 2 * L::U_BYTES, xb, yb, P0 + q, 4, g.sx, g.sy, g.sz)) {
            mbar_expect_tx(b, L::TX_BYTES);
            tma_load_4d(sp, &mu, xb, yb, P0 + q, 0, b);
            tma_load_4d(sp + L::U_BYTES, &muu, xb, yb, P0 + q, 0, b);
            tma_load_4d(sp + 2 * L::U_BYTES, &mnut, xb, yb, P0 + q, 0, b);
        } else {
            tma_reject(b, err, 7);
        }
    };
    // column constants of the two cells
    const T hyc = ldg(mv.m.h[1] + jc), hyn = ldg(mv.m.h[1] + jc + 1), hys = ldg(mv.m.h[1] + jc - 1);
    const T kyc = ldg(mv.m.k[1] + jc), kyn = ldg(mv.m.k[1] + jc + 1), kys = ldg(mv.m.k[1] + jc - 1);
    T hx[4], kxa[4];   // cells ic-1 .. ic+2
#pragma unroll
    for (int q = 0; q < 4; q++) { hx[q] = ldg(mv.m.h[0] + ic - 1 + q); kxa[q] = ldg(mv.m.k[0] + ic - 1 + q); }
    T2 Pc, Axe, Axw, Ayn, Ays, kxc, kxy;
    {
        T pc[2], axe[2], axw[2], ayn[2], ays[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const T hxc = hx[1 + e], kc_ = kxa[1 + e];
            const T P = hxc * hyc, Pe = hx[2 + e] * hyc, Pw = hx[e] * hyc, Pn = hxc * hyn, Ps = hxc * hys;
            const T kxc2 = kc_ * kc_, kyc2 = kyc * kyc;
            pc[e] = P;
            axe[e] = P * kxc2 + Pe * (kxa[2 + e] * kxa[2 + e]);
            axw[e] = P * kxc2 + Pw * (kxa[e] * kxa[e]);
            ayn[e] = P * kyc2 + Pn * (kyn * kyn);
            ays[e] = P * kyc2 + Ps * (kys * kys);
        }
        Pc = mk2(pc[0], pc[1]); Axe = mk2(axe[0], axe[1]); Axw = mk2(axw[0], axw[1]);
        Ayn = mk2(ayn[0], ayn[1]); Ays = mk2(ays[0], ays[1]);
        kxc = mk2(kxa[1], kxa[2]);
        kxy = mk2(kxa[1] * kyc, kxa[2] * kyc);
    }
    T hzb = ldg(mv.m.h[2] + P0 + 1), hzk = ldg(mv.m.h[2] + P0 + 2), kzb = ldg(mv.m.k[2] + P0 + 1), kzk = ldg(mv.m.k[2] + P0 + 2);
    unsigned colmask[2] = {0u, 0u};
    if (!ff && af.apcount > 0) {
#pragma unroll
        for (int e = 0; e < 2; e++)
#pragma unroll
            for (int t = 0; t < kMaxTurbines; t++)
                if (t < af.bs.n && (unsigned)(ic + e - af.bs.lo[t][0]) < (unsigned)af.bs.ext[t][0] &&
                    (unsigned)(jc - af.bs.lo[t][1]) < (unsigned)af.bs.ext[t][1])
                    colmask[e] |= 1u << t;
    }
    int issued = 0, waited = 0;
    if (threadIdx.x == 0) {
        prefetch_tmap(&mu); prefetch_tmap(&muu); prefetch_tmap(&mnut);
        for (int q = 0; q < NS; q++) mbar_init(bar + q, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const int first = min(NS, nplanes);
    if (threadIdx.x == 0)
        for (int q = 0; q < first; q++) issue(q);
    issued = first;
    auto wait_q = [&](int q) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + (q % NS), (q / NS) & 1, err); };
    bool fail = !wait_q(0);
    fail = !wait_q(1) || fail;
    fail = !wait_q(2) || fail;
    fail = !wait_q(3) || fail;
    waited = 4;
    T2 um2[3], um1[3], nutm1, uu2m1;
    if (__syncthreads_or(fail)) goto drain;
    {
        const T *U0 = (const T *)slot(0), *U1 = (const T *)slot(1);
        const T *UU1 = (const T *)(slot(1) + L::U_BYTES), *N1 = (const T *)(slot(1) + 2 * L::U_BYTES);
#pragma unroll
        for (int d = 0; d < 3; d++) { um2[d] = ld2(U0 + d * L::PE + o); um1[d] = ld2(U1 + d * L::PE + o); }
        nutm1 = ld2(N1 + o);
        uu2m1 = ld2(UU1 + 2 * L::PE + o);
    }
    __syncthreads();
    {
        const int upto = min(NS + 1, nplanes - 1);
        if (upto >= issued) {
            if (threadIdx.x == 0) {
                fence_proxy_async();
                for (int pl = issued; pl <= upto; pl++) issue(pl);
            }
            issued = upto + 1;
        }
    }
    for (int q = 2; q < nplanes - 2; q++) {
        fail = !(threadIdx.x >= 32 || mbar_wait(bar + s2, ph2, err));
        waited = q + 3;
        if (__syncthreads_or(fail)) goto drain;
        {
            const int upto = min(q - 1 + NS, nplanes - 1);
            if (upto >= issued) {
                if (threadIdx.x == 0) {
                    fence_proxy_async();
                    for (int pl = issued; pl <= upto; pl++) issue(pl);
                }
                issued = upto + 1;
            }
        }
        const int k = P0 + q;
        unsigned char *const sp0 = smem + s0 * L::SLOT, *const sp1 = smem + s1 * L::SLOT, *const sp2 = smem + s2 * L::SLOT;
        const T *U0 = (const T *)sp0, *UU0 = (const T *)(sp0 + L::U_BYTES), *N0 = (const T *)(sp0 + 2 * L::U_BYTES);
        const T *U1 = (const T *)sp1, *N1 = (const T *)(sp1 + 2 * L::U_BYTES);
        const T *U2 = (const T *)sp2;
        const T hzt = ldg(mv.m.h[2] + k + 1), kzt = ldg(mv.m.k[2] + k + 1);
        if (active) {
            const long long cc = g.id(i, j, k);
            const T hzkz2 = hzk * (kzk * kzk);
            const T Bzt = hzkz2 + hzt * (kzt * kzt), Bzb = hzkz2 + hzb * (kzb * kzb);
            const T2 ij = mul2(kxy, mk2(kzk, kzk));
            // face velocities: x faces of the pair from the cells i-1 .. i+1
            const T2 uxc = ld2(UU0 + o), uxm = ld2(UU0 + o - 2);
            const T2 UE = uxc, UW = mk2(uxm.y, uxc.x);
            const T2 VN = ld2(UU0 + L::PE + o), VS = ld2(UU0 + L::PE + o - L::BX);
            const T2 WT = ld2(UU0 + 2 * L::PE + o), WB = uu2m1;
            const T2 nc = ld2(N0 + o), nm = ld2(N0 + o - 2), np = ld2(N0 + o + 2);
            const T2 ne = mk2(nc.y, np.x), nw = mk2(nm.y, nc.x);
            const T2 nn = ld2(N0 + o + L::BX), ns = ld2(N0 + o - L::BX), nt = ld2(N1 + o);
            const T2 hzk2 = mk2(hzk, hzk), half = mk2(T(0.5), T(0.5)), rei = mk2(ReI, ReI);
            auto face = [&](T2 A, T2 nb) { return mul2(mul2(hzk2, A), add2(rei, mul2(half, add2(nc, nb)))); };
            const T2 ce = face(Axe, ne), cw = face(Axw, nw), cn = face(Ayn, nn), cs = face(Ays, ns);
            const T2 ct = mul2(mul2(Pc, mk2(Bzt, Bzt)), add2(rei, mul2(half, add2(nc, nt))));
            const T2 cb = mul2(mul2(Pc, mk2(Bzb, Bzb)), add2(rei, mul2(half, add2(nc, nutm1))));
            const T2 vscale = mul2(half, ij);
            T2 fv[3] = {mk2(T(0), T(0)), mk2(T(0), T(0)), mk2(T(0), T(0))};
            if (ff) {
                fv[0] = ld2(ff + cc); fv[1] = ld2(ff + cc + N); fv[2] = ld2(ff + cc + 2 * N);
            } else if (colmask[0] | colmask[1]) {
                const T *fbx = (const T *)af.fbox;
#pragma unroll
                for (int e = 0; e < 2; e++) {
#pragma unroll
                    for (int t = 0; t < kMaxTurbines; t++) {
                        const int lk = k - af.bs.lo[t][2];
                        if (((colmask[e] >> t) & 1u) && (unsigned)lk < (unsigned)af.bs.ext[t][2]) {
                            const long long qb = af.bs.off[t] + (i + e - af.bs.lo[t][0]) +
                                                 (long long)af.bs.ext[t][0] * ((j - af.bs.lo[t][1]) + (long long)af.bs.ext[t][1] * lk);
                            const T f0 = fbx[qb], f1 = fbx[qb + af.bs.total], f2 = fbx[qb + 2 * af.bs.total];
                            if (e == 0) { fv[0].x = f0; fv[1].x = f1; fv[2].x = f2; }
                            else { fv[0].y = f0; fv[1].y = f1; fv[2].y = f2; }
                            break;
                        }
                    }
                }
            }
            const T alpha = ADV == FALM_ADV_UTOPIA ? T(1. / 12.) : (ADV == FALM_ADV_KK ? T(1. / 4.) : T(1. / 24.));
            const T2 al = mk2(alpha, alpha);
            const T2 u0c = ld2(U0 + o), v0c = ld2(U0 + L::PE + o), w0c = ld2(U0 + 2 * L::PE + o);
            const T2 Ua = mul2(fabs2(mul2(u0c, kxc)), al), Va = mul2(fabs2(mul2(v0c, mk2(kyc, kyc))), al);
            const T2 Wa = mul2(fabs2(mul2(w0c, mk2(kzk, kzk))), al);
            const T2 c4 = mul2(mk2(T(0.5 / 24.), T(0.5 / 24.)), ij);
            const T2 dt2 = mk2(dt, dt);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const T *Ud = U0 + d * L::PE;
                const T2 C = ld2(Ud + o), M = ld2(Ud + o - 2), P = ld2(Ud + o + 2);
                const T2 xp1 = mk2(C.y, P.x), xm1 = mk2(M.y, C.x);
                const T2 un1 = ld2(Ud + o + L::BX), us1 = ld2(Ud + o - L::BX);
                const T2 un2 = ld2(Ud + o + 2 * L::BX), us2 = ld2(Ud + o - 2 * L::BX);
                const T2 ut1 = ld2(U1 + d * L::PE + o), ut2 = ld2(U2 + d * L::PE + o);
                const T2 ub1 = um1[d], ub2 = um2[d];
                const T2 ax = axis4p(C, xp1, P, xm1, M, Ua, UE, UW, c4);
                const T2 ay = axis4p(C, un1, un2, us1, us2, Va, VN, VS, c4);
                const T2 az = axis4p(C, ut1, ut2, ub1, ub2, Wa, WT, WB, c4);
                const T2 adv = add2(add2(ax, ay), az);
                const T2 dx = sub2(mul2(ce, sub2(xp1, C)), mul2(cw, sub2(C, xm1)));
                const T2 dy = sub2(mul2(cn, sub2(un1, C)), mul2(cs, sub2(C, us1)));
                const T2 dz = sub2(mul2(ct, sub2(ut1, C)), mul2(cb, sub2(C, ub1)));
                const T2 vis = mul2(add2(add2(dx, dy), dz), vscale);
                const T2 unv = un_is_u ? C : ld2(un + cc + d * N);
                st2(ua + cc + d * N, fma2(dt2, add2(sub2(vis, adv), fv[d]), unv));
            }
        }
        hzb = hzk; hzk = hzt; kzb = kzk; kzk = kzt;
#pragma unroll
        for (int d = 0; d < 3; d++) { um2[d] = um1[d]; um1[d] = ld2(U0 + d * L::PE + o); }
        nutm1 = ld2(N0 + o);
        uu2m1 = ld2(UU0 + 2 * L::PE + o);
        s0 = s1; s1 = s2;
        if (++s2 == NS) { s2 = 0; ph2 ^= 1; }
    }
    return;
drain:
    for (int q = waited; q < issued; q++) wait_q(q);
}

}  // namespace fb
