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
#include "tma.cuh"

namespace fb {

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

// race-free FSPseudoU (src/dev/FalmCFDDevCall.cu:10-301), same expressions as k_pseudo_u
template <typename T, int NS>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 2 : 3) k_pseudo_u_tma(Geom g, int kc, MetricView<T> mv,
    const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap muu,
    const __grid_constant__ CUtensorMap mnut, const T *__restrict__ un, int un_is_u, T *__restrict__ ua,
    const T *__restrict__ ff, AlmFuse af, T ReI, T dt, int adv, int *err) {
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
    auto wait_q = [&](int q) -> bool { return mbar_wait(bar + (q % NS), (q / NS) & 1, err); };
    bool fail = !wait_q(0);
    fail = !wait_q(1) || fail;
    waited = 2;
    T um2[3], um1[3], nutm1, uu2m1;
    {
        const T *U0 = (const T *)slot(0), *U1 = (const T *)slot(1);
        const T *UU1 = (const T *)(slot(1) + L::U_BYTES), *N1 = (const T *)(slot(1) + 2 * L::U_BYTES);
#pragma unroll
        for (int d = 0; d < 3; d++) { um2[d] = U0[d * L::PE + o]; um1[d] = U1[d * L::PE + o]; }
        nutm1 = N1[o];
        uu2m1 = UU1[2 * L::PE + o];
    }
    // every plane is waited for exactly once, before its first read: planes
    // 0..3 here (iteration q = 2 reads q, q+1, q+2), plane q+2 at iteration q
    fail = !wait_q(2) || fail;
    fail = !wait_q(3) || fail;
    waited = 4;
    if (__syncthreads_or(fail)) goto drain;
    if (threadIdx.x == 0) {
        fence_proxy_async();
        for (int q = NS; q < NS + 2 && q < nplanes; q++) issue(q);
    }
    issued = min(NS + 2, nplanes);
    for (int q = 2; q < nplanes - 2; q++) {
        // planes q (= k), q+1, q+2 must be resident; q+2 is the new one
        fail = !wait_q(q + 2);
        waited = q + 3;
        if (__syncthreads_or(fail)) goto drain;
        if (q >= 3 && q - 1 + NS < nplanes) {        // slot of plane q-1 is free: refill it
            if (threadIdx.x == 0) {
                fence_proxy_async();
                issue(q - 1 + NS);
            }
            issued = q - 1 + NS + 1;
        }
        const int k = P0 + q;
        const T *U0 = (const T *)slot(q), *UU0 = (const T *)(slot(q) + L::U_BYTES), *N0 = (const T *)(slot(q) + 2 * L::U_BYTES);
        const T *U1 = (const T *)slot(q + 1), *N1 = (const T *)(slot(q + 1) + 2 * L::U_BYTES);
        const T *U2 = (const T *)slot(q + 2);
        if (active) {
            const long long cc = g.id(i, j, k);
            const T Uabs = fabs(U0[o] * mv.kx(0, i));
            const T Vabs = fabs(U0[L::PE + o] * mv.kx(1, j));
            const T Wabs = fabs(U0[2 * L::PE + o] * mv.kx(2, k));
            const T UE = UU0[o], UW = UU0[o - 1], VN = UU0[L::PE + o], VS = UU0[L::PE + o - L::BX];
            const T WT = UU0[2 * L::PE + o], WB = uu2m1;
            const T nutcc = N0[o], nute1 = N0[o + 1], nutw1 = N0[o - 1], nutn1 = N0[o + L::BX], nuts1 = N0[o - L::BX];
            const T nutt1 = N1[o], nutb1 = nutm1;
            const T gxcc = mv.g(0, i, j, k), gxe1 = mv.g(0, i + 1, j, k), gxw1 = mv.g(0, i - 1, j, k);
            const T gycc = mv.g(1, i, j, k), gyn1 = mv.g(1, i, j + 1, k), gys1 = mv.g(1, i, j - 1, k);
            const T gzcc = mv.g(2, i, j, k), gzt1 = mv.g(2, i, j, k + 1), gzb1 = mv.g(2, i, j, k - 1);
            const T jacob = mv.ja(i, j, k);
            T fvec[3] = {0, 0, 0};
            if (ff) {
                fvec[0] = ff[cc]; fvec[1] = ff[cc + N]; fvec[2] = ff[cc + 2 * N];
            } else if (af.apcount > 0) {
                const double *bb = af.scal->bbox;
                double cx = (double)ldg(mv.m.x[0] + i), cy = (double)ldg(mv.m.x[1] + j), cz = (double)ldg(mv.m.x[2] + k);
                if (box_dist2(cx, bb[0], bb[1]) + box_dist2(cy, bb[2], bb[3]) + box_dist2(cz, bb[4], bb[5]) < af.rcut2) {
                    T ax = 0, ay = 0, az = 0;
                    const T te = (T)af.eta, e2 = (T)af.eps * (T)af.eps;
                    for (int a = 0; a < af.apcount; a++) {
                        T dx = (T)cx - (T)__ldg(af.xyz + 3 * a), dy = (T)cy - (T)__ldg(af.xyz + 3 * a + 1);
                        T dz = (T)cz - (T)__ldg(af.xyz + 3 * a + 2);
                        T rr2 = dx * dx + dy * dy + dz * dz;
                        if ((double)rr2 < af.rcut2) {
                            T ex = exp(-rr2 / e2);
                            ax += (T)__ldg(af.force + 3 * a) * te * ex;
                            ay += (T)__ldg(af.force + 3 * a + 1) * te * ex;
                            az += (T)__ldg(af.force + 3 * a + 2) * te * ex;
                        }
                    }
                    fvec[0] = ax; fvec[1] = ay; fvec[2] = az;
                }
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const T *Ud = U0 + d * L::PE;
                const T ucc = Ud[o];
                const T ue1 = Ud[o + 1], uw1 = Ud[o - 1], un1 = Ud[o + L::BX], us1 = Ud[o - L::BX];
                const T ut1 = U1[d * L::PE + o], ub1 = um1[d];
                T adv_v;
                if (adv == FALM_ADV_UPWIND1) {
                    adv_v = T(0);
                    adv_v += upwind_flux1(ucc, ue1, UE);
                    adv_v -= upwind_flux1(uw1, ucc, UW);
                    adv_v += upwind_flux1(ucc, un1, VN);
                    adv_v -= upwind_flux1(us1, ucc, VS);
                    adv_v += upwind_flux1(ucc, ut1, WT);
                    adv_v -= upwind_flux1(ub1, ucc, WB);
                    adv_v /= jacob;
                } else {
                    const T ue2 = Ud[o + 2], uw2 = Ud[o - 2], un2 = Ud[o + 2 * L::BX], us2 = Ud[o - 2 * L::BX];
                    const T ut2 = U2[d * L::PE + o], ub2 = um2[d];
                    if (adv == FALM_ADV_QUICK) {
                        adv_v = T(0.);
                        axis_quick(adv_v, ucc, ue1, ue2, uw1, uw2, UE, UW);
                        axis_quick(adv_v, ucc, un1, un2, us1, us2, VN, VS);
                        axis_quick(adv_v, ucc, ut1, ut2, ub1, ub2, WT, WB);
                        adv_v /= (T(16) * jacob);
                    } else {
                        const T alpha = adv == FALM_ADV_UTOPIA ? T(1. / 12.) : (adv == FALM_ADV_KK ? T(1. / 4.) : T(1. / 24.));
                        adv_v = T(0.0);
                        adv_v += axis4(alpha, ucc, ue1, ue2, uw1, uw2, Uabs, UE, UW, jacob);
                        adv_v += axis4(alpha, ucc, un1, un2, us1, us2, Vabs, VN, VS, jacob);
                        adv_v += axis4(alpha, ucc, ut1, ut2, ub1, ub2, Wabs, WT, WB, jacob);
                    }
                }
                T vis = T(0.0);
                vis += (gxcc + gxe1) * (ReI + T(0.5) * (nutcc + nute1)) * (ue1 - ucc);
                vis -= (gxcc + gxw1) * (ReI + T(0.5) * (nutcc + nutw1)) * (ucc - uw1);
                vis += (gycc + gyn1) * (ReI + T(0.5) * (nutcc + nutn1)) * (un1 - ucc);
                vis -= (gycc + gys1) * (ReI + T(0.5) * (nutcc + nuts1)) * (ucc - us1);
                vis += (gzcc + gzt1) * (ReI + T(0.5) * (nutcc + nutt1)) * (ut1 - ucc);
                vis -= (gzcc + gzb1) * (ReI + T(0.5) * (nutcc + nutb1)) * (ucc - ub1);
                vis /= (T(2) * jacob);
                const T unv = un_is_u ? ucc : un[cc + d * N];
                ua[cc + d * N] = unv + dt * (-adv_v + vis + fvec[d]);
            }
        }
        // the column's own values of plane k become the -1 neighbours of the next plane
#pragma unroll
        for (int d = 0; d < 3; d++) { um2[d] = um1[d]; um1[d] = U0[d * L::PE + o]; }
        nutm1 = N0[o];
        uu2m1 = UU0[2 * L::PE + o];
    }
    return;
drain:
    // a wait gave up: let this CTA's own copies land (bounded) before leaving
    for (int q = waited; q < issued; q++) wait_q(q);
}

}  // namespace fb
