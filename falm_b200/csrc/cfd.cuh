// FalmCFD kernels: pseudo-velocity (+ fused ALM body force), face velocity
// interpolation fused with the Poisson right-hand side, pressure projection,
// Smagorinsky/CSM eddy viscosity fused with the divergence norm.
//
// Each formula follows the reference expression by expression (same operand
// order) so that the FP64 path differs from the reference only by FMA
// contraction and reduction order.
#pragma once
#include "common.cuh"

namespace fb {

// ---------------------------------------------------------------- schemes
// src/FalmCFDScheme.h:8-31
template <typename T>
__device__ __forceinline__ T upwind_flux1(T ul, T ur, T UF) { return T(0.5) * (UF * (ur + ul) - fabs(UF) * (ur - ul)); }

// src/FalmCFDScheme.h:68-165 (Upwind3 alpha 1/24, UTOPIA 1/12, KK 1/4): one axis
template <typename T>
__device__ __forceinline__ T axis4(T alpha, T ucc, T up1, T up2, T um1, T um2, T Uabs, T JP, T JM, T jac) {
    T UDL = JP * (-up2 + T(27) * up1 - T(27) * ucc + um1) / T(24.);
    T UDR = JM * (-up1 + T(27) * ucc - T(27) * um1 + um2) / T(24.);
    T UD4 = Uabs * (up2 - T(4) * up1 + T(6) * ucc - T(4) * um1 + um2) * alpha;
    return T(.5) * (UDL + UDR) / jac + UD4;
}

// axis4 with its three divisions folded into multiplications: c = 1/(2*24*jac),
// Ua = |U| k_d alpha.  Same value up to rounding.
template <typename T>
__device__ __forceinline__ T axis4r(T ucc, T up1, T up2, T um1, T um2, T Ua, T JP, T JM, T c) {
    const T dl = -up2 + T(27) * up1 - T(27) * ucc + um1;
    const T dr = -up1 + T(27) * ucc - T(27) * um1 + um2;
    const T d4 = up2 - T(4) * up1 + T(6) * ucc - T(4) * um1 + um2;
    return (JP * dl + JM * dr) * c + Ua * d4;
}

// src/FalmCFDScheme.h:33-66, one axis, accumulated into adv in the reference's order
template <typename T>
__device__ __forceinline__ void axis_quick(T &adv, T ucc, T up1, T up2, T um1, T um2, T JP, T JM) {
    adv += JP * (-up2 + T(9) * up1 + T(9) * ucc - um1);
    adv += fabs(JP) * (up2 - T(3) * up1 + T(3) * ucc - um1);
    adv -= JM * (-up1 + T(9) * ucc + T(9) * um1 - um2);
    adv -= fabs(JM) * (up1 - T(3) * ucc + T(3) * um1 - um2);
}

// ---------------------------------------------------------------- ALM force inside the stencil

struct AlmFuse {
    int apcount;             // 0: no fused force
    const double *xyz;       // 3*apcount
    const double *force;     // 3*apcount
    const AlmScalars *scal;  // AP bounding box
    double eps, eta, rcut2;
    BoxSet bs;               // force boxes (read by the plane-streaming kernel)
    const void *fbox;
};

// Gaussian projection of src/alm/almDevCall.cu:255-294 truncated at rcut
// (contributions beyond rcut = 6 eps are below exp(-36) of the peak).
template <typename T>
__device__ __forceinline__ void alm_force_at(const double *s_ap, int apcount, double eps, double eta, double rcut2,
                                             T cx, T cy, T cz, T &fx, T &fy, T &fz) {
    T ax = 0, ay = 0, az = 0;
    const T te = (T)eta, e2 = (T)eps * (T)eps;
    for (int a = 0; a < apcount; a++) {
        T dx = cx - (T)s_ap[6 * a], dy = cy - (T)s_ap[6 * a + 1], dz = cz - (T)s_ap[6 * a + 2];
        T rr2 = dx * dx + dy * dy + dz * dz;
        if ((double)rr2 < rcut2) {
            T ex = exp(-rr2 / e2);
            ax += (T)s_ap[6 * a + 3] * te * ex;
            ay += (T)s_ap[6 * a + 4] * te * ex;
            az += (T)s_ap[6 * a + 5] * te * ex;
        }
    }
    fx = ax; fy = ay; fz = az;
}

__device__ __forceinline__ double box_dist2(double v, double lo, double hi) {
    double d = v < lo ? lo - v : (v > hi ? v - hi : 0.0);
    return d * d;
}

// ---------------------------------------------------------------- pseudo-velocity
// src/dev/FalmCFDDevCall.cu:10-301, race-free: ua must not alias u.
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_pseudo_u(Geom g, Region3 R, MetricView<T> mv,
    const T *__restrict__ un, const T *__restrict__ u, const T *__restrict__ uu, T *__restrict__ ua,
    const T *__restrict__ nut, const T *__restrict__ ff, AlmFuse af, T ReI, T dt, int adv) {
    __shared__ double s_ap[6 * kMaxFusedAp];
    const long long N = g.n;
    const int napf = af.apcount;
    if (napf > 0) {
        for (int a = threadIdx.x; a < napf; a += blockDim.x) {
            s_ap[6 * a] = af.xyz[3 * a]; s_ap[6 * a + 1] = af.xyz[3 * a + 1]; s_ap[6 * a + 2] = af.xyz[3 * a + 2];
            s_ap[6 * a + 3] = af.force[3 * a]; s_ap[6 * a + 4] = af.force[3 * a + 1]; s_ap[6 * a + 5] = af.force[3 * a + 2];
        }
        __syncthreads();
    }
    FB_FOR_ROWS(R, j, k) {
        bool row_force = false;
        double bx0 = 0, bx1 = 0;
        if (napf > 0) {
            const double *bb = af.scal->bbox;
            double cy = (double)ldg(mv.m.x[1] + j), cz = (double)ldg(mv.m.x[2] + k);
            row_force = box_dist2(cy, bb[2], bb[3]) + box_dist2(cz, bb[4], bb[5]) < af.rcut2;
            bx0 = bb[0]; bx1 = bb[1];
        }
        const T kyc = mv.kx(1, j), kzc = mv.kx(2, k);
        FB_FOR_I(R, i) {
            const long long cc = g.id(i, j, k);
            const long long e1 = cc + 1, w1 = cc - 1, e2 = cc + 2, w2 = cc - 2;
            const long long n1 = cc + g.sx, s1 = cc - g.sx, n2 = cc + 2 * g.sx, s2 = cc - 2 * g.sx;
            const long long sxy = (long long)g.sx * g.sy;
            const long long t1 = cc + sxy, b1 = cc - sxy, t2 = cc + 2 * sxy, b2 = cc - 2 * sxy;
            const T uc = u[cc], vc = u[cc + N], wc = u[cc + 2 * N];
            const T Uabs = fabs(uc * mv.kx(0, i));
            const T Vabs = fabs(vc * kyc);
            const T Wabs = fabs(wc * kzc);
            const T UE = uu[cc], UW = uu[w1], VN = uu[cc + N], VS = uu[s1 + N], WT = uu[cc + 2 * N], WB = uu[b1 + 2 * N];
            const T nutcc = nut[cc], nute1 = nut[e1], nutw1 = nut[w1], nutn1 = nut[n1], nuts1 = nut[s1];
            const T nutt1 = nut[t1], nutb1 = nut[b1];
            const T gxcc = mv.g(0, i, j, k), gxe1 = mv.g(0, i + 1, j, k), gxw1 = mv.g(0, i - 1, j, k);
            const T gycc = mv.g(1, i, j, k), gyn1 = mv.g(1, i, j + 1, k), gys1 = mv.g(1, i, j - 1, k);
            const T gzcc = mv.g(2, i, j, k), gzt1 = mv.g(2, i, j, k + 1), gzb1 = mv.g(2, i, j, k - 1);
            const T jacob = mv.ja(i, j, k);
            T fvec[3] = {0, 0, 0};
            if (ff) {
                fvec[0] = ff[cc]; fvec[1] = ff[cc + N]; fvec[2] = ff[cc + 2 * N];
            } else if (row_force) {
                double cx = (double)ldg(mv.m.x[0] + i);
                if (box_dist2(cx, bx0, bx1) + box_dist2((double)ldg(mv.m.x[1] + j), af.scal->bbox[2], af.scal->bbox[3]) +
                        box_dist2((double)ldg(mv.m.x[2] + k), af.scal->bbox[4], af.scal->bbox[5]) < af.rcut2)
                    alm_force_at<T>(s_ap, napf, af.eps, af.eta, af.rcut2, (T)cx, ldg(mv.m.x[1] + j),
                                    ldg(mv.m.x[2] + k), fvec[0], fvec[1], fvec[2]);
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const T *ud = u + d * N;
                const T ucc = ud[cc];
                const T ue1 = ud[e1], uw1 = ud[w1], un1 = ud[n1], us1 = ud[s1], ut1 = ud[t1], ub1 = ud[b1];
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
                    const T ue2 = ud[e2], uw2 = ud[w2], un2 = ud[n2], us2 = ud[s2], ut2 = ud[t2], ub2 = ud[b2];
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
                // src/FalmCFDScheme.h:167-191
                T vis = T(0.0);
                vis += (gxcc + gxe1) * (ReI + T(0.5) * (nutcc + nute1)) * (ue1 - ucc);
                vis -= (gxcc + gxw1) * (ReI + T(0.5) * (nutcc + nutw1)) * (ucc - uw1);
                vis += (gycc + gyn1) * (ReI + T(0.5) * (nutcc + nutn1)) * (un1 - ucc);
                vis -= (gycc + gys1) * (ReI + T(0.5) * (nutcc + nuts1)) * (ucc - us1);
                vis += (gzcc + gzt1) * (ReI + T(0.5) * (nutcc + nutt1)) * (ut1 - ucc);
                vis -= (gzcc + gzb1) * (ReI + T(0.5) * (nutcc + nutb1)) * (ucc - ub1);
                vis /= (T(2) * jacob);
                ua[cc + d * N] = un[cc + d * N] + dt * (-adv_v + vis + fvec[d]);
            }
        }
    }
}

// ---------------------------------------------------------------- face velocity (+ RHS)
// UtoCU (src/dev/FalmCFDDevCall.cu:303-325) + InterpolateCU (:327-349) in one
// pass over the face map; uc is rebuilt per face instead of round-tripping
// through HBM.  `uin` feeds interior cells, `ugh` guide cells (in the fused
// step the pseudo-velocity lives in a separate buffer whose guide cells are the
// previous velocity's, exactly what the reference reads from the aliased u).
// With RHS the divergence of the new faces, scaled by 1/(dt*maxdiag), is
// written at interior cells (src/FalmCFD.h:96-109); with CAVITY the wall-normal
// boundary faces are zero (app/lid3d/bcdev.cu:251-322) before the divergence.
template <typename T, bool RHS, bool CAVITY>
__global__ void __launch_bounds__(kRowThreads) k_utouu(Geom g, Region3 R, MetricView<T> mv,
    const T *__restrict__ uin, const T *__restrict__ ugh, T *__restrict__ uu, T *__restrict__ rhs, T rhs_scale) {
    const long long N = g.n;
    auto is_int = [&](int i, int j, int k) {
        return i >= g.gc && i < g.sx - g.gc && j >= g.gc && j < g.sy - g.gc && k >= g.gc && k < g.sz - g.gc;
    };
    auto ucv = [&](int d, int i, int j, int k) -> T {
        long long c = g.id(i, j, k);
        const T *src = is_int(i, j, k) ? uin : ugh;
        int idx = d == 0 ? i : (d == 1 ? j : k);
        return mv.ja(i, j, k) * mv.kx(d, idx) * src[c + d * N];
    };
    auto face = [&](int d, int i, int j, int k) -> T {
        if (CAVITY) {
            bool zero = false;
            if (d == 0) zero = (i == g.gc - 1 || i == g.sx - g.gc - 1) && j >= g.gc && j < g.sy - g.gc && k >= g.gc && k < g.sz - g.gc;
            if (d == 1) zero = (j == g.gc - 1 || j == g.sy - g.gc - 1) && i >= g.gc && i < g.sx - g.gc && k >= g.gc && k < g.sz - g.gc;
            if (d == 2) zero = ((k == g.gc - 1 && (g.zphys & 1)) || (k == g.sz - g.gc - 1 && (g.zphys & 2))) && i >= g.gc &&
                               i < g.sx - g.gc && j >= g.gc && j < g.sy - g.gc;   // slab interfaces keep their faces
            if (zero) return T(0);
        }
        T a = ucv(d, i, j, k);
        T b = d == 0 ? ucv(0, i + 1, j, k) : (d == 1 ? ucv(1, i, j + 1, k) : ucv(2, i, j, k + 1));
        return T(0.5) * (a + b);
    };
    FB_FOR_ROWS(R, j, k) {
        FB_FOR_I(R, i) {
            const long long cc = g.id(i, j, k);
            T UE = face(0, i, j, k), VN = face(1, i, j, k), WT = face(2, i, j, k);
            uu[cc] = UE; uu[cc + N] = VN; uu[cc + 2 * N] = WT;
            if (RHS && is_int(i, j, k)) {
                T UW = face(0, i - 1, j, k), VS = face(1, i, j - 1, k), WB = face(2, i, j, k - 1);
                T div = (UE - UW + VN - VS + WT - WB) / mv.ja(i, j, k);
                rhs[cc] = div * rhs_scale;
            }
        }
    }
}

// plain divergence of stored faces (src/dev/FalmCFDDevCall.cu:557-581), optionally scaled
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_divergence(Geom g, Region3 R, MetricView<T> mv,
    const T *__restrict__ uu, T *__restrict__ div, T scale, int apply_scale) {
    const long long N = g.n, sxy = (long long)g.sx * g.sy;
    FB_FOR_ROWS(R, j, k) {
        FB_FOR_I(R, i) {
            const long long c = g.id(i, j, k);
            T d = (uu[c] - uu[c - 1] + uu[c + N] - uu[c - g.sx + N] + uu[c + 2 * N] - uu[c - sxy + 2 * N]) / mv.ja(i, j, k);
            div[c] = apply_scale ? d * scale : d;
        }
    }
}

// ---------------------------------------------------------------- projection
// ProjectPGrid (src/dev/FalmCFDDevCall.cu:351-376) on interior cells and
// ProjectPFace (:378-407) on the face map, one pass.  u may alias ua, uu may alias uua.
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_project(Geom g, Region3 R, MetricView<T> mv,
    T *u, const T *ua, T *uu, const T *uua, const T *__restrict__ p, T dt) {
    const long long N = g.n, sxy = (long long)g.sx * g.sy;
    FB_FOR_ROWS(R, j, k) {
        FB_FOR_I(R, i) {
            const long long cc = g.id(i, j, k), e1 = cc + 1, n1 = cc + g.sx, t1 = cc + sxy;
            const T pcc = p[cc], pe = p[e1], pn = p[n1], pt = p[t1];
            T dpx = T(0.5) * (mv.g(0, i, j, k) + mv.g(0, i + 1, j, k)) * (pe - pcc);
            T dpy = T(0.5) * (mv.g(1, i, j, k) + mv.g(1, i, j + 1, k)) * (pn - pcc);
            T dpz = T(0.5) * (mv.g(2, i, j, k) + mv.g(2, i, j, k + 1)) * (pt - pcc);
            T f0 = uua[cc], f1 = uua[cc + N], f2 = uua[cc + 2 * N];
            bool in = i >= g.gc && j >= g.gc && k >= g.gc;   // upper bounds hold on the face map
            T a0 = 0, a1 = 0, a2 = 0, gx = 0, gy = 0, gz = 0;
            if (in) {
                a0 = ua[cc]; a1 = ua[cc + N]; a2 = ua[cc + 2 * N];
                gx = T(0.5) * mv.kx(0, i) * (pe - p[cc - 1]);
                gy = T(0.5) * mv.kx(1, j) * (pn - p[cc - g.sx]);
                gz = T(0.5) * mv.kx(2, k) * (pt - p[cc - sxy]);
            }
            uu[cc] = f0 - dt * dpx; uu[cc + N] = f1 - dt * dpy; uu[cc + 2 * N] = f2 - dt * dpz;
            if (in) { u[cc] = a0 - dt * gx; u[cc + N] = a1 - dt * gy; u[cc + 2 * N] = a2 - dt * gz; }
        }
    }
}

// ---------------------------------------------------------------- SGS (+ divergence norm)
// Smagorinsky src/dev/FalmCFDDevCall.cu:409-476, CSM :478-555.  With DIV the
// divergence of uu (:557-581) is evaluated in FP64 and its squared sum reduced
// on the device (app/nedo/main.cpp:194-197), optionally stored.
template <typename T, bool DIV>
__global__ void __launch_bounds__(kRowThreads) k_sgs_div(Geom g, Region3 R, MetricView<T> mv, Metric<double> m64,
    const T *__restrict__ u, T *__restrict__ nut, T Cs, int sgs, const T *__restrict__ uu, T *__restrict__ div_out,
    RedWork rw, double *divsum) {
    const long long N = g.n, sxy = (long long)g.sx * g.sy;
    double acc[1] = {0.0};
    FB_FOR_ROWS(R, j, k) {
        FB_FOR_I(R, i) {
            const long long cc = g.id(i, j, k);
            if (sgs != FALM_SGS_EMPTY) {
                const T kxx = mv.kx(0, i), kxy = mv.kx(1, j), kxz = mv.kx(2, k);
                T dd[3][3];
#pragma unroll
                for (int m = 0; m < 3; m++) {
                    const T *um = u + m * N;
                    dd[m][0] = T(0.5) * kxx * (um[cc + 1] - um[cc - 1]);
                    dd[m][1] = T(0.5) * kxy * (um[cc + g.sx] - um[cc - g.sx]);
                    dd[m][2] = T(0.5) * kxz * (um[cc + sxy] - um[cc - sxy]);
                }
                const T dux = dd[0][0], duy = dd[0][1], duz = dd[0][2];
                const T dvx = dd[1][0], dvy = dd[1][1], dvz = dd[1][2];
                const T dwx = dd[2][0], dwy = dd[2][1], dwz = dd[2][2];
                T d1 = T(2) * (dux * dux), d2 = T(2) * (dvy * dvy), d3 = T(2) * (dwz * dwz);
                T d4 = (duy + dvx) * (duy + dvx), d5 = (dvz + dwy) * (dvz + dwy), d6 = (duz + dwx) * (duz + dwx);
                T Du = sqrt(d1 + d2 + d3 + d4 + d5 + d6);
                T De = cbrt(mv.ja(i, j, k));
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
            if (DIV) {
                double UE = to_d(uu[cc]), UW = to_d(uu[cc - 1]), VN = to_d(uu[cc + N]), VS = to_d(uu[cc - g.sx + N]);
                double WT = to_d(uu[cc + 2 * N]), WB = to_d(uu[cc - sxy + 2 * N]);
                double ja = ldg(m64.h[0] + i) * ldg(m64.h[1] + j) * ldg(m64.h[2] + k);
                double dv = (UE - UW + VN - VS + WT - WB) / ja;
                if (div_out) div_out[cc] = (T)dv;
                acc[0] += dv * dv;
            }
        }
    }
    if (DIV) {
        double tot[1];
        if (grid_sum<1>(acc, rw, tot) && threadIdx.x == 0) *divsum = tot[0];
    }
}

}  // namespace fb
