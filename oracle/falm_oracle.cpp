/*
 * FALM LES step -- CPU oracle (test infrastructure only; see falm_oracle.h).
 *
 * Each function restates one reference routine and cites it.  Paths are
 * relative to the reference project root (ki2098/falm).  The arithmetic is
 * written in the same order as the reference so that the only differences to
 * the reference's CUDA build are floating-point contraction and summation
 * order.  Build with -ffp-contract=off (oracle/Makefile) so that the oracle
 * itself is deterministic across hosts.
 */
#include "falm_oracle.h"
#include <math.h>
#include <float.h>
#include <string.h>
#include <stdlib.h>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double kPi = M_PI;

struct Box {
    int sx, sy, sz, gc;
    long n;
    explicit Box(const or_case *c) : sx(c->sx), sy(c->sy), sz(c->sz), gc(c->gc), n((long)c->sx * c->sy * c->sz) {}
    inline long id(int i, int j, int k) const { return i + (long)j * sx + (long)k * sx * sy; }
};

inline double SQ(double a) { return a * a; }

/* src/FalmCFDScheme.h:8-31 */
inline double upwind_flux1(double ul, double ur, double UF) { return 0.5 * (UF * (ur + ul) - fabs(UF) * (ur - ul)); }
inline double scheme_upwind1(double ucc, double ue1, double uw1, double un1, double us1, double ut1, double ub1,
                             double JUE, double JUW, double JVN, double JVS, double JWT, double JWB, double jac) {
    double adv = 0.0;
    adv += upwind_flux1(ucc, ue1, JUE);
    adv -= upwind_flux1(uw1, ucc, JUW);
    adv += upwind_flux1(ucc, un1, JVN);
    adv -= upwind_flux1(us1, ucc, JVS);
    adv += upwind_flux1(ucc, ut1, JWT);
    adv -= upwind_flux1(ub1, ucc, JWB);
    adv /= jac;
    return adv;
}

/* src/FalmCFDScheme.h:33-66 */
inline double scheme_quick(double ucc, double ue1, double ue2, double uw1, double uw2, double un1, double un2,
                           double us1, double us2, double ut1, double ut2, double ub1, double ub2,
                           double JUE, double JUW, double JVN, double JVS, double JWT, double JWB, double jac) {
    double adv = 0.;
    adv += JUE*(- ue2 + 9*ue1 + 9*ucc - uw1);
    adv += fabs(JUE)*(ue2 - 3*ue1 + 3*ucc - uw1);
    adv -= JUW*(- ue1 + 9*ucc + 9*uw1 - uw2);
    adv -= fabs(JUW)*(ue1 - 3*ucc + 3*uw1 - uw2);
    adv += JVN*(- un2 + 9*un1 + 9*ucc - us1);
    adv += fabs(JVN)*(un2 - 3*un1 + 3*ucc - us1);
    adv -= JVS*(- un1 + 9*ucc + 9*us1 - us2);
    adv -= fabs(JVS)*(un1 - 3*ucc + 3*us1 - us2);
    adv += JWT*(- ut2 + 9*ut1 + 9*ucc - ub1);
    adv += fabs(JWT)*(ut2 - 3*ut1 + 3*ucc - ub1);
    adv -= JWB*(- ut1 + 9*ucc + 9*ub1 - ub2);
    adv -= fabs(JWB)*(ut1 - 3*ucc + 3*ub1 - ub2);
    adv /= (16*jac);
    return adv;
}

/* src/FalmCFDScheme.h:68-165: Upwind3 (alpha 1/24), UTOPIA (1/12), KK (1/4) share one form */
inline double scheme_4th(double alpha, double ucc, double ue1, double ue2, double uw1, double uw2, double un1, double un2,
                         double us1, double us2, double ut1, double ut2, double ub1, double ub2,
                         double Uabs, double Vabs, double Wabs,
                         double JUE, double JUW, double JVN, double JVS, double JWT, double JWB, double jac) {
    double adv = 0.0, UDL, UDR, UD4;
    UDL = JUE*(- ue2 + 27*ue1 - 27*ucc + uw1)/24.;
    UDR = JUW*(- ue1 + 27*ucc - 27*uw1 + uw2)/24.;
    UD4 = Uabs*(ue2 - 4*ue1 + 6*ucc - 4*uw1 + uw2)*alpha;
    adv += .5*(UDL + UDR)/jac + UD4;
    UDL = JVN*(- un2 + 27*un1 - 27*ucc + us1)/24.;
    UDR = JVS*(- un1 + 27*ucc - 27*us1 + us2)/24.;
    UD4 = Vabs*(un2 - 4*un1 + 6*ucc - 4*us1 + us2)*alpha;
    adv += .5*(UDL + UDR)/jac + UD4;
    UDL = JWT*(- ut2 + 27*ut1 - 27*ucc + ub1)/24.;
    UDR = JWB*(- ut1 + 27*ucc - 27*ub1 + ub2)/24.;
    UD4 = Wabs*(ut2 - 4*ut1 + 6*ucc - 4*ub1 + ub2)*alpha;
    adv += .5*(UDL + UDR)/jac + UD4;
    return adv;
}

/* src/FalmCFDScheme.h:167-191 */
inline double diffusion(double ReI, double ucc, double ue1, double uw1, double un1, double us1, double ut1, double ub1,
                        double nutcc, double nute1, double nutw1, double nutn1, double nuts1, double nutt1, double nutb1,
                        double gxcc, double gxe1, double gxw1, double gycc, double gyn1, double gys1,
                        double gzcc, double gzt1, double gzb1, double jac) {
    double vis = 0.0;
    vis += (gxcc + gxe1) * (ReI + 0.5 * (nutcc + nute1)) * (ue1 - ucc);
    vis -= (gxcc + gxw1) * (ReI + 0.5 * (nutcc + nutw1)) * (ucc - uw1);
    vis += (gycc + gyn1) * (ReI + 0.5 * (nutcc + nutn1)) * (un1 - ucc);
    vis -= (gycc + gys1) * (ReI + 0.5 * (nutcc + nuts1)) * (ucc - us1);
    vis += (gzcc + gzt1) * (ReI + 0.5 * (nutcc + nutt1)) * (ut1 - ucc);
    vis -= (gzcc + gzb1) * (ReI + 0.5 * (nutcc + nutb1)) * (ucc - ub1);
    vis /= (2 * jac);
    return vis;
}

/* deterministic interior sum: per-k partial sums, combined in k order */
template <typename F>
double interior_sum(const Box &b, F f) {
    int nk = b.sz - 2 * b.gc;
    std::vector<double> part(nk > 0 ? nk : 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int kk = 0; kk < nk; kk++) {
        int k = kk + b.gc;
        double s = 0.0;
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) s += f(b.id(i, j, k));
        part[kk] = s;
    }
    double s = 0.0;
    for (int kk = 0; kk < nk; kk++) s += part[kk];
    return s;
}

/* src/falmath.h:384-410 */
void frame_rotation(const double *x, const double *angle, int type, double *out) {
    double X = x[0], Y = x[1], Z = x[2];
    if (type == 1) {
        double C = cos(angle[0]), S = sin(angle[0]);
        out[0] = X; out[1] = C*Y + S*Z; out[2] = - S*Y + C*Z;
    } else if (type == 2) {
        double C = cos(angle[1]), S = sin(angle[1]);
        out[0] = C*X - S*Z; out[1] = Y; out[2] = S*X + C*Z;
    } else if (type == 3) {
        double C = cos(angle[2]), S = sin(angle[2]);
        out[0] = C*X + S*Y; out[1] = - S*X + C*Y; out[2] = Z;
    } else {
        out[0] = X; out[1] = Y; out[2] = Z;
    }
}

/* src/falmath.h:412-460 */
void frame_rotation_dt(const double *x, const double *v, const double *angle, const double *omega, int type, double *out) {
    double X = x[0], Y = x[1], Z = x[2], U = v[0], V = v[1], W = v[2];
    if (type == 1) {
        double C = cos(angle[0]), S = sin(angle[0]), O = omega[0];
        out[0] = 0. + U;
        out[1] = O*(- S*Y + C*Z) + (C*V + S*W);
        out[2] = O*(- C*Y - S*Z) + (- S*V + C*W);
    } else if (type == 2) {
        double C = cos(angle[1]), S = sin(angle[1]), O = omega[1];
        out[0] = O*(- S*X - C*Z) + (C*U - S*W);
        out[1] = 0. + V;
        out[2] = O*(  C*X - S*Z) + (S*U + C*W);
    } else if (type == 3) {
        double C = cos(angle[2]), S = sin(angle[2]), O = omega[2];
        out[0] = O*(-S*X + C*Y) + (C*U + S*V);
        out[1] = O*(-C*X - S*Y) + (- S*U + C*V);
        out[2] = 0. + W;
    } else {
        out[0] = U; out[1] = V; out[2] = W;
    }
}

/* src/alm/almDevCall.cu:12-26 */
int find_index(const double *seq, double value, int size) {
    if (value < seq[0]) return -1;
    if (value >= seq[size - 1]) return size - 1;
    for (int i = 0; i < size - 1; i++)
        if (seq[i] <= value && value < seq[i + 1]) return i;
    return size - 1;
}

/* src/alm/almDevCall.cu:28-41 */
double trilinear(double xd, double yd, double zd, double c0, double c1, double c2, double c3,
                 double c4, double c5, double c6, double c7) {
    double c01 = c0*(1. - xd) + c1*xd;
    double c23 = c2*(1. - xd) + c3*xd;
    double c45 = c4*(1. - xd) + c5*xd;
    double c67 = c6*(1. - xd) + c7*xd;
    double c0123 = c01*(1. - yd) + c23*yd;
    double c4567 = c45*(1. - yd) + c67*yd;
    return c0123*(1. - zd) + c4567*zd;
}

inline int isign(double a) { return (a > 0) - (a < 0); }

} // namespace

extern "C" {

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* src/falm.h:383-404: ja = hx*hy*hz, g = ja*kx*kx, kx = 1/h */
void oracle_metrics(const or_case *c, double *kx, double *g, double *ja) {
    Box b(c);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < b.sz; k++)
        for (int j = 0; j < b.sy; j++)
            for (int i = 0; i < b.sx; i++) {
                long idx = b.id(i, j, k);
                double px = c->hx[i], py = c->hy[j], pz = c->hz[k];
                double volume = px * py * pz;
                double dx = 1.0 / px, dy = 1.0 / py, dz = 1.0 / pz;
                ja[idx] = volume;
                g[idx] = volume * dx * dx;
                g[idx + b.n] = volume * dy * dy;
                g[idx + 2 * b.n] = volume * dz * dz;
                kx[idx] = dx; kx[idx + b.n] = dy; kx[idx + 2 * b.n] = dz;
            }
}

/* app/nedo/main.cpp:25-100 (channel: the x+ face keeps its east coefficient,
 * :55) and app/lid3d/main.cpp:22-92 (cavity: Neumann on every face); then
 * FalmMV::MaxDiag (src/MV.h:67-76) and ScaleMatrix by 1/maxdiag
 * (src/dev/MVDevCall.cu:506-522).  Columns c,w,e,s,n,b,t. */
double oracle_poisson_matrix(const or_case *c, const double *g, const double *ja, double *A) {
    Box b(c);
    memset(A, 0, sizeof(double) * 7 * b.n);
    int gc = b.gc;
    double maxdiag = 0.0;
    for (int k = gc; k < b.sz - gc; k++)
        for (int j = gc; j < b.sy - gc; j++)
            for (int i = gc; i < b.sx - gc; i++) {
                double ac = 0, ae = 0, aw = 0, an = 0, as = 0, at = 0, ab = 0;
                long cc = b.id(i, j, k);
                double gxcc = g[cc], gxe1 = g[b.id(i + 1, j, k)], gxw1 = g[b.id(i - 1, j, k)];
                double gycc = g[cc + b.n], gyn1 = g[b.id(i, j + 1, k) + b.n], gys1 = g[b.id(i, j - 1, k) + b.n];
                double gzcc = g[cc + 2 * b.n], gzt1 = g[b.id(i, j, k + 1) + 2 * b.n], gzb1 = g[b.id(i, j, k - 1) + 2 * b.n];
                double jacob = ja[cc], coef;
                coef = 0.5 * (gxcc + gxe1) / jacob;
                int east_limit = (c->bc == OR_BC_CHANNEL) ? b.sx - gc : b.sx - gc - 1;
                if (i < east_limit) { ac -= coef; ae = coef; }
                coef = 0.5 * (gxcc + gxw1) / jacob;
                if (i > gc) { ac -= coef; aw = coef; }
                coef = 0.5 * (gycc + gyn1) / jacob;
                if (j < b.sy - gc - 1) { ac -= coef; an = coef; }
                coef = 0.5 * (gycc + gys1) / jacob;
                if (j > gc) { ac -= coef; as = coef; }
                coef = 0.5 * (gzcc + gzt1) / jacob;
                if (k < b.sz - gc - 1) { ac -= coef; at = coef; }
                coef = 0.5 * (gzcc + gzb1) / jacob;
                if (k > gc) { ac -= coef; ab = coef; }
                A[cc] = ac; A[cc + b.n] = aw; A[cc + 2 * b.n] = ae; A[cc + 3 * b.n] = as;
                A[cc + 4 * b.n] = an; A[cc + 5 * b.n] = ab; A[cc + 6 * b.n] = at;
                if (fabs(ac) > maxdiag) maxdiag = fabs(ac);
            }
    double scale = 1.0 / maxdiag;
    for (long n = 0; n < 7 * b.n; n++) A[n] *= scale;
    return maxdiag;
}

/* src/dev/FalmCFDDevCall.cu:10-301 over the interior map, race-free call
 * convention (un and u are the previous velocity, ua is a separate output). */
void oracle_pseudo_u(const or_case *c, const double *un, const double *u, const double *uu,
                     double *ua, const double *nut, const double *kx, const double *g,
                     const double *ja, const double *ff) {
    Box b(c);
    const long N = b.n;
    const double ReI = 1.0 / c->Re, dt = c->dt;
    const int adv_type = c->adv;
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k);
                long e1 = b.id(i + 1, j, k), w1 = b.id(i - 1, j, k), n1 = b.id(i, j + 1, k), s1 = b.id(i, j - 1, k);
                long t1 = b.id(i, j, k + 1), b1 = b.id(i, j, k - 1);
                long e2 = b.id(i + 2, j, k), w2 = b.id(i - 2, j, k), n2 = b.id(i, j + 2, k), s2 = b.id(i, j - 2, k);
                long t2 = b.id(i, j, k + 2), b2 = b.id(i, j, k - 2);
                double Uabs = fabs(u[cc] * kx[cc]);
                double Vabs = fabs(u[cc + N] * kx[cc + N]);
                double Wabs = fabs(u[cc + 2 * N] * kx[cc + 2 * N]);
                double UE = uu[cc], UW = uu[w1], VN = uu[cc + N], VS = uu[s1 + N], WT = uu[cc + 2 * N], WB = uu[b1 + 2 * N];
                double nutcc = nut[cc], nute1 = nut[e1], nutw1 = nut[w1], nutn1 = nut[n1], nuts1 = nut[s1], nutt1 = nut[t1], nutb1 = nut[b1];
                double gxcc = g[cc], gxe1 = g[e1], gxw1 = g[w1];
                double gycc = g[cc + N], gyn1 = g[n1 + N], gys1 = g[s1 + N];
                double gzcc = g[cc + 2 * N], gzt1 = g[t1 + 2 * N], gzb1 = g[b1 + 2 * N];
                double jacob = ja[cc];
                for (int d = 0; d < 3; d++) {
                    const double *ud = u + d * N;
                    double ucc = ud[cc];
                    double ue1 = ud[e1], uw1 = ud[w1], un1 = ud[n1], us1 = ud[s1], ut1 = ud[t1], ub1 = ud[b1];
                    double ue2 = ud[e2], uw2 = ud[w2], un2 = ud[n2], us2 = ud[s2], ut2 = ud[t2], ub2 = ud[b2];
                    double adv;
                    if (adv_type == OR_ADV_UPWIND3)
                        adv = scheme_4th(1. / 24., ucc, ue1, ue2, uw1, uw2, un1, un2, us1, us2, ut1, ut2, ub1, ub2,
                                         Uabs, Vabs, Wabs, UE, UW, VN, VS, WT, WB, jacob);
                    else if (adv_type == OR_ADV_QUICK)
                        adv = scheme_quick(ucc, ue1, ue2, uw1, uw2, un1, un2, us1, us2, ut1, ut2, ub1, ub2,
                                           UE, UW, VN, VS, WT, WB, jacob);
                    else if (adv_type == OR_ADV_UTOPIA)
                        adv = scheme_4th(1. / 12., ucc, ue1, ue2, uw1, uw2, un1, un2, us1, us2, ut1, ut2, ub1, ub2,
                                         Uabs, Vabs, Wabs, UE, UW, VN, VS, WT, WB, jacob);
                    else if (adv_type == OR_ADV_KK)
                        adv = scheme_4th(1. / 4., ucc, ue1, ue2, uw1, uw2, un1, un2, us1, us2, ut1, ut2, ub1, ub2,
                                         Uabs, Vabs, Wabs, UE, UW, VN, VS, WT, WB, jacob);
                    else
                        adv = scheme_upwind1(ucc, ue1, uw1, un1, us1, ut1, ub1, UE, UW, VN, VS, WT, WB, jacob);
                    double vis = diffusion(ReI, ucc, ue1, uw1, un1, us1, ut1, ub1,
                                           nutcc, nute1, nutw1, nutn1, nuts1, nutt1, nutb1,
                                           gxcc, gxe1, gxw1, gycc, gyn1, gys1, gzcc, gzt1, gzb1, jacob);
                    ua[cc + d * N] = un[cc + d * N] + dt * (- adv + vis + ff[cc + d * N]);
                }
            }
}

/* src/FalmCFD.cpp:69-129: UtoCU (src/dev/FalmCFDDevCall.cu:303-325) on
 * Region(shape, gc-1), then InterpolateCU (:327-349) on the face map
 * (interior shape + 1, offset - 1). */
void oracle_utouu(const or_case *c, const double *u, double *uu, const double *kx, const double *ja) {
    Box b(c);
    const long N = b.n;
    std::vector<double> uc(3 * N, 0.0);
    int lo = b.gc - 1;
#pragma omp parallel for schedule(static)
    for (int k = lo; k < b.sz - lo; k++)
        for (int j = lo; j < b.sy - lo; j++)
            for (int i = lo; i < b.sx - lo; i++) {
                long idx = b.id(i, j, k);
                double jacob = ja[idx];
                uc[idx] = jacob * kx[idx] * u[idx];
                uc[idx + N] = jacob * kx[idx + N] * u[idx + N];
                uc[idx + 2 * N] = jacob * kx[idx + 2 * N] * u[idx + 2 * N];
            }
#pragma omp parallel for schedule(static)
    for (int k = lo; k < b.sz - b.gc; k++)
        for (int j = lo; j < b.sy - b.gc; j++)
            for (int i = lo; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k);
                uu[cc] = 0.5 * (uc[cc] + uc[b.id(i + 1, j, k)]);
                uu[cc + N] = 0.5 * (uc[cc + N] + uc[b.id(i, j + 1, k) + N]);
                uu[cc + 2 * N] = 0.5 * (uc[cc + 2 * N] + uc[b.id(i, j, k + 1) + 2 * N]);
            }
}

/* src/dev/FalmCFDDevCall.cu:557-581 on the interior map */
void oracle_divergence(const or_case *c, const double *uu, double *div, const double *ja) {
    Box b(c);
    const long N = b.n;
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k);
                double UE = uu[cc], UW = uu[b.id(i - 1, j, k)];
                double VN = uu[cc + N], VS = uu[b.id(i, j - 1, k) + N];
                double WT = uu[cc + 2 * N], WB = uu[b.id(i, j, k - 1) + 2 * N];
                div[cc] = (UE - UW + VN - VS + WT - WB) / ja[cc];
            }
}

/* src/FalmCFD.h:96-109: Divergence, then ScaleMatrix(rhs, 1/(dt*maxdiag)) over the whole array */
void oracle_poisson_rhs(const or_case *c, const double *uu, double *rhs, const double *ja, double maxdiag) {
    Box b(c);
    oracle_divergence(c, uu, rhs, ja);
    double scale = 1.0 / (c->dt * maxdiag);
    for (long n = 0; n < b.n; n++) rhs[n] *= scale;
}

/* src/FalmCFD.cpp:131-185: ProjectPGrid (src/dev/FalmCFDDevCall.cu:351-376) on
 * the interior, ProjectPFace (:378-407) on the face map. */
void oracle_project_p(const or_case *c, double *u, const double *ua, double *uu, const double *uua,
                      const double *p, const double *kx, const double *g) {
    Box b(c);
    const long N = b.n;
    const double dt = c->dt;
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k);
                double dpx = 0.5 * kx[cc] * (p[b.id(i + 1, j, k)] - p[b.id(i - 1, j, k)]);
                double dpy = 0.5 * kx[cc + N] * (p[b.id(i, j + 1, k)] - p[b.id(i, j - 1, k)]);
                double dpz = 0.5 * kx[cc + 2 * N] * (p[b.id(i, j, k + 1)] - p[b.id(i, j, k - 1)]);
                u[cc] = ua[cc] - dt * dpx;
                u[cc + N] = ua[cc + N] - dt * dpy;
                u[cc + 2 * N] = ua[cc + 2 * N] - dt * dpz;
            }
    int lo = b.gc - 1;
#pragma omp parallel for schedule(static)
    for (int k = lo; k < b.sz - b.gc; k++)
        for (int j = lo; j < b.sy - b.gc; j++)
            for (int i = lo; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k), e1 = b.id(i + 1, j, k), n1 = b.id(i, j + 1, k), t1 = b.id(i, j, k + 1);
                double pcc = p[cc];
                double dpx = 0.5 * (g[cc] + g[e1]) * (p[e1] - pcc);
                double dpy = 0.5 * (g[cc + N] + g[n1 + N]) * (p[n1] - pcc);
                double dpz = 0.5 * (g[cc + 2 * N] + g[t1 + 2 * N]) * (p[t1] - pcc);
                uu[cc] = uua[cc] - dt * dpx;
                uu[cc + N] = uua[cc + N] - dt * dpy;
                uu[cc + 2 * N] = uua[cc + 2 * N] - dt * dpz;
            }
}

/* src/dev/FalmCFDDevCall.cu:409-476 (Smagorinsky) and :478-555 (CSM) */
void oracle_sgs(const or_case *c, const double *u, double *nut, const double *kx, const double *ja) {
    Box b(c);
    const long N = b.n;
    if (c->sgs == OR_SGS_EMPTY) return;
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k);
                long e1 = b.id(i + 1, j, k), w1 = b.id(i - 1, j, k), n1 = b.id(i, j + 1, k), s1 = b.id(i, j - 1, k);
                long t1 = b.id(i, j, k + 1), b1 = b.id(i, j, k - 1);
                double kxx = kx[cc], kxy = kx[cc + N], kxz = kx[cc + 2 * N];
                double d[3][3];
                for (int m = 0; m < 3; m++) {
                    const double *um = u + m * N;
                    d[m][0] = 0.5 * kxx * (um[e1] - um[w1]);
                    d[m][1] = 0.5 * kxy * (um[n1] - um[s1]);
                    d[m][2] = 0.5 * kxz * (um[t1] - um[b1]);
                }
                double dux = d[0][0], duy = d[0][1], duz = d[0][2];
                double dvx = d[1][0], dvy = d[1][1], dvz = d[1][2];
                double dwx = d[2][0], dwy = d[2][1], dwz = d[2][2];
                double d1 = 2 * SQ(dux), d2 = 2 * SQ(dvy), d3 = 2 * SQ(dwz);
                double d4 = SQ(duy + dvx), d5 = SQ(dvz + dwy), d6 = SQ(duz + dwx);
                double Du = sqrt(d1 + d2 + d3 + d4 + d5 + d6);
                double De = cbrt(ja[cc]);
                if (c->sgs == OR_SGS_SMAGORINSKY) {
                    double lc = c->Cs * De;
                    nut[cc] = SQ(lc) * Du;
                } else {
                    double e = SQ(dux) + SQ(duy) + SQ(duz);
                    e += SQ(dvx) + SQ(dvy) + SQ(dvz);
                    e += SQ(dwx) + SQ(dwy) + SQ(dwz);
                    e *= 0.5;
                    double q = dux * dux + duy * dvx + duz * dwx;
                    q += dvx * duy + dvy * dvy + dvz * dwy;
                    q += dwx * duz + dwy * dvz + dwz * dwz;
                    q *= -0.5;
                    double fcs = (q + copysign(1e-9, q)) / (e + copysign(1e-9, e));
                    double CCsm = sqrt(fcs * fcs * fcs) * (1 - fcs) / 22.0;
                    nut[cc] = CCsm * SQ(De) * Du;
                }
            }
}

/* src/dev/MVDevCall.cu:152-183 on the interior map */
void oracle_mv(const or_case *c, const double *A, const double *x, double *ax) {
    Box b(c);
    const long N = b.n;
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k);
                double ac = A[cc], aw = A[cc + N], ae = A[cc + 2 * N], as = A[cc + 3 * N];
                double an = A[cc + 4 * N], ab = A[cc + 5 * N], at = A[cc + 6 * N];
                double xc = x[cc], xe = x[b.id(i + 1, j, k)], xw = x[b.id(i - 1, j, k)];
                double xn = x[b.id(i, j + 1, k)], xs = x[b.id(i, j - 1, k)];
                double xt = x[b.id(i, j, k + 1)], xb = x[b.id(i, j, k - 1)];
                ax[cc] = ac * xc + ae * xe + aw * xw + an * xn + as * xs + at * xt + ab * xb;
            }
}

/* src/dev/MVDevCall.cu:57-116 (interior dot) */
double oracle_dot(const or_case *c, const double *a, const double *bb) {
    Box b(c);
    return interior_sum(b, [&](long idx) { return a[idx] * bb[idx]; });
}

/* src/dev/MVDevCall.cu:118-179 (interior sum of squares over all columns) */
double oracle_normsq(const or_case *c, const double *a, int ncol) {
    Box b(c);
    return interior_sum(b, [&](long idx) {
        double t = 0.0;
        for (int d = 0; d < ncol; d++) t += a[idx + d * b.n] * a[idx + d * b.n];
        return t;
    });
}

/* src/dev/FalmEqDevCall.cu:54-85 */
void oracle_res(const or_case *c, const double *A, const double *x, const double *bvec, double *r) {
    Box b(c);
    const long N = b.n;
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                long cc = b.id(i, j, k);
                double ac = A[cc], aw = A[cc + N], ae = A[cc + 2 * N], as = A[cc + 3 * N];
                double an = A[cc + 4 * N], ab = A[cc + 5 * N], at = A[cc + 6 * N];
                double xc = x[cc], xe = x[b.id(i + 1, j, k)], xw = x[b.id(i - 1, j, k)];
                double xn = x[b.id(i, j + 1, k)], xs = x[b.id(i, j - 1, k)];
                double xt = x[b.id(i, j, k + 1)], xb = x[b.id(i, j, k - 1)];
                r[cc] = bvec[cc] - (ac * xc + ae * xe + aw * xw + an * xn + as * xs + at * xt + ab * xb);
            }
}

/* src/dev/FalmEqDevCall.cu:175-211: one red-black half sweep, colour
 * (i+j+k+sum(offset))%2 with a single rank (offset 0) */
void oracle_sor_sweep(const or_case *c, const double *A, double *x, const double *bvec, double omega, int color) {
    Box b(c);
    const long N = b.n;
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                if ((i + j + k) % 2 != color) continue;
                long cc = b.id(i, j, k);
                double ac = A[cc], aw = A[cc + N], ae = A[cc + 2 * N], as = A[cc + 3 * N];
                double an = A[cc + 4 * N], ab = A[cc + 5 * N], at = A[cc + 6 * N];
                double xc = x[cc], xe = x[b.id(i + 1, j, k)], xw = x[b.id(i - 1, j, k)];
                double xn = x[b.id(i, j + 1, k)], xs = x[b.id(i, j - 1, k)];
                double xt = x[b.id(i, j, k + 1)], xb = x[b.id(i, j, k - 1)];
                double cc_ = (bvec[cc] - (ac * xc + ae * xe + aw * xw + an * xn + as * xs + at * xt + ab * xb)) / ac;
                x[cc] = xc + omega * cc_;
            }
}

/* src/FalmEq.cpp:305-410 (PBiCGStab) with SORPC (:242-303) or JacobiPC
 * (:129-171; Jacobi sweep src/dev/FalmEqDevCall.cu:101-132) as preconditioner */
void oracle_pbicgstab(const or_case *c, const double *A, double *x, const double *bvec, double *r,
                      int *it_out, double *err_out) {
    Box b(c);
    const long N = b.n;
    const double gsize = (double)(b.sx - 2 * b.gc) * (b.sy - 2 * b.gc) * (b.sz - 2 * b.gc);
    std::vector<double> rr(N), p(N, 0.0), q(N, 0.0), s(N, 0.0), pp(N), ss(N), t(N, 0.0), xp(N);
    auto precondition = [&](double *z, const double *rhs) {
        if (c->pc_type == OR_PC_SOR) {
            for (int it = 0; it < c->pc_maxit; it++) {
                oracle_sor_sweep(c, A, z, rhs, c->pc_relax, 0);
                oracle_sor_sweep(c, A, z, rhs, c->pc_relax, 1);
            }
        } else if (c->pc_type == OR_PC_JACOBI) {
            for (int it = 0; it < c->pc_maxit; it++) {
                memcpy(xp.data(), z, sizeof(double) * N);
#pragma omp parallel for schedule(static)
                for (int k = b.gc; k < b.sz - b.gc; k++)
                    for (int j = b.gc; j < b.sy - b.gc; j++)
                        for (int i = b.gc; i < b.sx - b.gc; i++) {
                            long cc = b.id(i, j, k);
                            double ac = A[cc], aw = A[cc + N], ae = A[cc + 2 * N], as = A[cc + 3 * N];
                            double an = A[cc + 4 * N], ab = A[cc + 5 * N], at = A[cc + 6 * N];
                            const double *v = xp.data();
                            double xc = v[cc], xe = v[b.id(i + 1, j, k)], xw = v[b.id(i - 1, j, k)];
                            double xn = v[b.id(i, j + 1, k)], xs = v[b.id(i, j - 1, k)];
                            double xt = v[b.id(i, j, k + 1)], xb = v[b.id(i, j, k - 1)];
                            z[cc] = xc + (rhs[cc] - (ac * xc + ae * xe + aw * xw + an * xn + as * xs + at * xt + ab * xb)) / ac;
                        }
            }
        } else {
            /* no preconditioner: the reference then leaves pp = 0 (FalmEq.h:70-76);
               we keep that behaviour */
        }
    };
    oracle_res(c, A, x, bvec, r);
    double err = sqrt(oracle_normsq(c, r, 1)) / gsize;
    memcpy(rr.data(), r, sizeof(double) * N);
    double rrho = 1.0, alpha = 0.0, omega = 1.0, rho, beta;
    int it = 0;
    do {
        rho = oracle_dot(c, r, rr.data());
        if (fabs(rho) < FLT_MIN) { err = rho; break; }
        if (it == 0) {
            memcpy(p.data(), r, sizeof(double) * N);
        } else {
            beta = (rho * alpha) / (rrho * omega);
            interior_sum(b, [&](long idx) { p[idx] = r[idx] + beta * (p[idx] - omega * q[idx]); return 0.0; });
        }
        std::fill(pp.begin(), pp.end(), 0.0);
        precondition(pp.data(), p.data());
        oracle_mv(c, A, pp.data(), q.data());
        alpha = rho / oracle_dot(c, rr.data(), q.data());
        interior_sum(b, [&](long idx) { s[idx] = r[idx] - alpha * q[idx]; return 0.0; });
        std::fill(ss.begin(), ss.end(), 0.0);
        precondition(ss.data(), s.data());
        oracle_mv(c, A, ss.data(), t.data());
        omega = oracle_dot(c, t.data(), s.data()) / oracle_dot(c, t.data(), t.data());
        interior_sum(b, [&](long idx) { x[idx] += alpha * pp[idx] + omega * ss[idx]; return 0.0; });
        interior_sum(b, [&](long idx) { r[idx] = s[idx] - omega * t[idx]; return 0.0; });
        rrho = rho;
        err = sqrt(oracle_normsq(c, r, 1)) / gsize;
        it++;
    } while (it < c->ls_maxit && err > c->ls_tol);
    *it_out = it;
    *err_out = err;
}

/* The plain solvers of FalmEq::Solve: src/FalmEq.cpp:80-127 (Jacobi: xp = x
 * including ghosts, one sweep x = xp + (b - A xp)/ac as
 * src/dev/FalmEqDevCall.cu:101-132) and :173-240 (SOR: the Black half sweep,
 * then the Red one, with the solver's relaxation factor).  After each
 * iteration r = b - A x and err = ||r||_2 / N; the loop runs while
 * it < maxit && err > tol. */
void oracle_plain_solve(const or_case *c, int ls_type, double relax, const double *A, double *x,
                        const double *bvec, double *r, int *it_out, double *err_out) {
    Box b(c);
    const long N = b.n;
    const double gsize = (double)(b.sx - 2 * b.gc) * (b.sy - 2 * b.gc) * (b.sz - 2 * b.gc);
    std::vector<double> xp(N);
    int it = 0;
    double err = 0.0;
    do {
        if (ls_type == OR_PC_JACOBI) {
            memcpy(xp.data(), x, sizeof(double) * N);
            const double *v = xp.data();
#pragma omp parallel for schedule(static)
            for (int k = b.gc; k < b.sz - b.gc; k++)
                for (int j = b.gc; j < b.sy - b.gc; j++)
                    for (int i = b.gc; i < b.sx - b.gc; i++) {
                        long cc = b.id(i, j, k);
                        double ac = A[cc], aw = A[cc + N], ae = A[cc + 2 * N], as = A[cc + 3 * N];
                        double an = A[cc + 4 * N], ab = A[cc + 5 * N], at = A[cc + 6 * N];
                        double xc = v[cc], xe = v[b.id(i + 1, j, k)], xw = v[b.id(i - 1, j, k)];
                        double xn = v[b.id(i, j + 1, k)], xs = v[b.id(i, j - 1, k)];
                        double xt = v[b.id(i, j, k + 1)], xb = v[b.id(i, j, k - 1)];
                        x[cc] = xc + (bvec[cc] - (ac * xc + ae * xe + aw * xw + an * xn + as * xs + at * xt + ab * xb)) / ac;
                    }
        } else {
            oracle_sor_sweep(c, A, x, bvec, relax, 0);
            oracle_sor_sweep(c, A, x, bvec, relax, 1);
        }
        oracle_res(c, A, x, bvec, r);
        err = sqrt(oracle_normsq(c, r, 1)) / gsize;
        it++;
    } while (it < c->ls_maxit && err > c->ls_tol);
    *it_out = it;
    *err_out = err;
}

/* velocity ghost fill.  Channel: app/nedo/bcdevcall.cu:8-151 (inlet value
 * u_inlet as app/windtunnel/bcdevcall.cu:8-22, optionally perturbed by the
 * seeded inflow box); cavity: app/lid3d/bcdev.cu:11-105 (lid on y+). */
void oracle_ubc(const or_case *c, double *u, const double *uprev, double t) {
    Box b(c);
    const long N = b.n;
    const int gc = b.gc, sx = b.sx, sy = b.sy, sz = b.sz;
    if (c->bc == OR_BC_CHANNEL) {
        int nyi = sy - 2 * gc, nzi = sz - 2 * gc;
        double sfrac = 0.0; int s0 = 0, s1 = 0;
        if (c->inflow_box) {
            double xs = c->u_inlet * t / c->inflow_dx;
            double fl = floor(xs);
            sfrac = xs - fl;
            long s = (long)fl % c->inflow_nb;
            if (s < 0) s += c->inflow_nb;
            s0 = (int)s; s1 = (s0 + 1) % c->inflow_nb;
        }
        for (int k = gc; k < sz - gc; k++)
            for (int j = gc; j < sy - gc; j++) {
                /* inlet x- */
                double ub[3] = {c->u_inlet, 0.0, 0.0};
                if (c->inflow_box) {
                    long plane = (long)nyi * nzi;
                    long jk = (j - gc) + (long)(k - gc) * nyi;
                    for (int d = 0; d < 3; d++) {
                        const double *bx = c->inflow_box + (long)d * c->inflow_nb * plane;
                        ub[d] += (1.0 - sfrac) * bx[s0 * plane + jk] + sfrac * bx[s1 * plane + jk];
                    }
                }
                int i = gc - 1;
                for (int d = 0; d < 3; d++) { u[b.id(i, j, k) + d * N] = ub[d]; u[b.id(i - 1, j, k) + d * N] = ub[d]; }
                /* convective outlet x+ */
                i = sx - gc;
                long o1 = b.id(i, j, k), o2 = b.id(i + 1, j, k), i1 = b.id(i - 1, j, k), i2 = b.id(i - 2, j, k);
                double dxi = 1.0 / (c->x[i] - c->x[i - 1]);
                for (int d = 0; d < 3; d++) {
                    double du = 0.5 * dxi * (3 * uprev[o1 + d * N] - 4 * uprev[i1 + d * N] + uprev[i2 + d * N]);
                    double ubc = uprev[o1 + d * N] - c->dt * du;
                    u[o1 + d * N] = ubc;
                    u[o2 + d * N] = 2 * ubc - u[i1 + d * N];
                }
            }
        for (int k = gc; k < sz - gc; k++)
            for (int i = gc; i < sx - gc; i++) {
                /* slip y- and y+ */
                long o1 = b.id(i, gc - 1, k), o2 = b.id(i, gc - 2, k), i1 = b.id(i, gc, k);
                double ub[3] = {u[i1], 0.0, u[i1 + 2 * N]};
                for (int d = 0; d < 3; d++) { u[o1 + d * N] = ub[d]; u[o2 + d * N] = 2 * ub[d] - u[i1 + d * N]; }
                o1 = b.id(i, sy - gc, k); o2 = b.id(i, sy - gc + 1, k); i1 = b.id(i, sy - gc - 1, k);
                double vb[3] = {u[i1], 0.0, u[i1 + 2 * N]};
                for (int d = 0; d < 3; d++) { u[o1 + d * N] = vb[d]; u[o2 + d * N] = 2 * vb[d] - u[i1 + d * N]; }
            }
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++) {
                /* no-slip z- */
                long o1 = b.id(i, j, gc - 1), o2 = b.id(i, j, gc - 2), i1 = b.id(i, j, gc);
                for (int d = 0; d < 3; d++) { u[o1 + d * N] = 0.0; u[o2 + d * N] = 2 * 0.0 - u[i1 + d * N]; }
                /* slip z+ */
                o1 = b.id(i, j, sz - gc); o2 = b.id(i, j, sz - gc + 1); i1 = b.id(i, j, sz - gc - 1);
                double wb[3] = {u[i1], u[i1 + N], 0.0};
                for (int d = 0; d < 3; d++) { u[o1 + d * N] = wb[d]; u[o2 + d * N] = 2 * wb[d] - u[i1 + d * N]; }
            }
    } else {
        const double lid[3] = {1.0, 0.0, 0.0};
        for (int k = gc; k < sz - gc; k++)
            for (int j = gc; j < sy - gc; j++)
                for (int d = 0; d < 3; d++) {
                    double *ud = u + d * N;
                    ud[b.id(gc - 1, j, k)] = 2 * 0.0 - ud[b.id(gc, j, k)];
                    ud[b.id(gc - 2, j, k)] = 2 * 0.0 - ud[b.id(gc + 1, j, k)];
                    ud[b.id(sx - gc, j, k)] = 2 * 0.0 - ud[b.id(sx - gc - 1, j, k)];
                    ud[b.id(sx - gc + 1, j, k)] = 2 * 0.0 - ud[b.id(sx - gc - 2, j, k)];
                }
        for (int k = gc; k < sz - gc; k++)
            for (int i = gc; i < sx - gc; i++)
                for (int d = 0; d < 3; d++) {
                    double *ud = u + d * N;
                    ud[b.id(i, gc - 1, k)] = 2 * 0.0 - ud[b.id(i, gc, k)];
                    ud[b.id(i, gc - 2, k)] = 2 * 0.0 - ud[b.id(i, gc + 1, k)];
                    ud[b.id(i, sy - gc, k)] = 2 * lid[d] - ud[b.id(i, sy - gc - 1, k)];
                    ud[b.id(i, sy - gc + 1, k)] = 2 * lid[d] - ud[b.id(i, sy - gc - 2, k)];
                }
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++)
                for (int d = 0; d < 3; d++) {
                    double *ud = u + d * N;
                    ud[b.id(i, j, gc - 1)] = 2 * 0.0 - ud[b.id(i, j, gc)];
                    ud[b.id(i, j, gc - 2)] = 2 * 0.0 - ud[b.id(i, j, gc + 1)];
                    ud[b.id(i, j, sz - gc)] = 2 * 0.0 - ud[b.id(i, j, sz - gc - 1)];
                    ud[b.id(i, j, sz - gc + 1)] = 2 * 0.0 - ud[b.id(i, j, sz - gc - 2)];
                }
    }
}

/* pressure ghost fill: app/nedo/bcdevcall.cu:153-211 (Neumann, p = 0 at
 * x+), app/lid3d/bcdev.cu:143-213 (Neumann everywhere) */
void oracle_pbc(const or_case *c, double *p) {
    Box b(c);
    const int gc = b.gc, sx = b.sx, sy = b.sy, sz = b.sz;
    for (int k = gc; k < sz - gc; k++)
        for (int j = gc; j < sy - gc; j++) {
            p[b.id(gc - 1, j, k)] = p[b.id(gc, j, k)];
            p[b.id(sx - gc, j, k)] = (c->bc == OR_BC_CHANNEL) ? 0.0 : p[b.id(sx - gc - 1, j, k)];
        }
    for (int k = gc; k < sz - gc; k++)
        for (int i = gc; i < sx - gc; i++) {
            p[b.id(i, gc - 1, k)] = p[b.id(i, gc, k)];
            p[b.id(i, sy - gc, k)] = p[b.id(i, sy - gc - 1, k)];
        }
    for (int j = gc; j < sy - gc; j++)
        for (int i = gc; i < sx - gc; i++) {
            p[b.id(i, j, gc - 1)] = p[b.id(i, j, gc)];
            p[b.id(i, j, sz - gc)] = p[b.id(i, j, sz - gc - 1)];
        }
}

/* app/lid3d/bcdev.cu:251-322: zero wall-normal face flux (cavity only) */
void oracle_uubc(const or_case *c, double *uu) {
    if (c->bc != OR_BC_CAVITY) return;
    Box b(c);
    const long N = b.n;
    const int gc = b.gc, sx = b.sx, sy = b.sy, sz = b.sz;
    for (int k = gc; k < sz - gc; k++)
        for (int j = gc; j < sy - gc; j++) { uu[b.id(gc - 1, j, k)] = 0; uu[b.id(sx - gc - 1, j, k)] = 0; }
    for (int k = gc; k < sz - gc; k++)
        for (int i = gc; i < sx - gc; i++) { uu[b.id(i, gc - 1, k) + N] = 0; uu[b.id(i, sy - gc - 1, k) + N] = 0; }
    for (int j = gc; j < sy - gc; j++)
        for (int i = gc; i < sx - gc; i++) { uu[b.id(i, j, gc - 1) + 2 * N] = 0; uu[b.id(i, j, sz - gc - 1) + 2 * N] = 0; }
}

/* src/alm/bladeHandler.h:16-104 (AP tables from airfoil stations).  Station
 * polars st_cl/st_cd are row-major [station][attack]; outputs are the APFrame
 * layout (ap + atk*apcount, src/alm/apHandler.h:52-54). */
void oracle_build_aps(int n_station, const double *st_r, const double *st_chord, const double *st_twist,
                      const double *st_cl, const double *st_cd, int n_attack,
                      int apcount, int n_ap_per_blade, double radius, double hub_radius,
                      double *ap_r, double *ap_chord, double *ap_twist, double *ap_cl, double *ap_cd) {
    double dr = (radius - hub_radius) / n_ap_per_blade;
    for (int apid = 0; apid < apcount; apid++) {
        double apr = (apid % n_ap_per_blade + 0.5) * dr + hub_radius;
        double chord, twist;
        int lo = 0; double pw = 0.0; int mode;
        if (apr < st_r[0]) { mode = 0; }
        else if (apr >= st_r[n_station - 1]) { mode = 1; }
        else {
            mode = 2;
            int i;
            for (i = 0; i < n_station - 1; i++)
                if (st_r[i] <= apr && st_r[i + 1] > apr) { pw = (apr - st_r[i]) / (st_r[i + 1] - st_r[i]); break; }
            lo = i;
        }
        for (int a = 0; a < n_attack; a++) {
            double clv, cdv;
            if (mode == 0) { clv = st_cl[a]; cdv = st_cd[a]; }
            else if (mode == 1) { clv = st_cl[(n_station - 1) * n_attack + a]; cdv = st_cd[(n_station - 1) * n_attack + a]; }
            else {
                clv = (1. - pw) * st_cl[lo * n_attack + a] + pw * st_cl[(lo + 1) * n_attack + a];
                cdv = (1. - pw) * st_cd[lo * n_attack + a] + pw * st_cd[(lo + 1) * n_attack + a];
            }
            ap_cl[apid + (long)a * apcount] = clv;
            ap_cd[apid + (long)a * apcount] = cdv;
        }
        if (mode == 0) { chord = st_chord[0]; twist = st_twist[0]; }
        else if (mode == 1) { chord = st_chord[n_station - 1]; twist = st_twist[n_station - 1]; }
        else { chord = (1. - pw) * st_chord[lo] + pw * st_chord[lo + 1]; twist = (1. - pw) * st_twist[lo] + pw * st_twist[lo + 1]; }
        ap_r[apid] = apr; ap_chord[apid] = chord; ap_twist[apid] = twist;
    }
}

/* src/alm/alm.h:66-77 -> almDevCall.cu: UpdateTurbineAngles (:43-61),
 * UpdateAPX (:63-129), CalcAPForce (:131-253), DistributeAPForce (:255-294),
 * CalcTorqueAndThrust (:362-370).  Single rank. */
void oracle_alm(const or_case *c, const double *u, double *ff, double t,
                double *ap_xyz, double *ap_force, double *ap_torque, double *ap_thrust,
                double *turb_torque, double *turb_thrust) {
    Box b(c);
    const long N = b.n;
    const or_alm &a = c->alm;
    const int apcount = a.n_turbine * a.n_blade * a.n_ap_per_blade;
    const int nappt = a.n_ap_per_blade * a.n_blade;
    std::vector<double> angle(3 * a.n_turbine, 0.0), angvel(3 * a.n_turbine, 0.0);
    for (int tid = 0; tid < a.n_turbine; tid++) {
        int at = a.angle_type[tid];
        const double *m = a.motion + 3 * tid;
        if (at) {
            angle[3 * tid + at - 1] = m[0] * sin(m[1] * t + m[2]);
            angvel[3 * tid + at - 1] = m[0] * m[1] * cos(m[1] * t + m[2]);
        }
    }
    std::vector<int> ijk(3 * apcount), inside(apcount);
    const double dr = (a.radius - a.hub_radius) / a.n_ap_per_blade;
    for (int ap = 0; ap < apcount; ap++) {
        int tid = ap / nappt, bid = (ap % nappt) / a.n_ap_per_blade;
        double tip = a.tip_rate[tid];
        double theta = tip * t + (2 * kPi / a.n_blade) * bid;
        double apr = a.ap_r[ap];
        double c1[3] = {a.hub[3 * tid], a.hub[3 * tid + 1] + apr * cos(theta), a.hub[3 * tid + 2] + apr * sin(theta)};
        double nang[3] = {-angle[3 * tid], -angle[3 * tid + 1], -angle[3 * tid + 2]};
        double c0[3];
        frame_rotation(c1, nang, a.angle_type[tid], c0);
        for (int d = 0; d < 3; d++) c0[d] += a.base[3 * tid + d];
        for (int d = 0; d < 3; d++) ap_xyz[3 * ap + d] = c0[d];
        int I = find_index(c->x, c0[0], b.sx), J = find_index(c->y, c0[1], b.sy), K = find_index(c->z, c0[2], b.sz);
        ijk[3 * ap] = I; ijk[3 * ap + 1] = J; ijk[3 * ap + 2] = K;
        inside[ap] = (I >= b.gc - 1 && I < b.sx - b.gc - 1 && J >= b.gc - 1 && J < b.sy - b.gc - 1 &&
                      K >= b.gc - 1 && K < b.sz - b.gc - 1);
        if (!inside[ap]) {
            ap_force[3 * ap] = ap_force[3 * ap + 1] = ap_force[3 * ap + 2] = 0;
            ap_torque[ap] = 0; ap_thrust[ap] = 0;
            continue;
        }
        int i0 = I, i1 = I + 1, j0 = J, j1 = J + 1, k0 = K, k1 = K + 1;
        double xd = fabs(c0[0] - c->x[i0]) / fabs(c->x[i1] - c->x[i0]);
        double yd = fabs(c0[1] - c->y[j0]) / fabs(c->y[j1] - c->y[j0]);
        double zd = fabs(c0[2] - c->z[k0]) / fabs(c->z[k1] - c->z[k0]);
        long id0 = b.id(i0, j0, k0), id1 = b.id(i1, j0, k0), id2 = b.id(i0, j1, k0), id3 = b.id(i1, j1, k0);
        long id4 = b.id(i0, j0, k1), id5 = b.id(i1, j0, k1), id6 = b.id(i0, j1, k1), id7 = b.id(i1, j1, k1);
        double uvw[3];
        for (int d = 0; d < 3; d++) {
            const double *ud = u + d * N;
            uvw[d] = trilinear(xd, yd, zd, ud[id0], ud[id1], ud[id2], ud[id3], ud[id4], ud[id5], ud[id6], ud[id7]);
        }
        double rel[3] = {c0[0] - a.base[3 * tid], c0[1] - a.base[3 * tid + 1], c0[2] - a.base[3 * tid + 2]};
        double uvw_tt[3];
        frame_rotation_dt(rel, uvw, &angle[3 * tid], &angvel[3 * tid], a.angle_type[tid], uvw_tt);
        double ux = uvw_tt[0];
        double ut = tip * apr + uvw_tt[1] * sin(theta) - uvw_tt[2] * cos(theta);
        double urel2 = ux * ux + ut * ut;
        double phi = atan(ux / ut);
        /* src/alm/apHandler.h:121-141 */
        double chord = a.ap_chord[ap], twist = a.ap_twist[ap] + a.pitch;
        double attack = phi * 180. / kPi - twist;
        double clv = 0, cdv = 0;
        if (attack < a.attack[0]) { clv = a.cl[ap]; cdv = a.cd[ap]; }
        else if (attack >= a.attack[a.n_attack - 1]) {
            clv = a.cl[ap + (long)(a.n_attack - 1) * apcount]; cdv = a.cd[ap + (long)(a.n_attack - 1) * apcount];
        } else {
            for (int k = 0; k < a.n_attack - 1; k++)
                if (a.attack[k] <= attack && a.attack[k + 1] > attack) {
                    double pw = (attack - a.attack[k]) / (a.attack[k + 1] - a.attack[k]);
                    clv = (1. - pw) * a.cl[ap + (long)k * apcount] + pw * a.cl[ap + (long)(k + 1) * apcount];
                    cdv = (1. - pw) * a.cd[ap + (long)k * apcount] + pw * a.cd[ap + (long)(k + 1) * apcount];
                    break;
                }
        }
        double fl = .5 * clv * urel2 * chord * dr;
        double fd = .5 * cdv * urel2 * chord * dr;
        double fx = fl * cos(phi) + fd * sin(phi);
        double ft = fl * sin(phi) - fd * sin(phi);
        ft *= isign(tip);
        double f_tt[3] = {-fx, ft * sin(theta), -ft * cos(theta)};
        frame_rotation(f_tt, nang, a.angle_type[tid], ap_force + 3 * ap);
        ap_torque[ap] = fabs(ft) * apr;
        ap_thrust[ap] = fx;
    }
    const double eps = a.euler_eps;
    const double eta = 1. / ((eps * sqrt(kPi)) * (eps * sqrt(kPi)) * (eps * sqrt(kPi)));
#pragma omp parallel for schedule(static)
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                double cx = c->x[i], cy = c->y[j], cz = c->z[k];
                double fx = 0., fy = 0., fz = 0.;
                for (int ap = 0; ap < apcount; ap++) {
                    double rr2 = SQ(cx - ap_xyz[3 * ap]) + SQ(cy - ap_xyz[3 * ap + 1]) + SQ(cz - ap_xyz[3 * ap + 2]);
                    double ex = exp(-rr2 / SQ(eps));
                    fx += ap_force[3 * ap] * eta * ex;
                    fy += ap_force[3 * ap + 1] * eta * ex;
                    fz += ap_force[3 * ap + 2] * eta * ex;
                }
                long cid = b.id(i, j, k);
                ff[cid] = fx; ff[cid + N] = fy; ff[cid + 2 * N] = fz;
            }
    for (int tid = 0; tid < a.n_turbine; tid++) {
        double tq = 0, th = 0;
        for (int k = 0; k < nappt; k++) { tq += ap_torque[tid * nappt + k]; th += ap_thrust[tid * nappt + k]; }
        turb_torque[tid] = tq; turb_thrust[tid] = th;
    }
}

/* app/nedo/main.cpp:150-204 (channel) and app/lid3d/main.cpp:121-168
 * (cavity, uubc after UtoUU), with the race-free pseudo-velocity call
 * FSPseudoU(un=u_prev, u=u_prev, uu, ua=u). */
/* src/rmcp/bladeHandler.h:83-96 (find_position) and :98-107 (interpolate) */
static int rmcp_find(const double *m, double x, int n) {
    if (x < m[0]) return -1;
    if (x >= m[n - 1]) return n - 1;
    for (int i = 0; i < n - 1; i++)
        if (m[i] <= x && m[i + 1] > x) return i;
    return -2;
}
static double rmcp_interp(const double *m, const double *d, double x, int i, int n) {
    if (i < 0) return d[0];
    if (i >= n - 1) return d[n - 1];
    double p = (x - m[i]) / (m[i + 1] - m[i]);
    return (1. - p) * d[i] + p * d[i + 1];
}
/* src/rmcp/bladeHandler.h:109-131 (get_airfoil_params) */
static void rmcp_airfoil(const or_rmcp *r, double rr, double phi, double *chord, double *twist, double *cl, double *cd) {
    const int nr = r->n_station, na = r->n_attack;
    int rid = rmcp_find(r->st_r, rr, nr);
    *chord = rmcp_interp(r->st_r, r->st_chord, rr, rid, nr);
    *twist = rmcp_interp(r->st_r, r->st_twist, rr, rid, nr);
    double attack = phi - *twist;
    int aid = rmcp_find(r->attack, attack, na);
    if (rid < 0) {
        *cl = rmcp_interp(r->attack, r->cl, attack, aid, na);
        *cd = rmcp_interp(r->attack, r->cd, attack, aid, na);
    } else if (rid >= nr - 1) {
        *cl = rmcp_interp(r->attack, r->cl + (long)(nr - 1) * na, attack, aid, na);
        *cd = rmcp_interp(r->attack, r->cd + (long)(nr - 1) * na, attack, aid, na);
    } else {
        double p = (rr - r->st_r[rid]) / (r->st_r[rid + 1] - r->st_r[rid]);
        double cl0 = rmcp_interp(r->attack, r->cl + (long)rid * na, attack, aid, na);
        double cl1 = rmcp_interp(r->attack, r->cl + (long)(rid + 1) * na, attack, aid, na);
        double cd0 = rmcp_interp(r->attack, r->cd + (long)rid * na, attack, aid, na);
        double cd1 = rmcp_interp(r->attack, r->cd + (long)(rid + 1) * na, attack, aid, na);
        *cl = (1. - p) * cl0 + p * cl1;
        *cd = (1. - p) * cd0 + p * cd1;
    }
}

void oracle_rmcp(const or_case *c, const or_rmcp *r, const double *u, double *ff, int *flag, double t,
                 double *torque, double *thrust) {
    Box b(c);
    const long N = b.n;
    const double Pi = 3.14159265358979323846;
    const int Nb = r->n_blade;
    for (int q = 0; q < r->n_turbine; q++) { torque[q] = 0; thrust[q] = 0; }
    for (int k = b.gc; k < b.sz - b.gc; k++)
    for (int j = b.gc; j < b.sy - b.gc; j++)
    for (int i = b.gc; i < b.sx - b.gc; i++) {
        const long id = b.id(i, j, k);
        const double point[3] = {c->x[i], c->y[j], c->z[k]};
        /* the flag: src/rmcp/almDevCall.cu:13-65 */
        int f = 0;
        for (int tid = 0; tid < r->n_turbine; tid++) {
            double d0[3] = {point[0] - r->base[3 * tid], point[1] - r->base[3 * tid + 1], point[2] - r->base[3 * tid + 2]}, d[3];
            frame_rotation(d0, &r->angle[3 * tid], r->angle_type[tid], d);
            for (int a = 0; a < 3; a++) d[a] -= r->hub[3 * tid + a];
            double dx = d[0], dy = d[1], dz = d[2];
            double rr = sqrt(dy * dy + dz * dz);
            double th = atan2(dz, dy);
            if (th < 0) th += 2 * Pi;
            double rt = r->tip_rate[tid] * t;
            for (int bid = 0; bid < Nb; bid++) {
                double rtblade = rt + (bid * 2. / Nb) * Pi;
                double x_ = th - rtblade, thblade = x_ - floor(x_ / (2. * Pi)) * (2. * Pi);
                bool isblade = (rr <= r->radius && rr > r->hub_radius);
                isblade = isblade && (thblade >= (Nb - 1) * Pi / (Nb * 2)) && (thblade <= (Nb + 1) * Pi / (Nb * 2));
                isblade = isblade && (rr <= r->width / (2 * cos(thblade)) || rr <= r->width / (2 * cos(thblade + Pi)));
                isblade = isblade && dx >= 0 && dx < r->thick;
                if (isblade) f = tid + 1;
            }
        }
        if (flag) flag[id] = f;
        /* the force: src/rmcp/almDevCall.cu:144-209 */
        if (f > 0) {
            const int tid = f - 1;
            double xyz0[3] = {point[0] - r->base[3 * tid], point[1] - r->base[3 * tid + 1], point[2] - r->base[3 * tid + 2]}, xyz[3];
            double uvw0[3] = {u[id], u[id + N], u[id + 2 * N]}, uvw[3];
            const double omega0[3] = {0, 0, 0};
            frame_rotation(xyz0, &r->angle[3 * tid], r->angle_type[tid], xyz);
            frame_rotation_dt(xyz, uvw0, &r->angle[3 * tid], omega0, r->angle_type[tid], uvw);
            double dy = xyz[1] - r->hub[3 * tid + 1], dz = xyz[2] - r->hub[3 * tid + 2];
            double th = atan2(dz, dy);
            double rr = sqrt(dy * dy + dz * dz);
            double ux = uvw[0];
            double ut = r->tip_rate[tid] * rr + uvw[1] * sin(th) - uvw[2] * cos(th);
            double urel2 = ux * ux + ut * ut;
            double phi = atan(ux / ut);
            double chord, twist, cl, cd;
            rmcp_airfoil(r, rr, phi * 180. / Pi, &chord, &twist, &cl, &cd);
            double ps = (rr > r->width) ? asin(0.5 * r->width / rr) : 0.5 * Pi / Nb;
            double Cf = 0.5 * chord / (2 * rr * ps * r->thick);
            double ffx = fabs((cl * cos(phi) + cd * sin(phi)) * Cf * urel2);
            double fft = fabs((cl * sin(phi) - cd * cos(phi)) * Cf * urel2);
            double loc[3] = {-ffx, fft * sin(th), -fft * cos(th)}, nang[3], out[3];
            for (int a = 0; a < 3; a++) nang[a] = -r->angle[3 * tid + a];
            frame_rotation(loc, nang, r->angle_type[tid], out);
            ff[id] = out[0]; ff[id + N] = out[1]; ff[id + 2 * N] = out[2];
            torque[tid] += rr * fft;
            thrust[tid] += ffx;
        } else {
            ff[id] = 0; ff[id + N] = 0; ff[id + 2 * N] = 0;
        }
    }
}

void oracle_step(const or_case *c, double *u, double *uu, double *p, double *nut, double *ff,
                 const double *kx, const double *g, const double *ja, const double *A, double maxdiag,
                 double t, or_stats *st) {
    Box b(c);
    const long N = b.n;
    std::vector<double> uprev(u, u + 3 * N), rhs(N, 0.0), res(N, 0.0), div(N, 0.0);
    memset(st, 0, sizeof(*st));
    if (c->alm_on) {
        int apcount = c->alm.n_turbine * c->alm.n_blade * c->alm.n_ap_per_blade;
        std::vector<double> xyz(3 * apcount), f(3 * apcount), tq(apcount), th(apcount);
        oracle_alm(c, u, ff, t, xyz.data(), f.data(), tq.data(), th.data(), st->torque, st->thrust);
    }
    oracle_pseudo_u(c, uprev.data(), uprev.data(), uu, u, nut, kx, g, ja, ff);
    oracle_utouu(c, u, uu, kx, ja);
    oracle_uubc(c, uu);
    oracle_poisson_rhs(c, uu, rhs.data(), ja, maxdiag);
    oracle_pbicgstab(c, A, p, rhs.data(), res.data(), &st->it, &st->err);
    oracle_pbc(c, p);
    oracle_project_p(c, u, u, uu, uu, p, kx, g);
    oracle_ubc(c, u, uprev.data(), t);
    oracle_sgs(c, u, nut, kx, ja);
    oracle_divergence(c, uu, div.data(), ja);
    double nsq = oracle_normsq(c, div.data(), 1);
    st->divnorm = sqrt(nsq) / ((double)(b.sx - 2 * b.gc) * (b.sy - 2 * b.gc) * (b.sz - 2 * b.gc));
}

} // extern "C"

/* ========================================================================
 * Discrete adjoint of oracle_step (FP64).  No reference counterpart: this is
 * the adjoint of this project's own discretisation of the step, used to check
 * the device adjoint.  The Poisson solve is treated as exact (p = A^-1 rhs),
 * so its adjoint is one solve with the transposed operator.  Supported:
 * channel and cavity boundaries, the 4th-order schemes (Upwind3, UTOPIA, KK),
 * Smagorinsky or no SGS model.
 * ======================================================================== */
namespace {

struct ApTape {
    int inside, I, J, K, seg;
    double xd, yd, zd, theta, apr, ux, ut, urel2, phi, attack, clv, cdv, chord, fl, fd, fx, ft, sgn;
    double M[3][3];     /* d uvw_tt / d uvw */
    double nang[3];
    int tid, type;
};

/* recompute the AP state of oracle_alm at time t, keeping what the adjoint needs */
void alm_tape(const or_case *c, const double *u, double t, std::vector<ApTape> &tp, std::vector<double> &xyz,
              std::vector<double> &force) {
    Box b(c);
    const long N = b.n;
    const or_alm &a = c->alm;
    const int apcount = a.n_turbine * a.n_blade * a.n_ap_per_blade;
    const int nappt = a.n_ap_per_blade * a.n_blade;
    tp.assign(apcount, ApTape());
    xyz.assign(3 * apcount, 0.0);
    force.assign(3 * apcount, 0.0);
    std::vector<double> angle(3 * a.n_turbine, 0.0), angvel(3 * a.n_turbine, 0.0);
    for (int tid = 0; tid < a.n_turbine; tid++) {
        int at = a.angle_type[tid];
        const double *m = a.motion + 3 * tid;
        if (at) {
            angle[3 * tid + at - 1] = m[0] * sin(m[1] * t + m[2]);
            angvel[3 * tid + at - 1] = m[0] * m[1] * cos(m[1] * t + m[2]);
        }
    }
    const double dr = (a.radius - a.hub_radius) / a.n_ap_per_blade;
    for (int ap = 0; ap < apcount; ap++) {
        ApTape &T = tp[ap];
        int tid = ap / nappt, bid = (ap % nappt) / a.n_ap_per_blade;
        T.tid = tid; T.type = a.angle_type[tid];
        double tip = a.tip_rate[tid];
        double theta = tip * t + (2 * kPi / a.n_blade) * bid;
        double apr = a.ap_r[ap];
        T.theta = theta; T.apr = apr;
        double c1[3] = {a.hub[3 * tid], a.hub[3 * tid + 1] + apr * cos(theta), a.hub[3 * tid + 2] + apr * sin(theta)};
        double nang[3] = {-angle[3 * tid], -angle[3 * tid + 1], -angle[3 * tid + 2]};
        for (int d = 0; d < 3; d++) T.nang[d] = nang[d];
        double c0[3];
        frame_rotation(c1, nang, a.angle_type[tid], c0);
        for (int d = 0; d < 3; d++) c0[d] += a.base[3 * tid + d];
        for (int d = 0; d < 3; d++) xyz[3 * ap + d] = c0[d];
        int I = find_index(c->x, c0[0], b.sx), J = find_index(c->y, c0[1], b.sy), K = find_index(c->z, c0[2], b.sz);
        T.I = I; T.J = J; T.K = K;
        T.inside = (I >= b.gc - 1 && I < b.sx - b.gc - 1 && J >= b.gc - 1 && J < b.sy - b.gc - 1 &&
                    K >= b.gc - 1 && K < b.sz - b.gc - 1);
        if (!T.inside) continue;
        T.xd = fabs(c0[0] - c->x[I]) / fabs(c->x[I + 1] - c->x[I]);
        T.yd = fabs(c0[1] - c->y[J]) / fabs(c->y[J + 1] - c->y[J]);
        T.zd = fabs(c0[2] - c->z[K]) / fabs(c->z[K + 1] - c->z[K]);
        long id[8] = {b.id(I, J, K), b.id(I + 1, J, K), b.id(I, J + 1, K), b.id(I + 1, J + 1, K),
                      b.id(I, J, K + 1), b.id(I + 1, J, K + 1), b.id(I, J + 1, K + 1), b.id(I + 1, J + 1, K + 1)};
        double uvw[3];
        for (int d = 0; d < 3; d++) {
            const double *ud = u + d * N;
            uvw[d] = trilinear(T.xd, T.yd, T.zd, ud[id[0]], ud[id[1]], ud[id[2]], ud[id[3]], ud[id[4]], ud[id[5]], ud[id[6]], ud[id[7]]);
        }
        double rel[3] = {c0[0] - a.base[3 * tid], c0[1] - a.base[3 * tid + 1], c0[2] - a.base[3 * tid + 2]};
        double tt[3], t0[3], zero[3] = {0, 0, 0};
        frame_rotation_dt(rel, uvw, &angle[3 * tid], &angvel[3 * tid], a.angle_type[tid], tt);
        /* the map uvw -> uvw_tt is affine: its matrix from unit vectors */
        frame_rotation_dt(rel, zero, &angle[3 * tid], &angvel[3 * tid], a.angle_type[tid], t0);
        for (int q = 0; q < 3; q++) {
            double e[3] = {0, 0, 0}, o[3];
            e[q] = 1.0;
            frame_rotation_dt(rel, e, &angle[3 * tid], &angvel[3 * tid], a.angle_type[tid], o);
            for (int d = 0; d < 3; d++) T.M[d][q] = o[d] - t0[d];
        }
        T.ux = tt[0];
        T.ut = tip * apr + tt[1] * sin(theta) - tt[2] * cos(theta);
        T.urel2 = T.ux * T.ux + T.ut * T.ut;
        T.phi = atan(T.ux / T.ut);
        T.chord = a.ap_chord[ap];
        double twist = a.ap_twist[ap] + a.pitch;
        T.attack = T.phi * 180. / kPi - twist;
        T.seg = -1;
        if (T.attack < a.attack[0]) { T.clv = a.cl[ap]; T.cdv = a.cd[ap]; }
        else if (T.attack >= a.attack[a.n_attack - 1]) {
            T.clv = a.cl[ap + (long)(a.n_attack - 1) * apcount]; T.cdv = a.cd[ap + (long)(a.n_attack - 1) * apcount];
        } else {
            for (int k = 0; k < a.n_attack - 1; k++)
                if (a.attack[k] <= T.attack && a.attack[k + 1] > T.attack) {
                    double pw = (T.attack - a.attack[k]) / (a.attack[k + 1] - a.attack[k]);
                    T.clv = (1. - pw) * a.cl[ap + (long)k * apcount] + pw * a.cl[ap + (long)(k + 1) * apcount];
                    T.cdv = (1. - pw) * a.cd[ap + (long)k * apcount] + pw * a.cd[ap + (long)(k + 1) * apcount];
                    T.seg = k;
                    break;
                }
        }
        T.fl = .5 * T.clv * T.urel2 * T.chord * dr;
        T.fd = .5 * T.cdv * T.urel2 * T.chord * dr;
        T.fx = T.fl * cos(T.phi) + T.fd * sin(T.phi);
        T.sgn = isign(tip);
        T.ft = (T.fl * sin(T.phi) - T.fd * sin(T.phi)) * T.sgn;
        double f_tt[3] = {-T.fx, T.ft * sin(theta), -T.ft * cos(theta)};
        frame_rotation(f_tt, nang, a.angle_type[tid], &force[3 * ap]);
    }
}

/* adjoint of alm_tape + projection + the weighted power wP * sum_t tip_t torque_t:
   aff is the adjoint of the projected force field (interior); adds to au and the gradients */
void alm_adjoint(const or_case *c, const std::vector<ApTape> &tp, const std::vector<double> &xyz, const double *aff,
                 double wP, double *au, double *g_pitch, double *g_chord, double *g_twist) {
    Box b(c);
    const long N = b.n;
    const or_alm &a = c->alm;
    const int apcount = (int)tp.size();
    const double dr = (a.radius - a.hub_radius) / a.n_ap_per_blade;
    const double eps = a.euler_eps;
    const double eta = 1. / ((eps * sqrt(kPi)) * (eps * sqrt(kPi)) * (eps * sqrt(kPi)));
    /* adjoint of the projection ff(c) = sum_ap F_ap eta exp(-r^2/eps^2) */
    std::vector<double> aF(3 * apcount, 0.0);
    for (int k = b.gc; k < b.sz - b.gc; k++)
        for (int j = b.gc; j < b.sy - b.gc; j++)
            for (int i = b.gc; i < b.sx - b.gc; i++) {
                long cid = b.id(i, j, k);
                double a0 = aff[cid], a1 = aff[cid + N], a2 = aff[cid + 2 * N];
                if (a0 == 0 && a1 == 0 && a2 == 0) continue;
                for (int ap = 0; ap < apcount; ap++) {
                    double rr2 = SQ(c->x[i] - xyz[3 * ap]) + SQ(c->y[j] - xyz[3 * ap + 1]) + SQ(c->z[k] - xyz[3 * ap + 2]);
                    double w = eta * exp(-rr2 / SQ(eps));
                    aF[3 * ap] += a0 * w; aF[3 * ap + 1] += a1 * w; aF[3 * ap + 2] += a2 * w;
                }
            }
    for (int ap = 0; ap < apcount; ap++) {
        const ApTape &T = tp[ap];
        if (!T.inside) continue;
        /* force = R(nang) f_tt: R is orthogonal, its adjoint is the rotation by -nang */
        double an[3] = {-T.nang[0], -T.nang[1], -T.nang[2]};
        double aftt[3];
        /* transpose of frame_rotation by nang = frame_rotation by -nang (single-axis rotations) */
        frame_rotation(&aF[3 * ap], an, T.type, aftt);
        double afx = -aftt[0];
        double aft = aftt[1] * sin(T.theta) - aftt[2] * cos(T.theta);
        /* objective: wP * tip * |ft| * r */
        aft += wP * a.tip_rate[T.tid] * (double)isign(T.ft) * T.apr;
        double aft0 = aft * T.sgn;                       /* ft = ft0 * sgn */
        double s = sin(T.phi), co = cos(T.phi);
        double afl = afx * co + aft0 * s;
        double afd = afx * s - aft0 * s;
        double aphi = afx * (-T.fl * s + T.fd * co) + aft0 * (T.fl - T.fd) * co;
        double aclv = afl * .5 * T.urel2 * T.chord * dr, acdv = afd * .5 * T.urel2 * T.chord * dr;
        double aurel2 = afl * .5 * T.clv * T.chord * dr + afd * .5 * T.cdv * T.chord * dr;
        double achord = afl * .5 * T.clv * T.urel2 * dr + afd * .5 * T.cdv * T.urel2 * dr;
        double aattack = 0.0;
        if (T.seg >= 0) {
            int k = T.seg;
            double dA = a.attack[k + 1] - a.attack[k];
            aattack = aclv * (a.cl[ap + (long)(k + 1) * apcount] - a.cl[ap + (long)k * apcount]) / dA +
                      acdv * (a.cd[ap + (long)(k + 1) * apcount] - a.cd[ap + (long)k * apcount]) / dA;
        }
        aphi += aattack * 180. / kPi;
        g_twist[ap] += -aattack;
        *g_pitch += -aattack;
        g_chord[ap] += achord;
        /* phi = atan(ux/ut), urel2 = ux^2 + ut^2 */
        double aux = aphi * T.ut / T.urel2 + 2 * T.ux * aurel2;
        double aut = -aphi * T.ux / T.urel2 + 2 * T.ut * aurel2;
        double att[3] = {aux, aut * sin(T.theta), -aut * cos(T.theta)};
        double auvw[3];
        for (int q = 0; q < 3; q++) auvw[q] = T.M[0][q] * att[0] + T.M[1][q] * att[1] + T.M[2][q] * att[2];
        const double xd = T.xd, yd = T.yd, zd = T.zd;
        const double wts[8] = {(1 - xd) * (1 - yd) * (1 - zd), xd * (1 - yd) * (1 - zd), (1 - xd) * yd * (1 - zd), xd * yd * (1 - zd),
                               (1 - xd) * (1 - yd) * zd, xd * (1 - yd) * zd, (1 - xd) * yd * zd, xd * yd * zd};
        const int I = T.I, J = T.J, K = T.K;
        long id[8] = {b.id(I, J, K), b.id(I + 1, J, K), b.id(I, J + 1, K), b.id(I + 1, J + 1, K),
                      b.id(I, J, K + 1), b.id(I + 1, J, K + 1), b.id(I, J + 1, K + 1), b.id(I + 1, J + 1, K + 1)};
        for (int d = 0; d < 3; d++)
            for (int q = 0; q < 8; q++) au[id[q] + d * N] += auvw[d] * wts[q];
    }
}

inline double sgnd(double v) { return (v > 0) - (v < 0); }

}  // namespace

extern "C" {

/* A^T of a 7-column matrix over the interior (entries towards cells outside the interior dropped) */
void oracle_transpose_matrix(const or_case *c, const double *A, double *AT) {
    Box b(c);
    const long N = b.n;
    memset(AT, 0, sizeof(double) * 7 * N);
    const int gc = b.gc;
    auto in = [&](int i, int j, int k) { return i >= gc && i < b.sx - gc && j >= gc && j < b.sy - gc && k >= gc && k < b.sz - gc; };
    for (int k = gc; k < b.sz - gc; k++)
        for (int j = gc; j < b.sy - gc; j++)
            for (int i = gc; i < b.sx - gc; i++) {
                long cc = b.id(i, j, k);
                AT[cc] = A[cc];
                /* columns: c w e s n b t; AT(c, west) = A(west cell, east) */
                if (in(i - 1, j, k)) AT[cc + N] = A[b.id(i - 1, j, k) + 2 * N];
                if (in(i + 1, j, k)) AT[cc + 2 * N] = A[b.id(i + 1, j, k) + N];
                if (in(i, j - 1, k)) AT[cc + 3 * N] = A[b.id(i, j - 1, k) + 4 * N];
                if (in(i, j + 1, k)) AT[cc + 4 * N] = A[b.id(i, j + 1, k) + 3 * N];
                if (in(i, j, k - 1)) AT[cc + 5 * N] = A[b.id(i, j, k - 1) + 6 * N];
                if (in(i, j, k + 1)) AT[cc + 6 * N] = A[b.id(i, j, k + 1) + 5 * N];
            }
}

int oracle_step_adjoint(const or_case *c, const double *u0, const double *uu0, const double *nut0, const double *p0,
                        const double *kx, const double *g, const double *ja, const double *A, const double *AT,
                        double maxdiag, double t, double wP, double *au, double *auu, double *anut,
                        double *g_pitch, double *g_chord, double *g_twist) {
    Box b(c);
    const long N = b.n;
    const int gc = b.gc, sx = b.sx, sy = b.sy, sz = b.sz;
    if (c->adv != OR_ADV_UPWIND3 && c->adv != OR_ADV_UTOPIA && c->adv != OR_ADV_KK) return 1;
    if (c->sgs != OR_SGS_EMPTY && c->sgs != OR_SGS_SMAGORINSKY) return 1;
    const double dt = c->dt, ReI = 1.0 / c->Re;
    const double alpha = c->adv == OR_ADV_UTOPIA ? 1. / 12. : (c->adv == OR_ADV_KK ? 1. / 4. : 1. / 24.);
    const bool chan = c->bc == OR_BC_CHANNEL;
    auto interior = [&](int i, int j, int k) { return i >= gc && i < sx - gc && j >= gc && j < sy - gc && k >= gc && k < sz - gc; };
    auto facemap = [&](int i, int j, int k) { return i >= gc - 1 && i < sx - gc && j >= gc - 1 && j < sy - gc && k >= gc - 1 && k < sz - gc; };
    /* ---------------- forward recomputation */
    std::vector<double> ff(3 * N, 0.0), xyz, force;
    std::vector<ApTape> tp;
    if (c->alm_on) {
        alm_tape(c, u0, t, tp, xyz, force);
        int apcount = (int)tp.size();
        std::vector<double> x2(3 * apcount), f2(3 * apcount), tq(apcount), th(apcount);
        double ttq[8], tth[8];
        oracle_alm(c, u0, ff.data(), t, x2.data(), f2.data(), tq.data(), th.data(), ttq, tth);
    }
    std::vector<double> ua(u0, u0 + 3 * N);
    oracle_pseudo_u(c, u0, u0, uu0, ua.data(), nut0, kx, g, ja, ff.data());
    std::vector<double> uu1(uu0, uu0 + 3 * N), rhs(N, 0.0), res(N, 0.0), p(p0, p0 + N);
    oracle_utouu(c, ua.data(), uu1.data(), kx, ja);
    oracle_uubc(c, uu1.data());
    oracle_poisson_rhs(c, uu1.data(), rhs.data(), ja, maxdiag);
    int it; double err;
    oracle_pbicgstab(c, A, p.data(), rhs.data(), res.data(), &it, &err);
    oracle_pbc(c, p.data());
    std::vector<double> un(ua), uun(uu1);
    oracle_project_p(c, un.data(), un.data(), uun.data(), uun.data(), p.data(), kx, g);
    oracle_ubc(c, un.data(), u0, t);
    /* ---------------- reverse */
    std::vector<double> au0(3 * N, 0.0), auu0(3 * N, 0.0), anut0(N, 0.0);
    /* nut ghosts (and, without an SGS model, every cell) are not written by the step: identity */
    for (int k = 0; k < sz; k++)
        for (int j = 0; j < sy; j++)
            for (int i = 0; i < sx; i++)
                if (!interior(i, j, k) || c->sgs == OR_SGS_EMPTY) anut0[b.id(i, j, k)] += anut[b.id(i, j, k)];
    /* (9) SGS on the new velocity */
    if (c->sgs == OR_SGS_SMAGORINSKY) {
        for (int k = gc; k < sz - gc; k++)
            for (int j = gc; j < sy - gc; j++)
                for (int i = gc; i < sx - gc; i++) {
                    long cc = b.id(i, j, k);
                    double an = anut[cc];
                    if (an == 0) continue;
                    long e1 = b.id(i + 1, j, k), w1 = b.id(i - 1, j, k), n1 = b.id(i, j + 1, k), s1 = b.id(i, j - 1, k);
                    long t1 = b.id(i, j, k + 1), b1 = b.id(i, j, k - 1);
                    double kk[3] = {kx[cc], kx[cc + N], kx[cc + 2 * N]};
                    double d[3][3];
                    for (int m = 0; m < 3; m++) {
                        const double *um = un.data() + m * N;
                        d[m][0] = 0.5 * kk[0] * (um[e1] - um[w1]);
                        d[m][1] = 0.5 * kk[1] * (um[n1] - um[s1]);
                        d[m][2] = 0.5 * kk[2] * (um[t1] - um[b1]);
                    }
                    double dux = d[0][0], duy = d[0][1], duz = d[0][2], dvx = d[1][0], dvy = d[1][1], dvz = d[1][2];
                    double dwx = d[2][0], dwy = d[2][1], dwz = d[2][2];
                    double S = 2 * SQ(dux) + 2 * SQ(dvy) + 2 * SQ(dwz) + SQ(duy + dvx) + SQ(dvz + dwy) + SQ(duz + dwx);
                    double Du = sqrt(S);
                    if (Du == 0) continue;
                    double lc = c->Cs * cbrt(ja[cc]);
                    double aS = an * SQ(lc) * 0.5 / Du;
                    double ad[3][3];
                    ad[0][0] = aS * 4 * dux; ad[1][1] = aS * 4 * dvy; ad[2][2] = aS * 4 * dwz;
                    ad[0][1] = ad[1][0] = aS * 2 * (duy + dvx);
                    ad[1][2] = ad[2][1] = aS * 2 * (dvz + dwy);
                    ad[0][2] = ad[2][0] = aS * 2 * (duz + dwx);
                    for (int m = 0; m < 3; m++) {
                        double *am = au + m * N;
                        am[e1] += 0.5 * kk[0] * ad[m][0]; am[w1] -= 0.5 * kk[0] * ad[m][0];
                        am[n1] += 0.5 * kk[1] * ad[m][1]; am[s1] -= 0.5 * kk[1] * ad[m][1];
                        am[t1] += 0.5 * kk[2] * ad[m][2]; am[b1] -= 0.5 * kk[2] * ad[m][2];
                    }
                }
    }
    /* (8) velocity boundary conditions, in reverse order of oracle_ubc */
    std::vector<char> written(N, 0);
    if (chan) {
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++) {
                long o1 = b.id(i, j, sz - gc), o2 = b.id(i, j, sz - gc + 1), i1 = b.id(i, j, sz - gc - 1);
                /* slip z+: wb = (u, v, 0) of i1; o1 = wb; o2 = 2 wb - u(i1) */
                for (int d = 0; d < 2; d++) { au[i1 + d * N] += au[o1 + d * N] + au[o2 + d * N]; }
                au[i1 + 2 * N] += -au[o2 + 2 * N];
                for (int d = 0; d < 3; d++) { au[o1 + d * N] = 0; au[o2 + d * N] = 0; }
                written[o1] = written[o2] = 1;
                o1 = b.id(i, j, gc - 1); o2 = b.id(i, j, gc - 2); i1 = b.id(i, j, gc);
                for (int d = 0; d < 3; d++) { au[i1 + d * N] += -au[o2 + d * N]; au[o1 + d * N] = 0; au[o2 + d * N] = 0; }
                written[o1] = written[o2] = 1;
            }
        for (int k = gc; k < sz - gc; k++)
            for (int i = gc; i < sx - gc; i++) {
                for (int side = 1; side >= 0; side--) {
                    long o1, o2, i1;
                    if (side == 1) { o1 = b.id(i, sy - gc, k); o2 = b.id(i, sy - gc + 1, k); i1 = b.id(i, sy - gc - 1, k); }
                    else { o1 = b.id(i, gc - 1, k); o2 = b.id(i, gc - 2, k); i1 = b.id(i, gc, k); }
                    /* slip: (u, 0, w) of i1 */
                    au[i1] += au[o1] + au[o2];
                    au[i1 + N] += -au[o2 + N];
                    au[i1 + 2 * N] += au[o1 + 2 * N] + au[o2 + 2 * N];
                    for (int d = 0; d < 3; d++) { au[o1 + d * N] = 0; au[o2 + d * N] = 0; }
                    written[o1] = written[o2] = 1;
                }
            }
        for (int k = gc; k < sz - gc; k++)
            for (int j = gc; j < sy - gc; j++) {
                int i = sx - gc;
                long o1 = b.id(i, j, k), o2 = b.id(i + 1, j, k), i1 = b.id(i - 1, j, k), i2 = b.id(i - 2, j, k);
                double dxi = 1.0 / (c->x[i] - c->x[i - 1]);
                for (int d = 0; d < 3; d++) {
                    double aub = au[o1 + d * N] + 2 * au[o2 + d * N];
                    au[i1 + d * N] += -au[o2 + d * N];
                    au0[o1 + d * N] += aub * (1 - dt * 0.5 * dxi * 3);
                    au0[i1 + d * N] += aub * (dt * 0.5 * dxi * 4);
                    au0[i2 + d * N] += aub * (-dt * 0.5 * dxi);
                    au[o1 + d * N] = 0; au[o2 + d * N] = 0;
                }
                written[o1] = written[o2] = 1;
                i = gc - 1;
                long g1 = b.id(i, j, k), g2 = b.id(i - 1, j, k);
                for (int d = 0; d < 3; d++) { au[g1 + d * N] = 0; au[g2 + d * N] = 0; }
                written[g1] = written[g2] = 1;
            }
    } else {
        /* cavity: every face reflects about a wall value (lid constant) */
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++)
                for (int d = 0; d < 3; d++) {
                    double *a = au + d * N;
                    long g4[4] = {b.id(i, j, gc - 1), b.id(i, j, gc - 2), b.id(i, j, sz - gc), b.id(i, j, sz - gc + 1)};
                    long s4[4] = {b.id(i, j, gc), b.id(i, j, gc + 1), b.id(i, j, sz - gc - 1), b.id(i, j, sz - gc - 2)};
                    for (int q = 3; q >= 0; q--) { a[s4[q]] += -a[g4[q]]; a[g4[q]] = 0; written[g4[q]] = 1; }
                }
        for (int k = gc; k < sz - gc; k++)
            for (int i = gc; i < sx - gc; i++)
                for (int d = 0; d < 3; d++) {
                    double *a = au + d * N;
                    long g4[4] = {b.id(i, gc - 1, k), b.id(i, gc - 2, k), b.id(i, sy - gc, k), b.id(i, sy - gc + 1, k)};
                    long s4[4] = {b.id(i, gc, k), b.id(i, gc + 1, k), b.id(i, sy - gc - 1, k), b.id(i, sy - gc - 2, k)};
                    for (int q = 3; q >= 0; q--) { a[s4[q]] += -a[g4[q]]; a[g4[q]] = 0; written[g4[q]] = 1; }
                }
        for (int k = gc; k < sz - gc; k++)
            for (int j = gc; j < sy - gc; j++)
                for (int d = 0; d < 3; d++) {
                    double *a = au + d * N;
                    long g4[4] = {b.id(gc - 1, j, k), b.id(gc - 2, j, k), b.id(sx - gc, j, k), b.id(sx - gc + 1, j, k)};
                    long s4[4] = {b.id(gc, j, k), b.id(gc + 1, j, k), b.id(sx - gc - 1, j, k), b.id(sx - gc - 2, j, k)};
                    for (int q = 3; q >= 0; q--) { a[s4[q]] += -a[g4[q]]; a[g4[q]] = 0; written[g4[q]] = 1; }
                }
    }
    /* cells the step never writes carry the previous velocity: identity */
    for (long n = 0; n < N; n++) {
        int i = (int)(n % sx), j = (int)((n / sx) % sy), k = (int)(n / ((long)sx * sy));
        if (!interior(i, j, k) && !written[n])
            for (int d = 0; d < 3; d++) { au0[n + d * N] += au[n + d * N]; au[n + d * N] = 0; }
    }
    /* (7) projection: u = ua - dt kx dp/2 (interior), uu = uu1 - dt g dp (face map) */
    std::vector<double> aua(3 * N, 0.0), auu1(3 * N, 0.0), ap(N, 0.0);
    for (int k = gc; k < sz - gc; k++)
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++) {
                long cc = b.id(i, j, k);
                long nb[3][2] = {{b.id(i + 1, j, k), b.id(i - 1, j, k)}, {b.id(i, j + 1, k), b.id(i, j - 1, k)}, {b.id(i, j, k + 1), b.id(i, j, k - 1)}};
                for (int d = 0; d < 3; d++) {
                    double a = au[cc + d * N];
                    aua[cc + d * N] += a;
                    ap[nb[d][0]] += -dt * 0.5 * kx[cc + d * N] * a;
                    ap[nb[d][1]] += dt * 0.5 * kx[cc + d * N] * a;
                }
            }
    for (long n = 0; n < N; n++) {
        int i = (int)(n % sx), j = (int)((n / sx) % sy), k = (int)(n / ((long)sx * sy));
        if (!facemap(i, j, k)) {   /* uu cells outside the face map carry over */
            for (int d = 0; d < 3; d++) auu0[n + d * N] += auu[n + d * N];
            continue;
        }
        long nb[3] = {b.id(i + 1, j, k), b.id(i, j + 1, k), b.id(i, j, k + 1)};
        for (int d = 0; d < 3; d++) {
            double a = auu[n + d * N];
            auu1[n + d * N] += a;
            double cf = dt * 0.5 * (g[n + d * N] + g[nb[d] + d * N]);
            ap[nb[d]] += -cf * a;
            ap[n] += cf * a;
        }
    }
    /* (5) pressure boundary conditions, in reverse order of oracle_pbc */
    for (int j = gc; j < sy - gc; j++)
        for (int i = gc; i < sx - gc; i++) {
            ap[b.id(i, j, sz - gc - 1)] += ap[b.id(i, j, sz - gc)]; ap[b.id(i, j, sz - gc)] = 0;
            ap[b.id(i, j, gc)] += ap[b.id(i, j, gc - 1)]; ap[b.id(i, j, gc - 1)] = 0;
        }
    for (int k = gc; k < sz - gc; k++)
        for (int i = gc; i < sx - gc; i++) {
            ap[b.id(i, sy - gc - 1, k)] += ap[b.id(i, sy - gc, k)]; ap[b.id(i, sy - gc, k)] = 0;
            ap[b.id(i, gc, k)] += ap[b.id(i, gc - 1, k)]; ap[b.id(i, gc - 1, k)] = 0;
        }
    for (int k = gc; k < sz - gc; k++)
        for (int j = gc; j < sy - gc; j++) {
            if (chan) ap[b.id(sx - gc, j, k)] = 0;
            else { ap[b.id(sx - gc - 1, j, k)] += ap[b.id(sx - gc, j, k)]; ap[b.id(sx - gc, j, k)] = 0; }
            ap[b.id(gc, j, k)] += ap[b.id(gc - 1, j, k)]; ap[b.id(gc - 1, j, k)] = 0;
        }
    for (long n = 0; n < N; n++) {   /* remaining ghost entries of p are not read by the projection of interior data */
        int i = (int)(n % sx), j = (int)((n / sx) % sy), k = (int)(n / ((long)sx * sy));
        if (!interior(i, j, k)) ap[n] = 0;
    }
    /* (4) transposed Poisson solve: arhs = A^-T ap */
    std::vector<double> arhs(N, 0.0), r2(N, 0.0);
    oracle_pbicgstab(c, AT, arhs.data(), ap.data(), r2.data(), &it, &err);
    /* (3) rhs = div(uu1)/ja / (dt maxdiag) on the interior */
    const double scale = 1.0 / (dt * maxdiag);
    for (int k = gc; k < sz - gc; k++)
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++) {
                long cc = b.id(i, j, k);
                double a = arhs[cc] * scale / ja[cc];
                auu1[cc] += a; auu1[b.id(i - 1, j, k)] -= a;
                auu1[cc + N] += a; auu1[b.id(i, j - 1, k) + N] -= a;
                auu1[cc + 2 * N] += a; auu1[b.id(i, j, k - 1) + 2 * N] -= a;
            }
    if (c->bc == OR_BC_CAVITY) {   /* uubc zeroes the wall-normal faces */
        for (int k = gc; k < sz - gc; k++)
            for (int j = gc; j < sy - gc; j++) { auu1[b.id(gc - 1, j, k)] = 0; auu1[b.id(sx - gc - 1, j, k)] = 0; }
        for (int k = gc; k < sz - gc; k++)
            for (int i = gc; i < sx - gc; i++) { auu1[b.id(i, gc - 1, k) + N] = 0; auu1[b.id(i, sy - gc - 1, k) + N] = 0; }
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++) { auu1[b.id(i, j, gc - 1) + 2 * N] = 0; auu1[b.id(i, j, sz - gc - 1) + 2 * N] = 0; }
    }
    /* UtoUU: uu1 = 0.5 (uc(c) + uc(c+e_d)) on the face map, uc = ja kx ua on [gc-1, s-gc] */
    for (int k = gc - 1; k < sz - gc; k++)
        for (int j = gc - 1; j < sy - gc; j++)
            for (int i = gc - 1; i < sx - gc; i++) {
                long cc = b.id(i, j, k);
                long nb[3] = {b.id(i + 1, j, k), b.id(i, j + 1, k), b.id(i, j, k + 1)};
                for (int d = 0; d < 3; d++) {
                    double a = 0.5 * auu1[cc + d * N];
                    aua[cc + d * N] += a * ja[cc] * kx[cc + d * N];
                    aua[nb[d] + d * N] += a * ja[nb[d]] * kx[nb[d] + d * N];
                }
            }
    /* (2) pseudo-velocity: ua = u0 + dt(-adv + vis + ff) on the interior; ghosts of ua are u0's */
    std::vector<double> aff(3 * N, 0.0);
    for (long n = 0; n < N; n++) {
        int i = (int)(n % sx), j = (int)((n / sx) % sy), k = (int)(n / ((long)sx * sy));
        if (!interior(i, j, k))
            for (int d = 0; d < 3; d++) au0[n + d * N] += aua[n + d * N];
    }
    for (int k = gc; k < sz - gc; k++)
        for (int j = gc; j < sy - gc; j++)
            for (int i = gc; i < sx - gc; i++) {
                long cc = b.id(i, j, k);
                long e1 = b.id(i + 1, j, k), w1 = b.id(i - 1, j, k), n1 = b.id(i, j + 1, k), s1 = b.id(i, j - 1, k);
                long t1 = b.id(i, j, k + 1), b1 = b.id(i, j, k - 1);
                long e2 = b.id(i + 2, j, k), w2 = b.id(i - 2, j, k), n2 = b.id(i, j + 2, k), s2 = b.id(i, j - 2, k);
                long t2 = b.id(i, j, k + 2), b2 = b.id(i, j, k - 2);
                const long nbp[3][2] = {{e1, e2}, {n1, n2}, {t1, t2}}, nbm[3][2] = {{w1, w2}, {s1, s2}, {b1, b2}};
                const long facep[3] = {cc, cc + N, cc + 2 * N}, facem[3] = {w1, s1 + N, b1 + 2 * N};
                const long gm[3] = {w1, s1, b1}, gp[3] = {e1, n1, t1};
                double jac = ja[cc];
                double Uc[3], Ua[3];
                for (int q = 0; q < 3; q++) { Uc[q] = u0[cc + q * N] * kx[cc + q * N]; Ua[q] = fabs(Uc[q]); }
                double aUa[3] = {0, 0, 0};
                for (int d = 0; d < 3; d++) {
                    double a = aua[cc + d * N];
                    if (a == 0) continue;
                    const double *ud = u0 + d * N;
                    double *aud = au0.data() + d * N;
                    aud[cc] += a;
                    aff[cc + d * N] += dt * a;
                    double aadv = -dt * a, avis = dt * a / (2 * jac);
                    double ucc = ud[cc];
                    for (int ax = 0; ax < 3; ax++) {
                        double up1 = ud[nbp[ax][0]], up2 = ud[nbp[ax][1]], um1 = ud[nbm[ax][0]], um2 = ud[nbm[ax][1]];
                        double JP = uu0[facep[ax]], JM = uu0[facem[ax]];
                        double L = -up2 + 27 * up1 - 27 * ucc + um1, R = -up1 + 27 * ucc - 27 * um1 + um2;
                        double D = up2 - 4 * up1 + 6 * ucc - 4 * um1 + um2;
                        double f = 0.5 / (24. * jac);
                        auu0[facep[ax]] += aadv * f * L;
                        auu0[facem[ax]] += aadv * f * R;
                        aUa[ax] += aadv * D * alpha;
                        double s = Ua[ax] * alpha;
                        aud[nbp[ax][1]] += aadv * (-f * JP + s);
                        aud[nbp[ax][0]] += aadv * (f * (27 * JP - JM) - 4 * s);
                        aud[cc] += aadv * (f * (-27 * JP + 27 * JM) + 6 * s);
                        aud[nbm[ax][0]] += aadv * (f * (JP - 27 * JM) - 4 * s);
                        aud[nbm[ax][1]] += aadv * (f * JM + s);
                        /* diffusion faces +ax and -ax */
                        double Gp = g[cc + ax * N] + g[gp[ax] + ax * N], Gm = g[cc + ax * N] + g[gm[ax] + ax * N];
                        double Np = ReI + 0.5 * (nut0[cc] + nut0[gp[ax]]), Nm = ReI + 0.5 * (nut0[cc] + nut0[gm[ax]]);
                        double dp = up1 - ucc, dm = ucc - um1;
                        aud[nbp[ax][0]] += avis * Gp * Np; aud[cc] -= avis * Gp * Np;
                        aud[cc] -= avis * Gm * Nm; aud[nbm[ax][0]] += avis * Gm * Nm;
                        anut0[cc] += avis * 0.5 * (Gp * dp - Gm * dm);
                        anut0[gp[ax]] += avis * 0.5 * Gp * dp;
                        anut0[gm[ax]] -= avis * 0.5 * Gm * dm;
                    }
                }
                for (int q = 0; q < 3; q++) au0[cc + q * N] += aUa[q] * sgnd(Uc[q]) * kx[cc + q * N];
            }
    /* (1) ALM force and the power term of the objective */
    if (c->alm_on) alm_adjoint(c, tp, xyz, aff.data(), wP, au0.data(), g_pitch, g_chord, g_twist);
    memcpy(au, au0.data(), sizeof(double) * 3 * N);
    memcpy(auu, auu0.data(), sizeof(double) * 3 * N);
    memcpy(anut, anut0.data(), sizeof(double) * N);
    return 0;
}

} // extern "C"
