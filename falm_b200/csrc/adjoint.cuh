// Discrete adjoint of one time step.  No reference counterpart: this is
// the adjoint of this library's own discretisation of the step, with the
// Poisson solve treated as exact (p = A^-1 rhs), so that its adjoint is one
// solve with the transposed operator.  Each kernel below is the transpose of
// one forward stage, applied in reverse order; scatters from a cell to its
// stencil neighbours use double-precision atomics.
//
// Arrays: au/auu/anut hold the adjoint of the state after the step (they are
// consumed), au0/auu0/anut0 collect the adjoint of the state before it.  The
// adjoint is FP64 throughout; the forward state it is evaluated at (u, uu, nut
// of type T) is FP64 or, for a mixed-precision context, FP32.
#pragma once
#include "common.cuh"
#include "alm_bc.cuh"

namespace fb {

// grid-stride loop over the cells of the box [i0,i1) x [j0,j1) x [k0,k1)
#define ADJ_FOR_BOX(I0, I1, J0, J1, K0, K1, I, J, K)                                                             \
    for (long long _q = blockIdx.x * (long long)blockDim.x + threadIdx.x, _ni = (I1) - (I0), _nj = (J1) - (J0),  \
                   _tot = _ni * _nj * (long long)((K1) - (K0));                                                  \
         _q < _tot; _q += (long long)gridDim.x * blockDim.x)                                                     \
        for (int I = (I0) + (int)(_q % _ni), J = (J0) + (int)((_q / _ni) % _nj), K = (K0) + (int)(_q / (_ni * _nj)), \
                 _once = 1;                                                                                      \
             _once; _once = 0)

__device__ __forceinline__ bool adj_interior(const Geom &g, int i, int j, int k) {
    return i >= g.gc && i < g.sx - g.gc && j >= g.gc && j < g.sy - g.gc && k >= g.gc && k < g.sz - g.gc;
}
__device__ __forceinline__ bool adj_facemap(const Geom &g, int i, int j, int k) {
    return i >= g.gc - 1 && i < g.sx - g.gc && j >= g.gc - 1 && j < g.sy - g.gc && k >= g.gc - 1 && k < g.sz - g.gc;
}
__device__ __forceinline__ double adj_sgn(double v) { return (v > 0) - (v < 0); }

// (9) Smagorinsky eddy viscosity of the new velocity (SgsDivBody / k_sgs_div)
template <typename T>
__global__ void k_adj_sgs(Geom g, MetricView<double> mv, const T *__restrict__ un, const double *__restrict__ anut,
                          double *au, double Cs) {
    const long long N = g.n;
    ADJ_FOR_BOX(g.gc, g.sx - g.gc, g.gc, g.sy - g.gc, g.gc, g.sz - g.gc, i, j, k) {
        const long long cc = g.id(i, j, k);
        const double an = anut[cc];
        if (an == 0.0) continue;
        const long long nbp[3] = {g.id(i + 1, j, k), g.id(i, j + 1, k), g.id(i, j, k + 1)};
        const long long nbm[3] = {g.id(i - 1, j, k), g.id(i, j - 1, k), g.id(i, j, k - 1)};
        const double kk[3] = {mv.kx(0, i), mv.kx(1, j), mv.kx(2, k)};
        double d[3][3];
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int a = 0; a < 3; a++) d[m][a] = 0.5 * kk[a] * (to_d(un[nbp[a] + m * N]) - to_d(un[nbm[a] + m * N]));
        const double S = 2 * (d[0][0] * d[0][0]) + 2 * (d[1][1] * d[1][1]) + 2 * (d[2][2] * d[2][2]) + (d[0][1] + d[1][0]) * (d[0][1] + d[1][0]) +
                         (d[1][2] + d[2][1]) * (d[1][2] + d[2][1]) + (d[0][2] + d[2][0]) * (d[0][2] + d[2][0]);
        const double Du = sqrt(S);
        if (Du == 0.0) continue;
        const double lc = Cs * cbrt(mv.ja(i, j, k));
        const double aS = an * (lc * lc) * 0.5 / Du;
        double ad[3][3];
        ad[0][0] = aS * 4 * d[0][0]; ad[1][1] = aS * 4 * d[1][1]; ad[2][2] = aS * 4 * d[2][2];
        ad[0][1] = ad[1][0] = aS * 2 * (d[0][1] + d[1][0]);
        ad[1][2] = ad[2][1] = aS * 2 * (d[1][2] + d[2][1]);
        ad[0][2] = ad[2][0] = aS * 2 * (d[0][2] + d[2][0]);
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int a = 0; a < 3; a++) {
                atomicAdd(au + nbp[a] + m * N, 0.5 * kk[a] * ad[m][a]);
                atomicAdd(au + nbm[a] + m * N, -0.5 * kk[a] * ad[m][a]);
            }
    }
}

// (8) velocity boundary conditions (k_ubc), one face pair per blockIdx.y
__global__ void k_adj_ubc(Geom g, int kind, double *au, double *au0, const double *xc, double dt) {
    const long long N = g.n;
    const int gc = g.gc, sx = g.sx, sy = g.sy, sz = g.sz;
    const int pair = blockIdx.y;
    const int na = pair == 0 ? sy - 2 * gc : sx - 2 * gc;
    const int nb = pair == 2 ? sy - 2 * gc : sz - 2 * gc;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)na * nb; q += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(q % na) + gc, b = (int)(q / na) + gc;
        if (kind == FALM_BC_CHANNEL) {
            if (pair == 0) {
                const int j = a, k = b;
                for (int d = 0; d < 3; d++) { au[g.id(gc - 1, j, k) + d * N] = 0; au[g.id(gc - 2, j, k) + d * N] = 0; }   // inlet: fixed values
                const int i = sx - gc;
                const double dxi = 1.0 / (xc[i] - xc[i - 1]);
                const long long o1 = g.id(i, j, k), o2 = g.id(i + 1, j, k), i1 = g.id(i - 1, j, k), i2 = g.id(i - 2, j, k);
                for (int d = 0; d < 3; d++) {
                    const double aub = au[o1 + d * N] + 2 * au[o2 + d * N];
                    atomicAdd(au + i1 + d * N, -au[o2 + d * N]);
                    atomicAdd(au0 + o1 + d * N, aub * (1 - dt * 0.5 * dxi * 3));
                    atomicAdd(au0 + i1 + d * N, aub * (dt * 0.5 * dxi * 4));
                    atomicAdd(au0 + i2 + d * N, aub * (-dt * 0.5 * dxi));
                    au[o1 + d * N] = 0; au[o2 + d * N] = 0;
                }
            } else if (pair == 1) {
                const int i = a, k = b;
                for (int side = 0; side < 2; side++) {
                    long long o1, o2, i1;
                    if (side) { o1 = g.id(i, sy - gc, k); o2 = g.id(i, sy - gc + 1, k); i1 = g.id(i, sy - gc - 1, k); }
                    else { o1 = g.id(i, gc - 1, k); o2 = g.id(i, gc - 2, k); i1 = g.id(i, gc, k); }
                    atomicAdd(au + i1, au[o1] + au[o2]);
                    atomicAdd(au + i1 + N, -au[o2 + N]);
                    atomicAdd(au + i1 + 2 * N, au[o1 + 2 * N] + au[o2 + 2 * N]);
                    for (int d = 0; d < 3; d++) { au[o1 + d * N] = 0; au[o2 + d * N] = 0; }
                }
            } else {
                const int i = a, j = b;
                long long o1 = g.id(i, j, gc - 1), o2 = g.id(i, j, gc - 2), i1 = g.id(i, j, gc);
                for (int d = 0; d < 3; d++) { atomicAdd(au + i1 + d * N, -au[o2 + d * N]); au[o1 + d * N] = 0; au[o2 + d * N] = 0; }
                o1 = g.id(i, j, sz - gc); o2 = g.id(i, j, sz - gc + 1); i1 = g.id(i, j, sz - gc - 1);
                for (int d = 0; d < 2; d++) atomicAdd(au + i1 + d * N, au[o1 + d * N] + au[o2 + d * N]);
                atomicAdd(au + i1 + 2 * N, -au[o2 + 2 * N]);
                for (int d = 0; d < 3; d++) { au[o1 + d * N] = 0; au[o2 + d * N] = 0; }
            }
        } else {
            // cavity: every guide cell is 2 * wall value - a mirror interior cell
            for (int d = 0; d < 3; d++) {
                double *ad = au + d * N;
                long long gs[4], ss[4];
                if (pair == 0) {
                    const int j = a, k = b;
                    gs[0] = g.id(gc - 1, j, k); ss[0] = g.id(gc, j, k); gs[1] = g.id(gc - 2, j, k); ss[1] = g.id(gc + 1, j, k);
                    gs[2] = g.id(sx - gc, j, k); ss[2] = g.id(sx - gc - 1, j, k); gs[3] = g.id(sx - gc + 1, j, k); ss[3] = g.id(sx - gc - 2, j, k);
                } else if (pair == 1) {
                    const int i = a, k = b;
                    gs[0] = g.id(i, gc - 1, k); ss[0] = g.id(i, gc, k); gs[1] = g.id(i, gc - 2, k); ss[1] = g.id(i, gc + 1, k);
                    gs[2] = g.id(i, sy - gc, k); ss[2] = g.id(i, sy - gc - 1, k); gs[3] = g.id(i, sy - gc + 1, k); ss[3] = g.id(i, sy - gc - 2, k);
                } else {
                    const int i = a, j = b;
                    gs[0] = g.id(i, j, gc - 1); ss[0] = g.id(i, j, gc); gs[1] = g.id(i, j, gc - 2); ss[1] = g.id(i, j, gc + 1);
                    gs[2] = g.id(i, j, sz - gc); ss[2] = g.id(i, j, sz - gc - 1); gs[3] = g.id(i, j, sz - gc + 1); ss[3] = g.id(i, j, sz - gc - 2);
                }
                for (int q2 = 0; q2 < 4; q2++) { atomicAdd(ad + ss[q2], -ad[gs[q2]]); ad[gs[q2]] = 0; }
            }
        }
    }
}

// guide cells the step never writes (edges and corners: two or more indices
// outside the interior) carry the previous value: move their adjoint across
__global__ void k_adj_carry_edges(Geom g, double *src, double *dst, int ncomp) {
    const long long N = g.n;
    ADJ_FOR_BOX(0, g.sx, 0, g.sy, 0, g.sz, i, j, k) {
        const int out = (i < g.gc || i >= g.sx - g.gc) + (j < g.gc || j >= g.sy - g.gc) + (k < g.gc || k >= g.sz - g.gc);
        if (out < 2) continue;
        const long long cc = g.id(i, j, k);
        for (int d = 0; d < ncomp; d++) { dst[cc + d * N] += src[cc + d * N]; src[cc + d * N] = 0; }
    }
}

// (7) projection (ProjectBody / k_project): u = ua - dt kx dp/2 on the interior,
// uu = uu1 - dt (g_c + g_+)/2 (p_+ - p_c) on the face map; other uu cells carry over
__global__ void k_adj_project(Geom g, MetricView<double> mv, const double *au, const double *auu, double *aua,
                              double *auu1, double *auu0, double *ap, double dt) {
    const long long N = g.n;
    ADJ_FOR_BOX(0, g.sx, 0, g.sy, 0, g.sz, i, j, k) {
        const long long cc = g.id(i, j, k);
        if (adj_interior(g, i, j, k)) {
            const long long nbp[3] = {g.id(i + 1, j, k), g.id(i, j + 1, k), g.id(i, j, k + 1)};
            const long long nbm[3] = {g.id(i - 1, j, k), g.id(i, j - 1, k), g.id(i, j, k - 1)};
            const int idx[3] = {i, j, k};
            for (int d = 0; d < 3; d++) {
                const double a = au[cc + d * N];
                aua[cc + d * N] += a;
                const double f = dt * 0.5 * mv.kx(d, idx[d]) * a;
                atomicAdd(ap + nbp[d], -f);
                atomicAdd(ap + nbm[d], f);
            }
        }
        if (adj_facemap(g, i, j, k)) {
            const long long nb[3] = {g.id(i + 1, j, k), g.id(i, j + 1, k), g.id(i, j, k + 1)};
            const double gc3[3] = {mv.g(0, i, j, k), mv.g(1, i, j, k), mv.g(2, i, j, k)};
            const double gp3[3] = {mv.g(0, i + 1, j, k), mv.g(1, i, j + 1, k), mv.g(2, i, j, k + 1)};
            for (int d = 0; d < 3; d++) {
                const double a = auu[cc + d * N];
                auu1[cc + d * N] += a;
                const double f = dt * 0.5 * (gc3[d] + gp3[d]) * a;
                atomicAdd(ap + nb[d], -f);
                atomicAdd(ap + cc, f);
            }
        } else {
            for (int d = 0; d < 3; d++) auu0[cc + d * N] += auu[cc + d * N];
        }
    }
}

// (5) pressure boundary conditions (k_pbc), one face pair per blockIdx.y
__global__ void k_adj_pbc(Geom g, int kind, double *ap) {
    const int gc = g.gc, sx = g.sx, sy = g.sy, sz = g.sz;
    const int pair = blockIdx.y;
    const int na = pair == 0 ? sy - 2 * gc : sx - 2 * gc;
    const int nb = pair == 2 ? sy - 2 * gc : sz - 2 * gc;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)na * nb; q += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(q % na) + gc, b = (int)(q / na) + gc;
        long long g0, s0, g1, s1;
        if (pair == 0) { g0 = g.id(gc - 1, a, b); s0 = g.id(gc, a, b); g1 = g.id(sx - gc, a, b); s1 = g.id(sx - gc - 1, a, b); }
        else if (pair == 1) { g0 = g.id(a, gc - 1, b); s0 = g.id(a, gc, b); g1 = g.id(a, sy - gc, b); s1 = g.id(a, sy - gc - 1, b); }
        else { g0 = g.id(a, b, gc - 1); s0 = g.id(a, b, gc); g1 = g.id(a, b, sz - gc); s1 = g.id(a, b, sz - gc - 1); }
        atomicAdd(ap + s0, ap[g0]);
        if (!(pair == 0 && kind == FALM_BC_CHANNEL)) atomicAdd(ap + s1, ap[g1]);   // channel x+: p = 0
    }
}

__global__ void k_adj_zero_ghosts(Geom g, double *a) {
    ADJ_FOR_BOX(0, g.sx, 0, g.sy, 0, g.sz, i, j, k) {
        if (!adj_interior(g, i, j, k)) a[g.id(i, j, k)] = 0;
    }
}

// transposed 7-column operator over the interior (columns c w e s n b t)
__global__ void k_adj_transpose_op(Geom g, Op7<double> op, double *AT) {
    const long long N = g.n;
    ADJ_FOR_BOX(0, g.sx, 0, g.sy, 0, g.sz, i, j, k) {
        const long long cc = g.id(i, j, k);
        double r[7] = {0, 0, 0, 0, 0, 0, 0};
        if (adj_interior(g, i, j, k)) {
            double ac, aw, ae, as, an, ab, at;
            op.get(i, j, k, cc, ac, aw, ae, as, an, ab, at);
            r[0] = ac;
            const int nb[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
            const int opp[6] = {2, 1, 4, 3, 6, 5};   // the neighbour's coefficient towards this cell
            for (int q = 0; q < 6; q++) {
                const int x = nb[q][0], y = nb[q][1], z = nb[q][2];
                if (!adj_interior(g, x, y, z)) continue;
                double v[7];
                op.get(x, y, z, g.id(x, y, z), v[0], v[1], v[2], v[3], v[4], v[5], v[6]);
                r[q + 1] = v[opp[q]];
            }
        }
        for (int q = 0; q < 7; q++) AT[cc + q * N] = r[q];
    }
}

// (3) right-hand side rhs = div(uu1) / ja * scale on the interior
__global__ void k_adj_rhs(Geom g, MetricView<double> mv, const double *arhs, double *auu1, double scale) {
    const long long N = g.n;
    ADJ_FOR_BOX(g.gc, g.sx - g.gc, g.gc, g.sy - g.gc, g.gc, g.sz - g.gc, i, j, k) {
        const long long cc = g.id(i, j, k);
        const double a = arhs[cc] * scale / mv.ja(i, j, k);
        atomicAdd(auu1 + cc, a); atomicAdd(auu1 + g.id(i - 1, j, k), -a);
        atomicAdd(auu1 + cc + N, a); atomicAdd(auu1 + g.id(i, j - 1, k) + N, -a);
        atomicAdd(auu1 + cc + 2 * N, a); atomicAdd(auu1 + g.id(i, j, k - 1) + 2 * N, -a);
    }
}

// cavity uubc zeroes the wall-normal faces
__global__ void k_adj_uubc(Geom g, double *auu1) {
    const long long N = g.n;
    const int gc = g.gc;
    ADJ_FOR_BOX(gc - 1, g.sx - gc, gc - 1, g.sy - gc, gc - 1, g.sz - gc, i, j, k) {
        const bool ji = j >= gc && j < g.sy - gc, ki = k >= gc && k < g.sz - gc, ii = i >= gc && i < g.sx - gc;
        const long long cc = g.id(i, j, k);
        if ((i == gc - 1 || i == g.sx - gc - 1) && ji && ki) auu1[cc] = 0;
        if ((j == gc - 1 || j == g.sy - gc - 1) && ii && ki) auu1[cc + N] = 0;
        if ((k == gc - 1 || k == g.sz - gc - 1) && ii && ji) auu1[cc + 2 * N] = 0;
    }
}

// face velocity: uu1 = (uc_c + uc_{c+e_d}) / 2 on the face map, uc = ja kx ua
__global__ void k_adj_utouu(Geom g, MetricView<double> mv, const double *auu1, double *aua) {
    const long long N = g.n;
    ADJ_FOR_BOX(g.gc - 1, g.sx - g.gc, g.gc - 1, g.sy - g.gc, g.gc - 1, g.sz - g.gc, i, j, k) {
        const long long cc = g.id(i, j, k);
        const int nbi[3][3] = {{i + 1, j, k}, {i, j + 1, k}, {i, j, k + 1}};
        const int idx[3] = {i, j, k};
        for (int d = 0; d < 3; d++) {
            const double a = 0.5 * auu1[cc + d * N];
            if (a == 0.0) continue;
            const int x = nbi[d][0], y = nbi[d][1], z = nbi[d][2];
            atomicAdd(aua + cc + d * N, a * mv.ja(i, j, k) * mv.kx(d, idx[d]));
            atomicAdd(aua + g.id(x, y, z) + d * N, a * mv.ja(x, y, z) * mv.kx(d, idx[d] + 1));
        }
    }
}

// the pseudo-velocity buffer's guide cells hold the previous velocity
__global__ void k_adj_carry_ghosts(Geom g, const double *aua, double *au0) {
    const long long N = g.n;
    ADJ_FOR_BOX(0, g.sx, 0, g.sy, 0, g.sz, i, j, k) {
        if (adj_interior(g, i, j, k)) continue;
        const long long cc = g.id(i, j, k);
        for (int d = 0; d < 3; d++) au0[cc + d * N] += aua[cc + d * N];
    }
}

// (2) pseudo-velocity with a 4th-order scheme: ua = u0 + dt (-adv + vis + ff)
template <typename T>
__global__ void k_adj_pseudo_u(Geom g, MetricView<double> mv, const T *u0, const T *uu0, const T *nut0,
                               const double *aua, double *au0, double *auu0, double *anut0, double *aff,
                               double ReI, double dt, double alpha) {
    const long long N = g.n;
    ADJ_FOR_BOX(g.gc, g.sx - g.gc, g.gc, g.sy - g.gc, g.gc, g.sz - g.gc, i, j, k) {
        const long long cc = g.id(i, j, k);
        const long long e1 = g.id(i + 1, j, k), w1 = g.id(i - 1, j, k), n1 = g.id(i, j + 1, k), s1 = g.id(i, j - 1, k);
        const long long t1 = g.id(i, j, k + 1), b1 = g.id(i, j, k - 1);
        const long long nbp[3][2] = {{e1, g.id(i + 2, j, k)}, {n1, g.id(i, j + 2, k)}, {t1, g.id(i, j, k + 2)}};
        const long long nbm[3][2] = {{w1, g.id(i - 2, j, k)}, {s1, g.id(i, j - 2, k)}, {b1, g.id(i, j, k - 2)}};
        const long long facep[3] = {cc, cc + N, cc + 2 * N}, facem[3] = {w1, s1 + N, b1 + 2 * N};
        const int idx[3] = {i, j, k};
        const double jac = mv.ja(i, j, k);
        double Uc[3], Ua[3], Gp[3], Gm[3], Np[3], Nm[3];
        for (int q = 0; q < 3; q++) {
            Uc[q] = to_d(u0[cc + q * N]) * mv.kx(q, idx[q]);
            Ua[q] = fabs(Uc[q]);
            const int ip[3] = {i + (q == 0), j + (q == 1), k + (q == 2)}, im[3] = {i - (q == 0), j - (q == 1), k - (q == 2)};
            Gp[q] = mv.g(q, i, j, k) + mv.g(q, ip[0], ip[1], ip[2]);
            Gm[q] = mv.g(q, i, j, k) + mv.g(q, im[0], im[1], im[2]);
            Np[q] = ReI + 0.5 * (to_d(nut0[cc]) + to_d(nut0[nbp[q][0]]));
            Nm[q] = ReI + 0.5 * (to_d(nut0[cc]) + to_d(nut0[nbm[q][0]]));
        }
        double aUa[3] = {0, 0, 0};
        const double f = 0.5 / (24. * jac);
        for (int d = 0; d < 3; d++) {
            const double a = aua[cc + d * N];
            if (a == 0.0) continue;
            const T *ud = u0 + d * N;
            double *aud = au0 + d * N;
            atomicAdd(aud + cc, a);
            aff[cc + d * N] += dt * a;
            const double aadv = -dt * a, avis = dt * a / (2 * jac);
            const double ucc = to_d(ud[cc]);
            for (int ax = 0; ax < 3; ax++) {
                const double up1 = to_d(ud[nbp[ax][0]]), up2 = to_d(ud[nbp[ax][1]]), um1 = to_d(ud[nbm[ax][0]]), um2 = to_d(ud[nbm[ax][1]]);
                const double JP = to_d(uu0[facep[ax]]), JM = to_d(uu0[facem[ax]]);
                const double L = -up2 + 27 * up1 - 27 * ucc + um1, R = -up1 + 27 * ucc - 27 * um1 + um2;
                const double D = up2 - 4 * up1 + 6 * ucc - 4 * um1 + um2;
                atomicAdd(auu0 + facep[ax], aadv * f * L);
                atomicAdd(auu0 + facem[ax], aadv * f * R);
                aUa[ax] += aadv * D * alpha;
                const double s = Ua[ax] * alpha;
                const double dp = up1 - ucc, dm = ucc - um1;
                atomicAdd(aud + nbp[ax][1], aadv * (-f * JP + s));
                atomicAdd(aud + nbp[ax][0], aadv * (f * (27 * JP - JM) - 4 * s) + avis * Gp[ax] * Np[ax]);
                atomicAdd(aud + cc, aadv * (f * (-27 * JP + 27 * JM) + 6 * s) - avis * (Gp[ax] * Np[ax] + Gm[ax] * Nm[ax]));
                atomicAdd(aud + nbm[ax][0], aadv * (f * (JP - 27 * JM) - 4 * s) + avis * Gm[ax] * Nm[ax]);
                atomicAdd(aud + nbm[ax][1], aadv * (f * JM + s));
                atomicAdd(anut0 + cc, avis * 0.5 * (Gp[ax] * dp - Gm[ax] * dm));
                atomicAdd(anut0 + nbp[ax][0], avis * 0.5 * Gp[ax] * dp);
                atomicAdd(anut0 + nbm[ax][0], -avis * 0.5 * Gm[ax] * dm);
            }
        }
        for (int q = 0; q < 3; q++)
            if (aUa[q] != 0.0) atomicAdd(au0 + cc + q * N, aUa[q] * adj_sgn(Uc[q]) * mv.kx(q, idx[q]));
    }
}

// (1a) adjoint of the truncated Gaussian projection: one block per AP, summing
// aff eta exp(-r^2/eps^2) over the cells of its turbine's force box within the cutoff
__global__ void __launch_bounds__(256) k_adj_alm_project(Geom g, AlmDev a, const double *xc, const double *yc, const double *zc,
                                                         const double *aff, double *aF) {
    const long long N = g.n;
    const int ap = blockIdx.x;
    const int nappt = a.n_ap_per_blade * a.n_blade, tid = ap / nappt;
    const double eps = a.euler_eps, sq = sqrt(3.14159265358979323846) * eps, eta = 1. / (sq * sq * sq), e2 = eps * eps;
    const double px = a.ap_xyz[3 * ap], py = a.ap_xyz[3 * ap + 1], pz = a.ap_xyz[3 * ap + 2];
    int lo[3] = {0, 0, 0}, ex[3] = {0, 0, 0};
#pragma unroll
    for (int s = 0; s < kMaxTurbines; s++)
        if (s == tid) { for (int d = 0; d < 3; d++) { lo[d] = a.bs.lo[s][d]; ex[d] = a.bs.ext[s][d]; } }
    double acc[3] = {0, 0, 0};
    const long long tot = (long long)ex[0] * ex[1] * ex[2];
    for (long long q = threadIdx.x; q < tot; q += blockDim.x) {
        const int i = lo[0] + (int)(q % ex[0]), j = lo[1] + (int)((q / ex[0]) % ex[1]), k = lo[2] + (int)(q / ((long long)ex[0] * ex[1]));
        const double dx = xc[i] - px, dy = yc[j] - py, dz = zc[k] - pz;
        const double rr2 = dx * dx + dy * dy + dz * dz;
        if (rr2 < a.rcut2) {
            const double w = eta * exp(-rr2 / e2);
            const long long cc = g.id(i, j, k);
            acc[0] += aff[cc] * w; acc[1] += aff[cc + N] * w; acc[2] += aff[cc + 2 * N] * w;
        }
    }
    __shared__ double red[3][256];
    for (int d = 0; d < 3; d++) red[d][threadIdx.x] = acc[d];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int d = 0; d < 3; d++) red[d][threadIdx.x] += red[d][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; d++) aF[3 * ap + d] = red[d][0];
}

// (1b) per AP: recompute k_alm_force's chain and apply its transpose, plus the
// objective term wP * tip * |ft| * r; gradients: grad[0] pitch, grad[1 + ap]
// chord, grad[1 + apcount + ap] twist
template <typename T>
__global__ void __launch_bounds__(128) k_adj_alm_ap(Geom g, AlmDev a, const double *xc, const double *yc, const double *zc,
                                                    const T *u0, double t, const double *aF, double wP, double *au0,
                                                    double *grad) {
    const long long N = g.n;
    const int nappt = a.n_ap_per_blade * a.n_blade;
    const double dr = (a.radius - a.hub_radius) / a.n_ap_per_blade;
    const double Pi = 3.14159265358979323846;
    const int ap = blockIdx.x * blockDim.x + threadIdx.x;
    if (ap >= a.apcount) return;
    const int tid = ap / nappt, bid = (ap % nappt) / a.n_ap_per_blade;
    const int at = a.angle_type[tid];
    double angle[3] = {0, 0, 0}, angvel[3] = {0, 0, 0};
    const double *m = a.motion + 3 * tid;
    if (at) {
        angle[at - 1] = m[0] * sin(m[1] * t + m[2]);
        angvel[at - 1] = m[0] * m[1] * cos(m[1] * t + m[2]);
    }
    const double tip = a.tip_rate[tid];
    const double theta = tip * t + (2 * Pi / a.n_blade) * bid;
    const double apr = a.ap_r[ap];
    const double c1[3] = {a.hub[3 * tid], a.hub[3 * tid + 1] + apr * cos(theta), a.hub[3 * tid + 2] + apr * sin(theta)};
    const double nang[3] = {-angle[0], -angle[1], -angle[2]};
    double c0[3];
    rot(c1, nang, at, c0);
    for (int d = 0; d < 3; d++) c0[d] += a.base[3 * tid + d];
    const int I = find_index(xc, c0[0], g.sx), J = find_index(yc, c0[1], g.sy), K = find_index(zc, c0[2], g.sz);
    const bool inside = I >= g.gc - 1 && I < g.sx - g.gc - 1 && J >= g.gc - 1 && J < g.sy - g.gc - 1 && K >= g.gc - 1 && K < g.sz - g.gc - 1;
    if (!inside) return;
    const double xd = fabs(c0[0] - xc[I]) / fabs(xc[I + 1] - xc[I]);
    const double yd = fabs(c0[1] - yc[J]) / fabs(yc[J + 1] - yc[J]);
    const double zd = fabs(c0[2] - zc[K]) / fabs(zc[K + 1] - zc[K]);
    const long long id[8] = {g.id(I, J, K), g.id(I + 1, J, K), g.id(I, J + 1, K), g.id(I + 1, J + 1, K),
                             g.id(I, J, K + 1), g.id(I + 1, J, K + 1), g.id(I, J + 1, K + 1), g.id(I + 1, J + 1, K + 1)};
    const double wts[8] = {(1 - xd) * (1 - yd) * (1 - zd), xd * (1 - yd) * (1 - zd), (1 - xd) * yd * (1 - zd), xd * yd * (1 - zd),
                           (1 - xd) * (1 - yd) * zd, xd * (1 - yd) * zd, (1 - xd) * yd * zd, xd * yd * zd};
    double uvw[3];
    for (int d = 0; d < 3; d++) {
        const T *ud = u0 + d * N;
        const double c01 = to_d(ud[id[0]]) * (1. - xd) + to_d(ud[id[1]]) * xd, c23 = to_d(ud[id[2]]) * (1. - xd) + to_d(ud[id[3]]) * xd;
        const double c45 = to_d(ud[id[4]]) * (1. - xd) + to_d(ud[id[5]]) * xd, c67 = to_d(ud[id[6]]) * (1. - xd) + to_d(ud[id[7]]) * xd;
        uvw[d] = (c01 * (1. - yd) + c23 * yd) * (1. - zd) + (c45 * (1. - yd) + c67 * yd) * zd;
    }
    const double rel[3] = {c0[0] - a.base[3 * tid], c0[1] - a.base[3 * tid + 1], c0[2] - a.base[3 * tid + 2]};
    double tt[3], t0[3], M[3][3];
    const double zero[3] = {0, 0, 0};
    rot_dt(rel, uvw, angle, angvel, at, tt);
    rot_dt(rel, zero, angle, angvel, at, t0);   // uvw -> tt is affine: its matrix from unit vectors
    for (int q = 0; q < 3; q++) {
        double e[3] = {0, 0, 0}, o[3];
        e[q] = 1.0;
        rot_dt(rel, e, angle, angvel, at, o);
        for (int d = 0; d < 3; d++) M[d][q] = o[d] - t0[d];
    }
    const double ux = tt[0];
    const double ut = tip * apr + tt[1] * sin(theta) - tt[2] * cos(theta);
    const double urel2 = ux * ux + ut * ut;
    const double phi = atan(ux / ut);
    const double chord = a.ap_chord[ap], twist = a.ap_twist[ap] + a.pitch;
    const double attack = phi * 180. / Pi - twist;
    const int na = a.n_attack;
    double clv, cdv, slope_l = 0, slope_d = 0;
    if (attack < a.attack[0]) { clv = a.cl[ap]; cdv = a.cd[ap]; }
    else if (attack >= a.attack[na - 1]) { clv = a.cl[ap + (long long)(na - 1) * a.apcount]; cdv = a.cd[ap + (long long)(na - 1) * a.apcount]; }
    else {
        int lo = 0, hi = na - 1;
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (a.attack[mid] <= attack) lo = mid; else hi = mid; }
        const double dA = a.attack[lo + 1] - a.attack[lo];
        const double pw = (attack - a.attack[lo]) / dA;
        const double l0 = a.cl[ap + (long long)lo * a.apcount], l1 = a.cl[ap + (long long)(lo + 1) * a.apcount];
        const double d0 = a.cd[ap + (long long)lo * a.apcount], d1 = a.cd[ap + (long long)(lo + 1) * a.apcount];
        clv = (1. - pw) * l0 + pw * l1;
        cdv = (1. - pw) * d0 + pw * d1;
        slope_l = (l1 - l0) / dA;
        slope_d = (d1 - d0) / dA;
    }
    const double fl = .5 * clv * urel2 * chord * dr, fd = .5 * cdv * urel2 * chord * dr;
    const double s = sin(phi), co = cos(phi);
    const double sgn = (double)((tip > 0) - (tip < 0));
    const double ft = (fl * s - fd * s) * sgn;
    // force = R(nang) f_tt; the transpose of a single-axis rotation is the rotation by -nang
    double aftt[3];
    rot(aF + 3 * ap, angle, at, aftt);
    const double afx = -aftt[0];
    double aft = aftt[1] * sin(theta) - aftt[2] * cos(theta);
    aft += wP * tip * adj_sgn(ft) * apr;
    const double aft0 = aft * sgn;
    const double afl = afx * co + aft0 * s, afd = afx * s - aft0 * s;
    double aphi = afx * (-fl * s + fd * co) + aft0 * (fl - fd) * co;
    const double aclv = afl * .5 * urel2 * chord * dr, acdv = afd * .5 * urel2 * chord * dr;
    const double aurel2 = afl * .5 * clv * chord * dr + afd * .5 * cdv * chord * dr;
    const double achord = afl * .5 * clv * urel2 * dr + afd * .5 * cdv * urel2 * dr;
    const double aattack = aclv * slope_l + acdv * slope_d;
    aphi += aattack * 180. / Pi;
    atomicAdd(grad, -aattack);
    grad[1 + ap] += achord;
    grad[1 + a.apcount + ap] += -aattack;
    const double aux = aphi * ut / urel2 + 2 * ux * aurel2;
    const double aut = -aphi * ux / urel2 + 2 * ut * aurel2;
    const double att[3] = {aux, aut * sin(theta), -aut * cos(theta)};
    for (int d = 0; d < 3; d++) {
        const double auvw = M[0][d] * att[0] + M[1][d] * att[1] + M[2][d] * att[2];
        if (auvw != 0.0)
            for (int q = 0; q < 8; q++) atomicAdd(au0 + id[q] + d * N, auvw * wts[q]);
    }
}

}  // namespace fb
