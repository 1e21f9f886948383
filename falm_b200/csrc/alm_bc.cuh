// Actuator line model (src/alm/almDevCall.cu) and the application boundary
// kernels (app/nedo/bcdevcall.cu, app/windtunnel/bcdevcall.cu, app/lid3d/bcdev.cu).
#pragma once
#include "common.cuh"

namespace fb {

// ---------------------------------------------------------------- rotations (src/falmath.h:384-460)
__device__ inline void rot(const double *x, const double *angle, int type, double *o) {
    double X = x[0], Y = x[1], Z = x[2];
    if (type == 1) { double C = cos(angle[0]), S = sin(angle[0]); o[0] = X; o[1] = C * Y + S * Z; o[2] = -S * Y + C * Z; }
    else if (type == 2) { double C = cos(angle[1]), S = sin(angle[1]); o[0] = C * X - S * Z; o[1] = Y; o[2] = S * X + C * Z; }
    else if (type == 3) { double C = cos(angle[2]), S = sin(angle[2]); o[0] = C * X + S * Y; o[1] = -S * X + C * Y; o[2] = Z; }
    else { o[0] = X; o[1] = Y; o[2] = Z; }
}

__device__ inline void rot_dt(const double *x, const double *v, const double *angle, const double *om, int type, double *o) {
    double X = x[0], Y = x[1], Z = x[2], U = v[0], V = v[1], W = v[2];
    if (type == 1) {
        double C = cos(angle[0]), S = sin(angle[0]), O = om[0];
        o[0] = 0. + U; o[1] = O * (-S * Y + C * Z) + (C * V + S * W); o[2] = O * (-C * Y - S * Z) + (-S * V + C * W);
    } else if (type == 2) {
        double C = cos(angle[1]), S = sin(angle[1]), O = om[1];
        o[0] = O * (-S * X - C * Z) + (C * U - S * W); o[1] = 0. + V; o[2] = O * (C * X - S * Z) + (S * U + C * W);
    } else if (type == 3) {
        double C = cos(angle[2]), S = sin(angle[2]), O = om[2];
        o[0] = O * (-S * X + C * Y) + (C * U + S * V); o[1] = O * (-C * X - S * Y) + (-S * U + C * V); o[2] = 0. + W;
    } else { o[0] = U; o[1] = V; o[2] = W; }
}

// src/alm/almDevCall.cu:12-26 (a bisection gives the same index on a strictly
// increasing coordinate table)
__device__ inline int find_index(const double *seq, double v, int n) {
    if (v < seq[0]) return -1;
    if (v >= seq[n - 1]) return n - 1;
    int lo = 0, hi = n - 1;            // seq[lo] <= v < seq[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (seq[mid] <= v) lo = mid; else hi = mid;
    }
    return lo;
}

// One block evaluates every actuator point: UpdateTurbineAngles (:43-61),
// UpdateAPX (:63-129), CalcAPForce (:131-253), then CalcTorqueAndThrust
// (:362-370) and the AP bounding box used to truncate the projection.
// FP64 arithmetic in both precision modes (O(apcount) work).
// The cell-centre coordinates are staged in shared memory when `stage` (the
// bisections then run there), and the per-AP results the block reduces at the
// end are kept in shared memory too (up to kMaxFusedAp points).
template <typename T>
__global__ void __launch_bounds__(256) k_alm_force(Geom g, AlmDev a, const double *xc_g, const double *yc_g, const double *zc_g,
                                                 const T *__restrict__ u, double t_arg, int stage, const double *t_dev) {
    const double t = t_dev ? *t_dev : t_arg;   // a recorded step (CUDA graph) reads its time from device memory
    extern __shared__ double s_coord[];
    __shared__ double s_xyz[3 * kMaxFusedAp], s_tq[kMaxFusedAp], s_th[kMaxFusedAp];
    const bool keep = a.apcount <= kMaxFusedAp;
    const double *xc = xc_g, *yc = yc_g, *zc = zc_g;
    if (stage) {
        for (int q = threadIdx.x; q < g.sx; q += blockDim.x) s_coord[q] = xc_g[q];
        for (int q = threadIdx.x; q < g.sy; q += blockDim.x) s_coord[g.sx + q] = yc_g[q];
        for (int q = threadIdx.x; q < g.sz; q += blockDim.x) s_coord[g.sx + g.sy + q] = zc_g[q];
        __syncthreads();
        xc = s_coord; yc = s_coord + g.sx; zc = s_coord + g.sx + g.sy;
    }
    const long long N = g.n;
    const int nappt = a.n_ap_per_blade * a.n_blade;
    const double dr = (a.radius - a.hub_radius) / a.n_ap_per_blade;
    const double Pi = 3.14159265358979323846;
    for (int ap = threadIdx.x; ap < a.apcount; ap += blockDim.x) {
        int tid = ap / nappt, bid = (ap % nappt) / a.n_ap_per_blade;
        int at = a.angle_type[tid];
        double angle[3] = {0, 0, 0}, angvel[3] = {0, 0, 0};
        const double *m = a.motion + 3 * tid;
        if (at) {
            angle[at - 1] = m[0] * sin(m[1] * t + m[2]);
            angvel[at - 1] = m[0] * m[1] * cos(m[1] * t + m[2]);
        }
        double tip = a.tip_rate[tid];
        double theta = tip * t + (2 * Pi / a.n_blade) * bid;
        double apr = a.ap_r[ap];
        double c1[3] = {a.hub[3 * tid], a.hub[3 * tid + 1] + apr * cos(theta), a.hub[3 * tid + 2] + apr * sin(theta)};
        double nang[3] = {-angle[0], -angle[1], -angle[2]};
        double c0[3];
        rot(c1, nang, at, c0);
        for (int d = 0; d < 3; d++) c0[d] += a.base[3 * tid + d];
        for (int d = 0; d < 3; d++) a.ap_xyz[3 * ap + d] = c0[d];
        if (keep) for (int d = 0; d < 3; d++) s_xyz[3 * ap + d] = c0[d];
        int I = find_index(xc, c0[0], g.sx), J = find_index(yc, c0[1], g.sy), K = find_index(zc, c0[2], g.sz);
        // a slab evaluates the points whose lower interpolation plane K it owns:
        // its interior planes, and the guide plane below at a physical face
        const int klo = (g.zphys & 1) ? g.gc - 1 : g.gc, khi = (g.zphys & 2) ? g.sz - g.gc - 1 : g.sz - g.gc;
        bool inside = I >= g.gc - 1 && I < g.sx - g.gc - 1 && J >= g.gc - 1 && J < g.sy - g.gc - 1 && K >= klo && K < khi;
        if (!inside) {
            for (int d = 0; d < 3; d++) a.ap_force[3 * ap + d] = 0;
            a.ap_torque[ap] = 0; a.ap_thrust[ap] = 0;
            if (keep) { s_tq[ap] = 0; s_th[ap] = 0; }
            continue;
        }
        double xd = fabs(c0[0] - xc[I]) / fabs(xc[I + 1] - xc[I]);
        double yd = fabs(c0[1] - yc[J]) / fabs(yc[J + 1] - yc[J]);
        double zd = fabs(c0[2] - zc[K]) / fabs(zc[K + 1] - zc[K]);
        long long id0 = g.id(I, J, K), id1 = g.id(I + 1, J, K), id2 = g.id(I, J + 1, K), id3 = g.id(I + 1, J + 1, K);
        long long id4 = g.id(I, J, K + 1), id5 = g.id(I + 1, J, K + 1), id6 = g.id(I, J + 1, K + 1), id7 = g.id(I + 1, J + 1, K + 1);
        double uvw[3];
        for (int d = 0; d < 3; d++) {
            const T *ud = u + d * N;
            double c01 = to_d(ud[id0]) * (1. - xd) + to_d(ud[id1]) * xd;
            double c23 = to_d(ud[id2]) * (1. - xd) + to_d(ud[id3]) * xd;
            double c45 = to_d(ud[id4]) * (1. - xd) + to_d(ud[id5]) * xd;
            double c67 = to_d(ud[id6]) * (1. - xd) + to_d(ud[id7]) * xd;
            double c0123 = c01 * (1. - yd) + c23 * yd;
            double c4567 = c45 * (1. - yd) + c67 * yd;
            uvw[d] = c0123 * (1. - zd) + c4567 * zd;
        }
        double rel[3] = {c0[0] - a.base[3 * tid], c0[1] - a.base[3 * tid + 1], c0[2] - a.base[3 * tid + 2]};
        double utt[3];
        rot_dt(rel, uvw, angle, angvel, at, utt);
        double ux = utt[0];
        double ut = tip * apr + utt[1] * sin(theta) - utt[2] * cos(theta);
        double urel2 = ux * ux + ut * ut;
        double phi = atan(ux / ut);
        // src/alm/apHandler.h:121-141 (pitch offset is 0 for the reference's behaviour)
        double chord = a.ap_chord[ap], twist = a.ap_twist[ap] + a.pitch;
        double attack = phi * 180. / Pi - twist;
        const int na = a.n_attack;
        double clv = 0, cdv = 0;
        if (attack < a.attack[0]) { clv = a.cl[ap]; cdv = a.cd[ap]; }
        else if (attack >= a.attack[na - 1]) { clv = a.cl[ap + (long long)(na - 1) * a.apcount]; cdv = a.cd[ap + (long long)(na - 1) * a.apcount]; }
        else {
            int lo = 0, hi = na - 1;
            while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (a.attack[mid] <= attack) lo = mid; else hi = mid; }
            double pw = (attack - a.attack[lo]) / (a.attack[lo + 1] - a.attack[lo]);
            clv = (1. - pw) * a.cl[ap + (long long)lo * a.apcount] + pw * a.cl[ap + (long long)(lo + 1) * a.apcount];
            cdv = (1. - pw) * a.cd[ap + (long long)lo * a.apcount] + pw * a.cd[ap + (long long)(lo + 1) * a.apcount];
        }
        double fl = .5 * clv * urel2 * chord * dr;
        double fd = .5 * cdv * urel2 * chord * dr;
        double fx = fl * cos(phi) + fd * sin(phi);
        double ft = fl * sin(phi) - fd * sin(phi);        // src/alm/almDevCall.cu:239 (sic)
        ft *= (double)((tip > 0) - (tip < 0));
        double ftt[3] = {-fx, ft * sin(theta), -ft * cos(theta)};
        rot(ftt, nang, at, a.ap_force + 3 * ap);
        a.ap_torque[ap] = fabs(ft) * apr;
        a.ap_thrust[ap] = fx;
        if (keep) { s_tq[ap] = fabs(ft) * apr; s_th[ap] = fx; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double *pxyz = keep ? s_xyz : a.ap_xyz, *ptq = keep ? s_tq : a.ap_torque, *pth = keep ? s_th : a.ap_thrust;
        double bb[6] = {1e300, -1e300, 1e300, -1e300, 1e300, -1e300};
        for (int ap = 0; ap < a.apcount; ap++)
            for (int d = 0; d < 3; d++) {
                bb[2 * d] = fmin(bb[2 * d], pxyz[3 * ap + d]);
                bb[2 * d + 1] = fmax(bb[2 * d + 1], pxyz[3 * ap + d]);
            }
        for (int q = 0; q < 6; q++) a.scal->bbox[q] = bb[q];
        for (int tid = 0; tid < a.n_turbine && tid < kMaxTurbines; tid++) {
            double tq = 0, th = 0;
            for (int q = 0; q < nappt; q++) { tq += ptq[tid * nappt + q]; th += pth[tid * nappt + q]; }
            a.scal->torque[tid] = tq;
            a.scal->thrust[tid] = th;
        }
    }
}

// per-turbine torque and thrust from the per-AP arrays (CalcTorqueAndThrust,
// src/alm/almDevCall.cu:362-370), in the order k_alm_force sums them; run
// after the per-AP arrays were summed over the slabs of a decomposed grid
__global__ void k_alm_turbine_sums(AlmDev a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nappt = a.n_ap_per_blade * a.n_blade;
    for (int tid = 0; tid < a.n_turbine && tid < kMaxTurbines; tid++) {
        double tq = 0, th = 0;
        for (int q = 0; q < nappt; q++) { tq += a.ap_torque[tid * nappt + q]; th += a.ap_thrust[tid * nappt + q]; }
        a.scal->torque[tid] = tq;
        a.scal->thrust[tid] = th;
    }
}

// the cutoff test (double)v < r2 of a value v of type T as v < cut_bound<T>(r2):
// in FP32 the bound is the smallest float not below r2 (rounded up), so both
// tests agree for every float v
template <typename T>
__device__ __forceinline__ T cut_bound(double r2) {
    if constexpr (sizeof(T) == 4) return __double2float_ru(r2);
    else return r2;
}

// the APs' positions and forces, converted to T once per block
template <typename T>
__device__ __forceinline__ void stage_aps(const AlmDev &a, T *s_ap) {
    for (int q = threadIdx.x; q < a.apcount; q += blockDim.x) {
        for (int d = 0; d < 3; d++) { s_ap[6 * q + d] = (T)a.ap_xyz[3 * q + d]; s_ap[6 * q + 3 + d] = (T)a.ap_force[3 * q + d]; }
    }
}

// DistributeAPForce (src/alm/almDevCall.cu:255-294) as a stored field, truncated at rcut
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_alm_project(Geom g, Region3 R, MetricView<T> mv, AlmDev a, T *__restrict__ ff) {
    __shared__ T s_ap[6 * kMaxFusedAp];
    const int na = a.apcount;
    stage_aps<T>(a, s_ap);
    __syncthreads();
    const T rcut2 = cut_bound<T>(a.rcut2);
    const double eps = a.euler_eps, sq = sqrt(3.14159265358979323846) * eps, eta = 1. / (sq * sq * sq);
    const long long N = g.n;
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        T cx = ldg(mv.m.x[0] + i), cy = ldg(mv.m.x[1] + j), cz = ldg(mv.m.x[2] + k);
        T fx = 0, fy = 0, fz = 0;
        const T te = (T)eta, e2 = (T)eps * (T)eps;
        for (int q = 0; q < na; q++) {
            T dx = cx - s_ap[6 * q], dy = cy - s_ap[6 * q + 1], dz = cz - s_ap[6 * q + 2];
            T rr2 = dx * dx + dy * dy + dz * dz;
            if (rr2 < rcut2) {
                T ex = exp(-rr2 / e2);
                fx += s_ap[6 * q + 3] * te * ex;
                fy += s_ap[6 * q + 4] * te * ex;
                fz += s_ap[6 * q + 5] * te * ex;
            }
        }
        ff[c] = fx; ff[c + N] = fy; ff[c + 2 * N] = fz;
    }
}

// The same truncated Gaussian sum for the cells of the force boxes only; cells
// farther than the cutoff from the AP bounding box get zero without the AP loop.
template <typename T>
__global__ void __launch_bounds__(256) k_alm_box(AlmDev a, const double *xc, const double *yc, const double *zc) {
    __shared__ T s_ap[6 * kMaxFusedAp];
    const int na = a.apcount;
    stage_aps<T>(a, s_ap);
    __syncthreads();
    const T rcut2 = cut_bound<T>(a.rcut2);
    const double eps = a.euler_eps, sq = sqrt(3.14159265358979323846) * eps, eta = 1. / (sq * sq * sq);
    const double *bb = a.scal->bbox;
    const double b0 = bb[0], b1 = bb[1], b2 = bb[2], b3 = bb[3], b4 = bb[4], b5 = bb[5];
    // force boxes hold far fewer than 2^31 cells: 32-bit index arithmetic
    const int tot = (int)a.bs.total;
    T *f = (T *)a.fbox;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) {
        int l0 = 0, l1 = 0, l2 = 0, e0 = 1, e1 = 1, o = 0;
#pragma unroll
        for (int s = 0; s < kMaxTurbines; s++)
            if (s < a.bs.n && q >= a.bs.off[s]) {
                l0 = a.bs.lo[s][0]; l1 = a.bs.lo[s][1]; l2 = a.bs.lo[s][2];
                e0 = a.bs.ext[s][0]; e1 = a.bs.ext[s][1]; o = (int)a.bs.off[s];
            }
        int r = q - o;
        const int i = l0 + r % e0;
        r /= e0;
        const int j = l1 + r % e1, k = l2 + r / e1;
        const double cxd = xc[i], cyd = yc[j], czd = zc[k];
        T fx = 0, fy = 0, fz = 0;
        if (box_dist2(cxd, b0, b1) + box_dist2(cyd, b2, b3) + box_dist2(czd, b4, b5) < a.rcut2) {
            const T cx = (T)cxd, cy = (T)cyd, cz = (T)czd;
            const T te = (T)eta, e2 = (T)eps * (T)eps;
            for (int p = 0; p < na; p++) {
                T dx = cx - s_ap[6 * p], dy = cy - s_ap[6 * p + 1], dz = cz - s_ap[6 * p + 2];
                T rr2 = dx * dx + dy * dy + dz * dz;
                if (rr2 < rcut2) {
                    T ex = exp(-rr2 / e2);
                    fx += s_ap[6 * p + 3] * te * ex;
                    fy += s_ap[6 * p + 4] * te * ex;
                    fz += s_ap[6 * p + 5] * te * ex;
                }
            }
        }
        f[q] = fx; f[q + tot] = fy; f[q + 2 * tot] = fz;
    }
}

// ---------------------------------------------------------------- boundary conditions
// previous-velocity view for the convective outlet: full field or the
// compact 3-plane copy [d][plane][k][j], planes i = sx-gc-2, sx-gc-1, sx-gc
template <typename T>
struct UPrev {
    const T *p;
    int compact;
    __device__ __forceinline__ T at(const Geom &g, int d, int i, int j, int k) const {
        if (!compact) return p[g.id(i, j, k) + d * g.n];
        int pl = i - (g.sx - g.gc - 2);
        return p[(((long long)d * 3 + pl) * g.sz + k) * g.sy + j];
    }
};

template <typename T>
__global__ void k_save_outlet(Geom g, const T *__restrict__ u, T *__restrict__ out) {
    // one thread per (j, k, d): the three outlet-side cells are adjacent in x
    const int ns = g.sy * g.sz, tot = 3 * ns;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) {
        const int d = q / ns, jk = q - d * ns;
        const int j = jk % g.sy, k = jk / g.sy;
        const T *src = u + g.id(g.sx - g.gc - 2, j, k) + d * g.n;
        const T v0 = src[0], v1 = src[1], v2 = src[2];
        T *o = out + (long long)(3 * d) * ns + jk;
        o[0] = v0; o[ns] = v1; o[2 * ns] = v2;
    }
}

struct Inflow {
    const double *box;    // 3 x nb x nzi x nyi, or NULL
    int nb;
    double dx;
    const double *plane;  // streamed inlet velocity 3 x nzi x nyi for this call, or NULL
};

// ubc: blockIdx.y selects the x, y or z face pair; every face writes only its
// own guide cells and reads interior cells, so the three pairs are independent
// (the reference launches them on six concurrent streams).
template <typename T>
__global__ void k_ubc(Geom g, int kind, T *u, UPrev<T> up, const double *xc, double dt, double t_arg, double u_inlet, Inflow inf,
                      const double *t_dev) {
    const double t = t_dev ? *t_dev : t_arg;   // a recorded step (CUDA graph) reads its time from device memory
    const long long N = g.n;
    const int gc = g.gc, sx = g.sx, sy = g.sy, sz = g.sz;
    const int pair = blockIdx.y;
    const int na = pair == 0 ? sy - 2 * gc : sx - 2 * gc;
    const int nb = pair == 2 ? sy - 2 * gc : sz - 2 * gc;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na * nb; q += gridDim.x * blockDim.x) {
        const int a = q % na + gc, b = q / na + gc;
        if (kind == FALM_BC_CHANNEL) {
            if (pair == 0) {
                int j = a, k = b;
                double ub[3] = {u_inlet, 0.0, 0.0};
                if (inf.plane) {
                    long long plane = (long long)(sy - 2 * gc) * (sz - 2 * gc), jk = (j - gc) + (long long)(k - gc) * (sy - 2 * gc);
                    for (int d = 0; d < 3; d++) ub[d] = inf.plane[d * plane + jk];
                } else if (inf.box) {   // seeded inflow (no reference counterpart): frozen turbulence at x = U t
                    double xs = u_inlet * t / inf.dx, fl = floor(xs), fr = xs - fl;
                    long long s = (long long)fl % inf.nb;
                    if (s < 0) s += inf.nb;
                    int s0 = (int)s, s1 = (s0 + 1) % inf.nb;
                    // the box covers the whole grid's inlet plane (a slab reads its own planes)
                    long long plane = (long long)(sy - 2 * gc) * g.nzg, jk = (j - gc) + (long long)(k - gc + g.koff) * (sy - 2 * gc);
                    for (int d = 0; d < 3; d++) {
                        const double *bx = inf.box + (long long)d * inf.nb * plane;
                        ub[d] += (1.0 - fr) * bx[s0 * plane + jk] + fr * bx[s1 * plane + jk];
                    }
                }
                // inlet, app/windtunnel/bcdevcall.cu:8-22
                for (int d = 0; d < 3; d++) { u[g.id(gc - 1, j, k) + d * N] = (T)ub[d]; u[g.id(gc - 2, j, k) + d * N] = (T)ub[d]; }
                // convective outlet, app/nedo/bcdevcall.cu:25-43
                int i = sx - gc;
                double dxi = 1.0 / (xc[i] - xc[i - 1]);
                for (int d = 0; d < 3; d++) {
                    T uo1 = up.at(g, d, i, j, k), ui1 = up.at(g, d, i - 1, j, k), ui2 = up.at(g, d, i - 2, j, k);
                    T du = T(0.5) * (T)dxi * (T(3) * uo1 - T(4) * ui1 + ui2);
                    T ubc = uo1 - (T)dt * du;
                    u[g.id(i, j, k) + d * N] = ubc;
                    u[g.id(i + 1, j, k) + d * N] = T(2) * ubc - u[g.id(i - 1, j, k) + d * N];
                }
            } else if (pair == 1) {
                int i = a, k = b;   // slip y-, y+ (:46-79)
                long long in = g.id(i, gc, k);
                T v0[3] = {u[in], T(0), u[in + 2 * N]};
                for (int d = 0; d < 3; d++) { u[g.id(i, gc - 1, k) + d * N] = v0[d]; u[g.id(i, gc - 2, k) + d * N] = T(2) * v0[d] - u[in + d * N]; }
                in = g.id(i, sy - gc - 1, k);
                T v1[3] = {u[in], T(0), u[in + 2 * N]};
                for (int d = 0; d < 3; d++) { u[g.id(i, sy - gc, k) + d * N] = v1[d]; u[g.id(i, sy - gc + 1, k) + d * N] = T(2) * v1[d] - u[in + d * N]; }
            } else {
                int i = a, j = b;   // no-slip z- (:82-97), slip z+ (:100-115); slab interfaces are left alone
                long long in = g.id(i, j, gc);
                if (g.zphys & 1)
                    for (int d = 0; d < 3; d++) { u[g.id(i, j, gc - 1) + d * N] = T(0); u[g.id(i, j, gc - 2) + d * N] = T(2) * T(0) - u[in + d * N]; }
                in = g.id(i, j, sz - gc - 1);
                T w1[3] = {u[in], u[in + N], T(0)};
                if (g.zphys & 2)
                    for (int d = 0; d < 3; d++) { u[g.id(i, j, sz - gc) + d * N] = w1[d]; u[g.id(i, j, sz - gc + 1) + d * N] = T(2) * w1[d] - u[in + d * N]; }
            }
        } else {
            // cavity, app/lid3d/bcdev.cu:11-105: reflection about the wall value, lid on y+
            const T lid[3] = {T(1.0), T(0.0), T(0.0)};
            for (int d = 0; d < 3; d++) {
                T *ud = u + d * N;
                if (pair == 0) {
                    int j = a, k = b;
                    ud[g.id(gc - 1, j, k)] = T(2) * T(0) - ud[g.id(gc, j, k)];
                    ud[g.id(gc - 2, j, k)] = T(2) * T(0) - ud[g.id(gc + 1, j, k)];
                    ud[g.id(sx - gc, j, k)] = T(2) * T(0) - ud[g.id(sx - gc - 1, j, k)];
                    ud[g.id(sx - gc + 1, j, k)] = T(2) * T(0) - ud[g.id(sx - gc - 2, j, k)];
                } else if (pair == 1) {
                    int i = a, k = b;
                    ud[g.id(i, gc - 1, k)] = T(2) * T(0) - ud[g.id(i, gc, k)];
                    ud[g.id(i, gc - 2, k)] = T(2) * T(0) - ud[g.id(i, gc + 1, k)];
                    ud[g.id(i, sy - gc, k)] = T(2) * lid[d] - ud[g.id(i, sy - gc - 1, k)];
                    ud[g.id(i, sy - gc + 1, k)] = T(2) * lid[d] - ud[g.id(i, sy - gc - 2, k)];
                } else {
                    int i = a, j = b;
                    if (g.zphys & 1) {
                        ud[g.id(i, j, gc - 1)] = T(2) * T(0) - ud[g.id(i, j, gc)];
                        ud[g.id(i, j, gc - 2)] = T(2) * T(0) - ud[g.id(i, j, gc + 1)];
                    }
                    if (g.zphys & 2) {
                        ud[g.id(i, j, sz - gc)] = T(2) * T(0) - ud[g.id(i, j, sz - gc - 1)];
                        ud[g.id(i, j, sz - gc + 1)] = T(2) * T(0) - ud[g.id(i, j, sz - gc - 2)];
                    }
                }
            }
        }
    }
}

// pbc: app/nedo/bcdevcall.cu:153-211 (p = 0 on x+), app/lid3d/bcdev.cu:143-213
template <typename T>
__global__ void k_pbc(Geom g, int kind, T *p) {
    const int gc = g.gc, sx = g.sx, sy = g.sy, sz = g.sz;
    const int pair = blockIdx.y;
    const int na = pair == 0 ? sy - 2 * gc : sx - 2 * gc;
    const int nb = pair == 2 ? sy - 2 * gc : sz - 2 * gc;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na * nb; q += gridDim.x * blockDim.x) {
        const int a = q % na + gc, b = q / na + gc;
        if (pair == 0) {
            p[g.id(gc - 1, a, b)] = p[g.id(gc, a, b)];
            p[g.id(sx - gc, a, b)] = kind == FALM_BC_CHANNEL ? T(0.0) : p[g.id(sx - gc - 1, a, b)];
        } else if (pair == 1) {
            p[g.id(a, gc - 1, b)] = p[g.id(a, gc, b)];
            p[g.id(a, sy - gc, b)] = p[g.id(a, sy - gc - 1, b)];
        } else {
            if (g.zphys & 1) p[g.id(a, b, gc - 1)] = p[g.id(a, b, gc)];
            if (g.zphys & 2) p[g.id(a, b, sz - gc)] = p[g.id(a, b, sz - gc - 1)];
        }
    }
}

// uubc: app/lid3d/bcdev.cu:251-322
template <typename T>
__global__ void k_uubc(Geom g, T *uu) {
    const int gc = g.gc, sx = g.sx, sy = g.sy, sz = g.sz;
    const int pair = blockIdx.y;
    const int na = pair == 0 ? sy - 2 * gc : sx - 2 * gc;
    const int nb = pair == 2 ? sy - 2 * gc : sz - 2 * gc;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na * nb; q += gridDim.x * blockDim.x) {
        const int a = q % na + gc, b = q / na + gc;
        if (pair == 0) { uu[g.id(gc - 1, a, b)] = T(0); uu[g.id(sx - gc - 1, a, b)] = T(0); }
        else if (pair == 1) { uu[g.id(a, gc - 1, b) + g.n] = T(0); uu[g.id(a, sy - gc - 1, b) + g.n] = T(0); }
        else {
            if (g.zphys & 1) uu[g.id(a, b, gc - 1) + 2 * g.n] = T(0);
            if (g.zphys & 2) uu[g.id(a, b, sz - gc - 1) + 2 * g.n] = T(0);
        }
    }
}

}  // namespace fb
