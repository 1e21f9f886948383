// RMCP rotor model (src/rmcp/): the reference's alternate rotor forcing, in
// which the rotating blades of each turbine paint the cells they cover and
// every painted cell gets the blade-element force of its own velocity (no
// actuator points, no Gaussian projection).  The class surface is
// Rmcp::RmcpAlm (src/rmcp/alm.h:13-96) with its TurbineHandler and
// BladeHandler (turbineHandler.h:13-185, bladeHandler.h:11-185); the kernels
// restated here are kernel_SetALMFlag (almDevCall.cu:13-65) and kernel_ALM
// (:144-209) of that turbine description.
//
// One kernel runs over the cells of a per-turbine box (the cells within
// |hub| + radius + blade thickness of the turbine's base, which bounds every
// painted point since the turbine frame only rotates about the base): it
// tests the paint, evaluates the force where painted, writes the force field
// there (zero elsewhere in the box; the caller keeps the rest of the field at
// zero) and reduces each turbine's torque and thrust deterministically.
#pragma once
#include "common.cuh"
#include "alm_bc.cuh"

namespace fb {

struct RmcpDev {
    int n_turbine, n_blade, n_station, n_attack;
    double radius, hub_radius, width, thick;
    const double *base, *hub, *angle, *tip_rate;   // 3, 3, 3, 1 per turbine
    const int *angle_type;
    const double *st_r, *st_chord, *st_twist, *attack, *cl, *cd;
    BoxSet bs;
};

// bladeHandler.h:83-96 (a linear scan: -1 below the table, n - 1 at or above its end)
__device__ inline int rmcp_find(const double *m, double x, int n) {
    if (x < m[0]) return -1;
    if (x >= m[n - 1]) return n - 1;
    for (int i = 0; i < n - 1; i++)
        if (m[i] <= x && m[i + 1] > x) return i;
    return -2;
}

// bladeHandler.h:98-107
__device__ inline double rmcp_interp(const double *m, const double *d, double x, int i, int n) {
    if (i < 0) return d[0];
    if (i >= n - 1) return d[n - 1];
    const double p = (x - m[i]) / (m[i + 1] - m[i]);
    return (1. - p) * d[i] + p * d[i + 1];
}

// bladeHandler.h:109-131: chord and twist at radius r, lift and drag at the
// attack angle phi - twist, interpolated between the two stations around r
__device__ inline void rmcp_airfoil(const RmcpDev &a, double r, double phi, double &chord, double &twist, double &cl, double &cd) {
    const int nr = a.n_station, na = a.n_attack;
    const int rid = rmcp_find(a.st_r, r, nr);
    chord = rmcp_interp(a.st_r, a.st_chord, r, rid, nr);
    twist = rmcp_interp(a.st_r, a.st_twist, r, rid, nr);
    const double attack = phi - twist;
    const int aid = rmcp_find(a.attack, attack, na);
    if (rid < 0) {
        cl = rmcp_interp(a.attack, a.cl, attack, aid, na);
        cd = rmcp_interp(a.attack, a.cd, attack, aid, na);
    } else if (rid >= nr - 1) {
        cl = rmcp_interp(a.attack, a.cl + (long long)(nr - 1) * na, attack, aid, na);
        cd = rmcp_interp(a.attack, a.cd + (long long)(nr - 1) * na, attack, aid, na);
    } else {
        const double p = (r - a.st_r[rid]) / (a.st_r[rid + 1] - a.st_r[rid]);
        const double cl0 = rmcp_interp(a.attack, a.cl + (long long)rid * na, attack, aid, na);
        const double cl1 = rmcp_interp(a.attack, a.cl + (long long)(rid + 1) * na, attack, aid, na);
        const double cd0 = rmcp_interp(a.attack, a.cd + (long long)rid * na, attack, aid, na);
        const double cd1 = rmcp_interp(a.attack, a.cd + (long long)(rid + 1) * na, attack, aid, na);
        cl = (1. - p) * cl0 + p * cl1;
        cd = (1. - p) * cd0 + p * cd1;
    }
}

// the paint of a point at time t (almDevCall.cu:13-65): turbine + 1 of the
// last turbine whose blade strip (width `width` about the blade axis,
// thickness `thick` downstream of the rotor plane, hub_radius < r <= radius)
// holds it, else 0
__device__ inline int rmcp_flag(const RmcpDev &a, const double (&point)[3], double t) {
    const double Pi = 3.14159265358979323846;
    const int Nb = a.n_blade;
    int f = 0;
    for (int tid = 0; tid < a.n_turbine; tid++) {
        const double d0[3] = {point[0] - a.base[3 * tid], point[1] - a.base[3 * tid + 1], point[2] - a.base[3 * tid + 2]};
        double d[3];
        rot(d0, a.angle + 3 * tid, a.angle_type[tid], d);
        for (int q = 0; q < 3; q++) d[q] -= a.hub[3 * tid + q];
        const double dx = d[0], dy = d[1], dz = d[2];
        const double rr = sqrt(dy * dy + dz * dz);
        double th = atan2(dz, dy);
        if (th < 0) th += 2 * Pi;
        const double rt = a.tip_rate[tid] * t;
        for (int bid = 0; bid < Nb; bid++) {
            const double rtblade = rt + (bid * 2. / Nb) * Pi;
            const double xm = th - rtblade, thblade = xm - floor(xm / (2. * Pi)) * (2. * Pi);   // floormod (src/falmath.h:20-22)
            bool isblade = (rr <= a.radius && rr > a.hub_radius);
            isblade = isblade && (thblade >= (Nb - 1) * Pi / (Nb * 2)) && (thblade <= (Nb + 1) * Pi / (Nb * 2));
            isblade = isblade && (rr <= a.width / (2 * cos(thblade)) || rr <= a.width / (2 * cos(thblade + Pi)));
            isblade = isblade && dx >= 0 && dx < a.thick;
            if (isblade) f = tid + 1;
        }
    }
    return f;
}

// the force of a painted point (almDevCall.cu:144-209); r, |tangential| and
// |axial| force for the turbine sums
__device__ inline void rmcp_force(const RmcpDev &a, int tid, const double (&point)[3], const double (&u)[3], double (&f)[3], double &rr,
                                  double &fft, double &ffx) {
    const double Pi = 3.14159265358979323846;
    const double xyz0[3] = {point[0] - a.base[3 * tid], point[1] - a.base[3 * tid + 1], point[2] - a.base[3 * tid + 2]};
    double xyz[3], uvw[3];
    const double omega0[3] = {0, 0, 0};
    rot(xyz0, a.angle + 3 * tid, a.angle_type[tid], xyz);
    // the velocity is turned with the rotated position (sic), at zero angular velocity
    rot_dt(xyz, u, a.angle + 3 * tid, omega0, a.angle_type[tid], uvw);
    const double dy = xyz[1] - a.hub[3 * tid + 1], dz = xyz[2] - a.hub[3 * tid + 2];
    const double th = atan2(dz, dy);
    rr = sqrt(dy * dy + dz * dz);
    const double ux = uvw[0];
    const double ut = a.tip_rate[tid] * rr + uvw[1] * sin(th) - uvw[2] * cos(th);
    const double urel2 = ux * ux + ut * ut;
    const double phi = atan(ux / ut);
    double chord, twist, cl, cd;
    rmcp_airfoil(a, rr, phi * 180. / Pi, chord, twist, cl, cd);
    const double ps = (rr > a.width) ? asin(0.5 * a.width / rr) : 0.5 * Pi / a.n_blade;
    const double Cf = 0.5 * chord / (2 * rr * ps * a.thick);
    ffx = fabs((cl * cos(phi) + cd * sin(phi)) * Cf * urel2);
    fft = fabs((cl * sin(phi) - cd * cos(phi)) * Cf * urel2);
    const double loc[3] = {-ffx, fft * sin(th), -fft * cos(th)};
    const double nang[3] = {-a.angle[3 * tid], -a.angle[3 * tid + 1], -a.angle[3 * tid + 2]};
    rot(loc, nang, a.angle_type[tid], f);
}

// Over the cells of the boxes (a cell in several boxes is handled by the
// first): ff at the cell (zero where not painted), the paint in `flag` when
// given, and the sums of r |f_t| (torque) and |f_x| (thrust) per turbine into
// sums[0..kMaxTurbines) and sums[kMaxTurbines..2 kMaxTurbines).
template <typename T>
__global__ void __launch_bounds__(256) k_rmcp(Geom g, RmcpDev a, const double *xc, const double *yc, const double *zc,
                                              const T *__restrict__ u, T *__restrict__ ff, int *flag, double t_arg, RedWork rw,
                                              double *sums, const double *t_dev) {
    const double t = t_dev ? *t_dev : t_arg;   // a recorded step (CUDA graph) reads its time from device memory
    double acc[2 * kMaxTurbines];
#pragma unroll
    for (int q = 0; q < 2 * kMaxTurbines; q++) acc[q] = 0.0;
    const long long tot = a.bs.total;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int s = 0;
#pragma unroll
        for (int b = 0; b < kMaxTurbines; b++)
            if (b < a.bs.n && q >= a.bs.off[b]) s = b;
        long long r = q - a.bs.off[s];
        const int i = a.bs.lo[s][0] + (int)(r % a.bs.ext[s][0]);
        r /= a.bs.ext[s][0];
        const int j = a.bs.lo[s][1] + (int)(r % a.bs.ext[s][1]), k = a.bs.lo[s][2] + (int)(r / a.bs.ext[s][1]);
        bool first = true;
        for (int b = 0; b < s; b++)
            if ((unsigned)(i - a.bs.lo[b][0]) < (unsigned)a.bs.ext[b][0] && (unsigned)(j - a.bs.lo[b][1]) < (unsigned)a.bs.ext[b][1] &&
                (unsigned)(k - a.bs.lo[b][2]) < (unsigned)a.bs.ext[b][2])
                first = false;
        if (!first) continue;
        const long long c = g.id(i, j, k);
        const double point[3] = {xc[i], yc[j], zc[k]};
        const int f = rmcp_flag(a, point, t);
        if (flag) flag[c] = f;
        double fv[3] = {0, 0, 0};
        if (f > 0) {
            const double uv[3] = {to_d(u[c]), to_d(u[c + g.n]), to_d(u[c + 2 * g.n])};
            double rr, fft, ffx;
            rmcp_force(a, f - 1, point, uv, fv, rr, fft, ffx);
#pragma unroll
            for (int tq = 0; tq < kMaxTurbines; tq++)
                if (tq == f - 1) { acc[tq] += rr * fft; acc[kMaxTurbines + tq] += ffx; }
        }
        ff[c] = (T)fv[0]; ff[c + g.n] = (T)fv[1]; ff[c + 2 * g.n] = (T)fv[2];
    }
    double tot2[2 * kMaxTurbines];
    if (grid_sum<2 * kMaxTurbines>(acc, rw, tot2) && threadIdx.x == 0)
        for (int q = 0; q < 2 * kMaxTurbines; q++) sums[q] = tot2[q];
}

}  // namespace fb
