// FalmEq / FalmMV kernels: 7-point operator, residual, red-black SOR and
// Jacobi sweeps, and the right-preconditioned BiCGStab of src/FalmEq.cpp:305-410
// restructured so that every inner product is reduced on the device inside the
// kernel that produces its operands, and the scalars (alpha, beta, omega, rho,
// err) never leave the device:
//
//   k_bicg_p   p = r + beta(p - omega q); first SOR half-sweep of pp from zero
//   k_sor      remaining half-sweeps of the preconditioner
//   k_mv_dot1  q = A pp,  alpha = rho / (rr.q)
//   k_bicg_s   s = r - alpha q; first half-sweep of ss from zero
//   k_sor      ...
//   k_mv_dot2  t = A ss,  omega = (t.s)/(t.t)
//   k_bicg_xr  x += alpha pp + omega ss; r = s - omega t; ||r||, next rho, beta, stop test
//
// The first half-sweep of SOR from a zero start is pointwise (all neighbours
// are zero), so it is folded into the kernel that produces its right-hand side.
// Every kernel starts by reading the device `done` flag, so iterations can be
// queued ahead of the host's convergence check.
#pragma once
#include "common.cuh"

namespace fb {

// Poisson operator.  The reference stores 7 planes (src/falm.h:415); here the
// coefficients are separable 1D tables (a Cartesian control volume's face
// coefficient 0.5*(g_c+g_nb)/ja depends on one index only), or an explicit
// caller-owned 7-column matrix for general systems.
template <typename T>
struct Coef7 { T ac, aw, ae, as, an, ab, at; };

template <typename T>
struct Op7 {
    PoissonTables<T> t;
    const T *A;
    long long n;
    // x/y part of the table operator of one (i, j) column (hoisted out of a z
    // march): the four in-plane coefficients and the first three terms of the
    // diagonal's accumulation, so that at_col() rebuilds get() bit for bit
    struct Col { T aw, ae, as, an, dxy; };
    __device__ __forceinline__ Col column(int i, int j) const {
        Col r;
        if (A) { r.aw = r.ae = r.as = r.an = r.dxy = T(0); return r; }
        r.aw = ldg(t.cm[0] + i); r.ae = ldg(t.cp[0] + i);
        r.as = ldg(t.cm[1] + j); r.an = ldg(t.cp[1] + j);
        r.dxy = (ldg(t.dx0 + i) - ldg(t.up[1] + j)) - ldg(t.um[1] + j);
        return r;
    }
    __device__ __forceinline__ Coef7<T> at_col(const Col &cl, int k, long long c) const {
        Coef7<T> r;
        if (A) {
            r.ac = A[c]; r.aw = A[c + n]; r.ae = A[c + 2 * n]; r.as = A[c + 3 * n];
            r.an = A[c + 4 * n]; r.ab = A[c + 5 * n]; r.at = A[c + 6 * n];
        } else {
            r.aw = cl.aw; r.ae = cl.ae; r.as = cl.as; r.an = cl.an;
            r.ab = ldg(t.cm[2] + k); r.at = ldg(t.cp[2] + k);
            r.ac = ((cl.dxy - ldg(t.up[2] + k)) - ldg(t.um[2] + k)) * t.scale;
        }
        return r;
    }
    // z part of the table operator of one plane, shared by every column of a
    // tile: with a column's Col it gives at_col()'s coefficients
    struct ZPl { T ab, at, zp, zm; };
    __device__ __forceinline__ ZPl zplane(int k) const {
        ZPl z;
        if (A) { z.ab = z.at = z.zp = z.zm = T(0); return z; }
        z.ab = ldg(t.cm[2] + k); z.at = ldg(t.cp[2] + k); z.zp = ldg(t.up[2] + k); z.zm = ldg(t.um[2] + k);
        return z;
    }
    __device__ __forceinline__ T ac_col(const Col &cl, const ZPl &z) const { return ((cl.dxy - z.zp) - z.zm) * t.scale; }
    __device__ __forceinline__ void get(int i, int j, int k, long long c, T &ac, T &aw, T &ae, T &as, T &an, T &ab,
                                        T &at) const {
        if (A) {
            ac = A[c]; aw = A[c + n]; ae = A[c + 2 * n]; as = A[c + 3 * n];
            an = A[c + 4 * n]; ab = A[c + 5 * n]; at = A[c + 6 * n];
        } else {
            aw = ldg(t.cm[0] + i); ae = ldg(t.cp[0] + i);
            as = ldg(t.cm[1] + j); an = ldg(t.cp[1] + j);
            ab = ldg(t.cm[2] + k); at = ldg(t.cp[2] + k);
            // app/nedo/main.cpp:54-83 accumulates ac -= e, w, n, s, t, b in this order, then scales
            ac = ((((ldg(t.dx0 + i) - ldg(t.up[1] + j)) - ldg(t.um[1] + j)) - ldg(t.up[2] + k)) - ldg(t.um[2] + k)) * t.scale;
        }
    }
    __device__ __forceinline__ T diag(int i, int j, int k, long long c) const {
        if (A) return A[c];
        return ((((ldg(t.dx0 + i) - ldg(t.up[1] + j)) - ldg(t.um[1] + j)) - ldg(t.up[2] + k)) - ldg(t.um[2] + k)) * t.scale;
    }
    // the four terms of the diagonal's accumulation that are fixed along an x
    // row (j, k), so that diag_row() rebuilds diag() bit for bit
    struct RowD { T yp, ym, zp, zm; };
    __device__ __forceinline__ RowD row(int j, int k) const {
        RowD r;
        if (A) { r.yp = r.ym = r.zp = r.zm = T(0); return r; }
        r.yp = ldg(t.up[1] + j); r.ym = ldg(t.um[1] + j); r.zp = ldg(t.up[2] + k); r.zm = ldg(t.um[2] + k);
        return r;
    }
    __device__ __forceinline__ T diag_row(const RowD &rd, int i, long long c) const {
        if (A) return A[c];
        return ((((ldg(t.dx0 + i) - rd.yp) - rd.ym) - rd.zp) - rd.zm) * t.scale;
    }
};

// the SOR / Jacobi correction (b - Ax)/ac: IEEE division in FP64; in FP32
// (mixed precision) the numerator times the hardware reciprocal approximation
// (PTX rcp.approx, 1 ulp), within 2 ulp of the quotient
__device__ __forceinline__ float rcp_approx(float b) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    return r;
}
__device__ __forceinline__ double sor_div(double a, double b) { return a / b; }
__device__ __forceinline__ float sor_div(float a, float b) { return a * rcp_approx(b); }

// ac*xc + ae*xe + aw*xw + an*xn + as*xs + at*xt + ab*xb  (src/dev/MVDevCall.cu:181)
template <typename T, typename A>
__device__ __forceinline__ A apply7(const Op7<T> &op, const Geom &g, int i, int j, int k, long long c, const T *x) {
    T ac, aw, ae, as, an, ab, at;
    op.get(i, j, k, c, ac, aw, ae, as, an, ab, at);
    const long long sxy = (long long)g.sx * g.sy;
    return (A)ac * (A)x[c] + (A)ae * (A)x[c + 1] + (A)aw * (A)x[c - 1] + (A)an * (A)x[c + g.sx] +
           (A)as * (A)x[c - g.sx] + (A)at * (A)x[c + sxy] + (A)ab * (A)x[c - sxy];
}

// ---------------------------------------------------------------- generic MV / dot / norm
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_mv(Geom g, Region3 R, Op7<T> op, const T *__restrict__ x, T *__restrict__ ax) {
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        ax[c] = apply7<T, T>(op, g, i, j, k, c, x);
    }
}

// result slots: out[0..NV)
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_dot(Geom g, Region3 R, const T *__restrict__ a, const T *__restrict__ b,
                                                   int ncol, RedWork rw, double *out) {
    double acc[1] = {0.0};
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        if (b) acc[0] += to_d(a[c]) * to_d(b[c]);
        else for (int d = 0; d < ncol; d++) acc[0] += to_d(a[c + d * g.n]) * to_d(a[c + d * g.n]);
    }
    double tot[1];
    if (grid_sum<1>(acc, rw, tot) && threadIdx.x == 0) out[0] = tot[0];
}

// |a(:,col)| maximum over the interior (FalmMV::MaxDiag, src/MV.h:67-76)
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_absmax(Geom g, Region3 R, const T *__restrict__ a, unsigned long long *out) {
    double m = 0.0;
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) m = fmax(m, fabs(to_d(a[g.id(i, j, k)])));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

template <typename T>
__global__ void k_scale(T *a, long long n, T s) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) a[q] *= s;
}

// src/dev/MVDevCall.cu:678-695
template <typename T>
__global__ void k_axby(T a, const T *x, T b, const T *y, T *r, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        r[q] = a * x[q] + b * y[q];
}

// ---------------------------------------------------------------- BiCGStab scalars
// From the reduced totals of a kernel's products (one thread).
// start of a pass (src/FalmEq.cpp:329-336, 348-351): tot = {r.r (FP64), rr.r}
__device__ __forceinline__ void derive_res(SolverScalars *sc, const double (&tot)[2], int check_tol) {
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
// alpha = rho / (rr.q) (src/FalmEq.cpp:371)
__device__ __forceinline__ void derive_alpha(SolverScalars *sc, const double (&tot)[1]) {
    double alpha = sc->rho / tot[0];
    sc->alpha = alpha;
    if (!isfinite(alpha)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
}
__device__ __forceinline__ void derive_alpha(SolverScalars *sc, const double (&tot)[2]) {
    const double t1[1] = {tot[0]};
    derive_alpha(sc, t1);
}
// omega = (t.s) / (t.t) (src/FalmEq.cpp:389)
__device__ __forceinline__ void derive_omega(SolverScalars *sc, const double (&tot)[2]) {
    double omega = tot[0] / tot[1];
    sc->omega = omega;
    if (!isfinite(omega)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
}
// after x, r: tot = {r.r, r.rr}; the stop test (src/FalmEq.cpp:400-407) and,
// for the next iteration, rho and beta (:345-356)
__device__ __forceinline__ void derive_xr(SolverScalars *sc, const double (&tot)[2]) {
    double rho = sc->rho;
    sc->rrho = rho;
    double err = sqrt(tot[0]) / sc->gsize;
    sc->err = err;
    sc->it += 1;
    sc->first = 0;
    if (!isfinite(err)) { sc->done = 1; sc->status = FALM_ERR_NAN; return; }
    if (!(sc->it < sc->maxit && err > sc->tol)) {
        sc->done = 1;
        sc->status = err > sc->tol ? FALM_ERR_MAXIT : FALM_OK;
        return;
    }
    double rho_n = tot[1];
    if (fabs(rho_n) < FLT_MIN) {
        sc->err = rho_n;
        sc->done = 1;
        sc->status = err <= sc->tol ? FALM_OK : FALM_ERR_BREAKDOWN;
        return;
    }
    sc->beta = (rho_n * sc->alpha) / (rho * sc->omega);
    sc->rho = rho_n;
}

// ---------------------------------------------------------------- residual (+ solver start)
// src/dev/FalmEqDevCall.cu:54-85; evaluated in FP64 whatever the storage type
// (the true-residual recomputation of the mixed-precision mode).  With sc !=
// NULL it also starts a BiCGStab pass: rr = r, rho = r.rr, err = ||r||/N
// (src/FalmEq.cpp:329-336).
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_res(Geom g, Region3 R, Op7<T> op, const T *__restrict__ x,
    const T *__restrict__ b, T *__restrict__ r, T *__restrict__ rr, RedWork rw, SolverScalars *sc, int check_tol) {
    double acc[2] = {0.0, 0.0};
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        double rv = to_d(b[c]) - apply7<T, double>(op, g, i, j, k, c, x);
        T rt = (T)rv;
        r[c] = rt;
        if (rr) rr[c] = rt;
        acc[0] += rv * rv;
        acc[1] += to_d(rt) * to_d(rt);
    }
    if (!sc) return;
    double tot[2];
    if (grid_sum<2>(acc, rw, tot) && threadIdx.x == 0) {
        if (sc->defer) { sc->red[0] = tot[0]; sc->red[1] = tot[1]; }
        else derive_res(sc, tot, check_tol);
    }
}

// residual of a plain Jacobi / SOR iteration and the loop test of
// src/FalmEq.cpp:121-126 (and :236-239): r = b - A x, err = ||r||_2 / N in
// FP64, it++, stop when err <= tol or it == maxit.  Every block returns at once
// once the solve has stopped (queued iterations).
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_res_plain(Geom g, Region3 R, Op7<T> op, const T *__restrict__ x,
    const T *__restrict__ b, T *__restrict__ r, RedWork rw, SolverScalars *sc) {
    if (sc->done) return;
    double acc[1] = {0.0};
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        double rv = to_d(b[c]) - apply7<T, double>(op, g, i, j, k, c, x);
        r[c] = (T)rv;
        acc[0] += rv * rv;
    }
    double tot[1];
    if (grid_sum<1>(acc, rw, tot) && threadIdx.x == 0) {
        const double err = sqrt(tot[0]) / sc->gsize;
        sc->err = err;
        sc->it += 1;
        if (!isfinite(err)) { sc->done = 1; sc->status = FALM_ERR_NAN; }
        else if (err <= sc->tol) { sc->done = 1; sc->status = FALM_OK; }
        else if (sc->it >= sc->maxit) { sc->done = 1; sc->status = FALM_ERR_MAXIT; }
    }
}

// ---------------------------------------------------------------- preconditioner sweeps
// red-black SOR half sweep, colour (i+j+k)%2 (src/dev/FalmEqDevCall.cu:175-211)
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_sor(Geom g, Region3 R, Op7<T> op, T *x, const T *__restrict__ b,
                                                   T omega, int color, const SolverScalars *sc) {
    if (sc && sc->done) return;
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        if (((i + j + k + g.koff) & 1) != color) continue;
        long long c = g.id(i, j, k);
        T ac, aw, ae, as, an, ab, at;
        op.get(i, j, k, c, ac, aw, ae, as, an, ab, at);
        const long long sxy = (long long)g.sx * g.sy;
        T xc = x[c];
        T cc = (b[c] - (ac * xc + ae * x[c + 1] + aw * x[c - 1] + an * x[c + g.sx] + as * x[c - g.sx] +
                        at * x[c + sxy] + ab * x[c - sxy])) / ac;
        x[c] = xc + omega * cc;
    }
}

// Jacobi sweep (src/dev/FalmEqDevCall.cu:101-132): x = xp + (b - A xp)/ac
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_jacobi(Geom g, Region3 R, Op7<T> op, T *__restrict__ x,
                                                      const T *__restrict__ xp, const T *__restrict__ b, const SolverScalars *sc) {
    if (sc && sc->done) return;
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        T ac, aw, ae, as, an, ab, at;
        op.get(i, j, k, c, ac, aw, ae, as, an, ab, at);
        const long long sxy = (long long)g.sx * g.sy;
        T xc = xp[c];
        x[c] = xc + (b[c] - (ac * xc + ae * xp[c + 1] + aw * xp[c - 1] + an * xp[c + g.sx] + as * xp[c - g.sx] +
                             at * xp[c + sxy] + ab * xp[c - sxy])) / ac;
    }
}

// first sweep of the preconditioner from z = 0, pointwise (k: the plane's global
// index, local k + Geom::koff, which only sets the colour):
//   SOR:    black cells z = omega*(v/ac), red cells z = 0
//   Jacobi: z = v/ac
template <typename T>
__device__ __forceinline__ T pc_first(int pc_type, int i, int j, int k, T v, T ac, T omega) {
    if (pc_type == FALM_LS_SOR) return (((i + j + k) & 1) == 0) ? omega * sor_div(v, ac) : T(0);
    if (pc_type == FALM_LS_JACOBI) return sor_div(v, ac);
    return T(0);
}

// The vector steps below walk an x row with the 32 lanes of a warp in chunks
// of 32*kRowILP cells (cell u of a chunk at i + 32u): the loads of a chunk are
// issued before any of its arithmetic, so a warp keeps kRowILP requests per
// operand in flight.
constexpr int kRowILP = 4;

// ---------------------------------------------------------------- BiCGStab steps
// p_in: the previous p (read unless first); p_out: the new p, or null when the
// caller reads r in its place (first iteration, p = r)
template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_bicg_p(Geom g, Region3 R, Op7<T> op, T *p_out, const T *p_in,
    const T *__restrict__ q, const T *__restrict__ r, T *__restrict__ pp, int pc_type, T pc_omega, const SolverScalars *sc) {
    if (sc->done) return;
    const int first = sc->first;
    const T beta = (T)sc->beta, omega = (T)sc->omega;
    FB_FOR_ROWS(R, j, k) {
        const typename Op7<T>::RowD rd = op.row(j, k);
        const long long c0 = g.id(0, j, k);
        for (int ib = R.i0 + (threadIdx.x & 31); ib < R.i1; ib += 32 * kRowILP) {
            T rv[kRowILP], pv[kRowILP], qv[kRowILP];
#pragma unroll
            for (int u = 0; u < kRowILP; u++) {
                const int i = ib + 32 * u;
                rv[u] = pv[u] = qv[u] = T(0);
                if (i < R.i1) {
                    rv[u] = r[c0 + i];
                    if (!first) { pv[u] = p_in[c0 + i]; qv[u] = q[c0 + i]; }
                }
            }
#pragma unroll
            for (int u = 0; u < kRowILP; u++) {
                const int i = ib + 32 * u;
                if (i < R.i1) {
                    const long long c = c0 + i;
                    const T v = first ? rv[u] : rv[u] + beta * (pv[u] - omega * qv[u]);   // src/dev/FalmEqDevCall.cu:261
                    if (p_out) p_out[c] = v;
                    pp[c] = pc_first<T>(pc_type, i, j, k + g.koff, v, op.diag_row(rd, i, c), pc_omega);
                }
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_mv_dot1(Geom g, Region3 R, Op7<T> op, const T *__restrict__ pp,
    T *__restrict__ q, const T *__restrict__ rr, RedWork rw, SolverScalars *sc) {
    if (sc->done) return;
    double acc[1] = {0.0};
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        T qv = apply7<T, T>(op, g, i, j, k, c, pp);
        q[c] = qv;
        acc[0] += to_d(rr[c]) * to_d(qv);
    }
    double tot[1];
    if (grid_sum<1>(acc, rw, tot) && threadIdx.x == 0) {
        if (sc->defer) sc->red[0] = tot[0];
        else derive_alpha(sc, tot);
    }
}

template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_bicg_s(Geom g, Region3 R, Op7<T> op, T *__restrict__ s,
    const T *__restrict__ q, const T *__restrict__ r, T *__restrict__ ss, int pc_type, T pc_omega, const SolverScalars *sc) {
    if (sc->done) return;
    const T alpha = (T)sc->alpha;
    FB_FOR_ROWS(R, j, k) {
        const typename Op7<T>::RowD rd = op.row(j, k);
        const long long c0 = g.id(0, j, k);
        for (int ib = R.i0 + (threadIdx.x & 31); ib < R.i1; ib += 32 * kRowILP) {
            T rv[kRowILP], qv[kRowILP];
#pragma unroll
            for (int u = 0; u < kRowILP; u++) {
                const int i = ib + 32 * u;
                rv[u] = qv[u] = T(0);
                if (i < R.i1) { rv[u] = r[c0 + i]; qv[u] = q[c0 + i]; }
            }
#pragma unroll
            for (int u = 0; u < kRowILP; u++) {
                const int i = ib + 32 * u;
                if (i < R.i1) {
                    const long long c = c0 + i;
                    const T sv = rv[u] - alpha * qv[u];                   // src/dev/FalmEqDevCall.cu:284
                    s[c] = sv;
                    ss[c] = pc_first<T>(pc_type, i, j, k + g.koff, sv, op.diag_row(rd, i, c), pc_omega);
                }
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_mv_dot2(Geom g, Region3 R, Op7<T> op, const T *__restrict__ ss,
    T *__restrict__ t, const T *__restrict__ s, RedWork rw, SolverScalars *sc) {
    if (sc->done) return;
    double acc[2] = {0.0, 0.0};
    FB_FOR_ROWS(R, j, k) FB_FOR_I(R, i) {
        long long c = g.id(i, j, k);
        T tv = apply7<T, T>(op, g, i, j, k, c, ss);
        t[c] = tv;
        double td = to_d(tv);
        acc[0] += td * to_d(s[c]);
        acc[1] += td * td;
    }
    double tot[2];
    if (grid_sum<2>(acc, rw, tot) && threadIdx.x == 0) {
        if (sc->defer) { sc->red[0] = tot[0]; sc->red[1] = tot[1]; }
        else derive_omega(sc, tot);
    }
}

template <typename T>
__global__ void __launch_bounds__(kRowThreads) k_bicg_xr(Geom g, Region3 R, T *__restrict__ x, const T *__restrict__ pp,
    const T *__restrict__ ss, T *__restrict__ r, const T *__restrict__ s, const T *__restrict__ t, const T *__restrict__ rr,
    RedWork rw, SolverScalars *sc) {
    if (sc->done) return;
    const T alpha = (T)sc->alpha, omega = (T)sc->omega;
    double acc[2] = {0.0, 0.0};
    FB_FOR_ROWS(R, j, k) {
        const long long c0 = g.id(0, j, k);
        for (int ib = R.i0 + (threadIdx.x & 31); ib < R.i1; ib += 32 * kRowILP) {
            T xv[kRowILP], ppv[kRowILP], ssv[kRowILP], sv[kRowILP], tv[kRowILP], rrv[kRowILP];
#pragma unroll
            for (int u = 0; u < kRowILP; u++) {
                const int i = ib + 32 * u;
                xv[u] = ppv[u] = ssv[u] = sv[u] = tv[u] = rrv[u] = T(0);
                if (i < R.i1) {
                    const long long c = c0 + i;
                    xv[u] = x[c]; ppv[u] = pp[c]; ssv[u] = ss[c]; sv[u] = s[c]; tv[u] = t[c]; rrv[u] = rr[c];
                }
            }
#pragma unroll
            for (int u = 0; u < kRowILP; u++) {
                const int i = ib + 32 * u;
                if (i < R.i1) {
                    const long long c = c0 + i;
                    x[c] = xv[u] + (alpha * ppv[u] + omega * ssv[u]);      // src/dev/FalmEqDevCall.cu:307
                    const T rv = sv[u] - omega * tv[u];                    // :330
                    r[c] = rv;
                    const double rd = to_d(rv);
                    acc[0] += rd * rd;
                    acc[1] += rd * to_d(rrv[u]);
                }
            }
        }
    }
    double tot[2];
    if (grid_sum<2>(acc, rw, tot) && threadIdx.x == 0) {
        if (sc->defer) { sc->red[0] = tot[0]; sc->red[1] = tot[1]; }
        else derive_xr(sc, tot);
    }
}

// The scalars of a slab-decomposed solve (SolverScalars::defer): the kernels
// above left their local totals in red[], the totals were summed over the
// slabs in place, and one thread derives the scalars from them.
// stage 0: pass start (k_res, check_tol 0), 1: check (k_res, check_tol 1),
// 2: alpha, 3: omega, 4: x/r update
__global__ void k_slab_derive(SolverScalars *sc, int stage) {
    if (stage >= 2 && sc->done) return;
    double tot[2] = {sc->red[0], sc->red[1]};
    if (stage <= 1) derive_res(sc, tot, stage);
    else if (stage == 2) derive_alpha(sc, tot);
    else if (stage == 3) derive_omega(sc, tot);
    else derive_xr(sc, tot);
}

}  // namespace fb
