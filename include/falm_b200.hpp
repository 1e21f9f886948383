/*
 * falm_b200.hpp -- C++ host shim with the reference's solver-class surface
 * (FalmCFD, FalmEq, FalmMV, Alm::AlmHandler; src/FalmCFD.h, src/FalmEq.h,
 * src/MV.h, src/alm/alm.h) over the C ABI of include/falm_b200.h.
 *
 * Method names, argument order and meaning follow the reference, so a driver
 * such as app/nedo/main.cpp:150-204 keeps its shape.  Differences:
 *  - Real is double (FP64 context) or float (mixed context); Matrix<T> is a
 *    device-first stand-in with the reference's .dev.ptr / .host.ptr members.
 *  - kx, g, ja are accepted for signature compatibility and ignored: the
 *    metrics are evaluated from the control-volume tables bound to the
 *    Context (what the reference builds those planes from).
 *  - CPM is one rank with no neighbours (no MPI); block / stream-array
 *    arguments are accepted and ignored (the library sizes its own launches).
 *  - The reference prints error codes and continues (src/error.h:20-26); here
 *    every call returns the falm_status and a failing call throws Falm::Error.
 */
#ifndef FALM_B200_HPP
#define FALM_B200_HPP

#include <cuda_runtime.h>
#include <stdexcept>
#include <string>
#include <vector>
#include "falm_b200.h"

namespace Falm {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const falm_ctx *ctx, const char *where) {
    if (rc != FALM_OK) throw Error(rc, std::string(where) + ": " + (ctx ? falm_last_error(ctx) : "error"));
}

typedef int Int;
typedef unsigned Flag;
struct Int3 { Int v[3]; Int &operator[](int i) { return v[i]; } const Int &operator[](int i) const { return v[i]; } };

/* Region (src/region.h:8-31) and a one-rank CPM (src/CPMBase.h) */
struct Region {
    Int3 shape, offset;
    Int size;
    Region() : shape{{0, 0, 0}}, offset{{0, 0, 0}}, size(0) {}
    Region(Int3 s, Int3 o) : shape(s), offset(o), size(s[0] * s[1] * s[2]) {}
};

struct CPM {
    int rank = 0, size = 1;
    Int gc = 2;
    Region global;
    std::vector<Region> pdm_list;
    CPM() {}
    CPM(Int3 shape, Int gc_) : gc(gc_), global(shape, Int3{{0, 0, 0}}), pdm_list(1, Region(shape, Int3{{0, 0, 0}})) {}
    bool validNeighbour(Int) const { return false; }
};

/* device-first field in the reference layout (src/matrix.h:129-188) */
template <typename T>
struct Matrix {
    struct Frame { T *ptr = nullptr; } host, dev;
    Int shape[2] = {0, 0};
    Int size = 0;
    std::string name;
    Matrix() {}
    Matrix(Int3 dom, Int ncol, const std::string &n = "") { alloc(dom, ncol, n); }
    Matrix(const Matrix &) = delete;
    Matrix &operator=(const Matrix &) = delete;
    ~Matrix() { release(); }
    void alloc(Int3 dom, Int ncol, const std::string &n = "") {
        shape[0] = dom[0] * dom[1] * dom[2];
        shape[1] = ncol;
        size = shape[0] * ncol;
        name = n;
        host.ptr = new T[size]();
        if (cudaMalloc(&dev.ptr, sizeof(T) * size) != cudaSuccess) throw Error(FALM_ERR_ALLOC, "Matrix::alloc " + n);
        cudaMemset(dev.ptr, 0, sizeof(T) * size);
    }
    void release() {
        delete[] host.ptr;
        host.ptr = nullptr;
        if (dev.ptr) cudaFree(dev.ptr);
        dev.ptr = nullptr;
    }
    T &operator()(Int idx) { return host.ptr[idx]; }
    T &operator()(Int row, Int col) { return host.ptr[row + col * shape[0]]; }
    void sync_to_device() { cudaMemcpy(dev.ptr, host.ptr, sizeof(T) * size, cudaMemcpyHostToDevice); }
    void sync_to_host() { cudaMemcpy(host.ptr, dev.ptr, sizeof(T) * size, cudaMemcpyDeviceToHost); }
    void copy(const Matrix &src) { cudaMemcpy(dev.ptr, src.dev.ptr, sizeof(T) * size, cudaMemcpyDeviceToDevice); }
    void clear() { cudaMemset(dev.ptr, 0, sizeof(T) * size); }
};

/* one falm_ctx: the grid and the metric tables (FalmCore::computation_init, src/falm.h:342-431) */
class Context {
public:
    falm_ctx *h = nullptr;
    CPM cpm;
    Context(const falm_grid &g, int precision) : cpm(Int3{{g.sx, g.sy, g.sz}}, g.gc) {
        check(falm_create(&g, precision, &h), nullptr, "falm_create");
    }
    ~Context() { if (h) falm_destroy(h); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
};

struct AdvectionSchemeType { static const Flag Upwind1 = 0, Upwind3 = 1, QUICK = 2, UTOPIA = 3, KK = 4; };
struct SGSType { static const Flag Empty = 0, Smagorinsky = 1, CSM = 2; };

/* FalmCFD (src/FalmCFD.h:15-109) */
template <typename Real>
class FalmCFD {
public:
    Context *c;
    Real Re = 0, ReI = 0, CSmagorinsky = 0.1;
    Flag AdvScheme = AdvectionSchemeType::Upwind3, SGSModel = SGSType::Smagorinsky;
    explicit FalmCFD(Context &ctx) : c(&ctx) {}
    void init(Real _Re, Flag adv, Flag sgs = SGSType::Smagorinsky, Real Cs = 0.1) {
        Re = _Re; ReI = 1 / _Re; AdvScheme = adv; SGSModel = sgs; CSmagorinsky = Cs;
        check(falm_cfd_init(c->h, _Re, adv, sgs, Cs), c->h, "FalmCFD::init");
    }
    void FSPseudoU(Matrix<Real> &un, Matrix<Real> &u, Matrix<Real> &uu, Matrix<Real> &ua, Matrix<Real> &nut,
                   Matrix<Real> &, Matrix<Real> &, Matrix<Real> &, Matrix<Real> &ff, Real dt, CPM &, dim3 = dim3(),
                   cudaStream_t * = nullptr, Int = 0) {
        check(falm_cfd_pseudo_u(c->h, un.dev.ptr, u.dev.ptr, uu.dev.ptr, ua.dev.ptr, nut.dev.ptr, ff.dev.ptr, dt, 0.0, nullptr), c->h,
              "FalmCFD::FSPseudoU");
        cudaDeviceSynchronize();
    }
    void UtoUU(Matrix<Real> &u, Matrix<Real> &uu, Matrix<Real> &, Matrix<Real> &, CPM &, dim3 = dim3(), cudaStream_t * = nullptr) {
        check(falm_cfd_utouu(c->h, u.dev.ptr, uu.dev.ptr, nullptr), c->h, "FalmCFD::UtoUU");
        cudaDeviceSynchronize();
    }
    void ProjectP(Matrix<Real> &u, Matrix<Real> &ua, Matrix<Real> &uu, Matrix<Real> &uua, Matrix<Real> &p, Matrix<Real> &,
                  Matrix<Real> &, Real dt, CPM &, dim3 = dim3(), cudaStream_t * = nullptr) {
        check(falm_cfd_project_p(c->h, u.dev.ptr, ua.dev.ptr, uu.dev.ptr, uua.dev.ptr, p.dev.ptr, dt, nullptr), c->h, "FalmCFD::ProjectP");
        cudaDeviceSynchronize();
    }
    void SGS(Matrix<Real> &u, Matrix<Real> &nut, Matrix<Real> &, Matrix<Real> &, Matrix<Real> &, CPM &, dim3 = dim3(),
             cudaStream_t * = nullptr) {
        check(falm_cfd_sgs(c->h, u.dev.ptr, nut.dev.ptr, nullptr), c->h, "FalmCFD::SGS");
        cudaDeviceSynchronize();
    }
    void Divergence(Matrix<Real> &uu, Matrix<Real> &dvr, Matrix<Real> &, CPM &, dim3 = dim3()) {
        check(falm_cfd_divergence(c->h, uu.dev.ptr, dvr.dev.ptr, nullptr), c->h, "FalmCFD::Divergence");
        cudaDeviceSynchronize();
    }
    void MACCalcPoissonRHS(Matrix<Real> &uu, Matrix<Real> &rhs, Matrix<Real> &, Real dt, CPM &, dim3 = dim3(), Real maxdiag = 1.0) {
        check(falm_cfd_poisson_rhs(c->h, uu.dev.ptr, rhs.dev.ptr, dt, maxdiag, nullptr), c->h, "FalmCFD::MACCalcPoissonRHS");
        cudaDeviceSynchronize();
    }
};

/* FalmEq (src/FalmEq.h:14-76) */
struct LSType { static const Flag Empty = 0, Jacobi = 1, SOR = 2, PBiCGStab = 4; };

template <typename Real>
class FalmEq {
public:
    Context *c;
    Int maxit = 0, it = 0, pc_maxit = 5;
    Real tol = 0, err = 0, relax_factor = 1, pc_relax_factor = 1;
    Flag type = LSType::PBiCGStab, pc_type = LSType::SOR;
    explicit FalmEq(Context &ctx) : c(&ctx) {}
    void init(Flag _type, Int _maxit, Real _tol, Real _relax, Flag _pc_type = LSType::Empty, Int _pc_maxit = 5, Real _pc_relax = 1.0) {
        type = _type; maxit = _maxit; tol = _tol; relax_factor = _relax; pc_type = _pc_type; pc_maxit = _pc_maxit; pc_relax_factor = _pc_relax;
        check(falm_eq_init(c->h, _type, _maxit, _tol, _relax, _pc_type, _pc_maxit, _pc_relax), c->h, "FalmEq::init");
    }
    /* the Poisson operator of the drivers (make_poisson_coefficient_matrix, app/nedo/main.cpp:25-100) */
    Real PoissonOperator(int bc_kind) {
        double md = 0;
        check(falm_eq_poisson_operator(c->h, bc_kind, &md), c->h, "FalmEq::PoissonOperator");
        return (Real)md;
    }
    /* Solve with the bound Poisson operator (a == nullptr) or an explicit 7-column matrix */
    void Solve(Matrix<Real> *a, Matrix<Real> &x, Matrix<Real> &b, Matrix<Real> &r, CPM &, dim3 = dim3(), cudaStream_t * = nullptr) {
        check(falm_eq_set_matrix(c->h, a ? a->dev.ptr : nullptr), c->h, "FalmEq::Solve");
        double e = 0;
        int rc = falm_eq_solve(c->h, x.dev.ptr, b.dev.ptr, r.dev.ptr, nullptr, &it, &e);
        err = (Real)e;
        if (rc != FALM_ERR_MAXIT && rc != FALM_ERR_BREAKDOWN) check(rc, c->h, "FalmEq::Solve");
    }
    void Res(Matrix<Real> &x, Matrix<Real> &b, Matrix<Real> &r, CPM &, dim3 = dim3(), cudaStream_t * = nullptr) {
        check(falm_eq_res(c->h, x.dev.ptr, b.dev.ptr, r.dev.ptr, nullptr), c->h, "FalmEq::Res");
        cudaDeviceSynchronize();
    }
};

/* FalmMV statics (src/MV.h:11-136) bound to a context */
template <typename Real>
struct FalmMV {
    static void MV(Context &c, Matrix<Real> &x, Matrix<Real> &ax) {
        check(falm_mv_mv(c.h, x.dev.ptr, ax.dev.ptr, nullptr), c.h, "FalmMV::MV");
        cudaDeviceSynchronize();
    }
    static Real DotProduct(Context &c, Matrix<Real> &a, Matrix<Real> &b) {
        double v = 0;
        check(falm_mv_dot(c.h, a.dev.ptr, b.dev.ptr, &v, nullptr), c.h, "FalmMV::DotProduct");
        return (Real)v;
    }
    static Real EuclideanNormSq(Context &c, Matrix<Real> &a) {
        double v = 0;
        check(falm_mv_normsq(c.h, a.dev.ptr, a.shape[1], &v, nullptr), c.h, "FalmMV::EuclideanNormSq");
        return (Real)v;
    }
    static Real MaxDiag(Context &c) {
        double v = 0;
        check(falm_mv_maxdiag(c.h, &v), c.h, "FalmMV::MaxDiag");
        return (Real)v;
    }
    static void ScaleMatrix(Context &c, Matrix<Real> &a, Real scale) {
        check(falm_mv_scale(c.h, a.dev.ptr, a.size, scale, nullptr), c.h, "FalmMV::ScaleMatrix");
        cudaDeviceSynchronize();
    }
};

/* application boundary routines (app/nedo/bc.h, app/windtunnel/bc.h, app/lid3d/bc.h) */
template <typename Real>
void ubc(Context &c, Matrix<Real> &u, Matrix<Real> &uprev, Real dt, Real t) {
    check(falm_bc_ubc(c.h, u.dev.ptr, uprev.dev.ptr, dt, t, nullptr), c.h, "ubc");
    cudaDeviceSynchronize();
}
template <typename Real>
void pbc(Context &c, Matrix<Real> &p) {
    check(falm_bc_pbc(c.h, p.dev.ptr, nullptr), c.h, "pbc");
    cudaDeviceSynchronize();
}
template <typename Real>
void uubc(Context &c, Matrix<Real> &uu) {
    check(falm_bc_uubc(c.h, uu.dev.ptr, nullptr), c.h, "uubc");
    cudaDeviceSynchronize();
}

namespace Alm {
/* AlmHandler (src/alm/alm.h:12-140); init takes the built AP tables instead of JSON files */
template <typename Real>
class AlmHandler {
public:
    Context *c;
    int n_turbine = 0;
    std::vector<double> torque, thrust, tip_rate;
    explicit AlmHandler(Context &ctx) : c(&ctx) {}
    void init(const falm_alm_desc &d) {
        check(falm_alm_init(c->h, &d), c->h, "AlmHandler::init");
        n_turbine = d.n_turbine;
        torque.assign(n_turbine, 0.0);
        thrust.assign(n_turbine, 0.0);
        tip_rate.assign(d.tip_rate, d.tip_rate + d.n_turbine);
    }
    /* AlmHandler::Alm (src/alm/alm.h:66-77); x, y, z come from the bound context */
    void Alm(Matrix<Real> &uvw, Matrix<Real> &ff, Real t) {
        check(falm_alm_run(c->h, uvw.dev.ptr, ff.dev.ptr, t, nullptr, torque.data(), thrust.data()), c->h, "AlmHandler::Alm");
    }
    /* power and thrust per turbine (writePowerThrust, src/alm/alm.h:126-138) */
    double power(int tid) const { return torque[tid] * tip_rate[tid]; }
};
}  // namespace Alm

}  // namespace Falm

#endif
