/*
 * falm_b200.hpp -- C++ host shim with the reference's solver-class surface
 * (FalmCFD, FalmEq, FalmMV, Alm::AlmHandler, Rmcp::RmcpAlm, CPMComm;
 * src/FalmCFD.h, src/FalmEq.h, src/MV.h, src/alm/alm.h, src/rmcp/alm.h,
 * src/CPMComm.h) over the C ABI of include/falm_b200.h.
 *
 * Method names, argument order and meaning follow the reference, so a driver
 * such as app/nedo/main.cpp:150-204 keeps its shape.  Differences:
 *  - Real is double (FP64 context) or float (mixed context); Matrix<T> is a
 *    device-first stand-in with the reference's .dev.ptr / .host.ptr members.
 *  - kx, g, ja are accepted for signature compatibility and ignored: the
 *    metrics are evaluated from the control-volume tables bound to the
 *    Context (what the reference builds those planes from).
 *  - CPM is one rank with no neighbours unless Context::slab makes the context
 *    one z-slab of a decomposed grid; CPMComm<T> then exchanges a field's z
 *    halo through the slab's transport (no MPI).  Block / stream-array
 *    arguments are accepted and ignored (the library sizes its own launches).
 *  - Rmcp::RmcpAlm (src/rmcp/alm.h) is the RMCP rotor model over
 *    falm_rmcp_init / falm_rmcp_run.
 *  - The reference prints error codes and continues (src/error.h:20-26); here
 *    every call returns the falm_status and a failing call throws Falm::Error.
 *  - FalmIO takes the Context where the reference takes CPM, writes vector
 *    files from the device columns of a Matrix on the context's writer thread
 *    (FalmIO::wait before reading them), and FalmSolver::TAvg is the free
 *    function TAvg.
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
    static const Int XMINUS = 0, XPLUS = 1, YMINUS = 2, YPLUS = 3, ZMINUS = 4, ZPLUS = 5, NFACE = 6;
    int rank = 0, size = 1;
    Int gc = 2;
    Region global;
    std::vector<Region> pdm_list;
    CPM() {}
    CPM(Int3 shape, Int gc_) : gc(gc_), global(shape, Int3{{0, 0, 0}}), pdm_list(1, Region(shape, Int3{{0, 0, 0}})) {}
    /* a z-slab decomposition (the reference splits x, src/CPMBase.h:36-112): the only
       neighbours are the slabs below (ZMINUS) and above (ZPLUS) */
    bool validNeighbour(Int fid) const {
        return (fid == ZMINUS && rank > 0) || (fid == ZPLUS && rank < size - 1);
    }
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
    /* make this context slab `rank` of `nranks` (falm_slab_init): the grid given to the
       constructor is the slab's, z_offset its first interior plane in the whole grid of
       nz_global interior planes; call before any other set-up */
    void slab(int rank, int nranks, int z_offset, int nz_global, const falm_transport &t) {
        check(falm_slab_init(h, rank, nranks, z_offset, nz_global, &t), h, "Context::slab");
        cpm.rank = rank;
        cpm.size = nranks;
    }
};

/* CPMComm<T> (src/CPMComm.h:95-364) over the slab halo exchange: the exchange is ordered on the
   stream and complete for the stream's later work when IExchange6Face returns, so Wait6Face and
   PostExchange6Face have nothing left to do.  margin is the reference's inner offset of the sent
   planes, which is the guide-cell depth here; only the z faces of a slab have neighbours. */
template <typename T>
class CPMComm {
public:
    Context *c;
    explicit CPMComm(Context &ctx) : c(&ctx) {}
    void IExchange6Face(T *data, Int thick, Int /*margin*/, int /*grp_tag*/, void *stream = nullptr) {
        if (c->cpm.size > 1)
            check(falm_slab_halo(c->h, data, 1, thick, stream), c->h, "CPMComm::IExchange6Face");
    }
    void Wait6Face() {}
    void PostExchange6Face(void * = nullptr) {}
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

/* FalmSnapshotInfo (src/typedef.h:35-39) */
struct FalmSnapshotInfo {
    size_t step;
    double time;
    bool tavg;
};

/* FalmIO (src/FalmIO.h) */
struct FalmIO {
    /* writeVectorFile (src/FalmIO.h:69-97) of the columns of v */
    template <typename Real>
    static void writeVectorFile(const std::string &fpath, Context &c, Matrix<Real> &v, size_t step, double time) {
        const void *f[1] = {v.dev.ptr};
        const int nc[1] = {(int)v.shape[1]};
        check(falm_io_write_vector_file(c.h, fpath.c_str(), f, nc, 1, step, time, 0, nullptr), c.h, "FalmIO::writeVectorFile");
    }
    /* the drivers' uvwp file (src/falm.h:446-460): the columns of u, then p */
    template <typename Real>
    static void writeUVWP(const std::string &fpath, Context &c, Matrix<Real> &u, Matrix<Real> &p, size_t step, double time) {
        const void *f[2] = {u.dev.ptr, p.dev.ptr};
        const int nc[2] = {(int)u.shape[1], (int)p.shape[1]};
        check(falm_io_write_vector_file(c.h, fpath.c_str(), f, nc, 2, step, time, 0, nullptr), c.h, "FalmIO::writeUVWP");
    }
    static void wait(Context &c) { check(falm_io_wait(c.h), c.h, "FalmIO::wait"); }
    /* writeIndexFile (src/FalmIO.h:25-67) */
    static void writeIndexFile(const std::string &fpath, Context &c, const std::vector<FalmSnapshotInfo> &list, int dsize = 8) {
        std::vector<unsigned long long> steps;
        std::vector<double> times;
        std::vector<int> tavg;
        for (const auto &s : list) { steps.push_back(s.step); times.push_back(s.time); tavg.push_back(s.tavg ? 1 : 0); }
        const Int3 &sh = c.cpm.global.shape;
        const Int gc = c.cpm.gc;
        check(falm_io_write_index_file(fpath.c_str(), sh[0] - 2 * gc, sh[1] - 2 * gc, sh[2] - 2 * gc, gc, steps.data(), times.data(),
                                       tavg.data(), (int)list.size(), dsize),
              c.h, "FalmIO::writeIndexFile");
    }
    /* writeControlVolumeFile (src/FalmIO.h:118-135) of the context's grid */
    static void writeControlVolumeFile(const std::string &path, Context &c) {
        check(falm_io_write_cv_file(c.h, path.c_str()), c.h, "FalmIO::writeControlVolumeFile");
    }
    /* readControlVolumeFile (src/FalmIO.h:99-116): idmax = {sx, sy, sz}, gc and the six tables */
    static void readControlVolumeFile(const std::string &path, std::vector<double> xyz[3], std::vector<double> h[3], Int3 &idmax, Int &gc) {
        int d[4];
        check(falm_io_read_cv_file(path.c_str(), d, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr), nullptr,
              "FalmIO::readControlVolumeFile");
        for (int q = 0; q < 3; q++) { idmax[q] = d[q]; xyz[q].assign(d[q], 0.0); h[q].assign(d[q], 0.0); }
        gc = d[3];
        check(falm_io_read_cv_file(path.c_str(), d, xyz[0].data(), h[0].data(), xyz[1].data(), h[1].data(), xyz[2].data(), h[2].data()),
              nullptr, "FalmIO::readControlVolumeFile");
    }
};

/* FalmSolver::TAvg (src/falm.h:433-444): avg = (1 - 1/count) avg + f / count */
template <typename Real>
void TAvg(Context &c, Matrix<Real> &avg, Matrix<Real> &f, Int count) {
    check(falm_tavg(c.h, avg.dev.ptr, f.dev.ptr, (int)f.shape[1], count, nullptr), c.h, "TAvg");
}

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

namespace Rmcp {
/* RmcpAlm (src/rmcp/alm.h:11-96); init takes the turbine and blade tables instead of a JSON
   file.  The cell centres come from the bound context, so the x argument is dropped.  init also
   makes RMCP the forcing of falm_step. */
template <typename Real>
class RmcpAlm {
public:
    Context *c;
    int n_turbine = 0;
    std::vector<double> torque, thrust;
    explicit RmcpAlm(Context &ctx) : c(&ctx) {}
    void init(const falm_rmcp_desc &d) {
        check(falm_rmcp_init(c->h, &d), c->h, "RmcpAlm::init");
        n_turbine = d.n_turbine;
        torque.assign(n_turbine, 0.0);
        thrust.assign(n_turbine, 0.0);
    }
    /* SetALMFlag (alm.h:53-63): the paint of the turbines' box cells at time t into flag */
    void SetALMFlag(Matrix<int> &flag, Matrix<Real> &u, Matrix<Real> &ff, Real t) {
        check(falm_rmcp_run(c->h, u.dev.ptr, ff.dev.ptr, t, nullptr, flag.dev.ptr, nullptr, nullptr), c->h, "RmcpAlm::SetALMFlag");
    }
    /* ALM (alm.h:35-52) + CalcTorque (alm.h:26-33): ff at the painted cells, and the turbine sums */
    void ALM(Matrix<Real> &u, Matrix<Real> &ff, Real t) {
        check(falm_rmcp_run(c->h, u.dev.ptr, ff.dev.ptr, t, nullptr, nullptr, torque.data(), thrust.data()), c->h, "RmcpAlm::ALM");
    }
};
}  // namespace Rmcp

}  // namespace Falm

#endif
