/*
 * Harness around the reference's own CUDA implementation (test
 * infrastructure only).  oracle/Makefile compiles this file together with the
 * reference's sources, where they lie, into oracle/_ref/libfalmref.so.  It
 * drives the reference's classes (FalmCFD, FalmEq, FalmMV, Alm::AlmHandler,
 * the application boundary kernels) on one rank, the way the application
 * drivers do (app/nedo/main.cpp:102-204, app/lid3d/main.cpp:22-168), so that
 * the CPU oracle and the B200 product can both be checked against the
 * reference's own step on identical inputs.
 *
 * Call convention for the pseudo-velocity: FSPseudoU(un=u_prev, u=u_prev, ...,
 * ua=u).  The drivers pass ua aliased to u (app/nedo/main.cpp:162), which makes
 * the kernel read neighbours that other threads are overwriting; u_prev is an
 * exact copy of u taken at the start of the step (:152), so this convention is
 * the race-free explicit-Euler update the drivers intend.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <vector>
#include <fstream>
#include "FalmCFD.h"
#include "FalmEq.h"
#include "MV.h"
#include "alm/alm.h"
#include "rmcp/alm.h"
#include "windtunnel/bcdevcall.h"
#include "lid3d/bcdev.h"
#include "FalmIO.h"
#include "mesher/mesher.hpp"
#include "falm_oracle.h"

using namespace Falm;

namespace {

struct RefCase {
    or_case c;
    std::vector<double> hx, hy, hz;
    CPM cpm;
    Matrix<Real> x, y, z;                  /* 1D coordinates (FalmBaseMesh) */
    Matrix<Real> xyz, kx, g, ja;
    Matrix<Real> u, uu, p, nut, poi_a, rhs, res, ff, div, u_prev;
    FalmCFD cfd;
    FalmEq eq;
    Alm::AlmHandler alm;
    bool alm_on = false;
    Rmcp::RmcpAlm rmcp;
    bool rmcp_on = false;
    Real maxdiag = 1.0;
    dim3 block{8, 8, 8};
    Stream streams[CPM::NFACE];
    std::string workdir;
};

void ubc_all(RefCase &R, double) {
    Region &pdm = R.cpm.pdm_list[0];
    Int gc = R.cpm.gc;
    if (R.c.bc == OR_BC_CHANNEL) {
        ubc_xminus(R.u, R.c.u_inlet, pdm, gc, R.streams[CPM::XMINUS]);
        ubc_xplus(R.u, R.u_prev, R.xyz, R.c.dt, pdm, gc, R.streams[CPM::XPLUS]);
        ubc_yminus(R.u, pdm, gc, R.streams[CPM::YMINUS]);
        ubc_yplus(R.u, pdm, gc, R.streams[CPM::YPLUS]);
        ubc_zminus(R.u, pdm, gc, R.streams[CPM::ZMINUS]);
        ubc_zplus(R.u, pdm, gc, R.streams[CPM::ZPLUS]);
    } else {
        LID3D::ubc_xminus(R.u, pdm, gc, R.streams[CPM::XMINUS]);
        LID3D::ubc_xplus(R.u, pdm, gc, R.streams[CPM::XPLUS]);
        LID3D::ubc_yminus(R.u, pdm, gc, R.streams[CPM::YMINUS]);
        LID3D::ubc_yplus(R.u, pdm, gc, R.streams[CPM::YPLUS]);
        LID3D::ubc_zminus(R.u, pdm, gc, R.streams[CPM::ZMINUS]);
        LID3D::ubc_zplus(R.u, pdm, gc, R.streams[CPM::ZPLUS]);
    }
    cudaDeviceSynchronize();
}

void pbc_all(RefCase &R) {
    Region &pdm = R.cpm.pdm_list[0];
    Int gc = R.cpm.gc;
    if (R.c.bc == OR_BC_CHANNEL) {
        pbc_xminus(R.p, pdm, gc, R.streams[CPM::XMINUS]);
        pbc_xplus(R.p, pdm, gc, R.streams[CPM::XPLUS]);
        pbc_yminus(R.p, pdm, gc, R.streams[CPM::YMINUS]);
        pbc_yplus(R.p, pdm, gc, R.streams[CPM::YPLUS]);
        pbc_zminus(R.p, pdm, gc, R.streams[CPM::ZMINUS]);
        pbc_zplus(R.p, pdm, gc, R.streams[CPM::ZPLUS]);
    } else {
        LID3D::pbc_xminus(R.p, pdm, gc, R.streams[CPM::XMINUS]);
        LID3D::pbc_xplus(R.p, pdm, gc, R.streams[CPM::XPLUS]);
        LID3D::pbc_yminus(R.p, pdm, gc, R.streams[CPM::YMINUS]);
        LID3D::pbc_yplus(R.p, pdm, gc, R.streams[CPM::YPLUS]);
        LID3D::pbc_zminus(R.p, pdm, gc, R.streams[CPM::ZMINUS]);
        LID3D::pbc_zplus(R.p, pdm, gc, R.streams[CPM::ZPLUS]);
    }
    cudaDeviceSynchronize();
}

void uubc_all(RefCase &R) {
    if (R.c.bc != OR_BC_CAVITY) return;
    Region &pdm = R.cpm.pdm_list[0];
    Int gc = R.cpm.gc;
    LID3D::uubc_xminus(R.uu, pdm, gc, R.streams[CPM::XMINUS]);
    LID3D::uubc_xplus(R.uu, pdm, gc, R.streams[CPM::XPLUS]);
    LID3D::uubc_yminus(R.uu, pdm, gc, R.streams[CPM::YMINUS]);
    LID3D::uubc_yplus(R.uu, pdm, gc, R.streams[CPM::YPLUS]);
    LID3D::uubc_zminus(R.uu, pdm, gc, R.streams[CPM::ZMINUS]);
    LID3D::uubc_zplus(R.uu, pdm, gc, R.streams[CPM::ZPLUS]);
    cudaDeviceSynchronize();
}

void copy_in(Matrix<Real> &m, const double *src) {
    if (!src) return;
    memcpy(m.host.ptr, src, sizeof(double) * m.size);
    m.sync(MCP::Hst2Dev);
}

void copy_out(Matrix<Real> &m, double *dst) {
    if (!dst) return;
    m.sync(MCP::Dev2Hst);
    memcpy(dst, m.host.ptr, sizeof(double) * m.size);
}

} // namespace

extern "C" {

/* Build a one-rank case.  Airfoil stations (n_station, row-major polars
 * [station][attack]) feed the reference's own BladeHandler::buildAP. */
void *ref_create(const or_case *c, int n_station, const double *st_r, const double *st_chord,
                 const double *st_twist, const double *st_cl, const double *st_cd, const char *workdir) {
    RefCase *R = new RefCase();
    R->c = *c;
    R->workdir = workdir ? workdir : ".";
    for (auto &s : R->streams) cudaStreamCreate(&s);
    Int3 shape{{c->sx, c->sy, c->sz}};
    CPM &cpm = R->cpm;
    cpm.rank = 0;
    cpm.size = 1;
    cpm.initPartition(shape, c->gc, Int3{{1, 1, 1}});
    Region &pdm = cpm.pdm_list[0];

    R->x.alloc(c->sx, 1, HDC::HstDev, "x");
    R->y.alloc(c->sy, 1, HDC::HstDev, "y");
    R->z.alloc(c->sz, 1, HDC::HstDev, "z");
    for (int i = 0; i < c->sx; i++) R->x(i) = c->x[i];
    for (int j = 0; j < c->sy; j++) R->y(j) = c->y[j];
    for (int k = 0; k < c->sz; k++) R->z(k) = c->z[k];
    R->x.sync(MCP::Hst2Dev); R->y.sync(MCP::Hst2Dev); R->z.sync(MCP::Hst2Dev);

    /* metrics exactly as FalmCore::computation_init (src/falm.h:383-404) */
    R->xyz.alloc(shape, 3, HDC::HstDev, "coordinate");
    R->kx.alloc(shape, 3, HDC::HstDev, "kx");
    R->g.alloc(shape, 3, HDC::HstDev, "g");
    R->ja.alloc(shape, 1, HDC::HstDev, "ja");
    for (Int k = 0; k < shape[2]; k++)
    for (Int j = 0; j < shape[1]; j++)
    for (Int i = 0; i < shape[0]; i++) {
        Int idx = IDX(i, j, k, shape);
        R->xyz(idx, 0) = c->x[i]; R->xyz(idx, 1) = c->y[j]; R->xyz(idx, 2) = c->z[k];
        Real3 pitch;
        pitch[0] = c->hx[i]; pitch[1] = c->hy[j]; pitch[2] = c->hz[k];
        Real volume = PRODUCT3(pitch);
        Real3 dkdx = Real(1) / pitch;
        R->ja(idx) = volume;
        R->g(idx, 0) = volume * dkdx[0] * dkdx[0];
        R->g(idx, 1) = volume * dkdx[1] * dkdx[1];
        R->g(idx, 2) = volume * dkdx[2] * dkdx[2];
        R->kx(idx, 0) = dkdx[0]; R->kx(idx, 1) = dkdx[1]; R->kx(idx, 2) = dkdx[2];
    }
    R->xyz.sync(MCP::Hst2Dev); R->kx.sync(MCP::Hst2Dev); R->g.sync(MCP::Hst2Dev); R->ja.sync(MCP::Hst2Dev);

    R->u.alloc(shape, 3, HDC::HstDev, "u");
    R->uu.alloc(shape, 3, HDC::HstDev, "uu");
    R->p.alloc(shape, 1, HDC::HstDev, "p");
    R->nut.alloc(shape, 1, HDC::HstDev, "nut");
    R->poi_a.alloc(shape, 7, HDC::HstDev, "A", StencilMatrix::D3P7);
    R->rhs.alloc(shape, 1, HDC::HstDev, "rhs");
    R->res.alloc(shape, 1, HDC::HstDev, "res");
    R->ff.alloc(shape, 3, HDC::HstDev, "ff");
    R->div.alloc(shape, 1, HDC::HstDev, "div");
    R->u_prev.alloc(shape, 3, HDC::HstDev, "u_prev");

    R->cfd.init(c->Re, (Flag)c->adv, (Flag)c->sgs, c->Cs);
    R->cfd.alloc(shape);
    Flag pc = c->pc_type == OR_PC_SOR ? LSType::SOR : (c->pc_type == OR_PC_JACOBI ? LSType::Jacobi : LSType::Empty);
    R->eq.init(LSType::PBiCGStab, c->ls_maxit, c->ls_tol, 1.0, pc, c->pc_maxit, c->pc_relax);
    R->eq.alloc(shape);

    /* Poisson operator: the drivers' host assembly (app/nedo/main.cpp:25-100,
       app/lid3d/main.cpp:22-92), then the reference's MaxDiag and ScaleMatrix */
    for (Int k = cpm.gc; k < pdm.shape[2] - cpm.gc; k++)
    for (Int j = cpm.gc; j < pdm.shape[1] - cpm.gc; j++)
    for (Int i = cpm.gc; i < pdm.shape[0] - cpm.gc; i++) {
        Real ac = 0, ae = 0, aw = 0, an = 0, as = 0, at = 0, ab = 0;
        Int cc = IDX(i, j, k, pdm.shape);
        Real gxcc = R->g(cc, 0), gxe1 = R->g(IDX(i + 1, j, k, pdm.shape), 0), gxw1 = R->g(IDX(i - 1, j, k, pdm.shape), 0);
        Real gycc = R->g(cc, 1), gyn1 = R->g(IDX(i, j + 1, k, pdm.shape), 1), gys1 = R->g(IDX(i, j - 1, k, pdm.shape), 1);
        Real gzcc = R->g(cc, 2), gzt1 = R->g(IDX(i, j, k + 1, pdm.shape), 2), gzb1 = R->g(IDX(i, j, k - 1, pdm.shape), 2);
        Real jacob = R->ja(cc), coef;
        Int east_limit = (c->bc == OR_BC_CHANNEL) ? cpm.global.shape[0] - cpm.gc : cpm.global.shape[0] - cpm.gc - 1;
        coef = 0.5 * (gxcc + gxe1) / jacob;
        if (i < east_limit) { ac -= coef; ae = coef; }
        coef = 0.5 * (gxcc + gxw1) / jacob;
        if (i > cpm.gc) { ac -= coef; aw = coef; }
        coef = 0.5 * (gycc + gyn1) / jacob;
        if (j < cpm.global.shape[1] - cpm.gc - 1) { ac -= coef; an = coef; }
        coef = 0.5 * (gycc + gys1) / jacob;
        if (j > cpm.gc) { ac -= coef; as = coef; }
        coef = 0.5 * (gzcc + gzt1) / jacob;
        if (k < cpm.global.shape[2] - cpm.gc - 1) { ac -= coef; at = coef; }
        coef = 0.5 * (gzcc + gzb1) / jacob;
        if (k > cpm.gc) { ac -= coef; ab = coef; }
        R->poi_a(cc, 0) = ac; R->poi_a(cc, 1) = aw; R->poi_a(cc, 2) = ae; R->poi_a(cc, 3) = as;
        R->poi_a(cc, 4) = an; R->poi_a(cc, 5) = ab; R->poi_a(cc, 6) = at;
    }
    R->poi_a.sync(MCP::Hst2Dev);
    R->maxdiag = FalmMV::MaxDiag(R->poi_a, cpm, R->block);
    FalmMV::ScaleMatrix(R->poi_a, 1.0 / R->maxdiag, R->block);

    if (c->alm_on) {
        const or_alm &a = c->alm;
        Json blade;
        blade["attacks"] = std::vector<double>(a.attack, a.attack + a.n_attack);
        Json afs = Json::array();
        for (int s = 0; s < n_station; s++) {
            Json af;
            af["r/R"] = st_r[s];
            af["chord/R"] = st_chord[s];
            af["twist[deg]"] = st_twist[s];
            af["Cl"] = std::vector<double>(st_cl + (long)s * a.n_attack, st_cl + (long)(s + 1) * a.n_attack);
            af["Cd"] = std::vector<double>(st_cd + (long)s * a.n_attack, st_cd + (long)(s + 1) * a.n_attack);
            afs.push_back(af);
        }
        blade["airfoils"] = afs;
        Json prop;
        prop["radius"] = a.radius;
        prop["hubRadius"] = a.hub_radius;
        prop["bladeNumber"] = a.n_blade;
        prop["overhang"] = -a.hub[0];
        prop["tower"] = a.hub[2];
        prop["bladeProperties"] = blade;
        std::string prop_path = R->workdir + "/ref_turbine_properties.json";
        std::ofstream pf(prop_path);
        pf << prop.dump(2);
        pf.close();
        Json arr = Json::array();
        for (int t = 0; t < a.n_turbine; t++) {
            Json tj;
            tj["tipRate"] = a.tip_rate[t];
            tj["baseLocation"] = {a.base[3 * t], a.base[3 * t + 1], a.base[3 * t + 2]};
            Json ang = {0.0, 0.0, 0.0};
            int at = a.angle_type[t];
            if (at) {
                const double *m = a.motion + 3 * t;
                if (m[1] == 0.0) {
                    ang[at - 1] = m[0] * 180.0 / M_PI;
                } else {
                    Json mo;
                    mo["amplitude"] = m[0] * 180.0 / M_PI;
                    mo["period"] = 2.0 * M_PI / m[1];
                    mo["phase"] = m[2] * 180.0 / M_PI;
                    ang[at - 1] = mo;
                }
            }
            tj["angle"] = ang;
            arr.push_back(tj);
        }
        Json params;
        params["projectionWidth"] = a.euler_eps;
        params["bladePointNumber"] = a.n_ap_per_blade;
        params["turbineProperties"] = "ref_turbine_properties.json";
        params["apFile"] = "ref_ap.json";
        params["turbineArray"] = arr;
        params["writePowerThrust"] = false;
        R->alm.init(R->workdir, params, cpm, R->workdir + "/ref_PT.csv");
        R->alm_on = true;
    }
    cudaDeviceSynchronize();
    return R;
}

void ref_destroy(void *h) {
    RefCase *R = (RefCase *)h;
    if (!R) return;
    if (R->alm_on) R->alm.finalize();
    if (R->rmcp_on) R->rmcp.finalize();
    R->cfd.release();
    R->eq.release();
    for (auto &s : R->streams) cudaStreamDestroy(s);
    FalmMV::release();
    delete R;
}

double ref_maxdiag(void *h) { return ((RefCase *)h)->maxdiag; }

/* field ids for ref_set / ref_get */
enum { RF_U, RF_UU, RF_P, RF_NUT, RF_FF, RF_RHS, RF_RES, RF_UPREV, RF_DIV, RF_A, RF_KX, RF_G, RF_JA };

static Matrix<Real> *field(RefCase *R, int id) {
    switch (id) {
    case RF_U: return &R->u; case RF_UU: return &R->uu; case RF_P: return &R->p; case RF_NUT: return &R->nut;
    case RF_FF: return &R->ff; case RF_RHS: return &R->rhs; case RF_RES: return &R->res; case RF_UPREV: return &R->u_prev;
    case RF_DIV: return &R->div; case RF_A: return &R->poi_a; case RF_KX: return &R->kx; case RF_G: return &R->g;
    case RF_JA: return &R->ja;
    }
    return nullptr;
}

int ref_set(void *h, int id, const double *src) {
    Matrix<Real> *m = field((RefCase *)h, id);
    if (!m) return 1;
    copy_in(*m, src);
    return (int)cudaDeviceSynchronize();
}

int ref_get(void *h, int id, double *dst) {
    Matrix<Real> *m = field((RefCase *)h, id);
    if (!m) return 1;
    copy_out(*m, dst);
    return (int)cudaDeviceSynchronize();
}

/* single operations of the step, on the harness's own fields */
enum { RO_PSEUDO_U, RO_UTOUU, RO_RHS, RO_SOLVE, RO_PBC, RO_PROJECT, RO_UBC, RO_SGS, RO_DIV, RO_ALM, RO_UUBC };

int ref_op(void *h, int op, double t, or_stats *st) {
    RefCase *R = (RefCase *)h;
    switch (op) {
    case RO_PSEUDO_U:
        R->u_prev.copy(R->u, HDC::Device);
        R->cfd.FSPseudoU(R->u_prev, R->u_prev, R->uu, R->u, R->nut, R->kx, R->g, R->ja, R->ff, R->c.dt, R->cpm, R->block, R->streams, 1);
        break;
    case RO_UTOUU: R->cfd.UtoUU(R->u, R->uu, R->kx, R->ja, R->cpm, R->block, R->streams); break;
    case RO_UUBC: uubc_all(*R); break;
    case RO_RHS: R->cfd.MACCalcPoissonRHS(R->uu, R->rhs, R->ja, R->c.dt, R->cpm, R->block, R->maxdiag); break;
    case RO_SOLVE:
        R->eq.Solve(R->poi_a, R->p, R->rhs, R->res, R->cpm, R->block, R->streams);
        if (st) { st->it = R->eq.it; st->err = R->eq.err; }
        break;
    case RO_PBC: pbc_all(*R); break;
    case RO_PROJECT: R->cfd.ProjectP(R->u, R->u, R->uu, R->uu, R->p, R->kx, R->g, R->c.dt, R->cpm, R->block, R->streams); break;
    case RO_UBC: ubc_all(*R, t); break;
    case RO_SGS: R->cfd.SGS(R->u, R->nut, R->xyz, R->kx, R->ja, R->cpm, R->block, R->streams); break;
    case RO_DIV: {
        R->cfd.Divergence(R->uu, R->div, R->ja, R->cpm, R->block);
        double nsq = FalmMV::EuclideanNormSq(R->div, R->cpm, R->block);
        if (st) st->divnorm = sqrt(nsq) / PRODUCT3(R->cpm.pdm_list[0].shape - Int(2 * R->cpm.gc));
        break;
    }
    case RO_ALM:
        if (!R->alm_on) return 2;
        R->alm.Alm(R->x, R->y, R->z, R->u, R->ff, t, R->block);
        if (st)
            for (size_t tid = 0; tid < R->alm.turbines.n_turbine && tid < 8; tid++) {
                st->torque[tid] = R->alm.turbines.host.torque[tid];
                st->thrust[tid] = R->alm.turbines.host.thrust[tid];
            }
        break;
    default: return 1;
    }
    return (int)cudaDeviceSynchronize();
}

/* FalmEq::Solve with the plain Jacobi (ls_type 1) or red-black SOR (2) solver
 * (src/FalmEq.cpp:80-127, :173-240) on the harness's p (initial guess, then
 * solution), rhs and res */
int ref_plain_solve(void *h, int ls_type, double relax, int maxit, double tol, or_stats *st) {
    RefCase *R = (RefCase *)h;
    FalmEq eq;
    eq.init(ls_type == OR_PC_JACOBI ? LSType::Jacobi : LSType::SOR, maxit, tol, relax, LSType::Empty, 1, 1.0);
    eq.alloc(R->cpm.pdm_list[0].shape);
    eq.Solve(R->poi_a, R->p, R->rhs, R->res, R->cpm, R->block, R->streams);
    if (st) { st->it = eq.it; st->err = eq.err; }
    eq.release();
    return (int)cudaDeviceSynchronize();
}

/* FalmIO::writeVectorFile of the drivers' uvwp buffer (u, then p), as
 * FalmSolver::outputUVWP fills it (src/falm.h:446-460) */
int ref_write_uvwp(void *h, const char *path, unsigned long long step, double time) {
    RefCase *R = (RefCase *)h;
    Int3 shape = R->cpm.pdm_list[0].shape;
    Matrix<Real> uvwp;
    uvwp.alloc(shape, 4, HDC::Host, "uvwp");
    const size_t n = (size_t)PRODUCT3(shape);
    cudaMemcpy(&uvwp(0, 0), &R->u.dev(0), sizeof(Real) * n * 3, cudaMemcpyDeviceToHost);
    cudaMemcpy(&uvwp(0, 3), &R->p.dev(0), sizeof(Real) * n, cudaMemcpyDeviceToHost);
    FalmIO::writeVectorFile(path, R->cpm, uvwp, (size_t)step, time);
    uvwp.release();
    return (int)cudaDeviceSynchronize();
}

/* FalmIO::writeIndexFile for the harness's one-rank partition */
int ref_write_index(void *h, const char *path, const unsigned long long *steps, const double *times, const int *tavg, int n) {
    RefCase *R = (RefCase *)h;
    std::vector<FalmSnapshotInfo> list;
    for (int q = 0; q < n; q++) list.push_back(FalmSnapshotInfo{(size_t)steps[q], times[q], tavg && tavg[q] != 0});
    FalmIO::writeIndexFile(path, R->cpm, list);
    return 0;
}

/* FalmIO::writeControlVolumeFile of the case's grid */
int ref_write_cv(void *h, const char *path) {
    RefCase *R = (RefCase *)h;
    FalmBaseMesh mesh;
    mesh.alloc(R->c.sx, R->c.sy, R->c.sz, HDC::Host);
    for (int i = 0; i < R->c.sx; i++) { mesh.x(i) = R->c.x[i]; mesh.hx(i) = R->c.hx[i]; }
    for (int j = 0; j < R->c.sy; j++) { mesh.y(j) = R->c.y[j]; mesh.hy(j) = R->c.hy[j]; }
    for (int k = 0; k < R->c.sz; k++) { mesh.z(k) = R->c.z[k]; mesh.hz(k) = R->c.hz[k]; }
    Int3 idmax{{R->c.sx, R->c.sy, R->c.sz}};
    FalmIO::writeControlVolumeFile(path, mesh, idmax, R->c.gc);
    mesh.release();
    return 0;
}

/* Mesher::build_mesh (host only) */
int ref_build_mesh(const char *cvcenter, const char *meshpath, const char *outputfile, int gc) {
    Mesher::build_mesh(cvcenter, meshpath, outputfile, gc);
    return 0;
}

/* one time step in the drivers' order (app/nedo/main.cpp:150-204;
   app/lid3d/main.cpp:121-168 adds uubc after UtoUU and has no ALM) */
int ref_step(void *h, double t, or_stats *st) {
    RefCase *R = (RefCase *)h;
    or_stats local;
    memset(&local, 0, sizeof(local));
    R->u_prev.copy(R->u, HDC::Device);
    if (R->alm_on) ref_op(h, RO_ALM, t, &local);
    R->cfd.FSPseudoU(R->u_prev, R->u_prev, R->uu, R->u, R->nut, R->kx, R->g, R->ja, R->ff, R->c.dt, R->cpm, R->block, R->streams, 1);
    ref_op(h, RO_UTOUU, t, nullptr);
    ref_op(h, RO_UUBC, t, nullptr);
    ref_op(h, RO_RHS, t, nullptr);
    ref_op(h, RO_SOLVE, t, &local);
    ref_op(h, RO_PBC, t, nullptr);
    ref_op(h, RO_PROJECT, t, nullptr);
    ref_op(h, RO_UBC, t, nullptr);
    ref_op(h, RO_SGS, t, nullptr);
    ref_op(h, RO_DIV, t, &local);
    if (st) *st = local;
    return (int)cudaDeviceSynchronize();
}

/* The reference's RMCP model (src/rmcp/alm.h: RmcpAlm::init from the turbine parameters and
 * the blade property file it names, as its drivers do), on the harness's grid */
int ref_rmcp_init(void *h, const or_rmcp *r) {
    RefCase *R = (RefCase *)h;
    Json blade;
    blade["attacks"] = std::vector<double>(r->attack, r->attack + r->n_attack);
    Json afs = Json::array();
    for (int s = 0; s < r->n_station; s++) {
        Json af;
        af["r/R"] = r->st_r[s];
        af["chord/R"] = r->st_chord[s];
        af["twist[deg]"] = r->st_twist[s];
        af["Cl"] = std::vector<double>(r->cl + (long)s * r->n_attack, r->cl + (long)(s + 1) * r->n_attack);
        af["Cd"] = std::vector<double>(r->cd + (long)s * r->n_attack, r->cd + (long)(s + 1) * r->n_attack);
        afs.push_back(af);
    }
    blade["airfoils"] = afs;
    std::ofstream bf(R->workdir + "/rmcp_blade.json");
    bf << blade.dump(2);
    bf.close();
    Json params;
    params["radius"] = r->radius;
    params["hubRadius"] = r->hub_radius;
    params["bladeNumber"] = r->n_blade;
    params["overhang"] = -r->hub[0];
    params["tower"] = r->hub[2];
    params["bladeProperties"] = "rmcp_blade.json";
    Json arr = Json::array();
    for (int t = 0; t < r->n_turbine; t++) {
        Json tj;
        tj["tipRate"] = r->tip_rate[t];
        tj["baseLocation"] = {r->base[3 * t], r->base[3 * t + 1], r->base[3 * t + 2]};
        /* degrees, as the reference reads them (TurbineHandler::alloc converts with deg2rad) */
        tj["angle"] = {r->angle[3 * t] * 180.0 / M_PI, r->angle[3 * t + 1] * 180.0 / M_PI, r->angle[3 * t + 2] * 180.0 / M_PI};
        arr.push_back(tj);
    }
    params["turbineArray"] = arr;
    R->rmcp.init(R->cpm, params, R->workdir);
    R->rmcp_on = true;
    return (int)cudaDeviceSynchronize();
}

/* RmcpAlm::SetALMFlag + RmcpAlm::ALM at time t on the harness's u: ff (3N) and flag (N) out */
int ref_rmcp_run(void *h, double t, double *ff, int *flag) {
    RefCase *R = (RefCase *)h;
    if (!R->rmcp_on) return 2;
    R->rmcp.SetALMFlag(R->xyz, t, R->cpm);
    R->rmcp.ALM(R->u, R->xyz, R->ff, t, R->cpm);
    int rc = (int)cudaDeviceSynchronize();
    if (rc) return rc;
    copy_out(R->ff, ff);
    if (flag) cudaMemcpy(flag, R->rmcp.alm_flag.dev.ptr, sizeof(int) * R->rmcp.alm_flag.size, cudaMemcpyDeviceToHost);
    return (int)cudaDeviceSynchronize();
}

/* device copies of the APs after ref_op(RO_ALM): xyz (3*apcount), force (3*apcount) */
int ref_get_aps(void *h, double *xyz, double *force, double *torque, double *thrust) {
    RefCase *R = (RefCase *)h;
    if (!R->alm_on) return 2;
    size_t n = R->alm.aps.apcount;
    Alm::APFrame &d = R->alm.aps.dev;
    if (xyz) cudaMemcpy(xyz, d.xyz, sizeof(Real3) * n, cudaMemcpyDeviceToHost);
    if (force) cudaMemcpy(force, d.force, sizeof(Real3) * n, cudaMemcpyDeviceToHost);
    if (torque) cudaMemcpy(torque, d.torque, sizeof(Real) * n, cudaMemcpyDeviceToHost);
    if (thrust) cudaMemcpy(thrust, d.thrust, sizeof(Real) * n, cudaMemcpyDeviceToHost);
    return (int)cudaDeviceSynchronize();
}

} // extern "C"
