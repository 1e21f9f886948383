// nedo_driver: the time loop of app/nedo/main.cpp:150-204 written against the
// reference's class surface (include/falm_b200.hpp), FP64.
//
//   nedo_driver <case.bin> <out.bin> [<prefix> <interval> <tavg_start>]
//
// With a prefix the loop also averages u and p from step tavg_start on and
// writes the drivers' output (src/falm.h:433-475, app/nedo/main.cpp:199-200):
// every `interval` steps the u + p vector file <prefix>_000000_<it> (and
// <prefix>_tavg_000000_<it> of the averages while averaging), then
// <prefix>.json (index) and <prefix>.cv (control volumes) at the end.
//
// case.bin (little endian): int32 sx sy sz gc steps maxit pc_maxit adv sgs bc
// pc_type alm; float64 Re Cs dt tol pc_relax u_inlet; x y z hx hy hz; u (3N);
// with alm: int32 n_blade n_ap_per_blade n_attack angle_type; float64 radius
// hub_radius eps base[3] hub[3] tip motion[3]; ap_r ap_chord ap_twist (apc);
// attack (n_attack); cl cd (apc*n_attack).
// out.bin: u (3N), uu (3N), p (N), nut (N), then per step: it, err, divnorm, torque, thrust.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "falm_b200.hpp"

using namespace Falm;
typedef double Real;

namespace {
struct Reader {
    FILE *f;
    template <typename T> T get() { T v; if (fread(&v, sizeof(T), 1, f) != 1) throw Error(1, "short read"); return v; }
    std::vector<double> vec(size_t n) {
        std::vector<double> v(n);
        if (n && fread(v.data(), sizeof(double), n, f) != n) throw Error(1, "short read");
        return v;
    }
};
}  // namespace

int main(int argc, char **argv) {
    if (argc != 3 && argc != 6) {
        fprintf(stderr, "usage: %s case.bin out.bin [prefix interval tavg_start]\n", argv[0]);
        return 2;
    }
    const bool output = argc == 6;
    const std::string prefix = output ? argv[3] : "";
    const int interval = output ? atoi(argv[4]) : 0, tavg_start = output ? atoi(argv[5]) : 0;
    if (output && interval < 1) {
        fprintf(stderr, "nedo_driver: interval must be >= 1\n");
        return 2;
    }
    try {
        Reader rd{fopen(argv[1], "rb")};
        if (!rd.f) throw Error(1, "cannot open case");
        int sx = rd.get<int>(), sy = rd.get<int>(), sz = rd.get<int>(), gc = rd.get<int>(), steps = rd.get<int>();
        int maxit = rd.get<int>(), pc_maxit = rd.get<int>(), adv = rd.get<int>(), sgs = rd.get<int>(), bc = rd.get<int>();
        int pc_type = rd.get<int>(), alm_on = rd.get<int>();
        double Re = rd.get<double>(), Cs = rd.get<double>(), dt = rd.get<double>(), tol = rd.get<double>();
        double pc_relax = rd.get<double>(), u_inlet = rd.get<double>();
        std::vector<double> x = rd.vec(sx), y = rd.vec(sy), z = rd.vec(sz), hx = rd.vec(sx), hy = rd.vec(sy), hz = rd.vec(sz);
        const long N = (long)sx * sy * sz;
        std::vector<double> u0 = rd.vec(3 * N);
        falm_grid grid{sx, sy, sz, gc, x.data(), y.data(), z.data(), hx.data(), hy.data(), hz.data()};

        // FalmCore::computation_init (src/falm.h:342-431)
        Context ctx(grid, FALM_FP64);
        CPM &cpm = ctx.cpm;
        Int3 shape{{sx, sy, sz}};
        Matrix<Real> u(shape, 3, "u"), uu(shape, 3, "uu"), p(shape, 1, "p"), nut(shape, 1, "nut"), ff(shape, 3, "ff");
        Matrix<Real> rhs(shape, 1, "rhs"), res(shape, 1, "res"), div(shape, 1, "div"), u_previous(shape, 3, "u_prev");
        Matrix<Real> &kx = div, &g = div, &ja = div;   // unused by the B200 path (metrics come from the grid tables)
        memcpy(u.host.ptr, u0.data(), sizeof(double) * 3 * N);
        u.sync_to_device();

        FalmCFD<Real> fcfd(ctx);
        fcfd.init(Re, adv, sgs, Cs);
        FalmEq<Real> feq(ctx);
        feq.init(LSType::PBiCGStab, maxit, tol, 1.0, pc_type, pc_maxit, pc_relax);
        check(falm_bc_init(ctx.h, bc, u_inlet), ctx.h, "falm_bc_init");
        Real maxdiag = feq.PoissonOperator(bc);

        std::vector<double> ap[9];
        Alm::AlmHandler<Real> alm(ctx);
        if (alm_on) {
            int nb = rd.get<int>(), napb = rd.get<int>(), na = rd.get<int>(), atype = rd.get<int>();
            double radius = rd.get<double>(), hub_r = rd.get<double>(), eps = rd.get<double>();
            std::vector<double> base = rd.vec(3), hub = rd.vec(3), tip = rd.vec(1), motion = rd.vec(3);
            int apc = nb * napb;
            std::vector<double> r = rd.vec(apc), chord = rd.vec(apc), twist = rd.vec(apc), attack = rd.vec(na);
            std::vector<double> cl = rd.vec((size_t)apc * na), cd = rd.vec((size_t)apc * na);
            falm_alm_desc d{1, nb, napb, na, radius, hub_r, eps, base.data(), hub.data(), tip.data(), motion.data(), &atype,
                            r.data(), chord.data(), twist.data(), attack.data(), cl.data(), cd.data(), 0.0};
            alm.init(d);
        }
        fclose(rd.f);

        // app/nedo/main.cpp:132-133
        fcfd.UtoUU(u, uu, kx, ja, cpm);
        fcfd.SGS(u, nut, div, kx, ja, cpm);

        FILE *out = fopen(argv[2], "wb");
        if (!out) throw Error(1, "cannot open output");
        std::vector<double> stats;
        Matrix<Real> utavg(shape, 3, "utavg"), ptavg(shape, 1, "ptavg");
        std::vector<FalmSnapshotInfo> slices;
        auto name = [&](const std::string &pre, int it) {
            char buf[64];
            snprintf(buf, sizeof(buf), "_%06d_%010d", 0, it);
            return pre + buf;
        };
        for (int it = 1; it <= steps; it++) {
            const Real t = dt * it;
            // main_loop, app/nedo/main.cpp:150-204 (race-free pseudo-velocity: un = u_previous, ua separate)
            u_previous.copy(u);
            if (alm_on) alm.Alm(u, ff, t);
            fcfd.FSPseudoU(u_previous, u_previous, uu, u, nut, kx, g, ja, ff, dt, cpm);
            fcfd.UtoUU(u, uu, kx, ja, cpm);
            if (bc == FALM_BC_CAVITY) uubc(ctx, uu);
            fcfd.MACCalcPoissonRHS(uu, rhs, ja, dt, cpm, dim3(), maxdiag);
            feq.Solve(nullptr, p, rhs, res, cpm);
            pbc(ctx, p);
            fcfd.ProjectP(u, u, uu, uu, p, kx, g, dt, cpm);
            ubc(ctx, u, u_previous, (Real)dt, t);
            fcfd.SGS(u, nut, div, kx, ja, cpm);
            fcfd.Divergence(uu, div, ja, cpm);
            Real divnorm = std::sqrt(FalmMV<Real>::EuclideanNormSq(ctx, div)) / ((double)(sx - 2 * gc) * (sy - 2 * gc) * (sz - 2 * gc));
            printf("%8d %12.5e, %12.5e, %3d, %12.5e\n", it, t, divnorm, feq.it, feq.err);
            stats.push_back(feq.it);
            stats.push_back(feq.err);
            stats.push_back(divnorm);
            stats.push_back(alm_on ? alm.torque[0] : 0.0);
            stats.push_back(alm_on ? alm.thrust[0] : 0.0);
            if (output) {
                // FalmSolver::TAvg, then FalmSolver::outputUVWP (src/falm.h:433-475)
                const bool averaging = it >= tavg_start;
                if (averaging) {
                    TAvg(ctx, utavg, u, it - tavg_start + 1);
                    TAvg(ctx, ptavg, p, it - tavg_start + 1);
                }
                if (it % interval == 0) {
                    FalmIO::writeUVWP(name(prefix, it), ctx, u, p, it, t);
                    if (averaging) FalmIO::writeUVWP(name(prefix + "_tavg", it), ctx, utavg, ptavg, it, t);
                    slices.push_back(FalmSnapshotInfo{(size_t)it, t, averaging});
                }
            }
        }
        if (output) {
            FalmIO::wait(ctx);
            FalmIO::writeIndexFile(prefix + ".json", ctx, slices);
            FalmIO::writeControlVolumeFile(prefix + ".cv", ctx);
        }
        u.sync_to_host(); uu.sync_to_host(); p.sync_to_host(); nut.sync_to_host();
        fwrite(u.host.ptr, sizeof(double), 3 * N, out);
        fwrite(uu.host.ptr, sizeof(double), 3 * N, out);
        fwrite(p.host.ptr, sizeof(double), N, out);
        fwrite(nut.host.ptr, sizeof(double), N, out);
        fwrite(stats.data(), sizeof(double), stats.size(), out);
        fclose(out);
    } catch (const Error &e) {
        fprintf(stderr, "nedo_driver: %s (status %d)\n", e.what(), e.code);
        return 1;
    }
    return 0;
}
