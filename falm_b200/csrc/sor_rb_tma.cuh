// Temporally blocked red-black SOR: H consecutive half sweeps (colours c1,
// c1^1, ...) of FalmEqDevCall::SORSweep (src/dev/FalmEqDevCall.cu:175-211) in
// one pass over HBM, out of place (x_in -> x_out).
//
// A CTA owns a 64 x 8 tile of columns and a chunk of z planes.  Half sweep h
// must be evaluated on the tile plus a ring of H-h cells (in x, y and z) for
// the last one to be exact on the tile, so every plane of x_in and b is staged
// as one (tile + halo) TMA box.  The z march is a wavefront: when raw plane q
// has landed, half sweep 1 updates plane q-1, half sweep 2 plane q-2, ...,
// half sweep H plane q-H, each in place in shared memory and only on its own
// colour (which reads only the other colour, so in-place is exact), then the
// tile of plane q-H is final and is written to x_out.  Reads come from x_in
// only, so neighbouring CTAs never see a partially updated field.
#pragma once
#include "poisson.cuh"
#include "tma.cuh"

namespace fb {

// the SOR correction (b - Ax)/ac: IEEE division in FP64; in FP32 (mixed
// precision) the fast division, within 2 ulp
__device__ __forceinline__ double sor_div(double a, double b) { return a / b; }
__device__ __forceinline__ float sor_div(float a, float b) { return __fdividef(a, b); }

template <typename T, int H>
struct RBTile {
    static constexpr int TX = 64, TY = 8;
    // x halo of the box: >= H, and box origin i0 - HX = 64 bx + 2 - HX on a
    // 16-byte boundary for gc = 2
    static constexpr int HX = (H <= 2) ? 2 : (sizeof(T) == 4 ? 6 : 4);
    static constexpr int BX = TX + 2 * HX, BY = TY + 2 * H, PE = BX * BY;
    static constexpr int PB = (PE * (int)sizeof(T) + 127) / 128 * 128;   // one field plane
    static constexpr int SLOT = 2 * PB;                                   // x plane, then b plane
    // H+2 resident planes + look-ahead; a power of two keeps the slot index a mask
    static constexpr int NS = 8;
    static constexpr int TAB = (3 * BX + 4 * BY) * (int)sizeof(T);
    static constexpr int SMEM = NS * SLOT + 128 + ((TAB + 127) / 128) * 128 + 128;
};

template <typename T, int H>
__global__ void __launch_bounds__(256) k_sor_rb_tma(Geom g, int kc, const __grid_constant__ CUtensorMap mx,
                                                   const __grid_constant__ CUtensorMap mb, PoissonTables<T> tb, T *__restrict__ xout,
                                                   T omega, int c1, const SolverScalars *sc, int *err) {
    using L = RBTile<T, H>;
    constexpr unsigned NS = L::NS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t *bar = (uint64_t *)(smem + NS * L::SLOT);
    T *tab = (T *)(smem + NS * L::SLOT + 128);
    if (sc && sc->done) return;
    const int i0 = g.gc + blockIdx.x * L::TX, j0 = g.gc + blockIdx.y * L::TY;
    const int k0 = g.gc + blockIdx.z * kc, k1 = min(k0 + kc, g.sz - g.gc);
    const int P0 = k0 - H, nplanes = (k1 + H) - P0;
    const int xb = max(0, box_origin(i0 - L::HX, L::BX, g.sx, 16 / (int)sizeof(T)));
    const int yb = max(0, box_origin(j0 - H, L::BY, g.sy, 1));
    // x/y operator tables of the box: aw, ae, dx0 per column; as, an, up1, um1 per row
    T *t_aw = tab, *t_ae = tab + L::BX, *t_dx = tab + 2 * L::BX;
    T *t_as = tab + 3 * L::BX, *t_an = t_as + L::BY, *t_up = t_an + L::BY, *t_um = t_up + L::BY;
    for (int q = threadIdx.x; q < L::BX; q += blockDim.x) {
        const int x = min(xb + q, g.sx - 1);
        t_aw[q] = ldg(tb.cm[0] + x); t_ae[q] = ldg(tb.cp[0] + x); t_dx[q] = ldg(tb.dx0 + x);
    }
    for (int q = threadIdx.x; q < L::BY; q += blockDim.x) {
        const int y = min(yb + q, g.sy - 1);
        t_as[q] = ldg(tb.cm[1] + y); t_an[q] = ldg(tb.cp[1] + y); t_up[q] = ldg(tb.up[1] + y); t_um[q] = ldg(tb.um[1] + y);
    }
    auto slot = [&](int q) { return smem + ((unsigned)q % NS) * L::SLOT; };
    // planes outside the tensor (z < 0 or z >= sz) are never read: complete their barrier without a copy
    auto issue = [&](int q) {
        uint64_t *b = bar + ((unsigned)q % NS);
        const int z = P0 + q;
        if (z < 0 || z >= g.sz) { mbar_arrive(b); return; }
        unsigned char *s = slot(q);
        if (tma_ok(s, xb, yb, z, (int)sizeof(T), g.sx, g.sy, g.sz) && tma_ok(s + L::PB, xb, yb, z, (int)sizeof(T), g.sx, g.sy, g.sz)) {
            mbar_expect_tx(b, 2 * L::PE * sizeof(T));
            tma_load_4d(s, &mx, xb, yb, z, 0, b);
            tma_load_4d(s + L::PB, &mb, xb, yb, z, 0, b);
        } else {
            tma_reject(b, err, 4);
        }
    };
    // warp 0 polls the barriers; the block barrier that follows makes the
    // landed planes visible to every thread
    auto wait_q = [&](int q) -> bool { return threadIdx.x >= 32 || mbar_wait(bar + ((unsigned)q % NS), ((unsigned)q / NS) & 1, err); };
    if (threadIdx.x == 0) {
        prefetch_tmap(&mx); prefetch_tmap(&mb);
        for (unsigned s = 0; s < NS; s++) mbar_init(bar + s, 1);
        mbar_fence_init();
    }
    __syncthreads();
    int issued = min((int)NS, nplanes), waited = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < issued; q++) issue(q);
    const int ilo = g.gc, ihi = g.sx - g.gc, jlo = g.gc, jhi = g.sy - g.gc, klo = g.gc, khi = g.sz - g.gc;
    const long long sxy = (long long)g.sx * g.sy;
    for (int q = 0; q < nplanes; q++) {
        bool fail = !wait_q(q);
        waited = q + 1;
        if (__syncthreads_or(fail)) goto drain;
        // half sweeps 1..H on planes q-1 .. q-H (wavefront, ascending h)
#pragma unroll
        for (int h = 1; h <= H; h++) {
            const int p = q - h, kp = P0 + p, ring = H - h;
            if (p >= 1 && kp >= max(klo, k0 - ring) && kp < min(khi, k1 + ring)) {
                const int color = (c1 + h - 1) & 1;
                T *X0 = (T *)slot(p);
                const T *Xm = (const T *)slot(p - 1), *Xp = (const T *)slot(p + 1);
                const T *B0 = (const T *)(slot(p) + L::PB);
                const T ab = ldg(tb.cm[2] + kp), at = ldg(tb.cp[2] + kp), up2 = ldg(tb.up[2] + kp), um2 = ldg(tb.um[2] + kp);
                const int xs = i0 - ring, ys = j0 - ring;
                const int Wr = L::TX + 2 * ring, Hh = L::TY + 2 * ring, M = (Wr + 1) >> 1;
                for (int s = threadIdx.x; s < Hh * M; s += blockDim.x) {
                    const int r = s / M, m = s - r * M;
                    const int y = ys + r;
                    const int x = xs + 2 * m + ((color ^ (xs + y + kp)) & 1);
                    if (x >= xs + Wr || x < ilo || x >= ihi || y < jlo || y >= jhi) continue;
                    const int ox = x - xb, oy = y - yb, o = oy * L::BX + ox;
                    const T aw = t_aw[ox], ae = t_ae[ox], as = t_as[oy], an = t_an[oy];
                    const T ac = ((((t_dx[ox] - t_up[oy]) - t_um[oy]) - up2) - um2) * tb.scale;
                    const T xc = X0[o];
                    const T r7 = ac * xc + ae * X0[o + 1] + aw * X0[o - 1] + an * X0[o + L::BX] + as * X0[o - L::BX] +
                                 at * Xp[o] + ab * Xm[o];
                    X0[o] = xc + omega * sor_div(B0[o] - r7, ac);
                }
            }
            __syncthreads();
        }
        // the tile of plane q-H is final
        {
            const int p = q - H, kp = P0 + p;
            if (p >= 0 && kp >= k0 && kp < k1) {
                const T *X0 = (const T *)slot(p);
                for (int s = threadIdx.x; s < L::TX * L::TY; s += blockDim.x) {
                    const int x = i0 + (s & (L::TX - 1)), y = j0 + s / L::TX;
                    if (x < ihi && y < jhi) xout[(long long)x + (long long)y * g.sx + kp * sxy] = X0[(y - yb) * L::BX + (x - xb)];
                }
            }
        }
        // plane q-H-1 was last read by half sweep H above and by the previous
        // iteration's write-out, both behind a barrier: refill its slot
        {
            const int qn = q - H - 1 + (int)NS;
            if (q - H - 1 >= 0 && qn < nplanes) {
                if (threadIdx.x == 0) { fence_proxy_async(); issue(qn); }
                issued = qn + 1;
            }
        }
    }
    return;
drain:
    for (int q = waited; q < issued; q++) wait_q(q);
}

}  // namespace fb
