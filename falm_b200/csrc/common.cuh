// Device helpers shared by every kernel of falm_b200.
//
// Work decomposition ("row kernels"): a region of the box is a set of rows
// along x.  Each warp owns whole rows (j,k) and its 32 lanes walk the row with
// stride 32, so every global load and store of a warp is one contiguous run of
// 32 elements (coalesced).  The grid is sized to the SM count (persistent
// style, grid-stride over rows), which keeps the per-block partials of the
// fused reductions small enough for a single-block final sum.
#pragma once
#include "falm_internal.cuh"
#include <math.h>
#include <float.h>

namespace fb {

struct Region3 {
    int i0, i1, j0, j1, k0, k1;   // half-open ranges
    __host__ __device__ inline int nrows() const { return (j1 - j0) * (k1 - k0); }
};

__host__ inline Region3 interior(const Geom &g) {
    return Region3{g.gc, g.sx - g.gc, g.gc, g.sy - g.gc, g.gc, g.sz - g.gc};
}
// face map of the reference: interior shape + 1, offset - 1 (src/FalmCFD.cpp:119-126)
__host__ inline Region3 facemap(const Geom &g) {
    return Region3{g.gc - 1, g.sx - g.gc, g.gc - 1, g.sy - g.gc, g.gc - 1, g.sz - g.gc};
}

// iterate rows of a region: f(j, k) called once per (warp, row)
#define FB_FOR_ROWS(R, J, K)                                                            \
    for (int _row = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5), _nr = (R).nrows(); \
         _row < _nr; _row += gridDim.x * kWarpsPerBlock)                                \
        for (int J = (R).j0 + _row % ((R).j1 - (R).j0), K = (R).k0 + _row / ((R).j1 - (R).j0), _once = 1; _once; _once = 0)

#define FB_FOR_I(R, I) for (int I = (R).i0 + (threadIdx.x & 31); I < (R).i1; I += 32)

template <typename T> __device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// ---------------------------------------------------------------- metrics
// Bitwise the values of the reference's metric planes (src/falm.h:390-403):
// volume = (hx*hy)*hz, g_d = (volume*kx_d)*kx_d, kx_d = 1/h_d.
template <typename T>
struct MetricView {
    Metric<T> m;
    __device__ __forceinline__ T kx(int d, int idx) const { return ldg(m.k[d] + idx); }
    __device__ __forceinline__ T ja(int i, int j, int k) const {
        return ldg(m.h[0] + i) * ldg(m.h[1] + j) * ldg(m.h[2] + k);
    }
    __device__ __forceinline__ T g(int d, int i, int j, int k) const {
        int idx = d == 0 ? i : (d == 1 ? j : k);
        T kd = ldg(m.k[d] + idx);
        return ja(i, j, k) * kd * kd;
    }
};

// ---------------------------------------------------------------- reductions
template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
    for (int d = 0; d < NV; d++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[d] += __shfl_down_sync(0xffffffffu, v[d], o);
}

// Deterministic grid reduction.  Every block stores one partial per value;
// the last block to arrive sums the partials in a fixed order and returns
// true (all its threads), with the totals in out[] (valid in every thread of
// that block).  Other blocks return false.  NW: warps per block.
template <int NV, int NW = kWarpsPerBlock>
__device__ bool grid_sum(double (&v)[NV], const RedWork &rw, double (&out)[NV]) {
    __shared__ double sm[NV][NW];
    __shared__ bool last;
    __shared__ double tot[NV];
    warp_sum<NV>(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int d = 0; d < NV; d++) sm[d][warp] = v[d];
    __syncthreads();
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int d = 0; d < NV; d++) {
            double s = 0.0;
            for (int w = 0; w < NW; w++) s += sm[d][w];
            rw.partials[d * rw.maxBlocks + bid] = s;
        }
        __threadfence();
        unsigned ticket = atomicAdd(rw.counter, 1u);
        last = (ticket == nblk - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int d = 0; d < NV; d++) {
        acc[d] = 0.0;
        for (int b = threadIdx.x; b < (int)nblk; b += blockDim.x) acc[d] += __ldcg(rw.partials + d * rw.maxBlocks + b);
    }
    warp_sum<NV>(acc);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int d = 0; d < NV; d++) sm[d][warp] = acc[d];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int d = 0; d < NV; d++) {
            double s = 0.0;
            for (int w = 0; w < NW; w++) s += sm[d][w];
            tot[d] = s;
        }
        *rw.counter = 0u;
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < NV; d++) out[d] = tot[d];
    return true;
}

__device__ __forceinline__ double to_d(double v) { return v; }
__device__ __forceinline__ double to_d(float v) { return (double)v; }

}  // namespace fb
