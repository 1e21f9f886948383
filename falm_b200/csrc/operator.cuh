// The Poisson operator of the step (separable tables, maxdiag, scaling).
// Included by falm_b200.cu inside its anonymous namespace (after the headers
// it includes and the code before this point); not a standalone header.
#pragma once

// Build the separable Poisson tables.  For a Cartesian control volume
//   0.5*(g_d(c) + g_d(c+e_d))/ja(c)  with g_d = ja*kx_d^2
// depends on the index along d only; the table entry is evaluated with the
// reference's arithmetic (src/falm.h:394-400, app/nedo/main.cpp:43-83) at the
// cell (i, gc, gc) (resp. (gc, j, gc), (gc, gc, k)).  A dropped (Neumann)
// coefficient is stored as 0.
int build_poisson(falm_ctx *ctx, int kind) {
    const Geom &g = ctx->geo;
    const std::vector<double> *h[3] = {ctx->hx, ctx->hy, ctx->hz};
    const int s[3] = {g.sx, g.sy, g.sz};
    std::vector<double> up[3], um[3];
    double maxdiag = 0.0;
    auto gmet = [&](int d, int i, int j, int k) {
        double vol = (*h[0])[i] * (*h[1])[j] * (*h[2])[k];
        int id = d == 0 ? i : (d == 1 ? j : k);
        double kd = 1.0 / (*h[d])[id];
        return vol * kd * kd;
    };
    for (int d = 0; d < 3; d++) {
        up[d].assign(s[d], 0.0);
        um[d].assign(s[d], 0.0);
        for (int q = g.gc; q < s[d] - g.gc; q++) {
            int c[3] = {g.gc, g.gc, g.gc};
            c[d] = q;
            int cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
            cp[d] += 1; cm[d] -= 1;
            double jac = (*h[0])[c[0]] * (*h[1])[c[1]] * (*h[2])[c[2]];
            double gc0 = gmet(d, c[0], c[1], c[2]);
            double coef_p = 0.5 * (gc0 + gmet(d, cp[0], cp[1], cp[2])) / jac;
            double coef_m = 0.5 * (gc0 + gmet(d, cm[0], cm[1], cm[2])) / jac;
            // app/nedo/main.cpp:55 keeps the x+ coefficient (p = 0 guide cell); every other
            // physical face is Neumann (:60-83, app/lid3d/main.cpp:52-80); a slab interface
            // keeps its coefficients (the neighbour's plane lies beyond it)
            int plus_limit = (d == 0 && kind == FALM_BC_CHANNEL) ? s[d] - g.gc : s[d] - g.gc - 1;
            if (d == 2 && !(g.zphys & 2)) plus_limit = s[d] - g.gc;
            if (q < plus_limit) up[d][q] = coef_p;
            if (q > g.gc || (d == 2 && !(g.zphys & 1))) um[d][q] = coef_m;
        }
    }
    // maxdiag over the interior: |ac| is separable as well, but take the
    // exact maximum of the reference's accumulation order
    for (int k = g.gc; k < g.sz - g.gc; k++)
        for (int j = g.gc; j < g.sy - g.gc; j++)
            for (int i = g.gc; i < g.sx - g.gc; i++) {
                double ac = ((((-up[0][i]) - um[0][i]) - up[1][j]) - um[1][j] - up[2][k]) - um[2][k];
                maxdiag = std::max(maxdiag, std::fabs(ac));
            }
    if (ctx->slab_on && ctx->slab_nranks > 1) {
        // the maximum over the slabs (a collective: every rank builds its operator)
        double *d = nullptr;
        if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) { cudaGetLastError(); return fail(ctx, FALM_ERR_ALLOC, "poisson: maxdiag"); }
        int rc = cudaMemcpy(d, &maxdiag, sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess ? FALM_OK : FALM_ERR_CUDA;
        if (!rc) rc = ctx->transport.allreduce(ctx->transport.user, d, 1, FALM_REDUCE_MAX, nullptr);
        if (!rc && (cudaMemcpy(&maxdiag, d, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)) rc = FALM_ERR_CUDA;
        cudaFree(d);
        if (rc) { cudaGetLastError(); return fail(ctx, rc, "poisson: maxdiag over the slabs"); }
    }
    double scale = 1.0 / maxdiag;
    // layout: for each d: cm, cp, um, up (s[d] each), then dx0 (sx)
    size_t tot = 0;
    for (int d = 0; d < 3; d++) tot += 4 * (size_t)s[d];
    tot += g.sx;
    std::vector<double> h64(tot);
    std::vector<float> h32(tot);
    size_t off = 0;
    size_t o_cm[3], o_cp[3], o_um[3], o_up[3], o_dx0;
    for (int d = 0; d < 3; d++) {
        o_cm[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = um[d][q] * scale; off += s[d];
        o_cp[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = up[d][q] * scale; off += s[d];
        o_um[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = um[d][q]; off += s[d];
        o_up[d] = off; for (int q = 0; q < s[d]; q++) h64[off + q] = up[d][q]; off += s[d];
    }
    o_dx0 = off;
    for (int q = 0; q < g.sx; q++) h64[off + q] = (-up[0][q]) - um[0][q];
    off += g.sx;
    for (size_t q = 0; q < tot; q++) h32[q] = (float)h64[q];
    if (ctx->op_mem) { cudaFree(ctx->op_mem); ctx->op_mem = nullptr; }
    void *mem = nullptr;
    if (cudaMalloc(&mem, tot * (sizeof(double) + sizeof(float))) != cudaSuccess) { cudaGetLastError(); return fail(ctx, FALM_ERR_ALLOC, "poisson tables"); }
    double *d64 = (double *)mem;
    float *d32 = (float *)(d64 + tot);
    if (cudaMemcpy(d64, h64.data(), tot * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d32, h32.data(), tot * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(ctx, FALM_ERR_CUDA, "poisson tables copy");
    ctx->op_mem = mem;
    for (int d = 0; d < 3; d++) {
        ctx->pt64.cm[d] = d64 + o_cm[d]; ctx->pt64.cp[d] = d64 + o_cp[d]; ctx->pt64.um[d] = d64 + o_um[d]; ctx->pt64.up[d] = d64 + o_up[d];
        ctx->pt32.cm[d] = d32 + o_cm[d]; ctx->pt32.cp[d] = d32 + o_cp[d]; ctx->pt32.um[d] = d32 + o_um[d]; ctx->pt32.up[d] = d32 + o_up[d];
    }
    ctx->pt64.dx0 = d64 + o_dx0; ctx->pt32.dx0 = d32 + o_dx0;
    ctx->pt64.scale = scale; ctx->pt32.scale = (float)scale;
    ctx->pt64.koff = ctx->pt32.koff = g.koff;
    ctx->maxdiag = maxdiag;
    ctx->op_ready = 1;
    ctx->bc_kind_op = kind;
    // the coefficient of cell q towards q+1 equals that of q+1 towards q on every
    // axis (uniform spacing): the operator is symmetric over the interior
    ctx->op_symmetric = 1;
    for (int d = 0; d < 3; d++)
        for (int q = g.gc; q + 1 < s[d] - g.gc; q++)
            if (std::fabs(up[d][q] - um[d][q + 1]) > 1e-13 * std::fabs(up[d][q])) ctx->op_symmetric = 0;
    return FALM_OK;
}
