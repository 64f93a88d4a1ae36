// k_warm.cu -- warm starts of the red-black projection.
//
// The reference starts every projection from u = u*, p = p_old (phi = 0,
// pressure_redblack.f90:63-84).  A warm start supplies a guess dp for the
// pressure increment of the projection and applies it the way the sweeps
// apply their phi (pressure_redblack.f90:188-241): with phi = dp*dt_gamma
// per cell, each face moves by -(phi_right - phi_left)/h * mu of that face,
// wall faces of a Neumann-pressure wall stay put, and p += dp.  The sweeps
// then continue to the same target as without a guess (relative to
// ||div u*||, measured before the guess), so a good guess only saves
// iterations.
//
// Every projection records its increment dp = p_after - p_before per RK
// substage (projections are numbered in call order, three per step); the
// guesses are
//   MDX_GUESS_PREVIOUS      dp of the same substage in the previous step
//   MDX_GUESS_EXTRAPOLATED  2*dp(n-1) - dp(n-2) of the same substage (the
//                           previous one while only one is recorded)
//   MDX_GUESS_LEARNED       the extrapolated guess plus the U-Net's
//                           correction (k_unet.cu) predicted from the
//                           divergence that guess leaves.
// A guess that does not lower ||div u|| below ||div u*|| is undone (the
// first guessed step after a start from p = 0 takes the whole pressure
// build-up of the step before as its guess).  Supported with periodic x and
// z and y periodic or Neumann-pressure walls; otherwise the guess is
// skipped.
#include "mdx_internal.cuh"

#include <algorithm>

namespace {

// Apply the increment guess g (cells, (nx,ny,nz) order) to u, v, w, p.
// MUM: 0 mu = 1, 1 z-invariant planes, 2 padded arrays.
template <int MUM, int PY>
__global__ void k_apply_guess(mdx_dims d, double dg, double idx, double idy, double idz, const double* __restrict__ gs,
                              const double* __restrict__ mu, double* __restrict__ u, double* __restrict__ v,
                              double* __restrict__ w, double* __restrict__ p) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long r = t / d.nx;
        const int j = (int)(r % d.ny) + 1;
        const int k = (int)(r / d.ny) + 1;
        const int im = i == 1 ? d.nx : i - 1;
        const int km = k == 1 ? d.nz : k - 1;
        const long long c = pidx(d, i, j, k);
        const double phi = __ldg(gs + t) * dg;
        const double phx = __ldg(gs + qidx(d, im, j, k)) * dg;
        const double phz = __ldg(gs + qidx(d, i, j, km)) * dg;
        double mu_u = 1.0, mu_v = 1.0, mu_w = 1.0;
        if (MUM == 1) {
            const long long np = (long long)d.nxp * d.nyp, q = i + (long long)d.nxp * j;
            mu_u = __ldg(mu + q);
            mu_v = __ldg(mu + np + q);
            mu_w = __ldg(mu + 2 * np + q);
        } else if (MUM == 2) {
            mu_u = __ldg(mu + c);
            mu_v = __ldg(mu + d.npad + c);
            mu_w = __ldg(mu + 2 * d.npad + c);
        }
        u[c] -= (phi - phx) * idx * mu_u;
        w[c] -= (phi - phz) * idz * mu_w;
        if (PY || j >= 2) {   // v(1) of a wall stays put
            const int jm = j == 1 ? d.ny : j - 1;
            const double phy = __ldg(gs + qidx(d, i, jm, k)) * dg;
            v[c] -= (phi - phy) * idy * mu_v;
        }
        p[c] += __ldg(gs + t);
    }
}

__global__ void k_record_increment(mdx_dims d, const double* __restrict__ p, const double* __restrict__ p0,
                                   double* __restrict__ dp) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long r = t / d.nx;
        const int j = (int)(r % d.ny) + 1;
        const int k = (int)(r / d.ny) + 1;
        const long long c = pidx(d, i, j, k);
        dp[t] = p[c] - p0[c];
    }
}

__global__ void k_extrapolate(long long n, const double* __restrict__ h1, const double* __restrict__ h2,
                              double* __restrict__ g) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        g[t] = 2.0 * h1[t] - h2[t];
}

}  // namespace

bool mdx_guess_supported(const mdx_ctx_t* ctx) {
    const mdx_bc_t& b = ctx->bc;
    if (!b.is_periodic[0] || !b.is_periodic[2]) return false;
    if (b.is_periodic[1]) return true;
    return b.bc_type[bci(2, 0, 0)] == 1 && b.bc_value[bci(2, 0, 0)] == 0.0 && b.bc_type[bci(2, 1, 0)] == 1 &&
           b.bc_value[bci(2, 1, 0)] == 0.0;
}

int mdx_warm_alloc(mdx_ctx_t* ctx) {
    const size_t n = (size_t)ctx->d.nint;
    for (int t = 0; t < 3; ++t) {
        if (!ctx->dp_hist[t]) MDX_CUDA(ctx, cudaMalloc(&ctx->dp_hist[t], sizeof(double) * n));
        if (!ctx->dp_hist2[t]) MDX_CUDA(ctx, cudaMalloc(&ctx->dp_hist2[t], sizeof(double) * n));
    }
    if (!ctx->p_before) MDX_CUDA(ctx, cudaMalloc(&ctx->p_before, sizeof(double) * ctx->d.npad));
    if (!ctx->guess) MDX_CUDA(ctx, cudaMalloc(&ctx->guess, sizeof(double) * n));
    return MDX_OK;
}

void mdx_warm_free(mdx_ctx_t* ctx) {
    for (int t = 0; t < 3; ++t) {
        cudaFree(ctx->dp_hist[t]);
        ctx->dp_hist[t] = nullptr;
        cudaFree(ctx->dp_hist2[t]);
        ctx->dp_hist2[t] = nullptr;
    }
    cudaFree(ctx->p_before);
    ctx->p_before = nullptr;
    cudaFree(ctx->guess);
    ctx->guess = nullptr;
    cudaFree(ctx->ckpt);
    ctx->ckpt = nullptr;
    ctx->ckpt_valid = -1;
    ctx->hist_valid = 0;
}

int mdx_warm_begin(mdx_ctx_t* ctx) {
    MDX_TRY(mdx_warm_alloc(ctx));
    MDX_CUDA(ctx, cudaMemcpyAsync(ctx->p_before, ctx->f[MDX_PN], sizeof(double) * ctx->d.npad, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
    return MDX_OK;
}

int mdx_warm_end(mdx_ctx_t* ctx, bool converged, int iterations) {
    const int s = (int)(ctx->proj_count % 3);
    const mdx_dims& d = ctx->d;
    const int nb = (int)std::min<long long>((d.nint + 255) / 256, 8192);
    std::swap(ctx->dp_hist[s], ctx->dp_hist2[s]);   // the previous step's increment moves back one
    if (ctx->hist_valid & (1 << s)) ctx->hist_valid |= 8 << s;
    else ctx->hist_valid &= ~(8 << s);
    MDX_LAUNCH(ctx, MDX_T_OTHER, "record increment", k_record_increment, nb, 256, 0, d, ctx->f[MDX_PN], ctx->p_before,
               ctx->dp_hist[s]);
    ctx->hist_valid |= 1 << s;
    if (ctx->unet) MDX_TRY(mdx_unet_finish(ctx, converged, iterations));
    ctx->proj_count++;
    return MDX_OK;
}

// Undo an applied guess: u <- u*, p <- p at the start of the projection.
int mdx_undo_guess(mdx_ctx_t* ctx) {
    double** f = ctx->f;
    const size_t bytes = sizeof(double) * ctx->d.npad;
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_UN], f[MDX_US], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_VN], f[MDX_VS], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_WN], f[MDX_WS], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_PN], ctx->p_before, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return MDX_OK;
}

// Apply the increment guess gs (cells) with the IBM factors of this
// projection (ctx->mu in mode ctx->mu_mode: 0 one, 1 planes, 2 padded).
int mdx_apply_guess(mdx_ctx_t* ctx, const double* gs, double dg) {
    const int mu_mode = ctx->mu_mode;
    const mdx_dims& d = ctx->d;
    const mdx_grid_t& g = ctx->g;
    double** f = ctx->f;
    const int py = ctx->bc.is_periodic[1] ? 1 : 0;
    const int nb = (int)std::min<long long>((d.nint + 255) / 256, 8192);
    auto kfn = mu_mode == 1 ? (py ? k_apply_guess<1, 1> : k_apply_guess<1, 0>)
                            : (mu_mode == 2 ? (py ? k_apply_guess<2, 1> : k_apply_guess<2, 0>)
                                            : (py ? k_apply_guess<0, 1> : k_apply_guess<0, 0>));
    MDX_LAUNCH(ctx, MDX_T_OTHER, "apply guess", kfn, nb, 256, 0, d, dg, 1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz, gs,
               ctx->mu, f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN]);
    return MDX_OK;
}

// The guess of this projection into ctx->guess; *made = false when none is
// available (no history yet, no trained network).
int mdx_make_guess(mdx_ctx_t* ctx, bool* made) {
    *made = false;
    if (ctx->guess_mode == MDX_GUESS_ZERO) return MDX_OK;
    const int s = (int)(ctx->proj_count % 3);
    if (!(ctx->hist_valid & (1 << s))) return MDX_OK;
    const long long n = ctx->d.nint;
    if (ctx->guess_mode != MDX_GUESS_PREVIOUS && (ctx->hist_valid & (8 << s))) {
        const int nb = (int)std::min<long long>((n + 255) / 256, 8192);
        MDX_LAUNCH(ctx, MDX_T_OTHER, "extrapolate increment", k_extrapolate, nb, 256, 0, n, ctx->dp_hist[s],
                   ctx->dp_hist2[s], ctx->guess);
    } else {
        MDX_CUDA(ctx, cudaMemcpyAsync(ctx->guess, ctx->dp_hist[s], sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
    }
    *made = true;
    return MDX_OK;
}

int mdx_guess_apply(mdx_ctx_t* ctx, double dg, double r0, bool* guessed, double* rg) {
    *guessed = false;
    *rg = r0;
    bool made = false;
    MDX_TRY(mdx_make_guess(ctx, &made));
    if (!made) return MDX_OK;
    MDX_TRY(mdx_apply_guess(ctx, ctx->guess, dg));
    double r = r0;
    if (ctx->opts.tol > 0.0) {   // a guess that does not lower the divergence is undone
        double linf = 0.0;
        MDX_TRY(mdx_k_div_norms(ctx, ctx->f[MDX_UN], ctx->f[MDX_VN], ctx->f[MDX_WN], &r, &linf));
        if (!(r < r0)) return mdx_undo_guess(ctx);
    }
    *guessed = true;
    *rg = r;
    const int s = (int)(ctx->proj_count % 3);
    if (ctx->unet && ctx->guess_mode != MDX_GUESS_PREVIOUS && (ctx->hist_valid & (8 << s)))
        MDX_TRY(mdx_unet_correct(ctx, dg, rg));
    return MDX_OK;
}

extern "C" int mdx_set_pressure_guess(mdx_ctx_t* ctx, int mode, int record) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (mode < MDX_GUESS_ZERO || mode > MDX_GUESS_EXTRAPOLATED) return mdx_fail(ctx, MDX_ERR_ARG, "unknown guess mode %d", mode);
    ctx->guess_mode = mode;
    ctx->record_increments = record != 0;
    return MDX_OK;
}

extern "C" int mdx_warm_checkpoint(mdx_ctx_t* ctx, int restore) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (!ctx->fields) return mdx_fail(ctx, MDX_ERR_STATE, "field data not entered");
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = (size_t)ctx->d.nint;
    if (!restore) {
        if (!ctx->dp_hist[0]) MDX_TRY(mdx_warm_alloc(ctx));
        if (!ctx->ckpt) MDX_CUDA(ctx, cudaMalloc(&ctx->ckpt, sizeof(double) * 6 * n));
        for (int t = 0; t < 3; ++t) {
            MDX_CUDA(ctx, cudaMemcpyAsync(ctx->ckpt + t * n, ctx->dp_hist[t], sizeof(double) * n,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
            MDX_CUDA(ctx, cudaMemcpyAsync(ctx->ckpt + (3 + t) * n, ctx->dp_hist2[t], sizeof(double) * n,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
        }
        ctx->ckpt_valid = ctx->hist_valid;
        ctx->ckpt_count = ctx->proj_count;
        return MDX_OK;
    }
    if (ctx->ckpt_valid < 0 || !ctx->ckpt || !ctx->dp_hist[0])
        return mdx_fail(ctx, MDX_ERR_STATE, "no warm-start checkpoint saved");
    for (int t = 0; t < 3; ++t) {
        MDX_CUDA(ctx, cudaMemcpyAsync(ctx->dp_hist[t], ctx->ckpt + t * n, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
        MDX_CUDA(ctx, cudaMemcpyAsync(ctx->dp_hist2[t], ctx->ckpt + (3 + t) * n, sizeof(double) * n,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
    }
    ctx->hist_valid = ctx->ckpt_valid;
    ctx->proj_count = ctx->ckpt_count;
    return MDX_OK;
}

extern "C" int mdx_get_increment(mdx_ctx_t* ctx, int substage, double* host) {
    if (!ctx || !host || substage < 0 || substage > 2) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_get_increment: bad argument");
    if (!(ctx->hist_valid & (1 << substage)) || !ctx->dp_hist[substage])
        return mdx_fail(ctx, MDX_ERR_STATE, "no increment recorded for substage %d", substage);
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    MDX_CUDA(ctx, cudaMemcpyAsync(host, ctx->dp_hist[substage], sizeof(double) * ctx->d.nint, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MDX_OK;
}
