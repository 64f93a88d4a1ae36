// k_sor.cu -- red-black SOR velocity-pressure projection,
// src/modules/pressure/pressure_redblack.f90:27-254.
//
// One launch per colour sweep, one thread per cell of that colour.  Cells of
// one colour share no face and each owns its p, so the parallel sweep is
// bit-for-bit the reference's sequential loop (compiled with -fmad=false and
// the reference's expression order).  The reference iterates a fixed nIter;
// with tol > 0 the sweeps continue until ||div u||_2 <= max(tol*||div u*||_2,
// atol), checked every `check_every` iterations by a deterministic reduction.
//
// HBM: the IBM factors mu = 1/(1+dt_gamma*coef) are computed once per
// projection (the reference recomputes six per cell per sweep, :117-122);
// when the coefficients do not vary along z -- both the reference geometry
// and the wavy channel depend on x and y only -- mu is one (nx+2)(ny+2)
// plane per component that stays in L2, otherwise a padded array.  The same
// formula gives the same bits.  Successive sweeps walk the z planes in
// opposite directions, so each starts on the planes the previous one left
// in the 126 MB L2.
#include "mdx_internal.cuh"

#include <algorithm>
#include <cmath>

struct mdx_sor_params {
    double dx, dy, dz, idx, idy, idz, idx2, idy2, idz2, idt, sor, dt_gamma;
};

enum { MU_ONE = 0, MU_PLANE = 1, MU_FULL = 2 };

// mu = 1/(1 + dt_gamma*coef) over n elements of each component.
__global__ void k_mu_tables(long long n, long long stride_in, double dg, const double* __restrict__ cu,
                            const double* __restrict__ cv, const double* __restrict__ cw, double* __restrict__ mu) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        mu[t] = 1.0 / (1.0 + dg * __ldg(cu + t));
        mu[n + t] = 1.0 / (1.0 + dg * __ldg(cv + t));
        mu[2 * n + t] = 1.0 / (1.0 + dg * __ldg(cw + t));
    }
    (void)stride_in;
}

template <int MU>
__global__ void __launch_bounds__(256)
k_sor_sweep(mdx_dims d, mdx_bc_dev bc, mdx_sor_params p, int parity, int reverse, double* __restrict__ un,
            double* __restrict__ vn, double* __restrict__ wn, double* __restrict__ pn,
            const double* __restrict__ mu) {
    const int ni = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int kk = blockIdx.z * blockDim.z + threadIdx.z + 1;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    if (ni > nx / 2 || j > ny || kk > nz) return;
    const int k = reverse ? nz + 1 - kk : kk;
    const int* T = bc.type;
    const double* V = bc.value;
    const bool perx = bc.per[0] != 0, pery = bc.per[1] != 0, perz = bc.per[2] != 0;
    int jp = j + 1;
    if (pery && jp > ny) jp = 1;
    int kp = k + 1;
    if (perz && kp > nz) kp = 1;
    const int iLo = 1 + ((j + k + parity) & 1);
    const int i = iLo + 2 * (ni - 1);
    int ip = i + 1;
    if (perx && ip > nx) ip = 1;
    const double dg = p.dt_gamma;
    const long long c = pidx(d, i, j, k);
    const long long cip = pidx(d, ip, j, k), cjp = pidx(d, i, jp, k), ckp = pidx(d, i, j, kp);

    (void)dg;
    double mu_u_i = 1.0, mu_u_ip = 1.0, mu_v_j = 1.0, mu_v_jp = 1.0, mu_w_k = 1.0, mu_w_kp = 1.0;
    if (MU == MU_PLANE) {  // :117-122, z-invariant coefficients
        const long long np = (long long)d.nxp * d.nyp;
        const long long q = i + (long long)d.nxp * j;
        mu_u_i = __ldg(mu + q);
        mu_u_ip = __ldg(mu + ip + (long long)d.nxp * j);
        mu_v_j = __ldg(mu + np + q);
        mu_v_jp = __ldg(mu + np + i + (long long)d.nxp * jp);
        mu_w_k = __ldg(mu + 2 * np + q);
        mu_w_kp = mu_w_k;
    } else if (MU == MU_FULL) {
        const long long np = d.npad;
        mu_u_i = __ldg(mu + c);
        mu_u_ip = __ldg(mu + cip);
        mu_v_j = __ldg(mu + np + c);
        mu_v_jp = __ldg(mu + np + cjp);
        mu_w_k = __ldg(mu + 2 * np + c);
        mu_w_kp = __ldg(mu + 2 * np + ckp);
    }
    const double denom = (mu_u_i + mu_u_ip) * p.idx2 + (mu_w_k + mu_w_kp) * p.idz2 + (mu_v_j + mu_v_jp) * p.idy2;

    if (!perx) {  // :128-144
        if (i < 2) {
            if (T[bci(1, 0, 1)] == 0) un[c] = V[bci(1, 0, 1)];
            else un[c] = un[cip] - V[bci(1, 0, 1)] * p.dx;
        }
        if (i >= nx) {
            if (T[bci(1, 1, 1)] == 0) un[cip] = V[bci(1, 1, 1)];
            else un[cip] = un[pidx(d, nx, j, k)] + V[bci(1, 1, 1)] * p.dx;
        }
    }
    if (!pery) {  // :146-162
        if (j < 2) {
            if (T[bci(2, 0, 2)] == 0) vn[c] = V[bci(2, 0, 2)];
            else vn[c] = vn[cjp] - V[bci(2, 0, 2)] * p.dy;
        }
        if (j >= ny) {
            if (T[bci(2, 1, 2)] == 0) vn[cjp] = V[bci(2, 1, 2)];
            else vn[cjp] = vn[c] + V[bci(2, 1, 2)] * p.dy;
        }
    }
    if (!perz) {  // :164-180
        if (k < 2) {
            if (T[bci(3, 0, 3)] == 0) wn[c] = V[bci(3, 0, 3)];
            else wn[c] = wn[ckp] - V[bci(3, 0, 3)] * p.dz;
        }
        if (k >= nz) {
            if (T[bci(3, 1, 3)] == 0) wn[ckp] = V[bci(3, 1, 3)];
            else wn[ckp] = wn[c] + V[bci(3, 1, 3)] * p.dz;
        }
    }
    double u_i = un[c], u_ip = un[cip], v_j = vn[c], v_jp = vn[cjp], w_k = wn[c], w_kp = wn[ckp];
    // :183-188
    const double phi = ((u_ip - u_i) * p.idx + (v_jp - v_j) * p.idy + (w_kp - w_k) * p.idz) * (-p.sor / denom);
    pn[c] = pn[c] + phi * p.idt;
    // :190-241
    u_i = u_i - phi * p.idx * mu_u_i;
    if (!perx && i == 1) {
        if (T[bci(1, 0, 0)] == 0) u_i = u_i + V[bci(1, 0, 0)] * p.idx * mu_u_i;
        else u_i = u_i + (phi * p.idx - V[bci(1, 0, 0)]) * mu_u_i;
    }
    un[c] = u_i;
    u_ip = u_ip + phi * p.idx * mu_u_ip;
    if (!perx && i == nx) {
        if (T[bci(1, 1, 0)] == 0) u_ip = u_ip - V[bci(1, 1, 0)] * p.idx * mu_u_ip;
        else u_ip = u_ip + (V[bci(1, 1, 0)] - phi * p.idx) * mu_u_ip;
    }
    un[cip] = u_ip;
    v_j = v_j - phi * p.idy * mu_v_j;
    if (!pery && j == 1) {
        if (T[bci(2, 0, 0)] == 0) v_j = v_j + V[bci(2, 0, 0)] * p.idy * mu_v_j;
        else v_j = v_j + (phi * p.idy - V[bci(2, 0, 0)]) * mu_v_j;
    }
    vn[c] = v_j;
    v_jp = v_jp + phi * p.idy * mu_v_jp;
    if (!pery && j == ny) {
        if (T[bci(2, 1, 0)] == 0) v_jp = v_jp - V[bci(2, 1, 0)] * p.idy * mu_v_jp;
        else v_jp = v_jp + (V[bci(2, 1, 0)] - phi * p.idy) * mu_v_jp;
    }
    vn[cjp] = v_jp;
    w_k = w_k - phi * p.idz * mu_w_k;
    if (!perz && k == 1) {
        if (T[bci(3, 0, 0)] == 0) w_k = w_k + V[bci(3, 0, 0)] * p.idz * mu_w_k;
        else w_k = w_k + (phi * p.idz - V[bci(3, 0, 0)]) * mu_w_k;
    }
    wn[c] = w_k;
    w_kp = w_kp + phi * p.idz * mu_w_kp;
    if (!perz && k == nz) {
        // :237 -- the Dirichlet branch of the reference has no mu factor
        if (T[bci(3, 1, 0)] == 0) w_kp = w_kp - V[bci(3, 1, 0)] * p.idz;
        else w_kp = w_kp + (V[bci(3, 1, 0)] - phi * p.idz) * mu_w_kp;
    }
    wn[ckp] = w_kp;
}

double mdx_div_floor(const mdx_ctx_t* ctx, double umax) {
    const double eps = 2.220446049250313e-16;
    const mdx_grid_t& g = ctx->g;
    return eps * std::sqrt((double)ctx->d.nint) * umax * (1.0 / g.dx + 1.0 / g.dy + 1.0 / g.dz);
}

static mdx_sor_params sor_params(const mdx_ctx_t* ctx, double dg) {
    const mdx_grid_t& g = ctx->g;
    mdx_sor_params p;
    p.dx = g.dx; p.dy = g.dy; p.dz = g.dz;
    p.idx = 1.0 / g.dx; p.idy = 1.0 / g.dy; p.idz = 1.0 / g.dz;   // :54-60
    p.idx2 = p.idx * p.idx; p.idy2 = p.idy * p.idy; p.idz2 = p.idz * p.idz;
    p.idt = 1.0 / dg;
    p.sor = ctx->opts.sor;
    p.dt_gamma = dg;
    return p;
}

static int sor_iteration(mdx_ctx_t* ctx, const mdx_sor_params& p) {
    const mdx_dims& d = ctx->d;
    double** f = ctx->f;
    const int na = d.nx / 2;
    dim3 block(32, 4, 2);
    dim3 grid((na + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
    for (int parity = 0; parity < 2; ++parity) {
        const int rev = parity;   // red sweeps walk k up, black sweeps walk k down
        if (ctx->mu_mode == MU_ONE)
            MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep", k_sor_sweep<MU_ONE>, grid, block, 0, d, ctx->bcd, p, parity,
                       rev, f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], ctx->mu);
        else if (ctx->mu_mode == MU_PLANE)
            MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep", k_sor_sweep<MU_PLANE>, grid, block, 0, d, ctx->bcd, p,
                       parity, rev, f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], ctx->mu);
        else
            MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep", k_sor_sweep<MU_FULL>, grid, block, 0, d, ctx->bcd, p,
                       parity, rev, f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], ctx->mu);
    }
    return MDX_OK;
}

// The IBM factors of this projection's dt_gamma.
static int mu_tables(mdx_ctx_t* ctx, double dg) {
    const mdx_dims& d = ctx->d;
    if (ctx->ibm_zero) {
        ctx->mu_mode = MU_ONE;
        return MDX_OK;
    }
    const bool plane = ctx->coef_zinv;
    const long long n = plane ? (long long)d.nxp * d.nyp : d.npad;
    if (!ctx->mu || ctx->mu_elems < 3 * n) {
        cudaFree(ctx->mu);
        ctx->mu = nullptr;
        MDX_CUDA(ctx, cudaMalloc(&ctx->mu, sizeof(double) * 3 * n));
        ctx->mu_elems = 3 * n;
    }
    ctx->mu_mode = plane ? MU_PLANE : MU_FULL;
    const int nb = (int)std::min<long long>((n + 255) / 256, 4096);
    MDX_LAUNCH(ctx, MDX_T_OTHER, "mu tables", k_mu_tables, nb, 256, 0, n, 0LL, dg, ctx->f[MDX_COEF_U],
               ctx->f[MDX_COEF_V], ctx->f[MDX_COEF_W], ctx->mu);
    return MDX_OK;
}

int mdx_k_projection_redblack(mdx_ctx_t* ctx, double dg, mdx_solve_stats_t* st) {
    const mdx_dims& d = ctx->d;
    double** f = ctx->f;
    const size_t bytes = sizeof(double) * d.npad;
    // :63-84 -- u <- u* over the whole padded arrays
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_UN], f[MDX_US], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_VN], f[MDX_VS], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_WN], f[MDX_WS], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_TRY(mu_tables(ctx, dg));
    const mdx_sor_params p = sor_params(ctx, dg);
    mdx_solve_stats_t s{};
    const mdx_solver_opts_t& o = ctx->opts;
    if (o.tol <= 0.0) {
        for (int it = 0; it < o.n_iter; ++it) MDX_TRY(sor_iteration(ctx, p));
        s.iterations = o.n_iter;
        s.status = MDX_OK;
    } else {
        double r0 = 0.0, linf = 0.0, r = 0.0, umax = 0.0;
        MDX_TRY(mdx_k_div_norms(ctx, f[MDX_UN], f[MDX_VN], f[MDX_WN], &r0, &linf, &umax));
        s.residual0 = r0;
        // converged when ||div u|| <= max(tol*||div u*||, atol); the default
        // atol is the round-off level of the divergence, below which a
        // relative target cannot be met once u* is nearly solenoidal
        const double atol = (o.atol < 0.0) ? mdx_div_floor(ctx, umax) : o.atol;
        s.atol = atol;
        const double target = std::max(o.tol * r0, atol);
        if (!std::isfinite(r0) || !std::isfinite(umax)) {
            s.status = MDX_ERR_NONFINITE;
        } else if (r0 <= target) {
            s.status = MDX_OK;
            s.residual = (r0 > 0.0) ? 1.0 : 0.0;
        } else {
            int it = 0;
            s.status = MDX_NOT_CONVERGED;
            r = r0;
            while (it < o.max_iter) {
                const int m = std::min(o.check_every, o.max_iter - it);
                for (int q = 0; q < m; ++q) MDX_TRY(sor_iteration(ctx, p));
                it += m;
                MDX_TRY(mdx_k_div_norms(ctx, f[MDX_UN], f[MDX_VN], f[MDX_WN], &r, &linf));
                if (!std::isfinite(r)) { s.status = MDX_ERR_NONFINITE; break; }
                if (r <= target) { s.status = MDX_OK; break; }
            }
            s.iterations = it;
            s.residual = r / r0;
        }
    }
    ctx->last = s;
    if (st) *st = s;
    return MDX_OK;
}
