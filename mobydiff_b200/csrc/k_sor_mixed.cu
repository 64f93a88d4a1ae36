// k_sor_mixed.cu -- red-black projection with FP32 sweeps inside an FP64
// defect-correction loop (MDX_PREC_MIXED).
//
// The FP64 state u, v, w, p stays authoritative.  Each outer iteration
//   1. computes the FP64 divergence r = div(u) (the red-black neighbour rule)
//      and its L2 norm, kept as FP32 r~ per cell;
//   2. runs FP32 red-black sweeps on corrections du, dv, dw, dp (zero at the
//      start) with the cell divergence r~ + div(du): the same update as
//      pressure_redblack.f90:117-241 with homogeneous boundary values;
//   3. adds the corrections to the FP64 state (u += du, p += dp).
// It stops when the FP64 residual meets max(tol*||div u*||, atol), the
// target of the FP64 path.  A sweep moves 36 B per cell instead of 64 B;
// the slowest mode sets the iteration count, so the total number of sweeps
// stays close to the FP64 count.
//
// Supported: periodic x and z; y periodic, or walls with v Dirichlet 0 and p
// Neumann 0 (the channel), where the correction equations are exactly the
// homogeneous ones (the wall faces v(1), v(ny+1) stay 0); IBM factors 1 or
// z-invariant.  Other boundary sets run the FP64 path.
#include "mdx_cell32.cuh"

#include <algorithm>
#include <cmath>

namespace {

enum { MU_ONE = 0, MU_PLANE = 1, MU_FULL = 2 };   // the IBM-factor modes of k_sor.cu

__device__ inline double nanmax2(double a, double b) { return (a != a || b != b) ? (a + b) : fmax(a, b); }

__device__ inline void block_reduce3(double& s, double& m, double& u) {
    __shared__ double ss[MDX_RED_THREADS / 32], sm[MDX_RED_THREADS / 32], su[MDX_RED_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        m = nanmax2(m, __shfl_down_sync(0xffffffffu, m, o));
        u = nanmax2(u, __shfl_down_sync(0xffffffffu, u, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { ss[w] = s; sm[w] = m; su[w] = u; }
    __syncthreads();
    if (w == 0) {
        s = (l < MDX_RED_THREADS / 32) ? ss[l] : 0.0;
        m = (l < MDX_RED_THREADS / 32) ? sm[l] : 0.0;
        u = (l < MDX_RED_THREADS / 32) ? su[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o);
            m = nanmax2(m, __shfl_down_sync(0xffffffffu, m, o));
            u = nanmax2(u, __shfl_down_sync(0xffffffffu, u, o));
        }
    }
}

// FP64 divergence of (u,v,w) per cell (periodic x and z; y periodic when
// PY), stored as FP32 in r; partial sums of r^2, max|r| and max(|u|,|v|,|w|).
template <int PY>
__global__ void __launch_bounds__(MDX_RED_THREADS)
k_mixed_residual(mdx_dims d, double idx, double idy, double idz, const double* __restrict__ u,
                 const double* __restrict__ v, const double* __restrict__ w, float* __restrict__ r,
                 double* __restrict__ part) {
    double s = 0.0, m = 0.0, um = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long rr = t / d.nx;
        const int j = (int)(rr % d.ny) + 1;
        const int k = (int)(rr / d.ny) + 1;
        const long long c = pidx(d, i, j, k);
        const double dv = mixed_residual_cell<PY>(d, idx, idy, idz, i, j, k, u, v, w, r);
        s += dv * dv;
        m = nanmax2(m, fabs(dv));
        um = nanmax2(um, nanmax2(fabs(__ldg(u + c)), nanmax2(fabs(__ldg(v + c)), fabs(__ldg(w + c)))));
    }
    block_reduce3(s, m, um);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s;
        part[3 * blockIdx.x + 1] = m;
        part[3 * blockIdx.x + 2] = um;
    }
}

// Residual of the correction problem, r~ + div(du), as partial sums.
template <int PY>
__global__ void __launch_bounds__(MDX_RED_THREADS)
k_mixed_corr_residual(mdx_dims d, mixed_params P, const float* __restrict__ du, const float* __restrict__ dv,
                      const float* __restrict__ dw, const float* __restrict__ r, double* __restrict__ part) {
    double s = 0.0, m = 0.0, z = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long rr = t / d.nx;
        const int j = (int)(rr % d.ny) + 1;
        const int k = (int)(rr / d.ny) + 1;
        const float e = corr_residual_cell<PY>(d, P, i, j, k, du, dv, dw, r);
        s += (double)e * (double)e;
        m = nanmax2(m, fabs((double)e));
    }
    block_reduce3(s, m, z);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s;
        part[3 * blockIdx.x + 1] = m;
        part[3 * blockIdx.x + 2] = 0.0;
    }
}

// FP32 IBM factors and -omega/denom per (i,j) column (z-invariant): the
// denominator of pressure_redblack.f90:124-126 in FP64, then rounded.
__global__ void k_mixed_tables(mdx_dims d, int py, double idx2, double idy2, double idz2, double sor,
                               const double* __restrict__ mu, int plane_mu, float* __restrict__ mu32,
                               float* __restrict__ fac32) {
    const long long np = (long long)d.nxp * d.nyp;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x)
        mixed_tables_elem(d, py, idx2, idy2, idz2, sor, plane_mu ? mu : nullptr, t, mu32, fac32);
}

// One FP32 colour sweep of the correction (periodic x and z), on the
// colour-split arrays.
template <int PY>
__global__ void __launch_bounds__(256)
k_sor_sweep32(mdx_dims d, mixed_params P, int parity, int reverse, float* __restrict__ du, float* __restrict__ dv,
              float* __restrict__ dw, float* __restrict__ dp, const float* __restrict__ r,
              const float* __restrict__ mu32, const float* __restrict__ fac32) {
    const int ni = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int kk = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (ni > d.nx / 2 || j > d.ny || kk > d.nz) return;
    const int k = reverse ? d.nz + 1 - kk : kk;
    const int i = 1 + ((j + k + parity) & 1) + 2 * (ni - 1);
    sweep32_cell<PY>(d, P, i, j, k, du, dv, dw, dp, r, mu32, fac32);
}

// u += du, v += dv, w += dw, p += dp over the padded arrays; corrections reset.
__global__ void k_mixed_apply(mdx_dims d, double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                              double* __restrict__ p, float* __restrict__ du, float* __restrict__ dv,
                              float* __restrict__ dw, float* __restrict__ dp) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.npad; t += (long long)gridDim.x * blockDim.x)
        mixed_apply_elem(d, t, u, v, w, p, du, dv, dw, dp);
}

bool mixed_supported(const mdx_ctx_t* ctx) {
    const mdx_bc_t& b = ctx->bc;
    if (!b.is_periodic[0] || !b.is_periodic[2]) return false;
    if (ctx->mu_mode == MU_FULL) return false;
    if (b.is_periodic[1]) return true;
    const int* T = b.bc_type;
    const double* V = b.bc_value;
    return T[bci(2, 0, 2)] == 0 && V[bci(2, 0, 2)] == 0.0 && T[bci(2, 1, 2)] == 0 && V[bci(2, 1, 2)] == 0.0 &&
           T[bci(2, 0, 0)] == 1 && V[bci(2, 0, 0)] == 0.0 && T[bci(2, 1, 0)] == 1 && V[bci(2, 1, 0)] == 0.0;
}

// One allocation for the five colour-split FP32 arrays and the tables, each
// part starting on a 256-byte boundary.
int mixed_alloc(mdx_ctx_t* ctx) {
    if (ctx->mx_du) return MDX_OK;
    const size_t n = (size_t)split_elems(ctx->d), np = (size_t)split_plane_elems(ctx->d);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t arr = up(sizeof(float) * n), mu = up(sizeof(float) * 3 * np), fac = up(sizeof(float) * np);
    const size_t total = 5 * arr + mu + fac;
    char* base = nullptr;
    MDX_CUDA(ctx, cudaMalloc(&base, total));
    MDX_CUDA(ctx, cudaMemsetAsync(base, 0, total, ctx->stream));
    float** arrs[5] = {&ctx->mx_du, &ctx->mx_dv, &ctx->mx_dw, &ctx->mx_dp, &ctx->mx_r};
    for (int a = 0; a < 5; ++a) *arrs[a] = reinterpret_cast<float*>(base + a * arr);
    ctx->mx_mu = reinterpret_cast<float*>(base + 5 * arr);
    ctx->mx_fac = reinterpret_cast<float*>(base + 5 * arr + mu);
    ctx->mx_bytes = total;
    return MDX_OK;
}


}  // namespace

void mdx_mixed_free(mdx_ctx_t* ctx) {
    cudaFree(ctx->mx_du);   // the base of the one allocation
    float** arrs[7] = {&ctx->mx_du, &ctx->mx_dv, &ctx->mx_dw, &ctx->mx_dp, &ctx->mx_r, &ctx->mx_mu, &ctx->mx_fac};
    for (auto a : arrs) *a = nullptr;
    ctx->mx_bytes = 0;
}

// Called after u <- u*, the FP64 IBM factors of this projection and any
// warm-start guess; r0 and umax are ||div u*|| and max|u*| before the guess,
// atol the absolute floor.
int mdx_k_projection_redblack_mixed(mdx_ctx_t* ctx, double dg, mdx_solve_stats_t* st, bool* handled, double r0,
                                    double umax, double atol) {
    *handled = false;
    if (!mixed_supported(ctx) || ctx->opts.tol <= 0.0) return MDX_OK;
    *handled = true;
    MDX_TRY(mixed_alloc(ctx));
    const mdx_dims& d = ctx->d;
    const mdx_grid_t& g = ctx->g;
    const mdx_solver_opts_t& o = ctx->opts;
    const int py = ctx->bc.is_periodic[1] ? 1 : 0;
    double** f = ctx->f;
    const double idx = 1.0 / g.dx, idy = 1.0 / g.dy, idz = 1.0 / g.dz;
    mixed_params P{(float)idx, (float)idy, (float)idz, (float)(1.0 / dg)};
    const int nbt = (int)std::min<long long>(((long long)d.nxp * d.nyp + 255) / 256, 1024);
    MDX_LAUNCH(ctx, MDX_T_OTHER, "mixed tables", k_mixed_tables, nbt, 256, 0, d, py, idx * idx, idy * idy, idz * idz,
               o.inner_sor > 0.0 ? o.inner_sor : o.sor, ctx->mu, ctx->mu_mode == MU_PLANE ? 1 : 0, ctx->mx_mu,
               ctx->mx_fac);
    MDX_TRY(mdx_reduce_init(ctx));

    auto residual = [&](double* l2, double* umax) -> int {
        if (py)
            MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "mixed residual", k_mixed_residual<1>, ctx->red_blocks, MDX_RED_THREADS,
                       0, d, idx, idy, idz, f[MDX_UN], f[MDX_VN], f[MDX_WN], ctx->mx_r, ctx->red_part);
        else
            MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "mixed residual", k_mixed_residual<0>, ctx->red_blocks, MDX_RED_THREADS,
                       0, d, idx, idy, idz, f[MDX_UN], f[MDX_VN], f[MDX_WN], ctx->mx_r, ctx->red_part);
        double s2 = 0.0, mx = 0.0, um = 0.0;
        MDX_TRY(mdx_reduce_partials(ctx, &s2, &mx, &um));
        *l2 = std::sqrt(s2);
        if (umax) *umax = um;
        return MDX_OK;
    };
    auto corr_residual = [&](double* l2) -> int {
        if (py)
            MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "mixed corr residual", k_mixed_corr_residual<1>, ctx->red_blocks,
                       MDX_RED_THREADS, 0, d, P, ctx->mx_du, ctx->mx_dv, ctx->mx_dw, ctx->mx_r, ctx->red_part);
        else
            MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "mixed corr residual", k_mixed_corr_residual<0>, ctx->red_blocks,
                       MDX_RED_THREADS, 0, d, P, ctx->mx_du, ctx->mx_dv, ctx->mx_dw, ctx->mx_r, ctx->red_part);
        double s2 = 0.0;
        MDX_TRY(mdx_reduce_partials(ctx, &s2, nullptr, nullptr));
        *l2 = std::sqrt(s2);
        return MDX_OK;
    };
    auto sweeps = [&](int iters) -> int {
        const int na = d.nx / 2;
        dim3 block(32, 4, 2);
        dim3 grid((na + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
        mdx_event_pair run{};
        mdx_sweep_run_begin(ctx, &run);
        for (int it = 0; it < iters; ++it)
            for (int parity = 0; parity < 2; ++parity) {
                auto kfn = py ? k_sor_sweep32<1> : k_sor_sweep32<0>;
                MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep fp32", kfn, grid, block, 0, d, P, parity, parity,
                           ctx->mx_du, ctx->mx_dv, ctx->mx_dw, ctx->mx_dp, ctx->mx_r, ctx->mx_mu, ctx->mx_fac);
            }
        mdx_sweep_run_end(ctx, &run);
        return MDX_OK;
    };

    mdx_solve_stats_t s{};
    double r = 0.0;
    MDX_TRY(residual(&r, nullptr));   // r~ of the current (possibly warm-started) state
    s.residual0 = r0;
    s.atol = atol;
    const double target = std::max(o.tol * r0, atol);
    int it = 0, outer = 0;
    s.status = MDX_NOT_CONVERGED;
    if (!std::isfinite(r0) || !std::isfinite(umax) || !std::isfinite(r)) {
        s.status = MDX_ERR_NONFINITE;
    } else if (r <= target) {
        s.status = MDX_OK;
        s.residual = r0 > 0.0 ? r / r0 : 0.0;
    } else {
        // FP32 resolves a correction to about 1e-5 of its right-hand side
        const double inner_rel = 1e-5;
        while (it < o.max_iter && outer < 16) {
            ++outer;
            const double inner_target = std::max(target, inner_rel * r);
            double e = r, best = r;
            int stale = 0;
            mdx_check_schedule cs;
            cs.start(o.check_every, o.check_mode, r);
            int block = cs.every;
            while (it < o.max_iter) {
                const int m = std::min(block, o.max_iter - it);
                MDX_TRY(sweeps(m));
                it += m;
                MDX_TRY(corr_residual(&e));
                if (!std::isfinite(e)) break;
                if (e <= inner_target) break;
                // FP32 stagnation: less than 0.1 % per check_every iterations for 20 x check_every
                if (e < std::pow(0.999, (double)m / cs.every) * best) { best = e; stale = 0; }
                else if ((stale += m) >= 20 * cs.every) break;
                block = cs.next(it, e, inner_target);
            }
            const long long n = d.npad;
            MDX_LAUNCH(ctx, MDX_T_OTHER, "mixed apply", k_mixed_apply, (int)std::min<long long>((n + 255) / 256, 8192),
                       256, 0, d, f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], ctx->mx_du, ctx->mx_dv, ctx->mx_dw,
                       ctx->mx_dp);
            MDX_TRY(residual(&r, nullptr));
            if (!std::isfinite(r)) { s.status = MDX_ERR_NONFINITE; break; }
            if (r <= target) { s.status = MDX_OK; break; }
        }
        s.residual = r / r0;
    }
    s.iterations = it;
    s.variant = 100 + outer;   // mixed path: 100 + outer FP64 corrections
    ctx->last = s;
    if (st) *st = s;
    return MDX_OK;
}
