// k_step.cu -- predictor (momentum), ghost-cell boundary conditions, CFL,
// cell-centre velocities and the seeded initial condition.
//
// Parity: this file is compiled with -fmad=false and every expression keeps
// the reference's Fortran evaluation order, so the predictor and the
// boundary conditions are bit-for-bit the reference arithmetic (x86-64
// gfortran -O2 has no FMA contraction).  Skipping the IBM factor when all
// coefficients are zero is exact: 1/(1+dt_gamma*0) == 1.
#include "mdx_cell.cuh"

// ---------------------------------------------------------------------------
// Predictor, src/modules/step.f90:76-204.  A block is a 32 x 8 (i, j) tile
// that walks MOM_KZ planes along z; each thread carries the values its
// stencil reuses from plane to plane in registers (u, v, w, p at the cell in
// planes k-1..k+1, u(i+1) and v(j+1) of plane k-1, w(i-1) and w(j-1) of
// plane k+1), so per cell it reads the five values of plane k+1 it will need
// and the in-plane x/y neighbours of plane k: 22 loads instead of 31.  Warps
// read 32 consecutive doubles of every array.  The arithmetic is
// momentum_vals, the same as the ensemble kernel's.
// ---------------------------------------------------------------------------
constexpr int MOM_KZ = 8;

// DTD: the three step scalars come from the device's dt (adaptive-dt graph);
// otherwise their values are kernel parameters.
template <bool IBM, bool DTD>
__global__ void __launch_bounds__(256, 4)
k_momentum(mdx_dims d, mdx_step_params p, mdx_dscal da, mdx_dscal db, mdx_dscal dg,
           const double* __restrict__ un, const double* __restrict__ vn, const double* __restrict__ wn,
           const double* __restrict__ pn, double* __restrict__ us, double* __restrict__ vs,
           double* __restrict__ ws, double* __restrict__ ou, double* __restrict__ ov, double* __restrict__ ow,
           const double* __restrict__ cu, const double* __restrict__ cv, const double* __restrict__ cw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k0 = blockIdx.z * MOM_KZ + 1;
    if (i > d.nx || j > d.ny) return;
    const double dt_alpha = DTD ? da.get() : da.v, dt_beta = DTD ? db.get() : db.v,
                 dt_gamma = DTD ? dg.get() : dg.v;
    const int k1 = min(k0 + MOM_KZ - 1, d.nz);
    const long long SX = 1, SY = d.nxp, SZ = (long long)d.nxp * d.nyp;
    long long c = pidx(d, i, j, k0);
    long long q = qidx(d, i, j, k0);
    const long long SQ = (long long)d.nx * d.ny;
    // planes k0-1 and k0
    double u_km = __ldg(un + c - SZ), u_c = __ldg(un + c), u_ip_km = __ldg(un + c + SX - SZ);
    double v_km = __ldg(vn + c - SZ), v_c = __ldg(vn + c), v_jp_km = __ldg(vn + c + SY - SZ);
    double w_km = __ldg(wn + c - SZ), w_c = __ldg(wn + c), w_im = __ldg(wn + c - SX), w_jm = __ldg(wn + c - SY);
    double p_km = __ldg(pn + c - SZ);
    for (int k = k0; k <= k1; ++k, c += SZ, q += SQ) {
        mdx_mom_nb n;
        // plane k+1
        n.u_kp_v = __ldg(un + c + SZ);
        n.v_kp_v = __ldg(vn + c + SZ);
        n.w_kp_v = __ldg(wn + c + SZ);
        n.w_im_kp_v = __ldg(wn + c - SX + SZ);
        n.w_jm_kp_v = __ldg(wn + c - SY + SZ);
        // plane k
        n.u_ip_v = __ldg(un + c + SX); n.u_im_v = __ldg(un + c - SX);
        n.u_jp_v = __ldg(un + c + SY); n.u_jm_v = __ldg(un + c - SY); n.u_ip_jm_v = __ldg(un + c + SX - SY);
        n.v_ip_v = __ldg(vn + c + SX); n.v_im_v = __ldg(vn + c - SX);
        n.v_jp_v = __ldg(vn + c + SY); n.v_jm_v = __ldg(vn + c - SY); n.v_im_jp_v = __ldg(vn + c - SX + SY);
        n.w_ip_v = __ldg(wn + c + SX); n.w_jp_v = __ldg(wn + c + SY);
        n.p_c_v = __ldg(pn + c); n.p_im_v = __ldg(pn + c - SX); n.p_jm_v = __ldg(pn + c - SY);
        // carried
        n.u_c_v = u_c; n.u_km_v = u_km; n.u_ip_km_v = u_ip_km;
        n.v_c_v = v_c; n.v_km_v = v_km; n.v_jp_km_v = v_jp_km;
        n.w_c_v = w_c; n.w_km_v = w_km; n.w_im_v = w_im; n.w_jm_v = w_jm;
        n.p_km_v = p_km;
        momentum_vals<IBM>(n, p, dt_alpha, dt_beta, dt_gamma, us, vs, ws, ou, ov, ow, cu, cv, cw, c, q, c, i, j, k);
        u_km = u_c; u_c = n.u_kp_v; u_ip_km = n.u_ip_v;
        v_km = v_c; v_c = n.v_kp_v; v_jp_km = n.v_jp_v;
        w_km = w_c; w_c = n.w_kp_v; w_im = n.w_im_kp_v; w_jm = n.w_jm_kp_v;
        p_km = n.p_c_v;
    }
}

mdx_step_params mdx_make_params(const mdx_ctx_t* ctx) {
    const mdx_grid_t& g = ctx->g;
    mdx_step_params p;
    p.dx = g.dx; p.dy = g.dy; p.dz = g.dz;
    const double dx2 = g.dx * g.dx, dy2 = g.dy * g.dy, dz2 = g.dz * g.dz;  // step.f90:57-67
    p.idx = 1.0 / g.dx; p.idy = 1.0 / g.dy; p.idz = 1.0 / g.dz;
    p.idx2 = 1.0 / dx2; p.idy2 = 1.0 / dy2; p.idz2 = 1.0 / dz2;
    p.ire = 1.0 / g.re;
    p.fx = g.forcing_x; p.fy = g.forcing_y; p.fz = g.forcing_z;
    p.nx0 = ctx->bc.is_periodic[0] ? 1 : 2;   // step.f90:71-73
    p.ny0 = ctx->bc.is_periodic[1] ? 1 : 2;
    p.nz0 = ctx->bc.is_periodic[2] ? 1 : 2;
    return p;
}

int mdx_k_momentum(mdx_ctx_t* ctx, mdx_dscal da, mdx_dscal db, mdx_dscal dg) {
    const mdx_dims& d = ctx->d;
    dim3 block(32, 8, 1);
    dim3 grid((d.nx + 31) / 32, (d.ny + 7) / 8, (d.nz + MOM_KZ - 1) / MOM_KZ);
    mdx_step_params p = mdx_make_params(ctx);
    double** f = ctx->f;
    const bool dev = da.p || db.p || dg.p;
    auto kfn = ctx->ibm_zero ? (dev ? k_momentum<false, true> : k_momentum<false, false>)
                             : (dev ? k_momentum<true, true> : k_momentum<true, false>);
    MDX_LAUNCH(ctx, MDX_T_MOMENTUM, "momentum", kfn, grid, block, 0, d, p, da, db, dg, f[MDX_UN], f[MDX_VN],
               f[MDX_WN], f[MDX_PN], f[MDX_US], f[MDX_VS], f[MDX_WS], f[MDX_OLDRHSU], f[MDX_OLDRHSV], f[MDX_OLDRHSW],
               f[MDX_COEF_U], f[MDX_COEF_V], f[MDX_COEF_W]);
    return MDX_OK;
}

// ---------------------------------------------------------------------------
// apply_bc of the FFT builds, src/modules/boundary.f90:23-170, as the
// reference's three sequential phases (y walls, x periodic, z periodic).
// Each phase writes only ghost planes (plus the v wall row) and reads
// interior or already-final values, so threads within a phase never race.
// ---------------------------------------------------------------------------
struct mdx_six { double *un, *vn, *wn, *us, *vs, *ws, *pn; };

__global__ void k_bc_walls_y(mdx_dims d, mdx_six f) {   // boundary.f90:48-67
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > d.nx + 1 || k > d.nz + 1) return;
    const int ny = d.ny;
    f.un[pidx(d, i, ny + 1, k)] = -f.un[pidx(d, i, ny, k)];
    f.vn[pidx(d, i, ny + 1, k)] = 0.0;
    f.wn[pidx(d, i, ny + 1, k)] = -f.wn[pidx(d, i, ny, k)];
    f.un[pidx(d, i, 0, k)] = -f.un[pidx(d, i, 1, k)];
    f.vn[pidx(d, i, 1, k)] = 0.0;
    f.wn[pidx(d, i, 0, k)] = -f.wn[pidx(d, i, 1, k)];
    f.us[pidx(d, i, ny + 1, k)] = -f.us[pidx(d, i, ny, k)];
    f.vs[pidx(d, i, ny + 1, k)] = 0.0;
    f.ws[pidx(d, i, ny + 1, k)] = -f.ws[pidx(d, i, ny, k)];
    f.us[pidx(d, i, 0, k)] = -f.us[pidx(d, i, 1, k)];
    f.vs[pidx(d, i, 1, k)] = 0.0;
    f.ws[pidx(d, i, 0, k)] = -f.ws[pidx(d, i, 1, k)];
}

__global__ void k_bc_periodic_x(mdx_dims d, mdx_six f) {   // boundary.f90:87-117
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y * blockDim.y + threadIdx.y;
    if (j > d.ny + 1 || k > d.nz + 1) return;
    const int nx = d.nx;
    f.un[pidx(d, 0, j, k)] = f.un[pidx(d, nx, j, k)];
    f.wn[pidx(d, 0, j, k)] = f.wn[pidx(d, nx, j, k)];
    f.un[pidx(d, nx + 1, j, k)] = f.un[pidx(d, 1, j, k)];
    f.wn[pidx(d, nx + 1, j, k)] = f.wn[pidx(d, 1, j, k)];
    f.us[pidx(d, 0, j, k)] = f.us[pidx(d, nx, j, k)];
    f.ws[pidx(d, 0, j, k)] = f.ws[pidx(d, nx, j, k)];
    f.us[pidx(d, nx + 1, j, k)] = f.us[pidx(d, 1, j, k)];
    f.ws[pidx(d, nx + 1, j, k)] = f.ws[pidx(d, 1, j, k)];
    if (j >= 1) {
        f.vn[pidx(d, 0, j, k)] = f.vn[pidx(d, nx, j, k)];
        f.vn[pidx(d, nx + 1, j, k)] = f.vn[pidx(d, 1, j, k)];
        f.vs[pidx(d, 0, j, k)] = f.vs[pidx(d, nx, j, k)];
        f.vs[pidx(d, nx + 1, j, k)] = f.vs[pidx(d, 1, j, k)];
    }
    if (j >= 1 && j <= d.ny) {
        f.pn[pidx(d, 0, j, k)] = f.pn[pidx(d, nx, j, k)];
        f.pn[pidx(d, nx + 1, j, k)] = f.pn[pidx(d, 1, j, k)];
    }
}

__global__ void k_bc_periodic_z(mdx_dims d, mdx_six f) {   // boundary.f90:137-168
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > d.nx + 1 || j > d.ny + 1) return;
    const int nz = d.nz;
    f.un[pidx(d, i, j, 0)] = f.un[pidx(d, i, j, nz)];
    f.wn[pidx(d, i, j, 0)] = f.wn[pidx(d, i, j, nz)];
    f.un[pidx(d, i, j, nz + 1)] = f.un[pidx(d, i, j, 1)];
    f.wn[pidx(d, i, j, nz + 1)] = f.wn[pidx(d, i, j, 1)];
    f.us[pidx(d, i, j, 0)] = f.us[pidx(d, i, j, nz)];
    f.ws[pidx(d, i, j, 0)] = f.ws[pidx(d, i, j, nz)];
    f.us[pidx(d, i, j, nz + 1)] = f.us[pidx(d, i, j, 1)];
    f.ws[pidx(d, i, j, nz + 1)] = f.ws[pidx(d, i, j, 1)];
    if (j >= 1) {
        f.vn[pidx(d, i, j, 0)] = f.vn[pidx(d, i, j, nz)];
        f.vn[pidx(d, i, j, nz + 1)] = f.vn[pidx(d, i, j, 1)];
        f.vs[pidx(d, i, j, 0)] = f.vs[pidx(d, i, j, nz)];
        f.vs[pidx(d, i, j, nz + 1)] = f.vs[pidx(d, i, j, 1)];
    }
    if (j >= 1 && j <= d.ny) {
        f.pn[pidx(d, i, j, 0)] = f.pn[pidx(d, i, j, nz)];
        f.pn[pidx(d, i, j, nz + 1)] = f.pn[pidx(d, i, j, 1)];
    }
}

__global__ void k_bcrb_y(mdx_dims d, mdx_bc_dev bc, double dy, mdx_four f);
__global__ void k_bcrb_x(mdx_dims d, mdx_bc_dev bc, double dx, mdx_four f);
__global__ void k_bcrb_z(mdx_dims d, mdx_bc_dev bc, double dz, mdx_four f);

int mdx_k_apply_bc(mdx_ctx_t* ctx) {
    const mdx_dims& d = ctx->d;
    double** a = ctx->f;
    if (ctx->fft_ext_x || ctx->fft_ext_z) {
        // walls in x or z on the FFT path: the general boundary routine
        // (apply_bc_redblack's face rules, which for walls in y with zero
        // velocity give apply_bc's values) on u, v, w, p and on u*, v*, w*,
        // whose wall faces the right-hand side reads
        dim3 b(32, 8);
        for (const mdx_four& f : {mdx_four{a[MDX_UN], a[MDX_VN], a[MDX_WN], a[MDX_PN]},
                                  mdx_four{a[MDX_US], a[MDX_VS], a[MDX_WS], a[MDX_PN]}}) {
            MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc y (walls)", k_bcrb_y, dim3((d.nx + 31) / 32, (d.nz + 7) / 8), b, 0, d,
                       ctx->bcd, ctx->g.dy, f);
            MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc x (walls)", k_bcrb_x, dim3((d.ny + 31) / 32, (d.nz + 7) / 8), b, 0, d,
                       ctx->bcd, ctx->g.dx, f);
            MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc z (walls)", k_bcrb_z, dim3((d.nx + 31) / 32, (d.ny + 7) / 8), b, 0, d,
                       ctx->bcd, ctx->g.dz, f);
        }
        return MDX_OK;
    }
    mdx_six f{a[MDX_UN], a[MDX_VN], a[MDX_WN], a[MDX_US], a[MDX_VS], a[MDX_WS], a[MDX_PN]};
    dim3 b(32, 8);
    MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc y", k_bc_walls_y, dim3((d.nxp + 31) / 32, (d.nzp + 7) / 8), b, 0, d, f);
    MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc x", k_bc_periodic_x, dim3((d.nyp + 31) / 32, (d.nzp + 7) / 8), b, 0, d, f);
    MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc z", k_bc_periodic_z, dim3((d.nxp + 31) / 32, (d.nyp + 7) / 8), b, 0, d, f);
    return MDX_OK;
}

// ---------------------------------------------------------------------------
// apply_bc_redblack, src/modules/boundary.f90:173-368.  The reference loops
// over the faces sequentially in the order bottom, top, left, right, front,
// back; faces of different directions read each other's values (e.g. the
// x-periodic copy reads the v wall row set by the y faces), so the three
// directions run as three ordered launches.  Within one direction the
// min and max faces of a column touch disjoint cells (ny, nx, nz >= 2).
// ---------------------------------------------------------------------------

__global__ void k_bcrb_y(mdx_dims d, mdx_bc_dev bc, double dy, mdx_four f) {   // :207-258
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > d.nx || k > d.nz) return;
    bcrb_y_col(d, bc, dy, f, i, k);
}

__global__ void k_bcrb_x(mdx_dims d, mdx_bc_dev bc, double dx, mdx_four f) {   // :259-310
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (j > d.ny || k > d.nz) return;
    bcrb_x_col(d, bc, dx, f, j, k);
}

__global__ void k_bcrb_z(mdx_dims d, mdx_bc_dev bc, double dz, mdx_four f) {   // :311-364
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > d.nx || j > d.ny) return;
    bcrb_z_col(d, bc, dz, f, i, j);
}

int mdx_k_apply_bc_redblack(mdx_ctx_t* ctx) {
    const mdx_dims& d = ctx->d;
    double** a = ctx->f;
    mdx_four f{a[MDX_UN], a[MDX_VN], a[MDX_WN], a[MDX_PN]};
    dim3 b(32, 8);
    MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc_redblack y", k_bcrb_y, dim3((d.nx + 31) / 32, (d.nz + 7) / 8), b, 0, d,
               ctx->bcd, ctx->g.dy, f);
    MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc_redblack x", k_bcrb_x, dim3((d.ny + 31) / 32, (d.nz + 7) / 8), b, 0, d,
               ctx->bcd, ctx->g.dx, f);
    MDX_LAUNCH(ctx, MDX_T_BC, "apply_bc_redblack z", k_bcrb_z, dim3((d.nx + 31) / 32, (d.ny + 7) / 8), b, 0, d,
               ctx->bcd, ctx->g.dz, f);
    return MDX_OK;
}

// ---------------------------------------------------------------------------
// Deterministic reductions: fixed grid, per-block partials in a fixed order,
// one final block.  Used by the CFL (max) and the divergence norms (sum of
// squares and max-abs).
// ---------------------------------------------------------------------------
#define MDX_RED_THREADS 256

// Block reduction of (sum, max, max) in a fixed order; NaN in a max slot wins.
__device__ inline double nanmax(double a, double b) { return (a != a || b != b) ? (a + b) : fmax(a, b); }

__device__ inline void block_reduce3(double& s, double& m, double& u) {
    __shared__ double ss[MDX_RED_THREADS / 32], sm[MDX_RED_THREADS / 32], su[MDX_RED_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        m = nanmax(m, __shfl_down_sync(0xffffffffu, m, o));
        u = nanmax(u, __shfl_down_sync(0xffffffffu, u, o));
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
            m = nanmax(m, __shfl_down_sync(0xffffffffu, m, o));
            u = nanmax(u, __shfl_down_sync(0xffffffffu, u, o));
        }
    }
}

// Divergence with the red-black neighbour rule (periodic wrap to 1):
// partials of sum(div^2), max|div| and max(|u|,|v|,|w|) over the cells.
// SPLIT: u, v, w in the colour-split layout (the FP64 sweeps' working copies);
// the same cells in the same order, so the same sums.
template <bool SPLIT>
__device__ __forceinline__ long long lay(const mdx_dims& d, int i, int j, int k) {
    return SPLIT ? cidx(d, i, j, k) : pidx(d, i, j, k);
}

template <bool SPLIT>
__global__ void __launch_bounds__(MDX_RED_THREADS)
k_div_partials(mdx_dims d, int perx, int pery, int perz, double idx, double idy, double idz,
               const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
               double* __restrict__ part) {
    double s = 0.0, m = 0.0, um = 0.0;
    const long long n = d.nint;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long r = t / d.nx;
        const int j = (int)(r % d.ny) + 1;
        const int k = (int)(r / d.ny) + 1;
        const int ip = (perx && i + 1 > d.nx) ? 1 : i + 1;
        const int jp = (pery && j + 1 > d.ny) ? 1 : j + 1;
        const int kp = (perz && k + 1 > d.nz) ? 1 : k + 1;
        const long long c = lay<SPLIT>(d, i, j, k);
        const double uc = __ldg(u + c), vc = __ldg(v + c), wc = __ldg(w + c);
        const double dv = (__ldg(u + lay<SPLIT>(d, ip, j, k)) - uc) * idx +
                          (__ldg(v + lay<SPLIT>(d, i, jp, k)) - vc) * idy +
                          (__ldg(w + lay<SPLIT>(d, i, j, kp)) - wc) * idz;
        s += dv * dv;
        m = nanmax(m, fabs(dv));
        um = nanmax(um, nanmax(fabs(uc), nanmax(fabs(vc), fabs(wc))));
    }
    block_reduce3(s, m, um);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s;
        part[3 * blockIdx.x + 1] = m;
        part[3 * blockIdx.x + 2] = um;
    }
}

__global__ void __launch_bounds__(MDX_RED_THREADS)
k_cfl_partials(long long n, double dx, double dy, double dz, const double* __restrict__ u,
               const double* __restrict__ v, const double* __restrict__ w, double* __restrict__ part) {
    double m = 0.0, s = 0.0, um = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        m = fmax(m, fabs(__ldg(u + t) / dx));
        m = fmax(m, fabs(__ldg(v + t) / dy));
        m = fmax(m, fabs(__ldg(w + t) / dz));
    }
    block_reduce3(s, m, um);
    if (threadIdx.x == 0) { part[3 * blockIdx.x] = 0.0; part[3 * blockIdx.x + 1] = m; part[3 * blockIdx.x + 2] = 0.0; }
}

__global__ void __launch_bounds__(MDX_RED_THREADS)
k_reduce_final(int nb, const double* __restrict__ part, double* __restrict__ out) {
    double s = 0.0, m = 0.0, um = 0.0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        s += part[3 * t];
        m = nanmax(m, part[3 * t + 1]);
        um = nanmax(um, part[3 * t + 2]);
    }
    block_reduce3(s, m, um);
    if (threadIdx.x == 0) { out[0] = s; out[1] = m; out[2] = um; }
}

int mdx_reduce_init(mdx_ctx_t* ctx) {
    if (ctx->red_part) return MDX_OK;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    ctx->red_blocks = sms * 4;
    MDX_CUDA(ctx, cudaMalloc(&ctx->red_part, sizeof(double) * 3 * ctx->red_blocks));
    MDX_CUDA(ctx, cudaMalloc(&ctx->red_out, sizeof(double) * 3));
    MDX_CUDA(ctx, cudaMallocHost(&ctx->red_host, sizeof(double) * 3));
    MDX_CUDA(ctx, cudaEventCreate(&ctx->tune_ev[0]));
    MDX_CUDA(ctx, cudaEventCreate(&ctx->tune_ev[1]));
    return MDX_OK;
}

// Enqueue the divergence-norm reduction; the result lands in red_host after
// the stream reaches it (caller synchronises).
int mdx_k_div_norms_async(mdx_ctx_t* ctx, const double* u, const double* v, const double* w) {
    MDX_TRY(mdx_reduce_init(ctx));
    const mdx_dims& d = ctx->d;
    const int* per = ctx->bc.is_periodic;
    auto kfn = ctx->split_norms ? k_div_partials<true> : k_div_partials<false>;
    MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "divergence partials", kfn, ctx->red_blocks, MDX_RED_THREADS, 0, d, per[0],
               per[1], per[2], 1.0 / ctx->g.dx, 1.0 / ctx->g.dy, 1.0 / ctx->g.dz, u, v, w, ctx->red_part);
    MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "reduce final", k_reduce_final, 1, MDX_RED_THREADS, 0, ctx->red_blocks,
               ctx->red_part, ctx->red_out);
    MDX_CUDA(ctx, cudaMemcpyAsync(ctx->red_host, ctx->red_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return MDX_OK;
}

// Reduce the per-block partials (sum, max, max) left in red_part by a
// kernel of another module and bring them to the host (synchronises).
int mdx_reduce_partials(mdx_ctx_t* ctx, double* sum, double* max1, double* max2) {
    MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "reduce final", k_reduce_final, 1, MDX_RED_THREADS, 0, ctx->red_blocks,
               ctx->red_part, ctx->red_out);
    MDX_CUDA(ctx, cudaMemcpyAsync(ctx->red_host, ctx->red_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (sum) *sum = ctx->red_host[0];
    if (max1) *max1 = ctx->red_host[1];
    if (max2) *max2 = ctx->red_host[2];
    return MDX_OK;
}

int mdx_k_div_norms(mdx_ctx_t* ctx, const double* u, const double* v, const double* w, double* l2, double* linf,
                    double* umax) {
    MDX_TRY(mdx_k_div_norms_async(ctx, u, v, w));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *l2 = sqrt(ctx->red_host[0]);
    *linf = ctx->red_host[1];
    if (umax) *umax = ctx->red_host[2];
    return MDX_OK;
}

// get_cfl, src/modules/step.f90:210-258: max over the padded arrays of
// |u/dx|, |v/dy|, |w/dz| (max is exact, so the result is order-independent).
// After a step of the adaptive-dt path (src/main.f90:67,92-97), on the
// device: t += dt (the step's dt), cfl = get_cfl's maximum (red[1]), and
// when cflmax > 0 and cfl > 0, dt = min(cflmax/cfl, dtmax).  s = {dt, t, cfl}.
__global__ void k_dt_update(const double* __restrict__ red, double* __restrict__ s, double cflmax, double dtmax) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dt = s[0];
    s[1] = s[1] + dt;
    const double cfl = red[1];
    s[2] = cfl;
    if (cflmax > 0.0 && cfl > 0.0) s[0] = fmin(cflmax / cfl, dtmax);
}

// get_cfl's reduction into red_out[1], left on the device.
static int cfl_launch(mdx_ctx_t* ctx) {
    MDX_TRY(mdx_reduce_init(ctx));
    const mdx_dims& d = ctx->d;
    MDX_LAUNCH(ctx, MDX_T_OTHER, "cfl partials", k_cfl_partials, ctx->red_blocks, MDX_RED_THREADS, 0, d.npad,
               ctx->g.dx, ctx->g.dy, ctx->g.dz, ctx->f[MDX_UN], ctx->f[MDX_VN], ctx->f[MDX_WN],
               ctx->red_part);
    MDX_LAUNCH(ctx, MDX_T_OTHER, "reduce final", k_reduce_final, 1, MDX_RED_THREADS, 0, ctx->red_blocks,
               ctx->red_part, ctx->red_out);
    return MDX_OK;
}

int mdx_k_dt_update(mdx_ctx_t* ctx, double* s, double cflmax, double dtmax) {
    MDX_TRY(cfl_launch(ctx));
    MDX_LAUNCH(ctx, MDX_T_OTHER, "dt update", k_dt_update, 1, 32, 0, ctx->red_out, s, cflmax, dtmax);
    return MDX_OK;
}

int mdx_k_cfl(mdx_ctx_t* ctx, double* cfl) {
    MDX_TRY(cfl_launch(ctx));
    MDX_CUDA(ctx, cudaMemcpyAsync(ctx->red_host, ctx->red_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *cfl = ctx->red_host[1];
    return MDX_OK;
}

// ---------------------------------------------------------------------------
// center_vel, src/modules/io.f90:196-216.
// ---------------------------------------------------------------------------
__global__ void k_center_vel(mdx_dims d, const double* __restrict__ u, const double* __restrict__ v,
                             const double* __restrict__ w, double* __restrict__ uc, double* __restrict__ vc,
                             double* __restrict__ wc) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nint) return;
    const int i = (int)(t % d.nx) + 1;
    const long long r = t / d.nx;
    const int j = (int)(r % d.ny) + 1;
    const int k = (int)(r / d.ny) + 1;
    const long long c = pidx(d, i, j, k);
    uc[t] = 0.5 * (u[c] + u[pidx(d, i + 1, j, k)]);
    vc[t] = 0.5 * (v[c] + v[pidx(d, i, j + 1, k)]);
    wc[t] = 0.5 * (w[c] + w[pidx(d, i, j, k + 1)]);
}

int mdx_k_center_vel(mdx_ctx_t* ctx, double* uc, double* vc, double* wc) {
    const mdx_dims& d = ctx->d;
    double* buf = nullptr;
    MDX_CUDA(ctx, cudaMallocAsync(&buf, sizeof(double) * 3 * d.nint, ctx->stream));
    const int nb = (int)((d.nint + 255) / 256);
    mdx_event_pair p{};
    mdx_timer_begin(ctx, MDX_T_OTHER, &p);
    k_center_vel<<<nb, 256, 0, ctx->stream>>>(d, ctx->f[MDX_UN], ctx->f[MDX_VN], ctx->f[MDX_WN], buf, buf + d.nint,
                                              buf + 2 * d.nint);
    mdx_timer_end(ctx, &p);
    int rc = mdx_check_launch(ctx, "center_vel");
    if (rc == MDX_OK) {
        cudaError_t e = cudaSuccess;
        if (uc && e == cudaSuccess) e = cudaMemcpyAsync(uc, buf, sizeof(double) * d.nint, cudaMemcpyDeviceToHost, ctx->stream);
        if (vc && e == cudaSuccess) e = cudaMemcpyAsync(vc, buf + d.nint, sizeof(double) * d.nint, cudaMemcpyDeviceToHost, ctx->stream);
        if (wc && e == cudaSuccess) e = cudaMemcpyAsync(wc, buf + 2 * d.nint, sizeof(double) * d.nint, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = mdx_fail(ctx, MDX_ERR_CUDA, "center_vel copy: %s", cudaGetErrorString(e));
    }
    cudaFreeAsync(buf, ctx->stream);
    return rc;
}

// ---------------------------------------------------------------------------
// Seeded channel initial condition (counter-based SplitMix64 finaliser of
// Steele, Lea & Flood 2014 on seed + golden*(field<<40 | padded index)).
// yc(x) per x index comes from the host so the profile is the host's libm.
// ---------------------------------------------------------------------------
__global__ void k_channel_ic(mdx_dims d, double dy, uint64_t seed, double amp_u, double amp_vw,
                             const double* __restrict__ yc, double* __restrict__ un, double* __restrict__ vn,
                             double* __restrict__ wn) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nint) return;
    const int i = (int)(t % d.nx) + 1;
    const long long r = t / d.nx;
    const int j = (int)(r % d.ny) + 1;
    const int k = (int)(r / d.ny) + 1;
    const long long c = pidx(d, i, j, k);
    const double y = ((double)j - 0.5) * dy;
    const double e = y - yc[i - 1];
    double base = 1.0 - e * e;
    if (base < 0.0) base = 0.0;
    un[c] = base + ic_uniform(seed, 0, (uint64_t)c, amp_u);
    vn[c] = (j == 1) ? 0.0 : ic_uniform(seed, 1, (uint64_t)c, amp_vw);
    wn[c] = ic_uniform(seed, 2, (uint64_t)c, amp_vw);
}

int mdx_k_channel_ic(mdx_ctx_t* ctx, uint64_t seed, double amp_u, double amp_vw, const double* yc_host) {
    const mdx_dims& d = ctx->d;
    double* yc = nullptr;
    MDX_CUDA(ctx, cudaMallocAsync(&yc, sizeof(double) * d.nx, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(yc, yc_host, sizeof(double) * d.nx, cudaMemcpyHostToDevice, ctx->stream));
    const int nb = (int)((d.nint + 255) / 256);
    k_channel_ic<<<nb, 256, 0, ctx->stream>>>(d, ctx->g.dy, seed, amp_u, amp_vw, yc, ctx->f[MDX_UN], ctx->f[MDX_VN],
                                              ctx->f[MDX_WN]);
    int rc = mdx_check_launch(ctx, "channel_ic");
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // host yc buffer must outlive the copy
    cudaFreeAsync(yc, ctx->stream);
    return rc;
}

__global__ void k_fill(double* p, long long n, double v) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        p[t] = v;
}

int mdx_k_fill(mdx_ctx_t* ctx, double* p, long long n, double v) {
    MDX_LAUNCH(ctx, MDX_T_OTHER, "fill", k_fill, 1024, 256, 0, p, n, v);
    return MDX_OK;
}
