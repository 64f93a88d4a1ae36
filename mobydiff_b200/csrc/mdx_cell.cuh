// mdx_cell.cuh -- per-cell arithmetic shared by the single-channel kernels
// and the batched ensemble kernel, so that both compute the same bits.
// Every file that includes it is compiled with -fmad=false and keeps the
// reference's Fortran evaluation order.
#pragma once

#include "mdx_internal.cuh"

struct mdx_four { double *un, *vn, *wn, *pn; };

struct mdx_sor_params {
    double dx, dy, dz, idx, idy, idz, idx2, idy2, idz2, idt, sor, dt_gamma;
};

enum { MU_ONE = 0, MU_PLANE = 1, MU_FULL = 2 };

// -omega/denom of one cell, pressure_redblack.f90:124-126,186.
__device__ __forceinline__ double sor_factor(double mu_u_i, double mu_u_ip, double mu_v_j, double mu_v_jp,
                                             double mu_w_k, double mu_w_kp, const mdx_sor_params& p) {
    const double denom = (mu_u_i + mu_u_ip) * p.idx2 + (mu_w_k + mu_w_kp) * p.idz2 + (mu_v_j + mu_v_jp) * p.idy2;
    return -p.sor / denom;
}

// The update of one cell, pressure_redblack.f90:128-241, on register copies
// of its six faces and p, given its factor -omega/denom.  In the reference's
// one-sided boundary formulas un(nx,j,k), vn(i,j,k) and wn(i,j,nz) are the
// cell's own u_i, v_j, w_k (those branches run only for i = nx, j = ny,
// k = nz).  PX/PY/PZ: 1 periodic, 0 not, -1 read from bc at run time.
template <int PX = -1, int PY = -1, int PZ = -1>
__device__ __forceinline__ void sor_cell_fac(double& u_i, double& u_ip, double& v_j, double& v_jp, double& w_k,
                                             double& w_kp, double& pc, double mu_u_i, double mu_u_ip, double mu_v_j,
                                             double mu_v_jp, double mu_w_k, double mu_w_kp, double fac,
                                             const mdx_sor_params& p, const mdx_bc_dev& bc, int i, int j, int k,
                                             int nx, int ny, int nz) {
    const int* T = bc.type;
    const double* V = bc.value;
    const bool perx = PX >= 0 ? PX != 0 : bc.per[0] != 0;
    const bool pery = PY >= 0 ? PY != 0 : bc.per[1] != 0;
    const bool perz = PZ >= 0 ? PZ != 0 : bc.per[2] != 0;
    if (!perx) {  // :128-144
        if (i < 2) {
            if (T[bci(1, 0, 1)] == 0) u_i = V[bci(1, 0, 1)];
            else u_i = u_ip - V[bci(1, 0, 1)] * p.dx;
        }
        if (i >= nx) {
            if (T[bci(1, 1, 1)] == 0) u_ip = V[bci(1, 1, 1)];
            else u_ip = u_i + V[bci(1, 1, 1)] * p.dx;
        }
    }
    if (!pery) {  // :146-162
        if (j < 2) {
            if (T[bci(2, 0, 2)] == 0) v_j = V[bci(2, 0, 2)];
            else v_j = v_jp - V[bci(2, 0, 2)] * p.dy;
        }
        if (j >= ny) {
            if (T[bci(2, 1, 2)] == 0) v_jp = V[bci(2, 1, 2)];
            else v_jp = v_j + V[bci(2, 1, 2)] * p.dy;
        }
    }
    if (!perz) {  // :164-180
        if (k < 2) {
            if (T[bci(3, 0, 3)] == 0) w_k = V[bci(3, 0, 3)];
            else w_k = w_kp - V[bci(3, 0, 3)] * p.dz;
        }
        if (k >= nz) {
            if (T[bci(3, 1, 3)] == 0) w_kp = V[bci(3, 1, 3)];
            else w_kp = w_k + V[bci(3, 1, 3)] * p.dz;
        }
    }
    // :183-188
    const double phi = ((u_ip - u_i) * p.idx + (v_jp - v_j) * p.idy + (w_kp - w_k) * p.idz) * fac;
    pc = pc + phi * p.idt;
    // :190-241
    u_i = u_i - phi * p.idx * mu_u_i;
    if (!perx && i == 1) {
        if (T[bci(1, 0, 0)] == 0) u_i = u_i + V[bci(1, 0, 0)] * p.idx * mu_u_i;
        else u_i = u_i + (phi * p.idx - V[bci(1, 0, 0)]) * mu_u_i;
    }
    u_ip = u_ip + phi * p.idx * mu_u_ip;
    if (!perx && i == nx) {
        if (T[bci(1, 1, 0)] == 0) u_ip = u_ip - V[bci(1, 1, 0)] * p.idx * mu_u_ip;
        else u_ip = u_ip + (V[bci(1, 1, 0)] - phi * p.idx) * mu_u_ip;
    }
    v_j = v_j - phi * p.idy * mu_v_j;
    if (!pery && j == 1) {
        if (T[bci(2, 0, 0)] == 0) v_j = v_j + V[bci(2, 0, 0)] * p.idy * mu_v_j;
        else v_j = v_j + (phi * p.idy - V[bci(2, 0, 0)]) * mu_v_j;
    }
    v_jp = v_jp + phi * p.idy * mu_v_jp;
    if (!pery && j == ny) {
        if (T[bci(2, 1, 0)] == 0) v_jp = v_jp - V[bci(2, 1, 0)] * p.idy * mu_v_jp;
        else v_jp = v_jp + (V[bci(2, 1, 0)] - phi * p.idy) * mu_v_jp;
    }
    w_k = w_k - phi * p.idz * mu_w_k;
    if (!perz && k == 1) {
        if (T[bci(3, 0, 0)] == 0) w_k = w_k + V[bci(3, 0, 0)] * p.idz * mu_w_k;
        else w_k = w_k + (phi * p.idz - V[bci(3, 0, 0)]) * mu_w_k;
    }
    w_kp = w_kp + phi * p.idz * mu_w_kp;
    if (!perz && k == nz) {
        // :237 -- the Dirichlet branch of the reference has no mu factor
        if (T[bci(3, 1, 0)] == 0) w_kp = w_kp - V[bci(3, 1, 0)] * p.idz;
        else w_kp = w_kp + (V[bci(3, 1, 0)] - phi * p.idz) * mu_w_kp;
    }
}

// The whole update of one cell, pressure_redblack.f90:117-241.
__device__ __forceinline__ void sor_cell(double& u_i, double& u_ip, double& v_j, double& v_jp, double& w_k,
                                         double& w_kp, double& pc, double mu_u_i, double mu_u_ip, double mu_v_j,
                                         double mu_v_jp, double mu_w_k, double mu_w_kp, const mdx_sor_params& p,
                                         const mdx_bc_dev& bc, int i, int j, int k, int nx, int ny, int nz) {
    const double fac = sor_factor(mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w_k, mu_w_kp, p);
    sor_cell_fac(u_i, u_ip, v_j, v_jp, w_k, w_kp, pc, mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w_k, mu_w_kp, fac, p, bc,
                 i, j, k, nx, ny, nz);
}


// The stencil of the predictor at one cell: u, v, w on the cell's faces and
// their neighbours, p at the cell and its three lower neighbours.  Suffixes
// name the offset: ip = (i+1), jm = (j-1), ip_km = (i+1, k-1), and so on.
// momentum_vals reads it through accessors, so a caller can hand it values
// held in registers (mdx_mom_nb) or read on demand from the padded arrays
// (mdx_mom_ld, each value loaded in the branch that uses it).
#define MDX_MOM_STENCIL(X)                                                            \
    X(u_c) X(u_ip) X(u_im) X(u_jp) X(u_jm) X(u_kp) X(u_km) X(u_ip_jm) X(u_ip_km)   \
    X(v_c) X(v_ip) X(v_im) X(v_jp) X(v_jm) X(v_kp) X(v_km) X(v_im_jp) X(v_jp_km)   \
    X(w_c) X(w_ip) X(w_im) X(w_jp) X(w_jm) X(w_kp) X(w_km) X(w_im_kp) X(w_jm_kp)   \
    X(p_c) X(p_im) X(p_jm) X(p_km)
struct mdx_mom_nb {
#define MDX_MOM_FIELD(n) double n##_v;
#define MDX_MOM_GET(n) __device__ __forceinline__ double n() const { return n##_v; }
    MDX_MOM_STENCIL(MDX_MOM_FIELD)
    MDX_MOM_STENCIL(MDX_MOM_GET)
#undef MDX_MOM_FIELD
#undef MDX_MOM_GET
};
struct mdx_mom_ld {
    const double *un, *vn, *wn, *pn;
    long long c, SX, SY, SZ;
    __device__ __forceinline__ double u_c() const { return __ldg(un + c); }
    __device__ __forceinline__ double u_ip() const { return __ldg(un + c + SX); }
    __device__ __forceinline__ double u_im() const { return __ldg(un + c - SX); }
    __device__ __forceinline__ double u_jp() const { return __ldg(un + c + SY); }
    __device__ __forceinline__ double u_jm() const { return __ldg(un + c - SY); }
    __device__ __forceinline__ double u_kp() const { return __ldg(un + c + SZ); }
    __device__ __forceinline__ double u_km() const { return __ldg(un + c - SZ); }
    __device__ __forceinline__ double u_ip_jm() const { return __ldg(un + c + SX - SY); }
    __device__ __forceinline__ double u_ip_km() const { return __ldg(un + c + SX - SZ); }
    __device__ __forceinline__ double v_c() const { return __ldg(vn + c); }
    __device__ __forceinline__ double v_ip() const { return __ldg(vn + c + SX); }
    __device__ __forceinline__ double v_im() const { return __ldg(vn + c - SX); }
    __device__ __forceinline__ double v_jp() const { return __ldg(vn + c + SY); }
    __device__ __forceinline__ double v_jm() const { return __ldg(vn + c - SY); }
    __device__ __forceinline__ double v_kp() const { return __ldg(vn + c + SZ); }
    __device__ __forceinline__ double v_km() const { return __ldg(vn + c - SZ); }
    __device__ __forceinline__ double v_im_jp() const { return __ldg(vn + c - SX + SY); }
    __device__ __forceinline__ double v_jp_km() const { return __ldg(vn + c + SY - SZ); }
    __device__ __forceinline__ double w_c() const { return __ldg(wn + c); }
    __device__ __forceinline__ double w_ip() const { return __ldg(wn + c + SX); }
    __device__ __forceinline__ double w_im() const { return __ldg(wn + c - SX); }
    __device__ __forceinline__ double w_jp() const { return __ldg(wn + c + SY); }
    __device__ __forceinline__ double w_jm() const { return __ldg(wn + c - SY); }
    __device__ __forceinline__ double w_kp() const { return __ldg(wn + c + SZ); }
    __device__ __forceinline__ double w_km() const { return __ldg(wn + c - SZ); }
    __device__ __forceinline__ double w_im_kp() const { return __ldg(wn + c - SX + SZ); }
    __device__ __forceinline__ double w_jm_kp() const { return __ldg(wn + c - SY + SZ); }
    __device__ __forceinline__ double p_c() const { return __ldg(pn + c); }
    __device__ __forceinline__ double p_im() const { return __ldg(pn + c - SX); }
    __device__ __forceinline__ double p_jm() const { return __ldg(pn + c - SY); }
    __device__ __forceinline__ double p_km() const { return __ldg(pn + c - SZ); }
};

// The predictor of one cell (i,j,k), src/modules/step.f90:76-204, from its
// stencil values; writes us/vs/ws[c] and the new oldrhs at q.  The IBM
// coefficients of the cell are cu/cv/cw[cc] (padded index, or the (i,j)
// plane index when they do not vary along z).
template <bool IBM, class NB>
__device__ __forceinline__ void momentum_vals(const NB& n, const mdx_step_params& p, double dt_alpha,
                                              double dt_beta, double dt_gamma, double* __restrict__ us,
                                              double* __restrict__ vs, double* __restrict__ ws,
                                              double* __restrict__ ou, double* __restrict__ ov,
                                              double* __restrict__ ow, const double* __restrict__ cu,
                                              const double* __restrict__ cv, const double* __restrict__ cw,
                                              long long c, long long q, long long cc, int i, int j, int k) {
    const double idx = p.idx, idy = p.idy, idz = p.idz, idx2 = p.idx2, idy2 = p.idy2, idz2 = p.idz2, ire = p.ire;
    const double u_c = n.u_c(), v_c = n.v_c(), w_c = n.w_c(), p_c = n.p_c();
    if (i >= p.nx0) {  // step.f90:106-136
        const double u_ip = n.u_ip(), u_im = n.u_im(), u_jp = n.u_jp(), u_jm = n.u_jm(), u_kp = n.u_kp(), u_km = n.u_km();
        double s;
        s = u_ip + u_c;
        const double uu_p = 0.25 * (s * s);
        s = u_c + u_im;
        const double uu_m = 0.25 * (s * s);
        const double uv_p = 0.25 * (u_jp + u_c) * (n.v_jp() + n.v_im_jp());
        const double uv_m = 0.25 * (u_c + u_jm) * (v_c + n.v_im());
        const double uw_p = 0.25 * (u_c + u_kp) * (n.w_kp() + n.w_im_kp());
        const double uw_m = 0.25 * (u_c + u_km) * (w_c + n.w_im());
        const double diff_ux = (u_im - 2.0 * u_c + u_ip) * idx2;
        const double diff_uy = (u_jm - 2.0 * u_c + u_jp) * idy2;
        const double diff_uz = (u_km - 2.0 * u_c + u_kp) * idz2;
        const double dpx = (p_c - n.p_im()) * idx;
        const double rhsu = -((uu_p - uu_m) * idx) - (uv_p - uv_m) * idy - (uw_p - uw_m) * idz + p.fx +
                            ire * (diff_ux + diff_uy + diff_uz);
        double val = u_c + dt_alpha * rhsu + dt_beta * ou[q] - dt_gamma * dpx;
        if (IBM) val = val * (1.0 / (1.0 + dt_gamma * __ldg(cu + cc)));
        us[c] = val;
        ou[q] = rhsu;
    }
    if (j >= p.ny0) {  // step.f90:138-168
        const double v_ip = n.v_ip(), v_im = n.v_im(), v_jp = n.v_jp(), v_jm = n.v_jm(), v_kp = n.v_kp(), v_km = n.v_km();
        double s;
        const double vu_p = 0.25 * (v_c + v_ip) * (n.u_ip() + n.u_ip_jm());
        const double vu_m = 0.25 * (v_c + v_im) * (u_c + n.u_jm());
        s = v_c + v_jp;
        const double vv_p = 0.25 * (s * s);
        s = v_c + v_jm;
        const double vv_m = 0.25 * (s * s);
        const double vw_p = 0.25 * (v_kp + v_c) * (n.w_kp() + n.w_jm_kp());
        const double vw_m = 0.25 * (v_km + v_c) * (w_c + n.w_jm());
        const double diff_vx = (v_im - 2.0 * v_c + v_ip) * idx2;
        const double diff_vy = (v_jm - 2.0 * v_c + v_jp) * idy2;
        const double diff_vz = (v_km - 2.0 * v_c + v_kp) * idz2;
        const double dpy = (p_c - n.p_jm()) * idy;
        const double rhsv = -((vu_p - vu_m) * idx) - (vv_p - vv_m) * idy - (vw_p - vw_m) * idz + p.fy +
                            ire * (diff_vx + diff_vy + diff_vz);
        double val = v_c + dt_alpha * rhsv + dt_beta * ov[q] - dt_gamma * dpy;
        if (IBM) val = val * (1.0 / (1.0 + dt_gamma * __ldg(cv + cc)));
        vs[c] = val;
        ov[q] = rhsv;
    }
    if (k >= p.nz0) {  // step.f90:170-200
        const double w_ip = n.w_ip(), w_im = n.w_im(), w_jp = n.w_jp(), w_jm = n.w_jm(), w_kp = n.w_kp(), w_km = n.w_km();
        double s;
        const double wu_p = 0.25 * (w_c + w_ip) * (n.u_ip() + n.u_ip_km());
        const double wu_m = 0.25 * (w_c + w_im) * (u_c + n.u_km());
        s = w_c + w_kp;
        const double ww_p = 0.25 * (s * s);
        s = w_c + w_km;
        const double ww_m = 0.25 * (s * s);
        const double wv_p = 0.25 * (w_c + w_jp) * (n.v_jp() + n.v_jp_km());
        const double wv_m = 0.25 * (w_c + w_jm) * (v_c + n.v_km());
        const double diff_wx = (w_im - 2.0 * w_c + w_ip) * idx2;
        const double diff_wy = (w_jm - 2.0 * w_c + w_jp) * idy2;
        const double diff_wz = (w_km - 2.0 * w_c + w_kp) * idz2;
        const double dpz = (p_c - n.p_km()) * idz;
        const double rhsw = -((wu_p - wu_m) * idx) - (wv_p - wv_m) * idy - (ww_p - ww_m) * idz + p.fz +
                            ire * (diff_wx + diff_wy + diff_wz);
        double val = w_c + dt_alpha * rhsw + dt_beta * ow[q] - dt_gamma * dpz;
        if (IBM) val = val * (1.0 / (1.0 + dt_gamma * __ldg(cw + cc)));
        ws[c] = val;
        ow[q] = rhsw;
    }
}

// The predictor of one cell with its stencil read from the padded arrays in
// the branches that use it (every offset stays inside the ghost layer for
// 1 <= i,j,k <= n).
template <bool IBM>
__device__ __forceinline__ void momentum_cell(const mdx_dims& d, const mdx_step_params& p, double dt_alpha,
                                              double dt_beta, double dt_gamma, const double* __restrict__ un,
                                              const double* __restrict__ vn, const double* __restrict__ wn,
                                              const double* __restrict__ pn, double* __restrict__ us,
                                              double* __restrict__ vs, double* __restrict__ ws,
                                              double* __restrict__ ou, double* __restrict__ ov,
                                              double* __restrict__ ow, const double* __restrict__ cu,
                                              const double* __restrict__ cv, const double* __restrict__ cw,
                                              long long cc, int i, int j, int k) {
    const long long c = pidx(d, i, j, k);
    const mdx_mom_ld n{un, vn, wn, pn, c, 1, d.nxp, (long long)d.nxp * d.nyp};
    momentum_vals<IBM>(n, p, dt_alpha, dt_beta, dt_gamma, us, vs, ws, ou, ov, ow, cu, cv, cw, c, qidx(d, i, j, k), cc,
                       i, j, k);
}

// apply_bc_redblack, src/modules/boundary.f90:207-364, one (i,k), (j,k) or
// (i,j) column of each of the three sequential phases.
__device__ __forceinline__ void bcrb_y_col(const mdx_dims& d, const mdx_bc_dev& bc, double dy, const mdx_four& f, int i, int k) {
    const int ny = d.ny;
    const int* T = bc.type;
    const double* V = bc.value;
    double *un = f.un, *vn = f.vn, *wn = f.wn, *pn = f.pn;
    if (bc.per[1]) {
        un[pidx(d, i, 0, k)] = un[pidx(d, i, ny, k)];
        vn[pidx(d, i, 0, k)] = vn[pidx(d, i, ny, k)];
        wn[pidx(d, i, 0, k)] = wn[pidx(d, i, ny, k)];
        pn[pidx(d, i, 0, k)] = pn[pidx(d, i, ny, k)];
    } else {
        if (T[bci(2, 0, 1)] == 0) un[pidx(d, i, 0, k)] = 2 * V[bci(2, 0, 1)] - un[pidx(d, i, 1, k)];
        else un[pidx(d, i, 0, k)] = un[pidx(d, i, 1, k)] - V[bci(2, 0, 1)] * dy;
        if (T[bci(2, 0, 2)] == 0) vn[pidx(d, i, 1, k)] = V[bci(2, 0, 2)];
        else vn[pidx(d, i, 1, k)] = vn[pidx(d, i, 2, k)] - V[bci(2, 0, 2)] * dy;
        if (T[bci(2, 0, 3)] == 0) wn[pidx(d, i, 0, k)] = 2 * V[bci(2, 0, 3)] - wn[pidx(d, i, 1, k)];
        else wn[pidx(d, i, 0, k)] = wn[pidx(d, i, 1, k)] - V[bci(2, 0, 3)] * dy;
    }
    if (bc.per[1]) {
        un[pidx(d, i, ny + 1, k)] = un[pidx(d, i, 1, k)];
        vn[pidx(d, i, ny + 1, k)] = vn[pidx(d, i, 1, k)];
        wn[pidx(d, i, ny + 1, k)] = wn[pidx(d, i, 1, k)];
        pn[pidx(d, i, ny + 1, k)] = pn[pidx(d, i, 1, k)];
    } else {
        if (T[bci(2, 1, 1)] == 0) un[pidx(d, i, ny + 1, k)] = 2 * V[bci(2, 1, 1)] - un[pidx(d, i, ny, k)];
        else un[pidx(d, i, ny + 1, k)] = un[pidx(d, i, ny, k)] + V[bci(2, 1, 1)] * dy;
        if (T[bci(2, 1, 2)] == 0) vn[pidx(d, i, ny + 1, k)] = V[bci(2, 1, 2)];
        else vn[pidx(d, i, ny + 1, k)] = vn[pidx(d, i, ny, k)] + V[bci(2, 1, 2)] * dy;
        if (T[bci(2, 1, 3)] == 0) wn[pidx(d, i, ny + 1, k)] = 2 * V[bci(2, 1, 3)] - wn[pidx(d, i, ny, k)];
        else wn[pidx(d, i, ny + 1, k)] = wn[pidx(d, i, ny, k)] + V[bci(2, 1, 3)] * dy;
    }
}

__device__ __forceinline__ void bcrb_x_col(const mdx_dims& d, const mdx_bc_dev& bc, double dx, const mdx_four& f, int j, int k) {
    const int nx = d.nx;
    const int* T = bc.type;
    const double* V = bc.value;
    double *un = f.un, *vn = f.vn, *wn = f.wn, *pn = f.pn;
    if (bc.per[0]) {
        un[pidx(d, 0, j, k)] = un[pidx(d, nx, j, k)];
        vn[pidx(d, 0, j, k)] = vn[pidx(d, nx, j, k)];
        wn[pidx(d, 0, j, k)] = wn[pidx(d, nx, j, k)];
        pn[pidx(d, 0, j, k)] = pn[pidx(d, nx, j, k)];
    } else {
        if (T[bci(1, 0, 1)] == 0) un[pidx(d, 1, j, k)] = V[bci(1, 0, 1)];
        else un[pidx(d, 1, j, k)] = un[pidx(d, 2, j, k)] - V[bci(1, 0, 1)] * dx;
        if (T[bci(1, 0, 2)] == 0) vn[pidx(d, 0, j, k)] = 2 * V[bci(1, 0, 2)] - vn[pidx(d, 1, j, k)];
        else vn[pidx(d, 0, j, k)] = vn[pidx(d, 1, j, k)] - V[bci(1, 0, 2)] * dx;
        if (T[bci(1, 0, 3)] == 0) wn[pidx(d, 0, j, k)] = 2 * V[bci(1, 0, 3)] - wn[pidx(d, 1, j, k)];
        else wn[pidx(d, 0, j, k)] = wn[pidx(d, 1, j, k)] - V[bci(1, 0, 3)] * dx;
    }
    if (bc.per[0]) {
        un[pidx(d, nx + 1, j, k)] = un[pidx(d, 1, j, k)];
        vn[pidx(d, nx + 1, j, k)] = vn[pidx(d, 1, j, k)];
        wn[pidx(d, nx + 1, j, k)] = wn[pidx(d, 1, j, k)];
        pn[pidx(d, nx + 1, j, k)] = pn[pidx(d, 1, j, k)];
    } else {
        if (T[bci(1, 1, 1)] == 0) un[pidx(d, nx + 1, j, k)] = V[bci(1, 1, 1)];
        else un[pidx(d, nx + 1, j, k)] = un[pidx(d, nx, j, k)] + V[bci(1, 1, 1)] * dx;
        if (T[bci(1, 1, 2)] == 0) vn[pidx(d, nx + 1, j, k)] = 2 * V[bci(1, 1, 2)] - vn[pidx(d, nx, j, k)];
        else vn[pidx(d, nx + 1, j, k)] = vn[pidx(d, nx, j, k)] + V[bci(1, 1, 2)] * dx;
        if (T[bci(1, 1, 3)] == 0) wn[pidx(d, nx + 1, j, k)] = 2 * V[bci(1, 1, 3)] - wn[pidx(d, nx, j, k)];
        else wn[pidx(d, nx + 1, j, k)] = wn[pidx(d, nx, j, k)] + V[bci(1, 1, 3)] * dx;
    }
}

__device__ __forceinline__ void bcrb_z_col(const mdx_dims& d, const mdx_bc_dev& bc, double dz, const mdx_four& f, int i, int j) {
    const int nz = d.nz;
    const int* T = bc.type;
    const double* V = bc.value;
    double *un = f.un, *vn = f.vn, *wn = f.wn, *pn = f.pn;
    if (bc.per[2]) {
        un[pidx(d, i, j, 0)] = un[pidx(d, i, j, nz)];
        vn[pidx(d, i, j, 0)] = vn[pidx(d, i, j, nz)];
        wn[pidx(d, i, j, 0)] = wn[pidx(d, i, j, nz)];
        pn[pidx(d, i, j, 0)] = pn[pidx(d, i, j, nz)];
    } else {
        if (T[bci(3, 0, 1)] == 0) un[pidx(d, i, j, 0)] = 2 * V[bci(3, 0, 1)] - un[pidx(d, i, j, 1)];
        else un[pidx(d, i, j, 0)] = un[pidx(d, i, j, 1)] - V[bci(3, 0, 1)] * dz;
        if (T[bci(3, 0, 2)] == 0) vn[pidx(d, i, j, 0)] = 2 * V[bci(3, 0, 2)] - vn[pidx(d, i, j, 1)];
        else vn[pidx(d, i, j, 0)] = vn[pidx(d, i, j, 1)] - V[bci(3, 0, 2)] * dz;
        if (T[bci(3, 0, 3)] == 0) wn[pidx(d, i, j, 1)] = V[bci(3, 0, 3)];
        else wn[pidx(d, i, j, 1)] = wn[pidx(d, i, j, 2)] - V[bci(3, 0, 3)] * dz;
    }
    if (bc.per[2]) {
        un[pidx(d, i, j, nz + 1)] = un[pidx(d, i, j, 1)];
        vn[pidx(d, i, j, nz + 1)] = vn[pidx(d, i, j, 1)];
        wn[pidx(d, i, j, nz + 1)] = wn[pidx(d, i, j, 1)];
        pn[pidx(d, i, j, nz + 1)] = pn[pidx(d, i, j, 1)];
    } else {
        if (T[bci(3, 1, 1)] == 0) un[pidx(d, i, j, nz + 1)] = 2 * V[bci(3, 1, 1)] - un[pidx(d, i, j, nz)];
        else un[pidx(d, i, j, nz + 1)] = un[pidx(d, i, j, nz)] + V[bci(3, 1, 1)] * dz;
        if (T[bci(3, 1, 2)] == 0) vn[pidx(d, i, j, nz + 1)] = 2 * V[bci(3, 1, 2)] - vn[pidx(d, i, j, nz)];
        else vn[pidx(d, i, j, nz + 1)] = vn[pidx(d, i, j, nz)] + V[bci(3, 1, 2)] * dz;
        if (T[bci(3, 1, 3)] == 0) wn[pidx(d, i, j, nz + 1)] = V[bci(3, 1, 3)];
        else wn[pidx(d, i, j, nz + 1)] = wn[pidx(d, i, j, nz)] + V[bci(3, 1, 3)] * dz;
    }
}

// Seeded channel initial condition (counter-based SplitMix64 finaliser of
// Steele, Lea & Flood 2014 on seed + golden*(field<<40 | padded index)).
__device__ __forceinline__ uint64_t ic_hash(uint64_t seed, uint64_t field, uint64_t lin) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * ((field << 40) | lin);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double ic_uniform(uint64_t seed, uint64_t field, uint64_t lin, double amp) {
    const double u01 = (double)(ic_hash(seed, field, lin) >> 11) * (1.0 / 9007199254740992.0);
    return amp * (2.0 * u01 - 1.0);
}

