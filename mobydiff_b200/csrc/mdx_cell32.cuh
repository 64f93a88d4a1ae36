// mdx_cell32.cuh -- per-cell arithmetic of the mixed-precision red-black
// projection (FP32 correction sweeps inside FP64 defect correction), shared by
// the single-channel kernels (k_sor_mixed.cu) and the ensemble kernel.
#pragma once

#include "mdx_internal.cuh"

struct mixed_params {
    float idx, idy, idz, idt;
};

// The FP32 arithmetic of the correction sweeps is written with explicit
// roundings (__fmul_rn, __fsub_rn, __fmaf_rn), so that every kernel that
// updates a cell -- the colour sweeps, the fused red+black pass, the ensemble
// -- rounds the same operations whatever its compile flags, and they agree
// bit for bit.
// Cell divergence plus residual: r~ + (u_ip-u_i)/dx + (v_jp-v_j)/dy + (w_kp-w_k)/dz.
__device__ __forceinline__ float sweep32_div(const mixed_params& P, float r, float ui, float uip, float vj, float vjp,
                                             float wk, float wkp) {
    return __fmaf_rn(__fsub_rn(wkp, wk), P.idz, __fmaf_rn(__fsub_rn(vjp, vj), P.idy, __fmaf_rn(__fsub_rn(uip, ui), P.idx, r)));
}

// The update of one cell from its six faces, its correction dp and its
// residual r~ (pressure_redblack.f90:117-241 with homogeneous boundary
// values): phi = fac * (r~ + div), dp += phi/dt_gamma, faces -+ phi/h mu.
// v_lo / v_hi false keep a wall face v(1) / v(ny+1) at its value (0).
__device__ __forceinline__ void sweep32_update(const mixed_params& P, float r, float& u_i, float& u_ip, float& v_j,
                                               float& v_jp, float& w_k, float& w_kp, float& dp, float mu_u_i,
                                               float mu_u_ip, float mu_v_j, float mu_v_jp, float mu_w, float fac,
                                               bool v_lo, bool v_hi) {
    const float ui = u_i, uip = u_ip, vj = v_j, vjp = v_jp, wk = w_k, wkp = w_kp;
    const float phi = __fmul_rn(sweep32_div(P, r, ui, uip, vj, vjp, wk, wkp), fac);
    dp = __fmaf_rn(phi, P.idt, dp);
    const float px = __fmul_rn(phi, P.idx), py = __fmul_rn(phi, P.idy), pz = __fmul_rn(phi, P.idz);
    u_i = __fmaf_rn(-px, mu_u_i, ui);
    u_ip = __fmaf_rn(px, mu_u_ip, uip);
    if (v_lo) v_j = __fmaf_rn(-py, mu_v_j, vj);
    if (v_hi) v_jp = __fmaf_rn(py, mu_v_jp, vjp);
    w_k = __fmaf_rn(-pz, mu_w, wk);
    w_kp = __fmaf_rn(pz, mu_w, wkp);
}

// One FP32 colour-sweep update of cell (i, j, k) of the correction problem
// (periodic x and z; y periodic when PY, else walls whose faces v(1),
// v(ny+1) stay 0).
template <int PY>
__device__ __forceinline__ void sweep32_cell(const mdx_dims& d, const mixed_params& P, int i, int j, int k,
                                             float* __restrict__ du, float* __restrict__ dv, float* __restrict__ dw,
                                             float* __restrict__ dp, const float* __restrict__ r,
                                             const float* __restrict__ mu32, const float* __restrict__ fac32) {
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int jp = (PY && j == ny) ? 1 : j + 1;
    const int kp = (k == nz) ? 1 : k + 1;
    const int ip = (i == nx) ? 1 : i + 1;
    const int np = split_plane_elems(d);
    const int q = pidx2(d, i, j);
    const long long c = cidx(d, i, j, k), cip = cidx(d, ip, j, k), cjp = cidx(d, i, jp, k), ckp = cidx(d, i, j, kp);
    const float mu_u_i = __ldg(mu32 + q), mu_u_ip = __ldg(mu32 + pidx2(d, ip, j));
    const float mu_v_j = __ldg(mu32 + np + q), mu_v_jp = __ldg(mu32 + np + pidx2(d, i, jp));
    const float mu_w = __ldg(mu32 + 2 * np + q);
    float u_i = du[c], u_ip = du[cip], v_j = dv[c], v_jp = dv[cjp], w_k = dw[c], w_kp = dw[ckp], p = dp[c];
    const bool v_lo = PY || j > 1, v_hi = PY || j < ny;   // wall faces v(1), v(ny+1) stay 0
    sweep32_update(P, __ldg(r + c), u_i, u_ip, v_j, v_jp, w_k, w_kp, p, mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w,
                   __ldg(fac32 + q), v_lo, v_hi);
    dp[c] = p;
    du[c] = u_i;
    du[cip] = u_ip;
    if (v_lo) dv[c] = v_j;
    if (v_hi) dv[cjp] = v_jp;
    dw[c] = w_k;
    dw[ckp] = w_kp;
}

// Residual of the correction problem at cell (i, j, k): r~ + div(du).
template <int PY>
__device__ __forceinline__ float corr_residual_cell(const mdx_dims& d, const mixed_params& P, int i, int j, int k,
                                                    const float* __restrict__ du, const float* __restrict__ dv,
                                                    const float* __restrict__ dw, const float* __restrict__ r) {
    const int ip = i == d.nx ? 1 : i + 1;
    const int jp = (PY && j == d.ny) ? 1 : j + 1;
    const int kp = k == d.nz ? 1 : k + 1;
    const long long c = cidx(d, i, j, k);
    return __ldg(r + c) + (__ldg(du + cidx(d, ip, j, k)) - __ldg(du + c)) * P.idx +
           (__ldg(dv + cidx(d, i, jp, k)) - __ldg(dv + c)) * P.idy +
           (__ldg(dw + cidx(d, i, j, kp)) - __ldg(dw + c)) * P.idz;
}

// FP64 divergence of (u, v, w) at cell (i, j, k) (the red-black neighbour
// rule), stored as FP32 r~; returned for the norms.
template <int PY>
__device__ __forceinline__ double mixed_residual_cell(const mdx_dims& d, double idx, double idy, double idz, int i,
                                                      int j, int k, const double* __restrict__ u,
                                                      const double* __restrict__ v, const double* __restrict__ w,
                                                      float* __restrict__ r) {
    const int ip = i == d.nx ? 1 : i + 1;
    const int jp = (PY && j == d.ny) ? 1 : j + 1;
    const int kp = k == d.nz ? 1 : k + 1;
    const long long c = pidx(d, i, j, k);
    const double dv = (__ldg(u + pidx(d, ip, j, k)) - __ldg(u + c)) * idx +
                      (__ldg(v + pidx(d, i, jp, k)) - __ldg(v + c)) * idy +
                      (__ldg(w + pidx(d, i, j, kp)) - __ldg(w + c)) * idz;
    r[cidx(d, i, j, k)] = (float)dv;
    return dv;
}

// u += du, v += dv, w += dw, p += dp at padded element t; corrections reset.
__device__ __forceinline__ void mixed_apply_elem(const mdx_dims& d, long long t, double* __restrict__ u,
                                                 double* __restrict__ v, double* __restrict__ w,
                                                 double* __restrict__ p, float* __restrict__ du,
                                                 float* __restrict__ dv, float* __restrict__ dw,
                                                 float* __restrict__ dp) {
    const int i = (int)(t % d.nxp);
    const long long rr = t / d.nxp;
    const int j = (int)(rr % d.nyp);
    const int k = (int)(rr / d.nyp);
    const long long c = cidx(d, i, j, k);
    u[t] += (double)du[c];
    v[t] += (double)dv[c];
    w[t] += (double)dw[c];
    p[t] += (double)dp[c];
    du[c] = 0.f;
    dv[c] = 0.f;
    dw[c] = 0.f;
    dp[c] = 0.f;
}

// FP32 IBM factors and -omega/denom of the (i, j) column at plane element t
// (z-invariant factors; mu = FP64 planes or null for none).
__device__ __forceinline__ void mixed_tables_elem(const mdx_dims& d, int py, double idx2, double idy2, double idz2,
                                                  double sor, const double* __restrict__ mu, long long t,
                                                  float* __restrict__ mu32, float* __restrict__ fac32) {
    const long long np = (long long)d.nxp * d.nyp;
    const int ps = split_plane_elems(d);
    const int i = (int)(t % d.nxp), j = (int)(t / d.nxp);
    double mu_u = 1.0, mu_v = 1.0, mu_w = 1.0;
    if (mu) {
        mu_u = mu[t];
        mu_v = mu[np + t];
        mu_w = mu[2 * np + t];
    }
    const int o = pidx2(d, i, j);
    mu32[o] = (float)mu_u;
    mu32[ps + o] = (float)mu_v;
    mu32[2 * ps + o] = (float)mu_w;
    double f = 0.0;
    if (i >= 1 && i <= d.nx && j >= 1 && j <= d.ny) {
        const int ip = i == d.nx ? 1 : i + 1;
        const int jp = (py && j == d.ny) ? 1 : j + 1;
        double mu_uip = 1.0, mu_vjp = 1.0;
        if (mu) {
            mu_uip = mu[ip + (long long)d.nxp * j];
            mu_vjp = mu[np + i + (long long)d.nxp * jp];
        }
        const double denom = (mu_u + mu_uip) * idx2 + (mu_w + mu_w) * idz2 + (mu_v + mu_vjp) * idy2;
        f = -sor / denom;
    }
    fac32[o] = (float)f;
}

// ---- potential form ----------------------------------------------------------
// Starting from zero corrections, the face updates of sweep32_update leave
// every face at h^-1 mu (Phi(low cell) - Phi(high cell)), Phi the sum of the
// phi a cell has taken, so the divergence the next update needs is a
// 7-point stencil of Phi: e = r~ + sum over the faces of a_f (Phi(c) -
// Phi(across)), a_f = h^-2 mu_f (0 for a wall face), and the update is
// Phi += fac e.  The cell arithmetic, FP32 roundings explicit, shared by the
// single-channel kernels (k_sor_mixed.cu) and the ensemble.
__device__ __forceinline__ float pot_e(float r, float c, float xl, float xr, float ym, float yp, float zm, float zp,
                                       float axl, float axr, float ayl, float ayr, float az) {
    float e = __fmaf_rn(axl, __fsub_rn(c, xl), r);
    e = __fmaf_rn(axr, __fsub_rn(c, xr), e);
    e = __fmaf_rn(ayl, __fsub_rn(c, ym), e);
    e = __fmaf_rn(ayr, __fsub_rn(c, yp), e);
    return __fmaf_rn(az, __fadd_rn(__fsub_rn(c, zm), __fsub_rn(c, zp)), e);
}

// e of cell (i, j, k) with Phi and r~ in the face form's colour-split layout
// (cidx) and the FP32 factor planes mu32: x and z periodic, y periodic when
// PY, else walls (rows 0 and ny+1 hold 0, their faces' a_y is 0).  Phi and r~
// change inside a persistent kernel, so they are read with coherent loads.
template <int PY>
__device__ __forceinline__ float pot_split_e(const mdx_dims& d, const mixed_params& P, int i, int j, int k, float c,
                                             const float* phi, const float* r, const float* mu32) {
    const int ip = i == d.nx ? 1 : i + 1, im = i == 1 ? d.nx : i - 1;
    const int kp = k == d.nz ? 1 : k + 1, km = k == 1 ? d.nz : k - 1;
    const int jp = (PY && j == d.ny) ? 1 : j + 1, jm = (PY && j == 1) ? d.ny : j - 1;
    const int np = split_plane_elems(d);
    const float ix2 = __fmul_rn(P.idx, P.idx), iy2 = __fmul_rn(P.idy, P.idy), iz2 = __fmul_rn(P.idz, P.idz);
    const float axl = __fmul_rn(ix2, mu32[pidx2(d, i, j)]);
    const float axr = __fmul_rn(ix2, mu32[pidx2(d, ip, j)]);
    const float ayl = (PY || j > 1) ? __fmul_rn(iy2, mu32[np + pidx2(d, i, j)]) : 0.f;
    const float ayr = (PY || j < d.ny) ? __fmul_rn(iy2, mu32[np + pidx2(d, i, jp)]) : 0.f;
    const float az = __fmul_rn(iz2, mu32[2 * np + pidx2(d, i, j)]);
    return pot_e(r[cidx(d, i, j, k)], c, phi[cidx(d, im, j, k)], phi[cidx(d, ip, j, k)], phi[cidx(d, i, jm, k)],
                 phi[cidx(d, i, jp, k)], phi[cidx(d, i, j, km)], phi[cidx(d, i, j, kp)], axl, axr, ayl, ayr, az);
}

// One potential-form update of cell (i, j, k), fac from the factor plane.
template <int PY>
__device__ __forceinline__ void pot_split_cell(const mdx_dims& d, const mixed_params& P, int i, int j, int k,
                                               float* phi, const float* r, const float* mu32, const float* fac32) {
    const long long c = cidx(d, i, j, k);
    const float v = phi[c];
    phi[c] = __fmaf_rn(fac32[pidx2(d, i, j)], pot_split_e<PY>(d, P, i, j, k, v, phi, r, mu32), v);
}

// u, v, w, p of cell (i, j, k) += the corrections Phi stands for, in FP64:
// its low faces (a wall face v(1) stays) and p += Phi/dt_gamma; mu = the
// FP64 factor planes (u, v, w, each (nx+2)(ny+2)) or null for none.
template <int PY>
__device__ __forceinline__ void pot_split_apply(const mdx_dims& d, int i, int j, int k, double idx, double idy,
                                                double idz, double idt, const double* mu, const float* phi,
                                                double* u, double* v, double* w, double* p) {
    const int im = i == 1 ? d.nx : i - 1, km = k == 1 ? d.nz : k - 1;
    const int jm = (PY && j == 1) ? d.ny : j - 1;
    const long long np = (long long)d.nxp * d.nyp, q = i + (long long)d.nxp * j;
    const double mu_u = mu ? mu[q] : 1.0, mu_v = mu ? mu[np + q] : 1.0, mu_w = mu ? mu[2 * np + q] : 1.0;
    const double c = (double)phi[cidx(d, i, j, k)];
    const long long a = pidx(d, i, j, k);
    u[a] += idx * mu_u * ((double)phi[cidx(d, im, j, k)] - c);
    if (PY || j > 1) v[a] += idy * mu_v * ((double)phi[cidx(d, i, jm, k)] - c);
    w[a] += idz * mu_w * ((double)phi[cidx(d, i, j, km)] - c);
    p[a] += c * idt;
}
