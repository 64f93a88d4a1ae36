// mdx_cell32.cuh -- per-cell arithmetic of the mixed-precision red-black
// projection (FP32 correction sweeps inside FP64 defect correction), shared by
// the single-channel kernels (k_sor_mixed.cu) and the ensemble kernel.
#pragma once

#include "mdx_internal.cuh"

struct mixed_params {
    float idx, idy, idz, idt;
};

// Colour-split layout of the FP32 arrays (du, dv, dw, dp, r): element
// (i, j, k) of the padded grid lives in half (i + j + k) & 1 at
// (k (ny+2) + j) (nx+2)/2 + i/2, so the cells of one colour in a row -- and
// the faces they own or share -- are consecutive: every access of a colour
// sweep is unit-stride.  A face belongs to the cell on its high side
// (u(i) to cell i).  nx is even, so (nx+2)/2 is whole.
__device__ __forceinline__ long long cidx(const mdx_dims& d, int i, int j, int k) {
    const int hx = d.nxp >> 1;
    return ((i + j + k) & 1) * ((long long)hx * d.nyp * d.nzp) + ((long long)k * d.nyp + j) * hx + (i >> 1);
}
// (i, j) planes of the IBM factors and sweep factors split by the parity of i.
__device__ __forceinline__ int pidx2(const mdx_dims& d, int i, int j) {
    const int hx = d.nxp >> 1;
    return (i & 1) * (hx * d.nyp) + j * hx + (i >> 1);
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
    const int np = d.nxp * d.nyp;
    const int q = pidx2(d, i, j);
    const long long c = cidx(d, i, j, k), cip = cidx(d, ip, j, k), cjp = cidx(d, i, jp, k), ckp = cidx(d, i, j, kp);
    const float mu_u_i = __ldg(mu32 + q), mu_u_ip = __ldg(mu32 + pidx2(d, ip, j));
    const float mu_v_j = __ldg(mu32 + np + q), mu_v_jp = __ldg(mu32 + np + pidx2(d, i, jp));
    const float mu_w = __ldg(mu32 + 2 * np + q);
    const float u_i = du[c], u_ip = du[cip], v_j = dv[c], v_jp = dv[cjp], w_k = dw[c], w_kp = dw[ckp];
    const float div = __ldg(r + c) + (u_ip - u_i) * P.idx + (v_jp - v_j) * P.idy + (w_kp - w_k) * P.idz;
    const float phi = div * __ldg(fac32 + q);
    dp[c] += phi * P.idt;
    du[c] = u_i - phi * P.idx * mu_u_i;
    du[cip] = u_ip + phi * P.idx * mu_u_ip;
    if (PY || j > 1) dv[c] = v_j - phi * P.idy * mu_v_j;         // wall face v(1) stays 0
    if (PY || j < ny) dv[cjp] = v_jp + phi * P.idy * mu_v_jp;    // wall face v(ny+1) stays 0
    dw[c] = w_k - phi * P.idz * mu_w;
    dw[ckp] = w_kp + phi * P.idz * mu_w;
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
    const int i = (int)(t % d.nxp), j = (int)(t / d.nxp);
    double mu_u = 1.0, mu_v = 1.0, mu_w = 1.0;
    if (mu) {
        mu_u = mu[t];
        mu_v = mu[np + t];
        mu_w = mu[2 * np + t];
    }
    const int o = pidx2(d, i, j);
    mu32[o] = (float)mu_u;
    mu32[np + o] = (float)mu_v;
    mu32[2 * np + o] = (float)mu_w;
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
