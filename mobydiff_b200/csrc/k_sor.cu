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
#include "mdx_cell.cuh"

#include <algorithm>
#include <cmath>

// mu = 1/(1 + dt_gamma*coef) over n elements of each component.
__global__ void k_mu_tables(long long n, double dg, const double* __restrict__ cu, const double* __restrict__ cv,
                            const double* __restrict__ cw, double* __restrict__ mu) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        mu[t] = 1.0 / (1.0 + dg * __ldg(cu + t));
        mu[n + t] = 1.0 / (1.0 + dg * __ldg(cv + t));
        mu[2 * n + t] = 1.0 / (1.0 + dg * __ldg(cw + t));
    }
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
    const bool perx = bc.per[0] != 0, pery = bc.per[1] != 0, perz = bc.per[2] != 0;
    int jp = j + 1;
    if (pery && jp > ny) jp = 1;
    int kp = k + 1;
    if (perz && kp > nz) kp = 1;
    const int iLo = 1 + ((j + k + parity) & 1);
    const int i = iLo + 2 * (ni - 1);
    int ip = i + 1;
    if (perx && ip > nx) ip = 1;
    const long long c = pidx(d, i, j, k);
    const long long cip = pidx(d, ip, j, k), cjp = pidx(d, i, jp, k), ckp = pidx(d, i, j, kp);
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
    double u_i = un[c], u_ip = un[cip], v_j = vn[c], v_jp = vn[cjp], w_k = wn[c], w_kp = wn[ckp], pc = pn[c];
    sor_cell(u_i, u_ip, v_j, v_jp, w_k, w_kp, pc, mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w_k, mu_w_kp, p, bc, i, j, k,
             nx, ny, nz);
    un[c] = u_i;
    un[cip] = u_ip;
    vn[c] = v_j;
    vn[cjp] = v_jp;
    wn[c] = w_k;
    wn[ckp] = w_kp;
    pn[c] = pc;
}

// ---------------------------------------------------------------------------
// One full red+black iteration in one pass (periodic x and z).
//
// Each block owns the cells of a TX x TY tile in x-y and a chunk of KZ z
// planes.  It walks its z range with a ring of four planes in shared memory
// holding u, v, w, p of the tile plus a two-cell halo ring in x and y; the
// plane two ahead is fetched with cp.async while the current ones compute.
// On plane q it runs the red update on every red cell of the halo region,
// then the black update of plane q-1 on the tile plus a one-cell ring, then
// writes the owned faces of plane q-1 (u(i), v(j), w(k) and p of the tile
// cells; v(ny+1) for a y wall).  All reads come from the old state (u0..p0)
// and all writes go to the new state (u1..p1), so blocks never see each
// other's updates; red cells of the halo are recomputed from the same old
// values their owners use, so every face ends with exactly the value of a
// red sweep followed by a black sweep.  The state crosses HBM once per
// iteration instead of twice.
//
// Shared-memory rows store even columns then odd columns, so the cells of
// one colour in a row (every other column) are contiguous: a warp's accesses
// fall in distinct banks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 8 : 0;   // 0 source bytes: the 8 destination bytes are zero-filled
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int TX, int TY, int NTH>
struct fused_geom {
    static constexpr int NT = NTH;
    static constexpr int WX = TX + 3, WY = TY + 3;   // halo: x in [x0-2, x0+TX], y in [y0-2, y0+TY]
    static constexpr int UX = WX + 1;                // u rows also hold the right face of the last cell
    static constexpr int H = (UX + 1) / 2;           // even columns, then odd columns
    static constexpr int R = 2 * H;                  // row stride
    static constexpr int NU = WY * R, NV = (WY + 1) * R, NC = WY * R;
    static constexpr int SLOT = NU + NV + 2 * NC;
    static constexpr int LU = WY * UX, LV = (WY + 1) * WX, LC = WY * WX;   // elements fetched per plane
    static constexpr int LTOT = LU + LV + 2 * LC;
    static constexpr int NLD = (LTOT + NT - 1) / NT;
    static constexpr int HR = (WX + 1) / 2;          // red candidates per row
    static constexpr int HB = (WX - 1) / 2;          // black candidates per row (columns 1..WX-2)
    __device__ static __forceinline__ int col(int lx) { return (lx & 1) * H + (lx >> 1); }
};

template <int MU, int PY, int TX, int TY, int NTH>
__global__ void __launch_bounds__(NTH)
k_sor_fused(mdx_dims d, mdx_bc_dev bc, mdx_sor_params P, int KZ, const double* __restrict__ u0,
            const double* __restrict__ v0, const double* __restrict__ w0, const double* __restrict__ p0,
            double* __restrict__ u1, double* __restrict__ v1, double* __restrict__ w1, double* __restrict__ p1,
            const double* __restrict__ mu) {
    using G = fused_geom<TX, TY, NTH>;
    constexpr int NT = G::NT, WX = G::WX, WY = G::WY, UX = G::UX, R = G::R;
    constexpr int NU = G::NU, NV = G::NV, NC = G::NC, SLOT = G::SLOT;
    constexpr int LU = G::LU, LV = G::LV, LC = G::LC, LTOT = G::LTOT, NLD = G::NLD;
    constexpr int HR = G::HR, HB = G::HB;
    static_assert(WY * HR <= NT && (WY - 2) * HB <= NT && TX * TY <= NT, "one cell per thread per phase");
    extern __shared__ double sm[];
    double* smu = sm + 4 * SLOT;              // mu_u (NU), mu_v (NV), mu_w (NC)  [MU_PLANE]
    double* sfac = smu + (MU == MU_PLANE ? NU + NV + NC : 0);   // -omega/denom per column (NC)
    int* gxt = (int*)(sfac + NC);             // global x of local column (UX)
    int* gyt = gxt + UX;                      // global y of local row (WY+1), -1 outside

    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int x0 = blockIdx.x * TX + 1, y0 = blockIdx.y * TY + 1;
    const int k0 = blockIdx.z * KZ + 1;
    const int k1 = min(k0 + KZ, nz + 1);
    const int tid = threadIdx.x;
    const long long plane = (long long)d.nxp * d.nyp;

    for (int t = tid; t < UX; t += NT) gxt[t] = ((x0 - 2 + t - 1) % nx + nx) % nx + 1;
    for (int t = tid; t <= WY; t += NT) {
        int g = y0 - 2 + t;
        if (PY) g = ((g - 1) % ny + ny) % ny + 1;
        else if (g < 0 || g > ny + 1) g = -1;
        gyt[t] = g;
    }
    __syncthreads();
    if (MU == MU_PLANE) {
        for (int t = tid; t < LU; t += NT) {
            const int ly = t / UX, lx = t - ly * UX, gy = gyt[ly];
            smu[ly * R + G::col(lx)] = gy >= 0 ? __ldg(mu + gxt[lx] + (long long)d.nxp * gy) : 1.0;
        }
        for (int t = tid; t < LV; t += NT) {
            const int ly = t / WX, lx = t - ly * WX, gy = gyt[ly];
            smu[NU + ly * R + G::col(lx)] = gy >= 0 ? __ldg(mu + plane + gxt[lx] + (long long)d.nxp * gy) : 1.0;
        }
        for (int t = tid; t < LC; t += NT) {
            const int ly = t / WX, lx = t - ly * WX, gy = gyt[ly];
            smu[NU + NV + ly * R + G::col(lx)] =
                gy >= 0 ? __ldg(mu + 2 * plane + gxt[lx] + (long long)d.nxp * gy) : 1.0;
        }
        __syncthreads();
    }
    // -omega/denom of every column (:124-126,186); z-invariant in both modes
    for (int t = tid; t < LC; t += NT) {
        const int ly = t / WX, lx = t - ly * WX;
        double mu_u_i = 1.0, mu_u_ip = 1.0, mu_v_j = 1.0, mu_v_jp = 1.0, mu_w = 1.0;
        if (MU == MU_PLANE) {
            mu_u_i = smu[ly * R + G::col(lx)];
            mu_u_ip = smu[ly * R + G::col(lx + 1)];
            mu_v_j = smu[NU + ly * R + G::col(lx)];
            mu_v_jp = smu[NU + (ly + 1) * R + G::col(lx)];
            mu_w = smu[NU + NV + ly * R + G::col(lx)];
        }
        sfac[ly * R + G::col(lx)] = sor_factor(mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, P);
    }

    // Per-thread fetch descriptors: plane-relative global offset (-1 outside
    // the domain: zero-filled) and the shared-memory index in a slot.
    int ldoff[NLD], lddst[NLD];
#pragma unroll
    for (int m = 0; m < NLD; ++m) {
        const int e = tid + m * NT;
        int off = -1, dst = -1;
        if (e < LTOT) {
            int lx, ly, base;
            if (e < LU) {
                ly = e / UX;
                lx = e - ly * UX;
                base = 0;
            } else if (e < LU + LV) {
                const int t = e - LU;
                ly = t / WX;
                lx = t - ly * WX;
                base = NU;
            } else {
                const int t = e - LU - LV;
                const int t2 = t < LC ? t : t - LC;
                ly = t2 / WX;
                lx = t2 - ly * WX;
                base = t < LC ? NU + NV : NU + NV + NC;
            }
            dst = base + ly * R + G::col(lx);
            const int gy = gyt[ly];
            if (gy >= 0) off = gxt[lx] + d.nxp * gy;
        }
        ldoff[m] = off;
        lddst[m] = dst;
    }
    auto slot = [&](int q) { return sm + ((q - k0 + 2) & 3) * SLOT; };
    auto issue = [&](int q, int gk) {
        double* s = slot(q);
        const long long pk = (long long)gk * plane;
#pragma unroll
        for (int m = 0; m < NLD; ++m) {
            const int e = tid + m * NT;
            if (e < LTOT) {
                const double* src = e < LU ? u0 : (e < LU + LV ? v0 : (e < LU + LV + LC ? w0 : p0));
                const int off = ldoff[m];
                cp_async8(s + lddst[m], off >= 0 ? src + pk + off : u0, off >= 0);
            }
        }
        cp_async_commit();
    };
    const int r_ly = tid / HR, r_m = tid % HR;
    const int b_ly = 1 + tid / HB, b_m = tid % HB;
    const bool r_ok = tid < WY * HR, b_ok = tid < (WY - 2) * HB;
    auto cell = [&](int q, int ly, int lx, int gy, int gk) {
        double* s = slot(q);
        double* su = s;
        double* sv = s + NU;
        double* sw = s + NU + NV;
        double* sp = s + NU + NV + NC;
        double* swn = slot(q + 1) + NU + NV;
        const int c0 = ly * R + G::col(lx), c1 = ly * R + G::col(lx + 1), cn = c0 + R;
        double mu_u_i = 1.0, mu_u_ip = 1.0, mu_v_j = 1.0, mu_v_jp = 1.0, mu_w = 1.0;
        if (MU == MU_PLANE) {
            mu_u_i = smu[c0];
            mu_u_ip = smu[c1];
            mu_v_j = smu[NU + c0];
            mu_v_jp = smu[NU + cn];
            mu_w = smu[NU + NV + c0];
        }
        double ui = su[c0], uip = su[c1], vj = sv[c0], vjp = sv[cn], wk = sw[c0], wkp = swn[c0], pc = sp[c0];
        sor_cell_fac<1, PY, 1>(ui, uip, vj, vjp, wk, wkp, pc, mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, sfac[c0],
                               P, bc, 0, gy, gk, nx, ny, nz);
        su[c0] = ui;
        su[c1] = uip;
        sv[c0] = vj;
        sv[cn] = vjp;
        sw[c0] = wk;
        swn[c0] = wkp;
        sp[c0] = pc;
    };
    auto red = [&](int q, int gk) {   // red: (i+j+k) odd, whole halo region
        if (!r_ok) return;
        const int gy = gyt[r_ly];
        if (gy < 1 || gy > ny) return;
        const int lx = ((x0 + gy + gk + 1) & 1) + 2 * r_m;
        if (lx < WX) cell(q, r_ly, lx, gy, gk);
    };
    auto black = [&](int q, int gk) {   // black: (i+j+k) even, tile plus one ring
        if (!b_ok) return;
        const int gy = gyt[b_ly];
        if (gy < 1 || gy > ny) return;
        const int lx = 1 + ((x0 + 1 + gy + gk) & 1) + 2 * b_m;
        if (lx < WX - 1) cell(q, b_ly, lx, gy, gk);
    };
    // owned cell of this thread
    const int o_gx = x0 + tid % TX, o_gy = y0 + tid / TX;
    const bool o_ok = o_gx <= nx && o_gy <= ny;
    const int o_s = (2 + tid / TX) * R + G::col(2 + tid % TX);
    const int o_off = o_gx + d.nxp * o_gy;
    auto store = [&](int q, int gk) {
        if (!o_ok) return;
        const double* s = slot(q);
        const long long c = (long long)gk * plane + o_off;
        u1[c] = s[o_s];
        v1[c] = s[NU + o_s];
        w1[c] = s[NU + NV + o_s];
        p1[c] = s[NU + NV + NC + o_s];
        if (!PY && o_gy == ny) v1[c + d.nxp] = s[NU + o_s + R];
    };
    auto wrapz = [&](int q) { return ((q - 1) % nz + nz) % nz + 1; };

    issue(k0 - 2, wrapz(k0 - 2));
    issue(k0 - 1, wrapz(k0 - 1));
    int gkm = wrapz(k0 - 3);   // plane q-1
    int gk = wrapz(k0 - 2);    // plane q
    for (int q = k0 - 2; q <= k1; ++q) {
        if (q + 2 <= k1 + 1) issue(q + 2, wrapz(q + 2));
        else cp_async_commit();           // empty group keeps the wait count uniform
        cp_async_wait1();                 // planes up to q+1 have landed
        __syncthreads();
        red(q, gk);                       // halo region of plane q
        __syncthreads();
        if (q - 1 >= k0 - 1) black(q - 1, gkm);   // tile + one ring of plane q-1
        __syncthreads();
        if (q - 1 >= k0) store(q - 1, gkm);
        __syncthreads();                  // slot of q-1 is refilled by the next issue
        gkm = gk;
        gk = gk == nz ? 1 : gk + 1;
    }
}

double mdx_div_floor(const mdx_ctx_t* ctx, double umax) {
    const double eps = 2.220446049250313e-16;
    const mdx_grid_t& g = ctx->g;
    return eps * std::sqrt((double)ctx->d.nint) * umax * (1.0 / g.dx + 1.0 / g.dy + 1.0 / g.dz);
}

// One colour sweep for periodic x and z (the configurations of every run
// here): boundary flags are compile-time constants, in-plane offsets are
// 32-bit, and registers are bounded for occupancy.
template <int MU, int PY>
__global__ void __launch_bounds__(256, 4)
k_sor_sweep_pxz(mdx_dims d, mdx_bc_dev bc, mdx_sor_params p, int parity, int reverse, double* __restrict__ un,
                double* __restrict__ vn, double* __restrict__ wn, double* __restrict__ pn,
                const double* __restrict__ mu) {
    const int ni = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int kk = blockIdx.z * blockDim.z + threadIdx.z + 1;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    if (ni > nx / 2 || j > ny || kk > nz) return;
    const int k = reverse ? nz + 1 - kk : kk;
    const int jp = (PY && j == ny) ? 1 : j + 1;
    const int kp = (k == nz) ? 1 : k + 1;
    const int i = 1 + ((j + k + parity) & 1) + 2 * (ni - 1);
    const int ip = (i == nx) ? 1 : i + 1;
    const long long plane = (long long)d.nxp * d.nyp;
    const int q = i + d.nxp * j, qip = ip + d.nxp * j, qjp = i + d.nxp * jp;
    double* U = un + k * plane;
    double* Vv = vn + k * plane;
    double* W = wn + k * plane;
    double* Wn = wn + kp * plane;
    double* Pp = pn + k * plane;
    double mu_u_i = 1.0, mu_u_ip = 1.0, mu_v_j = 1.0, mu_v_jp = 1.0, mu_w = 1.0;
    if (MU == MU_PLANE) {
        mu_u_i = __ldg(mu + q);
        mu_u_ip = __ldg(mu + qip);
        mu_v_j = __ldg(mu + plane + q);
        mu_v_jp = __ldg(mu + plane + qjp);
        mu_w = __ldg(mu + 2 * plane + q);
    }
    double u_i = U[q], u_ip = U[qip], v_j = Vv[q], v_jp = Vv[qjp], w_k = W[q], w_kp = Wn[q], pc = Pp[q];
    const double fac = sor_factor(mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, p);
    sor_cell_fac<1, PY, 1>(u_i, u_ip, v_j, v_jp, w_k, w_kp, pc, mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, fac, p,
                           bc, i, j, k, nx, ny, nz);
    U[q] = u_i;
    U[qip] = u_ip;
    Vv[q] = v_j;
    Vv[qjp] = v_jp;
    W[q] = w_k;
    Wn[q] = w_kp;
    Pp[q] = pc;
}

// ---------------------------------------------------------------------------
// The same colour sweep on colour-split copies of u, v, w, p (cidx): the
// cells of one colour in a row and every face they touch are consecutive, so
// a warp's loads and stores fill whole 32-byte sectors instead of every other
// element of them.  Same per-cell arithmetic as k_sor_sweep_pxz, so the
// same bits; the copies are made once per projection (k_split_copy).
// ---------------------------------------------------------------------------
template <int MU, int PY>
__global__ void __launch_bounds__(256, 4)
k_sor_sweep_split(mdx_dims d, mdx_bc_dev bc, mdx_sor_params p, int parity, int reverse, double* __restrict__ un,
                  double* __restrict__ vn, double* __restrict__ wn, double* __restrict__ pn,
                  const double* __restrict__ mu) {
    const int ni = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int kk = blockIdx.z * blockDim.z + threadIdx.z + 1;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    if (ni > nx / 2 || j > ny || kk > nz) return;
    const int k = reverse ? nz + 1 - kk : kk;
    const int jp = (PY && j == ny) ? 1 : j + 1;
    const int kp = (k == nz) ? 1 : k + 1;
    const int i = 1 + ((j + k + parity) & 1) + 2 * (ni - 1);
    const int ip = (i == nx) ? 1 : i + 1;
    const long long c = cidx(d, i, j, k), cip = cidx(d, ip, j, k), cjp = cidx(d, i, jp, k), ckp = cidx(d, i, j, kp);
    double mu_u_i = 1.0, mu_u_ip = 1.0, mu_v_j = 1.0, mu_v_jp = 1.0, mu_w = 1.0;
    if (MU == MU_PLANE) {
        const long long plane = (long long)d.nxp * d.nyp;
        const int q = i + d.nxp * j;
        mu_u_i = __ldg(mu + q);
        mu_u_ip = __ldg(mu + ip + d.nxp * j);
        mu_v_j = __ldg(mu + plane + q);
        mu_v_jp = __ldg(mu + plane + i + d.nxp * jp);
        mu_w = __ldg(mu + 2 * plane + q);
    }
    double u_i = un[c], u_ip = un[cip], v_j = vn[c], v_jp = vn[cjp], w_k = wn[c], w_kp = wn[ckp], pc = pn[c];
    const double fac = sor_factor(mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, p);
    sor_cell_fac<1, PY, 1>(u_i, u_ip, v_j, v_jp, w_k, w_kp, pc, mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, fac, p,
                           bc, i, j, k, nx, ny, nz);
    un[c] = u_i;
    un[cip] = u_ip;
    vn[c] = v_j;
    vn[cjp] = v_jp;
    wn[c] = w_k;
    wn[ckp] = w_kp;
    pn[c] = pc;
}

// The IBM factors (1 without IBM) and -omega/denom of every (i, j) column in
// colour-split planes (pidx2) for k_sor_sweep_splitv: [mu_u | mu_v | mu_w |
// fac], each split_plane_elems long.  fac is sor_factor of the column -- the
// FP64 expression the other kernels evaluate per cell; with z-invariant
// factors it is the same for every cell of the column, so the same bits.
template <int MU>
__global__ void k_split_tables(mdx_dims d, int py, mdx_sor_params p, const double* __restrict__ mu,
                               double* __restrict__ tab) {
    const long long np = (long long)d.nxp * d.nyp;
    const int ps = split_plane_elems(d);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nxp), j = (int)(t / d.nxp);
        double mu_u = 1.0, mu_v = 1.0, mu_w = 1.0;
        if (MU == MU_PLANE) {
            mu_u = __ldg(mu + t);
            mu_v = __ldg(mu + np + t);
            mu_w = __ldg(mu + 2 * np + t);
        }
        const int o = pidx2(d, i, j);
        tab[o] = mu_u;
        tab[ps + o] = mu_v;
        tab[2 * ps + o] = mu_w;
        double f = 0.0;
        if (i >= 1 && i <= d.nx && j >= 1 && j <= d.ny) {
            const int ip = i == d.nx ? 1 : i + 1;
            const int jp = (py && j == d.ny) ? 1 : j + 1;
            double mu_uip = 1.0, mu_vjp = 1.0;
            if (MU == MU_PLANE) {
                mu_uip = __ldg(mu + ip + (long long)d.nxp * j);
                mu_vjp = __ldg(mu + np + i + (long long)d.nxp * jp);
            }
            f = sor_factor(mu_u, mu_uip, mu_v, mu_vjp, mu_w, mu_w, p);
        }
        tab[3 * ps + o] = f;
    }
}

__device__ __forceinline__ void ld2(double (&a)[2], const double* q) {
    const double2 v = *reinterpret_cast<const double2*>(q);
    a[0] = v.x;
    a[1] = v.y;
}
__device__ __forceinline__ void ld2_ro(double (&a)[2], const double* __restrict__ q) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(q));
    a[0] = v.x;
    a[1] = v.y;
}
__device__ __forceinline__ void st2(double* q, const double (&a)[2]) {
    *reinterpret_cast<double2*>(q) = make_double2(a[0], a[1]);
}

// One FP64 colour sweep on the colour-split copies with two consecutive cells
// of the swept colour per thread, moved with 16-byte accesses: the layout
// and ownership of k_sor_sweep32v (k_sor_mixed.cu) -- a thread owns window w
// (positions 2w, 2w + 1) of its row in the swept colour's half and of the
// other half's rows (j + 1, k) and (j, k + 1); the x neighbours' faces u(i+1)
// are the window shifted by one in rows whose swept cells have odd i (window
// plus one scalar), the window itself in the others except the wrap of cell
// nx to position 0, and are stored one scalar per cell; positions without a
// swept cell are written back unchanged.  The factors come from
// k_split_tables.  The per-cell arithmetic is sor_cell_fac, as in
// k_sor_sweep_split, so the same bits.  Periodic x and z.
template <int PY>
__global__ void __launch_bounds__(128)
k_sor_sweep_splitv(mdx_dims d, mdx_bc_dev bc, mdx_sor_params p, int parity, int reverse, int nwin,
                   double* __restrict__ un, double* __restrict__ vn, double* __restrict__ wn,
                   double* __restrict__ pn, const double* __restrict__ tab) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per_plane = (long long)nwin * d.ny;
    if (g >= per_plane * d.nz) return;
    const int kk = (int)(g / per_plane);
    const int rem = (int)(g - (long long)kk * per_plane);
    const int j = rem / nwin + 1;
    const int p0 = 2 * (rem - (j - 1) * nwin);
    const int k = reverse ? d.nz - kk : kk + 1;
    const int cs = 1 - parity;            // colour (i + j + k) & 1 of the swept cells
    const int eo = (cs + j + k) & 1;      // i & 1 of the swept cells of this row
    const int half = d.nx / 2;
    const int jp = (PY && j == d.ny) ? 1 : j + 1;
    const int kp = (k == d.nz) ? 1 : k + 1;
    const long long H = (long long)d.hs * d.nyp * d.nzp;
    const long long own = cs * H + ((long long)k * d.nyp + j) * d.hs + p0;
    const long long oth = (1 - cs) * H + ((long long)k * d.nyp + j) * d.hs;
    const long long ojp = (1 - cs) * H + ((long long)k * d.nyp + jp) * d.hs + p0;
    const long long okp = (1 - cs) * H + ((long long)kp * d.nyp + j) * d.hs + p0;
    const int PH = d.hs * d.nyp, ps = 2 * PH;
    const int hp = (eo + j) & 1;
    const int mown = hp * PH + j * d.hs + p0;
    const int mox = (1 - hp) * PH + j * d.hs;
    const int mjp = (1 - hp) * PH + jp * d.hs + p0;

    double u0[2], ux[2], v0[2], vy[2], w0[2], wz[2], q[2];
    double mu_u[2], mu_ux[2], mu_v[2], mu_vy[2], mu_w[2], fc[2];
    ld2(u0, un + own);
    ld2(v0, vn + own);
    ld2(w0, wn + own);
    ld2(q, pn + own);
    ld2(ux, un + oth + p0);
    ld2(vy, vn + ojp);
    ld2(wz, wn + okp);
    ld2_ro(mu_u, tab + mown);
    ld2_ro(mu_v, tab + ps + mown);
    ld2_ro(mu_w, tab + 2 * ps + mown);
    ld2_ro(fc, tab + 3 * ps + mown);
    ld2_ro(mu_ux, tab + mox + p0);
    ld2_ro(mu_vy, tab + ps + mjp);
    const int xe = eo ? p0 + 2 : 0;
    const bool need_xe = eo ? (p0 + 2 < d.hs) : (half >= p0 && half < p0 + 2);
    double uxe = 0.0, muxe = 0.0;
    if (need_xe) {
        uxe = un[oth + xe];
        muxe = __ldg(tab + mox + xe);
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int pe = p0 + e;
        const bool valid = eo ? (pe < half) : (pe >= 1 && pe <= half);
        const bool wrap = !eo && pe == half;
        double u_ip, mu_ip;
        if (e == 0) {
            u_ip = eo ? ux[1] : (wrap ? uxe : ux[0]);
            mu_ip = eo ? mu_ux[1] : (wrap ? muxe : mu_ux[0]);
        } else {
            u_ip = (eo || wrap) ? uxe : ux[1];
            mu_ip = (eo || wrap) ? muxe : mu_ux[1];
        }
        if (valid) {
            const int i = 2 * pe + eo;
            sor_cell_fac<1, PY, 1>(u0[e], u_ip, v0[e], vy[e], w0[e], wz[e], q[e], mu_u[e], mu_ip, mu_v[e], mu_vy[e],
                                   mu_w[e], mu_w[e], fc[e], p, bc, i, j, k, d.nx, d.ny, d.nz);
            un[oth + (eo ? pe + 1 : (wrap ? 0 : pe))] = u_ip;
        }
    }
    st2(un + own, u0);
    st2(vn + own, v0);
    st2(wn + own, w0);
    st2(pn + own, q);
    st2(vn + ojp, vy);
    st2(wn + okp, wz);
}

// Every padded element of u, v, w, p between the reference layout and the
// colour-split copies (TO_SPLIT) or back.
template <bool TO_SPLIT>
__global__ void k_split_copy(mdx_dims d, double* __restrict__ a0, double* __restrict__ a1, double* __restrict__ a2,
                             double* __restrict__ a3, double* __restrict__ s0, double* __restrict__ s1,
                             double* __restrict__ s2, double* __restrict__ s3) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.npad; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nxp);
        const long long r = t / d.nxp;
        const int j = (int)(r % d.nyp);
        const int k = (int)(r / d.nyp);
        const long long c = cidx(d, i, j, k);
        if (TO_SPLIT) {
            s0[c] = a0[t]; s1[c] = a1[t]; s2[c] = a2[t]; s3[c] = a3[t];
        } else {
            a0[t] = s0[c]; a1[t] = s1[c]; a2[t] = s2[c]; a3[t] = s3[c];
        }
    }
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
    const bool pxz = ctx->bc.is_periodic[0] && ctx->bc.is_periodic[2] && ctx->mu_mode != MU_FULL;
    const bool py = ctx->bc.is_periodic[1] != 0;
    for (int parity = 0; parity < 2; ++parity) {
        const int rev = parity;   // red sweeps walk k up, black sweeps walk k down
        if (pxz) {
            auto kfn = ctx->mu_mode == MU_PLANE ? (py ? k_sor_sweep_pxz<MU_PLANE, 1> : k_sor_sweep_pxz<MU_PLANE, 0>)
                                                : (py ? k_sor_sweep_pxz<MU_ONE, 1> : k_sor_sweep_pxz<MU_ONE, 0>);
            MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep", kfn, grid, block, 0, d, ctx->bcd, p, parity, rev,
                       f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], ctx->mu);
        } else if (ctx->mu_mode == MU_ONE)
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

// ---- red-black kernel variants and their autotuner ---------------------------
// Variants (all bit-identical per iteration):
//   MDX_SORV_SWEEPS    one launch per colour sweep
//   MDX_SORV_FUSED8    fused red+black pass, 32x8 tiles, 256 threads
//   MDX_SORV_FUSED16   fused red+black pass, 32x16 tiles, 512 threads
//   MDX_SORV_SPLIT     one launch per colour sweep on colour-split copies
//                      (tol > 0 only: the copies cost two passes over u, v,
//                      w, p per projection)
//   MDX_SORV_SPLITV    the same with two cells per thread and 16-byte
//                      accesses, the column factors from tables
// All but the first need periodic x and z and mu = 1 or z-invariant.
// (the enum is in mdx_internal.cuh)

static int split_alloc(mdx_ctx_t* ctx) {
    const size_t bytes = sizeof(double) * (size_t)split_elems(ctx->d);
    for (int t = 0; t < 4; ++t)
        if (!ctx->split_f[t]) MDX_CUDA(ctx, cudaMalloc(&ctx->split_f[t], bytes));
    if (!ctx->split_tab) {
        const size_t tb = sizeof(double) * 4 * (size_t)split_plane_elems(ctx->d);
        MDX_CUDA(ctx, cudaMalloc(&ctx->split_tab, tb));
        MDX_CUDA(ctx, cudaMemsetAsync(ctx->split_tab, 0, tb, ctx->stream));
    }
    return MDX_OK;
}

// The column factors of this projection for k_sor_sweep_splitv.
static int split_tables(mdx_ctx_t* ctx, const mdx_sor_params& p) {
    const mdx_dims& d = ctx->d;
    const int py = ctx->bc.is_periodic[1] ? 1 : 0;
    const int nb = (int)std::min<long long>(((long long)d.nxp * d.nyp + 255) / 256, 1024);
    auto kfn = ctx->mu_mode == MU_PLANE ? k_split_tables<MU_PLANE> : k_split_tables<MU_ONE>;
    MDX_LAUNCH(ctx, MDX_T_OTHER, "split tables", kfn, nb, 256, 0, d, py, p, ctx->mu, ctx->split_tab);
    return MDX_OK;
}

static int sor_splitv_iteration(mdx_ctx_t* ctx, const mdx_sor_params& p) {
    const mdx_dims& d = ctx->d;
    double** s = ctx->split_f;
    const int nwin = (d.nx / 2 + 2) / 2;   // windows of two positions covering 0 .. nx/2
    const long long nthr = (long long)nwin * d.ny * d.nz;
    const int nb = (int)((nthr + 127) / 128);   // 128-thread blocks: 5 per SM at 92 registers
    auto kfn = ctx->bc.is_periodic[1] ? k_sor_sweep_splitv<1> : k_sor_sweep_splitv<0>;
    for (int parity = 0; parity < 2; ++parity)
        MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep split vec", kfn, nb, 128, 0, d, ctx->bcd, p, parity, parity, nwin,
                   s[0], s[1], s[2], s[3], ctx->split_tab);
    return MDX_OK;
}

// u, v, w, p into (to_split) or out of the colour-split copies.
static int split_copy(mdx_ctx_t* ctx, bool to_split) {
    const mdx_dims& d = ctx->d;
    double** f = ctx->f;
    double** s = ctx->split_f;
    const int nb = (int)std::min<long long>((d.npad + 255) / 256, 148 * 16);
    auto kfn = to_split ? k_split_copy<true> : k_split_copy<false>;
    MDX_LAUNCH(ctx, MDX_T_OTHER, "split copy", kfn, nb, 256, 0, d, f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], s[0],
               s[1], s[2], s[3]);
    ctx->split_norms = to_split;
    return MDX_OK;
}

static int sor_split_iteration(mdx_ctx_t* ctx, const mdx_sor_params& p) {
    const mdx_dims& d = ctx->d;
    double** s = ctx->split_f;
    dim3 block(32, 4, 2);
    dim3 grid((d.nx / 2 + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
    const bool py = ctx->bc.is_periodic[1] != 0;
    auto kfn = ctx->mu_mode == MU_PLANE ? (py ? k_sor_sweep_split<MU_PLANE, 1> : k_sor_sweep_split<MU_PLANE, 0>)
                                        : (py ? k_sor_sweep_split<MU_ONE, 1> : k_sor_sweep_split<MU_ONE, 0>);
    for (int parity = 0; parity < 2; ++parity)
        MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep split", kfn, grid, block, 0, d, ctx->bcd, p, parity, parity, s[0],
                   s[1], s[2], s[3], ctx->mu);
    return MDX_OK;
}

template <int MU, int TY, int NT>
static size_t fused_smem() {
    using G = fused_geom<32, TY, NT>;
    return sizeof(double) * (4 * G::SLOT + (MU == MU_PLANE ? G::NU + G::NV + G::NC : 0) + G::NC) +
           sizeof(int) * (G::UX + G::WY + 1);
}

static bool fused_ok(const mdx_ctx_t* ctx) {
    return ctx->bc.is_periodic[0] && ctx->bc.is_periodic[2] && ctx->mu_mode != MU_FULL;
}

template <int TY, int NT>
static int fused_attrs(mdx_ctx_t* ctx) {
    const int s_one = (int)fused_smem<MU_ONE, TY, NT>(), s_plane = (int)fused_smem<MU_PLANE, TY, NT>();
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_sor_fused<MU_ONE, 0, 32, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s_one));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_sor_fused<MU_ONE, 1, 32, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s_one));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_sor_fused<MU_PLANE, 0, 32, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s_plane));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_sor_fused<MU_PLANE, 1, 32, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s_plane));
    return MDX_OK;
}

static int fused_prepare(mdx_ctx_t* ctx) {
    const size_t bytes = sizeof(double) * ctx->d.npad;
    for (int t = 0; t < 4; ++t)
        if (!ctx->sor_alt[t]) MDX_CUDA(ctx, cudaMalloc(&ctx->sor_alt[t], bytes));
    // the second state starts as a copy, so faces the sweeps never touch
    // (ghosts) are equal in both
    const int ids[4] = {MDX_UN, MDX_VN, MDX_WN, MDX_PN};
    for (int t = 0; t < 4; ++t)
        MDX_CUDA(ctx, cudaMemcpyAsync(ctx->sor_alt[t], ctx->f[ids[t]], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    if (!ctx->fused_attr) {
        MDX_TRY((fused_attrs<8, 256>(ctx)));
        MDX_TRY((fused_attrs<16, 512>(ctx)));
        ctx->fused_attr = true;
    }
    return MDX_OK;
}

template <int TY, int NT>
static int sor_fused_iteration(mdx_ctx_t* ctx, const mdx_sor_params& p) {
    const mdx_dims& d = ctx->d;
    double** f = ctx->f;
    const int KZ = ctx->opts.sor_kz > 0 ? ctx->opts.sor_kz : 16;
    dim3 grid((d.nx + 31) / 32, (d.ny + TY - 1) / TY, (d.nz + KZ - 1) / KZ);
    double** a = ctx->sor_alt;
    const bool py = ctx->bc.is_periodic[1] != 0;
    const bool plane = ctx->mu_mode == MU_PLANE;
    auto kfn = plane ? (py ? k_sor_fused<MU_PLANE, 1, 32, TY, NT> : k_sor_fused<MU_PLANE, 0, 32, TY, NT>)
                     : (py ? k_sor_fused<MU_ONE, 1, 32, TY, NT> : k_sor_fused<MU_ONE, 0, 32, TY, NT>);
    const size_t smem = plane ? fused_smem<MU_PLANE, TY, NT>() : fused_smem<MU_ONE, TY, NT>();
    MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor fused", kfn, grid, NT, smem, d, ctx->bcd, p, KZ, f[MDX_UN], f[MDX_VN],
               f[MDX_WN], f[MDX_PN], a[0], a[1], a[2], a[3], ctx->mu);
    // the new state becomes the current one
    std::swap(f[MDX_UN], a[0]);
    std::swap(f[MDX_VN], a[1]);
    std::swap(f[MDX_WN], a[2]);
    std::swap(f[MDX_PN], a[3]);
    return MDX_OK;
}

static int sor_iterate(mdx_ctx_t* ctx, const mdx_sor_params& p, int variant) {
    if (variant == MDX_SORV_SPLIT) return sor_split_iteration(ctx, p);
    if (variant == MDX_SORV_SPLITV) return sor_splitv_iteration(ctx, p);
    if (variant == MDX_SORV_FUSED8) return sor_fused_iteration<8, 256>(ctx, p);
    if (variant == MDX_SORV_FUSED16) return sor_fused_iteration<16, 512>(ctx, p);
    return sor_iteration(ctx, p);
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
    MDX_LAUNCH(ctx, MDX_T_OTHER, "mu tables", k_mu_tables, nb, 256, 0, n, dg, ctx->f[MDX_COEF_U],
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
    const mdx_solver_opts_t& o = ctx->opts;
    // Residual scale of this projection, on u* before any guess: converged
    // when ||div u|| <= max(tol*||div u*||, atol); the default atol is the
    // round-off level of the divergence, below which a relative target
    // cannot be met once u* is nearly solenoidal.
    double r0 = 0.0, umax = 0.0, atol = 0.0, target = 0.0;
    if (o.tol > 0.0) {
        double linf = 0.0;
        MDX_TRY(mdx_k_div_norms(ctx, f[MDX_UN], f[MDX_VN], f[MDX_WN], &r0, &linf, &umax));
        atol = (o.atol < 0.0) ? mdx_div_floor(ctx, umax) : o.atol;
        target = std::max(o.tol * r0, atol);
    }
    // warm start: record this projection's increment; apply a guess
    const bool warm = mdx_guess_supported(ctx) && (ctx->guess_mode != MDX_GUESS_ZERO || ctx->record_increments);
    if (warm) MDX_TRY(mdx_warm_begin(ctx));
    bool guessed = false;
    double rg = r0;   // ||div u|| after the guess
    if (warm && ctx->guess_mode != MDX_GUESS_ZERO) MDX_TRY(mdx_guess_apply(ctx, dg, r0, &guessed, &rg));
    if (o.precision == MDX_PREC_MIXED) {   // FP32 sweeps in FP64 defect correction
        bool handled = false;
        MDX_TRY(mdx_k_projection_redblack_mixed(ctx, dg, st, &handled, r0, umax, atol));
        if (handled) {
            ctx->last.guessed = guessed ? 1 : 0;
            if (st) st->guessed = ctx->last.guessed;
            if (warm) MDX_TRY(mdx_warm_end(ctx, ctx->last.status == MDX_OK, ctx->last.iterations));
            return MDX_OK;
        }
    }
    // kernel variant: the requested one, the tuned one, or -- while tuning --
    // the next untried candidate for each residual-check block
    const bool fok = fused_ok(ctx);
    int want = ctx->opts.sor_variant;
    if (want < MDX_SORV_AUTO || want >= MDX_SORV_NUM) want = MDX_SORV_AUTO;
    if (want != MDX_SORV_SWEEPS && !fok) want = MDX_SORV_SWEEPS;
    if (want == MDX_SORV_AUTO || want == MDX_SORV_FUSED8 || want == MDX_SORV_FUSED16) MDX_TRY(fused_prepare(ctx));
    const bool splitv = want == MDX_SORV_AUTO || want == MDX_SORV_SPLITV;
    if (want == MDX_SORV_AUTO || want == MDX_SORV_SPLIT || splitv) MDX_TRY(split_alloc(ctx));
    const mdx_sor_params p = sor_params(ctx, dg);
    if (splitv) MDX_TRY(split_tables(ctx, p));
    // where u, v, w, p live while the sweeps run: the colour-split copies for
    // MDX_SORV_SPLIT blocks, the reference arrays for the others
    bool in_split = false;
    auto layout_for = [&](int v) -> int {
        if ((v == MDX_SORV_SPLIT || v == MDX_SORV_SPLITV) != in_split) {
            in_split = !in_split;
            MDX_TRY(split_copy(ctx, in_split));
        }
        return MDX_OK;
    };
    auto pick = [&]() -> int {
        if (want != MDX_SORV_AUTO) return want;
        if (ctx->sor_tuned > 0) return ctx->sor_tuned;
        for (int v = MDX_SORV_SWEEPS; v < MDX_SORV_NUM; ++v)
            if (ctx->sor_tune_ms[v] <= 0.0) return v;
        int best = MDX_SORV_SWEEPS;
        for (int v = MDX_SORV_SWEEPS; v < MDX_SORV_NUM; ++v)
            if (ctx->sor_tune_ms[v] < ctx->sor_tune_ms[best]) best = v;
        ctx->sor_tuned = best;
        return best;
    };
    mdx_solve_stats_t s{};
    s.guessed = guessed ? 1 : 0;
    if (o.tol <= 0.0) {
        const int v = (want == MDX_SORV_AUTO) ? (ctx->sor_tuned > 0 ? ctx->sor_tuned : MDX_SORV_SWEEPS) : want;
        MDX_TRY(layout_for(v));
        mdx_event_pair run{};
        mdx_sweep_run_begin(ctx, &run);
        for (int it = 0; it < o.n_iter; ++it) MDX_TRY(sor_iterate(ctx, p, v));
        mdx_sweep_run_end(ctx, &run);
        MDX_TRY(layout_for(MDX_SORV_SWEEPS));
        s.variant = v;
        s.iterations = o.n_iter;
        s.status = MDX_OK;
    } else {
        double linf = 0.0, r = rg;
        s.residual0 = r0;
        s.atol = atol;
        if (!std::isfinite(r0) || !std::isfinite(umax) || !std::isfinite(r)) {
            s.status = MDX_ERR_NONFINITE;
        } else if (r <= target) {
            s.status = MDX_OK;
            s.residual = (r0 > 0.0) ? r / r0 : 0.0;
        } else {
            int it = 0;
            s.status = MDX_NOT_CONVERGED;
            mdx_check_schedule cs;
            cs.start(o.check_every, o.check_mode, r);
            int block = cs.every;
            while (it < o.max_iter) {
                const int m = std::min(block, o.max_iter - it);
                const int v = pick();
                MDX_TRY(layout_for(v));
                const bool timing_block = want == MDX_SORV_AUTO && ctx->sor_tuned == 0;
                if (timing_block) MDX_CUDA(ctx, cudaEventRecord(ctx->tune_ev[0], ctx->stream));
                mdx_event_pair run{};
                mdx_sweep_run_begin(ctx, &run);
                for (int q = 0; q < m; ++q) MDX_TRY(sor_iterate(ctx, p, v));
                mdx_sweep_run_end(ctx, &run);
                if (timing_block) MDX_CUDA(ctx, cudaEventRecord(ctx->tune_ev[1], ctx->stream));
                it += m;
                s.variant = v;
                double** uvw = in_split ? ctx->split_f : nullptr;
                MDX_TRY(mdx_k_div_norms(ctx, uvw ? uvw[0] : f[MDX_UN], uvw ? uvw[1] : f[MDX_VN],
                                        uvw ? uvw[2] : f[MDX_WN], &r, &linf));
                if (timing_block) {   // the norms synchronised the stream; time per iteration
                    float ms = 0.f;
                    if (cudaEventElapsedTime(&ms, ctx->tune_ev[0], ctx->tune_ev[1]) == cudaSuccess)
                        ctx->sor_tune_ms[v] = ms > 0.f ? ms / m : 1e-9;
                }
                if (!std::isfinite(r)) { s.status = MDX_ERR_NONFINITE; break; }
                if (r <= target) { s.status = MDX_OK; break; }
                block = cs.next(it, r, target);
            }
            MDX_TRY(layout_for(MDX_SORV_SWEEPS));
            s.iterations = it;
            s.residual = r / r0;
        }
    }
    if (warm) MDX_TRY(mdx_warm_end(ctx, o.tol > 0.0 && s.status == MDX_OK, s.iterations));
    ctx->last = s;
    if (st) *st = s;
    return MDX_OK;
}
