// k_ensemble.cu -- batched ensemble: many independent wavy-wall channels of
// different sizes advanced together, one persistent cooperative launch per
// RK3 substage for all of them.  No counterpart in the reference, which
// advances one channel per process.
//
// Each member is a channel like the single-context path runs it: periodic
// x and z, no-slip walls in y (v Dirichlet 0, p Neumann 0), the wavy-wall
// IBM of set_ibm_coeff (geometry 1, coefficients independent of z) or none,
// the red-black projection in FP64, optionally warm-started from the
// extrapolated pressure increment.  The substage kernel runs, for every
// member, the phases of one substage with a grid-wide barrier between them:
//   momentum -> u <- u*, IBM factors -> ||div u*|| -> [guess, ||div||,
//   undo] -> red/black sweeps with a residual check every check_every
//   iterations until each member meets its own tolerance -> increment
//   record -> boundary conditions (y, x, z phases).
// The per-cell arithmetic is the single-context kernels' (mdx_cell.cuh,
// -fmad=false), so with a fixed iteration count every member's fields are
// bit-for-bit those of the single-context path; with a tolerance the
// residual sums run in another order, which moves the last bits of the norm.
//
// Work: every phase walks a list of 256-element tiles (member, first
// element), members back to back, with the blocks of the persistent grid
// striding over the list; members that have converged skip their sweep and
// residual tiles.  Loop decisions are read from device memory after a grid
// barrier, so every block takes the same path; all loops are bounded by
// max_iter.  The grid (threads per block, blocks per SM) comes from a timed
// autotuner whose choice is cached in a JSON file.
#include "mdx_cell.cuh"
#include "mdx_cell32.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace cg = cooperative_groups;

namespace {

constexpr int ETILE = 256;           // elements per work tile
// cells of one colour per sweep tile.  Measured on the 64-member C4
// ensemble: 1024 (the tile set-up spread over more cells per thread) 3 %
// slower -- late in a substage only the slowest members are swept, and
// fewer tiles keep fewer blocks busy -- and 128 (more tiles, set-up per
// cell) 13 % slower.
constexpr int HTILE = 256;
constexpr int MAX_THREADS = 512;

// n / d for 32-bit n by one multiply-high with c = ceil(2^64 / d) (Lemire,
// Kaser & Kurz, "Faster remainder by direct computation", 2019); d >= 2.
struct fdiv32 {
    unsigned long long c;
    unsigned d;
};
fdiv32 make_fdiv(unsigned d) { return fdiv32{~0ull / d + 1ull, d}; }
__device__ __forceinline__ unsigned fq(unsigned n, const fdiv32& f) {
    return (unsigned)__umul64hi(f.c, (unsigned long long)n);
}

struct ens_member {                  // per member, read-only in the kernel
    mdx_dims d;
    mdx_step_params p;
    mdx_sor_params sp;               // dt_gamma and idt set per projection
    mdx_bc_dev bc;
    double dt;
    double idx, idy, idz;            // 1/dx, 1/dy, 1/dz
    int ibm;                         // coefficient planes present (MU_PLANE)
    fdiv32 fx, fy, fh;               // division by nx, ny, nx/2
    double *un, *vn, *wn, *pn, *us, *vs, *ws, *ou, *ov, *ow;
    double *cu, *cv, *cw;            // (nx+2)(ny+2) planes
    double *mu;                      // 3 planes of this projection
    double *p0, *guess;
    double* h[3][2];                 // increment history per substage
    // mixed precision: FP32 corrections and residual (colour-split), FP32 factor planes
    float *du, *dv, *dw, *dp, *r32, *mu32, *fac32;
    // learned warm start: the last two increments of this substage (network
    // inputs) and the network's correction
    double *hl1, *hl2, *delta;
};

struct ens_state {                   // per member, updated in the kernel
    double r0, umax, atol, target, r, rg;
    int it, active, guessed, status, undo, has_guess, extrap;
    int hist_valid;                  // bit s: current increment of substage s; bit 3+s: the one before
    int flip;                        // bit s: h[s][1] is the current increment
    int last_iters;
    long long iters_total;
    double last_residual;
    // mixed precision: 0 FP64 residual (after applying the corrections), 1 FP32
    // sweeps, 2 done; outer FP64 corrections; inner stop state
    int phase, outer, stale;
    double e_best, inner_target;
    // learned warm start: this projection's correction (0 none, 1 kept, 2
    // undone, 3 being tried) and the counts over the run
    int lr_last;
    long long lr_corr, lr_rej;
    // the gate (gate_period > 0): per substage, averages of the iterations
    // with the correction (1) and without (0), their counts, projections
    // since the other choice was tried, this projection's choice (-1 none),
    // and the projections left to the extrapolated guess
    double g_ema[3][2];
    int g_n[3][2];
    int g_since[3];
    int g_arm;
    long long lr_gated;
    // the FP32 sweeps' scalars of this substage (1/dx, 1/dy, 1/dz, 1/dt_gamma),
    // set once at the substage start instead of per tile
    float p32[4];
};

struct ens_list {
    const int2* t;
    int n;
};

struct ens_args {
    const ens_member* mem;
    ens_state* st;
    int nmem;
    ens_list cell, half, pad, plane, bcy, bcx, bcz;
    const int* cell_begin;           // [nmem + 1]: each member's range of cell tiles
    const int* half_begin;           // [nmem + 1]: each member's range of sweep tiles
    int* act;                        // [2 (nmem + 1)]: prefix sums of the active members' sweep, then cell tiles
    double* part;                    // 3 doubles per cell tile
    double a, b, c;                  // RK3 coefficients of this substage
    int substage;
    int momentum;                    // 0: the t=0 projection (u* = u, dt_gamma = 1)
    int guess_mode;
    int n_iter, max_iter, check_every;
    double tol, atol;
    int mixed;                       // FP32 sweeps in FP64 defect correction
    int pot;                         // ... carrying each cell's phi (the potential form, Phi in dp; inner_form 2)
    double inner_sor;                // their over-relaxation
    // 0: the whole substage; 1: up to the warm start, then the network's
    // inputs; 2: from the learned correction on (the network ran between)
    int split;
    const int* learn_ok;             // per member: the network wrote a correction
    int gate_period;                 // > 0: apply it per substage only while it takes fewer iterations
};

// The gate's choice for an eligible projection of substage s: 0 the
// extrapolated guess alone, 1 with the learned correction (the rule of
// mdx_unet_correct: a baseline without it first, then with it, then the
// cheaper one, the other re-tried every period-th projection).
__device__ int gate_choose(ens_state& S, int s, int period) {
    if (S.g_n[s][0] == 0) return 0;
    if (S.g_n[s][1] == 0) return 1;
    const int pref = S.g_ema[s][1] <= S.g_ema[s][0] ? 1 : 0;
    if (++S.g_since[s] >= period) {
        S.g_since[s] = 0;
        return 1 - pref;
    }
    return pref;
}

__device__ __forceinline__ double nanmax(double a, double b) { return (a != a || b != b) ? (a + b) : fmax(a, b); }

// Block-wide (sum, max, max) for any blockDim <= MAX_THREADS; result in thread 0.
__device__ void block_reduce3(double& s, double& m, double& u) {
    __shared__ double sh[3][MAX_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        m = nanmax(m, __shfl_down_sync(0xffffffffu, m, o));
        u = nanmax(u, __shfl_down_sync(0xffffffffu, u, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (l == 0) {
        sh[0][w] = s;
        sh[1][w] = m;
        sh[2][w] = u;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < nw; ++q) {
            s += sh[0][q];
            m = nanmax(m, sh[1][q]);
            u = nanmax(u, sh[2][q]);
        }
    }
}

__device__ __forceinline__ void cell_ijk(const ens_member& M, unsigned t, int& i, int& j, int& k) {
    const unsigned r = fq(t, M.fx);
    i = (int)(t - r * M.fx.d) + 1;
    const unsigned kk = fq(r, M.fy);
    j = (int)(r - kk * M.fy.d) + 1;
    k = (int)kk + 1;
}

__device__ __forceinline__ double dg_of(const ens_args& A, const ens_member& M) {
    return A.momentum ? M.dt * A.c : 1.0;
}

// Prefix sums of the sweep and cell tiles of the members still active (one
// thread); a converged member's range is empty, so the sweeps and residual
// checks visit only live tiles however many members have finished.
__device__ void compact_active(const ens_args& A) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int h = 0, c = 0;
    int* ah = A.act;
    int* ac = A.act + A.nmem + 1;
    for (int m = 0; m < A.nmem; ++m) {
        ah[m] = h;
        ac[m] = c;
        if (A.st[m].active) {
            h += A.half_begin[m + 1] - A.half_begin[m];
            c += A.cell_begin[m + 1] - A.cell_begin[m];
        }
    }
    ah[A.nmem] = h;
    ac[A.nmem] = c;
}

// Virtual tile vt of a compacted prefix -> (member, tile of that member's range).
__device__ __forceinline__ int2 active_tile(const int* pref, const int* begin, int nmem, int vt) {
    int lo = 0, hi = nmem;   // pref[lo] <= vt < pref[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pref[mid] <= vt) lo = mid;
        else hi = mid;
    }
    return make_int2(lo, begin[lo] + (vt - pref[lo]));
}

// Partials of sum div^2, max|div|, max(|u|,|v|,|w|) of cell tile ti (the
// divergence of k_div_partials) into part[3 ti ..].
__device__ void residual_tile(const ens_args& A, int ti) {
    const int2 T = A.cell.t[ti];
    const ens_member& M = A.mem[T.x];
    const mdx_dims d = M.d;
    const double* __restrict__ un = M.un;
    const double* __restrict__ vn = M.vn;
    const double* __restrict__ wn = M.wn;
    const double idx = M.idx, idy = M.idy, idz = M.idz;
    const fdiv32 fx = M.fx, fy = M.fy;
    double s = 0.0, m = 0.0, um = 0.0;
    for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
        const unsigned t = (unsigned)T.y + e;
        if (t >= (unsigned)d.nint) break;
        const unsigned r = fq(t, fx);
        const int i = (int)(t - r * fx.d) + 1;
        const unsigned kq = fq(r, fy);
        const int j = (int)(r - kq * fy.d) + 1;
        const int k = (int)kq + 1;
        const int ip = i + 1 > d.nx ? 1 : i + 1;
        const int jp = j + 1;   // walls in y: v(ny+1) is the wall face
        const int kp = k + 1 > d.nz ? 1 : k + 1;
        const long long c = pidx(d, i, j, k);
        const double uc = un[c], vc = vn[c], wc = wn[c];
        const double dv = (un[pidx(d, ip, j, k)] - uc) * idx + (vn[pidx(d, i, jp, k)] - vc) * idy +
                          (wn[pidx(d, i, j, kp)] - wc) * idz;
        s += dv * dv;
        m = nanmax(m, fabs(dv));
        um = nanmax(um, nanmax(fabs(uc), nanmax(fabs(vc), fabs(wc))));
    }
    block_reduce3(s, m, um);
    if (threadIdx.x == 0) {
        A.part[3 * ti] = s;
        A.part[3 * ti + 1] = m;
        A.part[3 * ti + 2] = um;
    }
    __syncthreads();
}

// Residual partials of the members selected by `want`.
template <typename Want>
__device__ void residual_tiles(const ens_args& A, Want want) {
    for (int ti = blockIdx.x; ti < A.cell.n; ti += gridDim.x)
        if (want(A.cell.t[ti].x)) residual_tile(A, ti);   // uniform per block
}

// Residual partials of the active members (compacted ranges).
__device__ void residual_active(const ens_args& A) {
    const int* pref = A.act + A.nmem + 1;
    const int total = pref[A.nmem];
    for (int vt = blockIdx.x; vt < total; vt += gridDim.x)
        residual_tile(A, active_tile(pref, A.cell_begin, A.nmem, vt).y);
}

// Sum the tile partials of member m (block-wide, fixed order for a fixed
// block size): s = sum of squares, um = max |u|.
__device__ void member_sums(const ens_args& A, int m, double& s, double& um) {
    double ss = 0.0, mm = 0.0, uu = 0.0;
    for (int ti = A.cell_begin[m] + threadIdx.x; ti < A.cell_begin[m + 1]; ti += blockDim.x) {
        ss += A.part[3 * ti];
        mm = nanmax(mm, A.part[3 * ti + 1]);
        uu = nanmax(uu, A.part[3 * ti + 2]);
    }
    block_reduce3(ss, mm, uu);
    s = ss;
    um = uu;
}

// What a colour sweep of one member reads, copied to registers per tile so
// that stores through the field pointers do not force reloads.
struct sweep_view {
    mdx_dims d;
    double *un, *vn, *wn, *pn;
    const double* mu;
    int ibm;
    fdiv32 fy, fh;
};

__device__ __forceinline__ sweep_view make_view(const ens_member& M) {
    sweep_view v;
    v.d = M.d;
    v.un = M.un;
    v.vn = M.vn;
    v.wn = M.wn;
    v.pn = M.pn;
    v.mu = M.mu;
    v.ibm = M.ibm;
    v.fy = M.fy;
    v.fh = M.fh;
    return v;
}

// One colour sweep of a member's cell at sweep element t: the arithmetic of
// k_sor_sweep_pxz (periodic x and z, walls in y; the wall rows read the
// boundary values from bc).
__device__ __forceinline__ void sweep_cell(const sweep_view& v, const mdx_bc_dev& bc, const mdx_sor_params& p,
                                           int parity, unsigned t) {
    const mdx_dims& d = v.d;
    const unsigned r = fq(t, v.fh);
    const int ni = (int)(t - r * v.fh.d) + 1;
    const unsigned q = fq(r, v.fy);
    const int j = (int)(r - q * v.fy.d) + 1;
    const int kk = (int)q + 1;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int k = parity ? nz + 1 - kk : kk;
    const int jp = j + 1;
    int kp = k + 1;
    if (kp > nz) kp = 1;
    const int i = 1 + ((j + k + parity) & 1) + 2 * (ni - 1);
    int ip = i + 1;
    if (ip > nx) ip = 1;
    const long long c = pidx(d, i, j, k);
    const long long cip = pidx(d, ip, j, k), cjp = pidx(d, i, jp, k), ckp = pidx(d, i, j, kp);
    double mu_u_i = 1.0, mu_u_ip = 1.0, mu_v_j = 1.0, mu_v_jp = 1.0, mu_w = 1.0;
    if (v.ibm) {
        const double* mu = v.mu;
        const long long np = (long long)d.nxp * d.nyp;
        const long long qq = i + (long long)d.nxp * j;
        mu_u_i = mu[qq];
        mu_u_ip = mu[ip + (long long)d.nxp * j];
        mu_v_j = mu[np + qq];
        mu_v_jp = mu[np + i + (long long)d.nxp * jp];
        mu_w = mu[2 * np + qq];
    }
    double* __restrict__ un = v.un;
    double* __restrict__ vn = v.vn;
    double* __restrict__ wn = v.wn;
    double* __restrict__ pn = v.pn;
    double u_i = un[c], u_ip = un[cip], v_j = vn[c], v_jp = vn[cjp], w_k = wn[c], w_kp = wn[ckp], pc = pn[c];
    const double fac = sor_factor(mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, p);
    sor_cell_fac<1, 0, 1>(u_i, u_ip, v_j, v_jp, w_k, w_kp, pc, mu_u_i, mu_u_ip, mu_v_j, mu_v_jp, mu_w, mu_w, fac, p, bc,
                          i, j, k, nx, ny, nz);
    un[c] = u_i;
    un[cip] = u_ip;
    vn[c] = v_j;
    vn[cjp] = v_jp;
    wn[c] = w_k;
    wn[ckp] = w_kp;
    pn[c] = pc;
}

// ---- mixed precision -------------------------------------------------------
__device__ __forceinline__ mixed_params mixed_of(const ens_member& M, double dg) {
    return mixed_params{(float)M.idx, (float)M.idy, (float)M.idz, (float)(1.0 / dg)};
}

// FP64 residual of cell tile ti into r~ and partials (sum div^2, max|div|, max|u|).
__device__ void mixed_residual_tile(const ens_args& A, int ti) {
    const int2 T = A.cell.t[ti];
    const ens_member& M = A.mem[T.x];
    const mdx_dims d = M.d;
    const double *un = M.un, *vn = M.vn, *wn = M.wn;
    float* r = M.r32;
    const double idx = M.idx, idy = M.idy, idz = M.idz;
    const fdiv32 fx = M.fx, fy = M.fy;
    double s = 0.0, m = 0.0, um = 0.0;
    for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
        const unsigned t = (unsigned)T.y + e;
        if (t >= (unsigned)d.nint) break;
        const unsigned q = fq(t, fx);
        const int i = (int)(t - q * fx.d) + 1;
        const unsigned kq = fq(q, fy);
        const int j = (int)(q - kq * fy.d) + 1;
        const int k = (int)kq + 1;
        const double dv = mixed_residual_cell<0>(d, idx, idy, idz, i, j, k, un, vn, wn, r);
        if (A.pot) M.dp[cidx(d, i, j, k)] = 0.f;   // Phi starts from 0 (its corrections were applied)
        const long long c = pidx(d, i, j, k);
        s += dv * dv;
        m = nanmax(m, fabs(dv));
        um = nanmax(um, nanmax(fabs(un[c]), nanmax(fabs(vn[c]), fabs(wn[c]))));
    }
    block_reduce3(s, m, um);
    if (threadIdx.x == 0) {
        A.part[3 * ti] = s;
        A.part[3 * ti + 1] = m;
        A.part[3 * ti + 2] = um;
    }
    __syncthreads();
}

// FP32 correction residual of cell tile ti: partials of sum e^2 and max|e|.
__device__ void corr_residual_tile(const ens_args& A, int ti) {
    const int2 T = A.cell.t[ti];
    const ens_member& M = A.mem[T.x];
    const mdx_dims d = M.d;
    const float* p32 = A.st[T.x].p32;
    const mixed_params P{p32[0], p32[1], p32[2], p32[3]};
    const fdiv32 fx = M.fx, fy = M.fy;
    double s = 0.0, m = 0.0, z = 0.0;
    for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
        const unsigned t = (unsigned)T.y + e;
        if (t >= (unsigned)d.nint) break;
        const unsigned q = fq(t, fx);
        const int i = (int)(t - q * fx.d) + 1;
        const unsigned kq = fq(q, fy);
        const int j = (int)(q - kq * fy.d) + 1;
        const int k = (int)kq + 1;
        const float ev = A.pot ? pot_split_e<0>(d, P, i, j, k, M.dp[cidx(d, i, j, k)], M.dp, M.r32, M.mu32)
                               : corr_residual_cell<0>(d, P, i, j, k, M.du, M.dv, M.dw, M.r32);
        s += (double)ev * (double)ev;
        m = nanmax(m, fabs((double)ev));
    }
    block_reduce3(s, m, z);
    if (threadIdx.x == 0) {
        A.part[3 * ti] = s;
        A.part[3 * ti + 1] = m;
        A.part[3 * ti + 2] = 0.0;
    }
    __syncthreads();
}

// One FP32 colour sweep of sweep tile ti.
__device__ __forceinline__ void sweep32_tile(const ens_args& A, int parity, int ti) {
    const int2 T = A.half.t[ti];
    const ens_member& M = A.mem[T.x];
    const mdx_dims d = M.d;
    const float* p32 = A.st[T.x].p32;
    const mixed_params P{p32[0], p32[1], p32[2], p32[3]};
    const fdiv32 fy = M.fy, fh = M.fh;
    float *du = M.du, *dv = M.dv, *dw = M.dw, *dp = M.dp;
    const float *r = M.r32, *mu32 = M.mu32, *fac32 = M.fac32;
    const unsigned nh = (unsigned)((d.nx / 2) * d.ny * d.nz);
    for (int e = threadIdx.x; e < HTILE; e += blockDim.x) {
        const unsigned t = (unsigned)T.y + e;
        if (t >= nh) break;
        const unsigned q = fq(t, fh);
        const int ni = (int)(t - q * fh.d) + 1;
        const unsigned kq = fq(q, fy);
        const int j = (int)(q - kq * fy.d) + 1;
        const int kk = (int)kq + 1;
        const int k = parity ? d.nz + 1 - kk : kk;
        const int i = 1 + ((j + k + parity) & 1) + 2 * (ni - 1);
        if (A.pot) pot_split_cell<0>(d, P, i, j, k, dp, r, mu32, fac32);
        else sweep32_cell<0>(d, P, i, j, k, du, dv, dw, dp, r, mu32, fac32);
    }
}

__device__ void sweep32_active(const ens_args& A, int parity) {
    const int* pref = A.act;
    const int total = pref[A.nmem];
    for (int vt = blockIdx.x; vt < total; vt += gridDim.x)
        sweep32_tile(A, parity, active_tile(pref, A.half_begin, A.nmem, vt).y);
}

__device__ __forceinline__ mdx_sor_params proj_params(const ens_member& M, double dg) {
    mdx_sor_params p = M.sp;
    p.idt = 1.0 / dg;
    p.dt_gamma = dg;
    return p;
}

__device__ __forceinline__ void sweep_tile(const ens_args& A, int parity, int ti) {
    const int2 T = A.half.t[ti];
    const ens_member& M = A.mem[T.x];
    const sweep_view v = make_view(M);
    const unsigned nh = (unsigned)((v.d.nx / 2) * v.d.ny * v.d.nz);
    const mdx_sor_params p = proj_params(M, dg_of(A, M));
    for (int e = threadIdx.x; e < HTILE; e += blockDim.x) {
        const unsigned t = (unsigned)T.y + e;
        if (t >= nh) break;
        sweep_cell(v, M.bc, p, parity, t);
    }
}

// One colour sweep of every member.
__device__ void sweep_all(const ens_args& A, int parity) {
    for (int ti = blockIdx.x; ti < A.half.n; ti += gridDim.x) sweep_tile(A, parity, ti);
}

// One colour sweep of the active members (compacted ranges).
__device__ void sweep_active(const ens_args& A, int parity) {
    const int* pref = A.act;
    const int total = pref[A.nmem];
    for (int vt = blockIdx.x; vt < total; vt += gridDim.x)
        sweep_tile(A, parity, active_tile(pref, A.half_begin, A.nmem, vt).y);
}

template <typename F>
__device__ void pad_tiles(const ens_args& A, F f) {
    for (int ti = blockIdx.x; ti < A.pad.n; ti += gridDim.x) {
        const int2 T = A.pad.t[ti];
        const ens_member& M = A.mem[T.x];
        for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
            const long long t = (long long)T.y + e;
            if (t >= M.d.npad) break;
            f(T.x, M, t);
        }
    }
}

template <typename F>
__device__ void cell_tiles(const ens_args& A, F f) {
    for (int ti = blockIdx.x; ti < A.cell.n; ti += gridDim.x) {
        const int2 T = A.cell.t[ti];
        const ens_member& M = A.mem[T.x];
        for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
            const unsigned t = (unsigned)T.y + e;
            if (t >= (unsigned)M.d.nint) break;
            f(T.x, M, t);
        }
    }
}

// Apply member M's increment guess at cell t (k_apply_guess of k_warm.cu).
__device__ __forceinline__ void guess_cell(const ens_member& M, double dg, unsigned t, const double* gs) {
    const mdx_dims& d = M.d;
    int i, j, k;
    cell_ijk(M, t, i, j, k);
    const int im = i == 1 ? d.nx : i - 1;
    const int km = k == 1 ? d.nz : k - 1;
    const long long c = pidx(d, i, j, k);
    const double phi = gs[t] * dg;
    const double phx = gs[qidx(d, im, j, k)] * dg;
    const double phz = gs[qidx(d, i, j, km)] * dg;
    double mu_u = 1.0, mu_v = 1.0, mu_w = 1.0;
    if (M.ibm) {
        const long long np = (long long)d.nxp * d.nyp, q = i + (long long)d.nxp * j;
        mu_u = M.mu[q];
        mu_v = M.mu[np + q];
        mu_w = M.mu[2 * np + q];
    }
    M.un[c] -= (phi - phx) * M.idx * mu_u;
    M.wn[c] -= (phi - phz) * M.idz * mu_w;
    if (M.bc.per[1] || j >= 2) {
        const int jm = j == 1 ? d.ny : j - 1;
        const double phy = gs[qidx(d, i, jm, k)] * dg;
        M.vn[c] -= (phi - phy) * M.idy * mu_v;
    }
    M.pn[c] += gs[t];
}

// MINB 1: registers for the predictor (one block of 512 per SM); MINB 2:
// 64 registers (spills in the predictor), twice the resident warps for
// the latency-bound sweeps.  The autotuner picks one.
template <int MINB>
__global__ void __launch_bounds__(MAX_THREADS, MINB) k_ens_substage(ens_args A) {
    cg::grid_group grid = cg::this_grid();
    const int s = A.substage;
    const bool warm = A.momentum && A.guess_mode != MDX_GUESS_ZERO;
    const bool meas = A.tol > 0.0;

    if (A.split != 2) {
    // ---- predictor (or u* = u for the t=0 projection) ----
    if (A.momentum) {
        for (int ti = blockIdx.x; ti < A.cell.n; ti += gridDim.x) {
            const int2 T = A.cell.t[ti];
            const ens_member& M = A.mem[T.x];
            const mdx_dims d = M.d;
            const mdx_step_params p = M.p;
            const double dg = M.dt * A.c, da = M.dt * A.a, db = M.dt * A.b;
            const fdiv32 fx = M.fx, fy = M.fy;
            const double *un = M.un, *vn = M.vn, *wn = M.wn, *pn = M.pn;
            double *us = M.us, *vs = M.vs, *ws = M.ws, *ou = M.ou, *ov = M.ov, *ow = M.ow;
            const double *cu = M.cu, *cv = M.cv, *cw = M.cw;
            const int ibm = M.ibm;
            for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
                const unsigned t = (unsigned)T.y + e;
                if (t >= (unsigned)d.nint) break;
                const unsigned r = fq(t, fx);
                const int i = (int)(t - r * fx.d) + 1;
                const unsigned kq = fq(r, fy);
                const int j = (int)(r - kq * fy.d) + 1;
                const int k = (int)kq + 1;
                if (ibm)
                    momentum_cell<true>(d, p, da, db, dg, un, vn, wn, pn, us, vs, ws, ou, ov, ow, cu, cv, cw,
                                        i + (long long)d.nxp * j, i, j, k);
                else
                    momentum_cell<false>(d, p, da, db, dg, un, vn, wn, pn, us, vs, ws, ou, ov, ow, cu, cv, cw, 0, i,
                                         j, k);
            }
        }
    } else {
        pad_tiles(A, [&](int, const ens_member& M, long long t) {
            M.us[t] = M.un[t];
            M.vs[t] = M.vn[t];
            M.ws[t] = M.wn[t];
        });
    }
    grid.sync();

    // ---- projection set-up: u <- u*, p at the start, IBM factors ----
    pad_tiles(A, [&](int, const ens_member& M, long long t) {
        M.un[t] = M.us[t];
        M.vn[t] = M.vs[t];
        M.wn[t] = M.ws[t];
        if (warm) M.p0[t] = M.pn[t];
    });
    for (int ti = blockIdx.x; ti < A.plane.n; ti += gridDim.x) {
        const int2 T = A.plane.t[ti];
        const ens_member& M = A.mem[T.x];
        if (!M.ibm) continue;
        const long long np = (long long)M.d.nxp * M.d.nyp;
        const double dg = dg_of(A, M);
        for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
            const long long t = (long long)T.y + e;
            if (t >= np) break;
            M.mu[t] = 1.0 / (1.0 + dg * M.cu[t]);
            M.mu[np + t] = 1.0 / (1.0 + dg * M.cv[t]);
            M.mu[2 * np + t] = 1.0 / (1.0 + dg * M.cw[t]);
        }
    }
    if (blockIdx.x == 0)
        for (int m = threadIdx.x; m < A.nmem; m += blockDim.x) {
            ens_state& S = A.st[m];
            S.it = 0;
            S.guessed = 0;
            S.undo = 0;
            S.status = MDX_OK;
            S.active = !meas;
            const int h = S.hist_valid;
            S.has_guess = warm && (h & (1 << s));
            S.extrap = A.guess_mode != MDX_GUESS_PREVIOUS && (h & (8 << s));
            S.lr_last = 0;
            S.g_arm = -1;
            const mixed_params P = mixed_of(A.mem[m], dg_of(A, A.mem[m]));
            S.p32[0] = P.idx;
            S.p32[1] = P.idy;
            S.p32[2] = P.idz;
            S.p32[3] = P.idt;
        }
    grid.sync();

    // ---- ||div u*||, max|u*|, target (and the FP32 factor planes) ----
    if (meas) {
        if (A.mixed)
            for (int ti = blockIdx.x; ti < A.plane.n; ti += gridDim.x) {
                const int2 T = A.plane.t[ti];
                const ens_member& M = A.mem[T.x];
                const long long np = (long long)M.d.nxp * M.d.nyp;
                const double om = A.inner_sor > 0.0 ? A.inner_sor : M.sp.sor;
                for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
                    const long long t = (long long)T.y + e;
                    if (t >= np) break;
                    mixed_tables_elem(M.d, 0, M.sp.idx2, M.sp.idy2, M.sp.idz2, om, M.ibm ? M.mu : nullptr, t, M.mu32,
                                      M.fac32);
                }
            }
        residual_tiles(A, [](int) { return true; });
        grid.sync();
        for (int m = blockIdx.x; m < A.nmem; m += gridDim.x) {
            double s2, um;
            member_sums(A, m, s2, um);
            if (threadIdx.x == 0) {
                const ens_member& M = A.mem[m];
                ens_state& S = A.st[m];
                S.r0 = sqrt(s2);
                S.umax = um;
                S.atol = A.atol < 0.0 ? 2.220446049250313e-16 * sqrt((double)M.d.nint) * um * (M.idx + M.idy + M.idz)
                                      : A.atol;
                S.target = fmax(A.tol * S.r0, S.atol);
                S.r = S.r0;
                const bool fin = isfinite(S.r0) && isfinite(um);
                S.status = fin ? (S.r0 <= S.target ? MDX_OK : MDX_NOT_CONVERGED) : MDX_ERR_NONFINITE;
                S.active = S.status == MDX_NOT_CONVERGED;
            }
            __syncthreads();
        }
        grid.sync();
    }

    // ---- warm start: the previous or extrapolated increment ----
    if (warm) {
        cell_tiles(A, [&](int m, const ens_member& M, unsigned t) {
            const ens_state& S = A.st[m];
            if (!S.has_guess) return;
            const int cur = (S.flip >> s) & 1;
            const double h1 = M.h[s][cur][t];
            M.guess[t] = S.extrap ? 2.0 * h1 - M.h[s][cur ^ 1][t] : h1;
        });
        grid.sync();
        cell_tiles(A, [&](int m, const ens_member& M, unsigned t) {
            if (A.st[m].has_guess) guess_cell(M, dg_of(A, M), t, M.guess);
        });
        grid.sync();
        if (meas) {
            residual_tiles(A, [&](int m) { return A.st[m].has_guess != 0; });
            grid.sync();
            for (int m = blockIdx.x; m < A.nmem; m += gridDim.x) {
                if (!A.st[m].has_guess) continue;
                double s2, um;
                member_sums(A, m, s2, um);
                if (threadIdx.x == 0) {
                    ens_state& S = A.st[m];
                    const double rg = sqrt(s2);
                    S.rg = rg;
                    if (!(rg < S.r0)) {
                        S.undo = 1;
                    } else {
                        S.guessed = 1;
                        S.r = rg;
                        if (S.status == MDX_NOT_CONVERGED && rg <= S.target) {
                            S.status = MDX_OK;
                            S.active = 0;
                        }
                    }
                }
                __syncthreads();
            }
            grid.sync();
            pad_tiles(A, [&](int m, const ens_member& M, long long t) {
                if (!A.st[m].undo) return;
                M.un[t] = M.us[t];
                M.vn[t] = M.vs[t];
                M.wn[t] = M.ws[t];
                M.pn[t] = M.p0[t];
            });
            grid.sync();
        } else if (blockIdx.x == 0) {
            for (int m = threadIdx.x; m < A.nmem; m += blockDim.x) A.st[m].guessed = A.st[m].has_guess;
        }
    }
    if (A.split == 1) {   // the network's inputs: the last two increments of members that kept the extrapolated guess
        if (warm && meas)
            cell_tiles(A, [&](int m, const ens_member& M, unsigned t) {
                const ens_state& S = A.st[m];
                if (!(S.guessed && S.extrap)) return;
                const int cur = (S.flip >> s) & 1;
                M.hl1[t] = M.h[s][cur][t];
                M.hl2[t] = M.h[s][cur ^ 1][t];
            });
        return;
    }
    }   // split != 2

    // ---- the learned correction (the network ran between parts 1 and 2):
    // applied like a guess on top of the extrapolated one, kept when it
    // lowers ||div u||, else undone back to the extrapolated guess ----
    if (A.split == 2 && warm && meas) {
        if (blockIdx.x == 0)
            for (int m = threadIdx.x; m < A.nmem; m += blockDim.x) {
                ens_state& S = A.st[m];
                const bool elig = A.learn_ok[m] && S.guessed && S.extrap && S.status == MDX_NOT_CONVERGED;
                int arm = elig ? 1 : 0;
                if (elig && A.gate_period > 0) {
                    arm = gate_choose(S, s, A.gate_period);
                    S.g_arm = arm;
                    if (arm == 0) S.lr_gated++;
                }
                S.lr_last = arm == 1 ? 3 : 0;
            }
        grid.sync();
        cell_tiles(A, [&](int m, const ens_member& M, unsigned t) {
            if (A.st[m].lr_last == 3) guess_cell(M, dg_of(A, M), t, M.delta);
        });
        grid.sync();
        residual_tiles(A, [&](int m) { return A.st[m].lr_last == 3; });
        grid.sync();
        for (int m = blockIdx.x; m < A.nmem; m += gridDim.x) {
            if (A.st[m].lr_last != 3) continue;
            double s2, um;
            member_sums(A, m, s2, um);
            if (threadIdx.x == 0) {
                ens_state& S = A.st[m];
                const double rl = sqrt(s2);
                if (rl < S.rg) {
                    S.lr_last = 1;
                    S.lr_corr++;
                    S.rg = rl;
                    S.r = rl;
                    if (rl <= S.target) {
                        S.status = MDX_OK;
                        S.active = 0;
                    }
                } else {
                    S.lr_last = 2;
                    S.lr_rej++;
                }
            }
            __syncthreads();
        }
        grid.sync();
        pad_tiles(A, [&](int m, const ens_member& M, long long t) {
            if (A.st[m].lr_last != 2) return;
            M.un[t] = M.us[t];
            M.vn[t] = M.vs[t];
            M.wn[t] = M.ws[t];
            M.pn[t] = M.p0[t];
        });
        grid.sync();
        cell_tiles(A, [&](int m, const ens_member& M, unsigned t) {
            if (A.st[m].lr_last == 2) guess_cell(M, dg_of(A, M), t, M.guess);
        });
        grid.sync();
    }

    // ---- red-black iterations ----
    if (!meas) {
        for (int it = 0; it < A.n_iter; ++it) {
            for (int parity = 0; parity < 2; ++parity) {
                sweep_all(A, parity);
                grid.sync();
            }
        }
    } else if (A.mixed) {
        // FP32 sweeps in FP64 defect correction (k_sor_mixed.cu's loop), each
        // member on its own: phase 0 applies its corrections (none on the first
        // round) and takes the FP64 residual r~, phase 1 sweeps until the FP32
        // correction residual meets max(target, 1e-5 r) or stagnates
        if (blockIdx.x == 0)
            for (int m = threadIdx.x; m < A.nmem; m += blockDim.x) {
                ens_state& S = A.st[m];
                S.phase = S.active ? 0 : 2;
                S.outer = 0;
                S.it = 0;
                S.active = 0;   // sweeping members
            }
        grid.sync();
        const int max_rounds = A.max_iter / max(A.check_every, 1) + 64;
        for (int round = 0; round < max_rounds; ++round) {
            if (A.pot)
                cell_tiles(A, [&](int m, const ens_member& M, unsigned t) {
                    const ens_state& S = A.st[m];
                    if (S.phase == 0 && S.outer > 0) {
                        int i, j, k;
                        cell_ijk(M, t, i, j, k);
                        pot_split_apply<0>(M.d, i, j, k, M.idx, M.idy, M.idz, 1.0 / dg_of(A, M), M.ibm ? M.mu : nullptr,
                                           M.dp, M.un, M.vn, M.wn, M.pn);
                    }
                });
            else
                pad_tiles(A, [&](int m, const ens_member& M, long long t) {
                    const ens_state& S = A.st[m];
                    if (S.phase == 0 && S.outer > 0)
                        mixed_apply_elem(M.d, t, M.un, M.vn, M.wn, M.pn, M.du, M.dv, M.dw, M.dp);
                });
            grid.sync();
            for (int ti = blockIdx.x; ti < A.cell.n; ti += gridDim.x)
                if (A.st[A.cell.t[ti].x].phase == 0) mixed_residual_tile(A, ti);
            grid.sync();
            for (int m = blockIdx.x; m < A.nmem; m += gridDim.x) {
                if (A.st[m].phase != 0) continue;
                double s2, um;
                member_sums(A, m, s2, um);
                if (threadIdx.x == 0) {
                    ens_state& S = A.st[m];
                    S.r = sqrt(s2);
                    if (!isfinite(S.r)) {
                        S.status = MDX_ERR_NONFINITE;
                        S.phase = 2;
                    } else if (S.r <= S.target) {
                        S.status = MDX_OK;
                        S.phase = 2;
                    } else if (S.outer >= 16 || S.it >= A.max_iter) {
                        S.phase = 2;   // NOT_CONVERGED
                    } else {
                        S.outer++;
                        S.inner_target = fmax(S.target, 1e-5 * S.r);
                        S.e_best = S.r;
                        S.stale = 0;
                        S.phase = 1;
                    }
                    S.active = S.phase == 1;
                }
                __syncthreads();
            }
            grid.sync();
            compact_active(A);
            grid.sync();
            if (A.act[A.nmem] == 0) break;   // every member done
            const int mm = A.check_every;
            for (int q = 0; q < mm; ++q)
                for (int parity = 0; parity < 2; ++parity) {
                    sweep32_active(A, parity);
                    grid.sync();
                }
            for (int ti = blockIdx.x; ti < A.cell.n; ti += gridDim.x)
                if (A.st[A.cell.t[ti].x].phase == 1) corr_residual_tile(A, ti);
            grid.sync();
            for (int m = blockIdx.x; m < A.nmem; m += gridDim.x) {
                if (A.st[m].phase != 1) continue;
                double s2, um;
                member_sums(A, m, s2, um);
                if (threadIdx.x == 0) {
                    ens_state& S = A.st[m];
                    const double e = sqrt(s2);
                    S.it += mm;
                    bool stop = !isfinite(e) || e <= S.inner_target || S.it >= A.max_iter;
                    if (!stop) {
                        if (e < 0.999 * S.e_best) {
                            S.e_best = e;
                            S.stale = 0;
                        } else if (++S.stale >= 20) {
                            stop = true;   // FP32 stagnation
                        }
                    }
                    if (stop) S.phase = 0;
                }
                __syncthreads();
            }
            grid.sync();
        }
        if (blockIdx.x == 0)
            for (int m = threadIdx.x; m < A.nmem; m += blockDim.x) A.st[m].active = 0;
        grid.sync();
    } else {
        compact_active(A);
        grid.sync();
        int it = 0;
        // every block reads the same compacted prefix after the barrier
        while (it < A.max_iter && A.act[A.nmem] > 0) {
            const int mm = min(A.check_every, A.max_iter - it);
            for (int q = 0; q < mm; ++q)
                for (int parity = 0; parity < 2; ++parity) {
                    sweep_active(A, parity);
                    grid.sync();
                }
            it += mm;
            residual_active(A);
            grid.sync();
            for (int m = blockIdx.x; m < A.nmem; m += gridDim.x) {
                if (!A.st[m].active) continue;
                double s2, um;
                member_sums(A, m, s2, um);
                if (threadIdx.x == 0) {
                    ens_state& S = A.st[m];
                    S.r = sqrt(s2);
                    S.it = it;
                    if (!isfinite(S.r)) {
                        S.status = MDX_ERR_NONFINITE;
                        S.active = 0;
                    } else if (S.r <= S.target) {
                        S.status = MDX_OK;
                        S.active = 0;
                    } else if (it >= A.max_iter) {
                        S.active = 0;
                    }
                }
                __syncthreads();
            }
            grid.sync();
            compact_active(A);
            grid.sync();
        }
    }

    // ---- statistics, increment history ----
    if (blockIdx.x == 0)
        for (int m = threadIdx.x; m < A.nmem; m += blockDim.x) {
            ens_state& S = A.st[m];
            const int iters = meas ? S.it : A.n_iter;   // mixed: FP32 iterations
            S.last_iters = iters;
            S.iters_total += iters;
            if (S.g_arm >= 0) {   // the gate's sample
                if (S.status == MDX_OK) {
                    double& e = S.g_ema[s][S.g_arm];
                    e = S.g_n[s][S.g_arm] > 0 ? 0.5 * e + 0.5 * (double)iters : (double)iters;
                    S.g_n[s][S.g_arm]++;
                }
                S.g_arm = -1;
            }
            S.last_residual = meas ? (S.r0 > 0.0 ? S.r / S.r0 : 0.0) : 0.0;
            if (warm) {
                S.flip ^= 1 << s;
                if (S.hist_valid & (1 << s)) S.hist_valid |= 8 << s;
                else S.hist_valid &= ~(8 << s);
                S.hist_valid |= 1 << s;
            }
        }
    grid.sync();
    if (warm) {
        cell_tiles(A, [&](int m, const ens_member& M, unsigned t) {
            const int cur = (A.st[m].flip >> s) & 1;
            int i, j, k;
            cell_ijk(M, t, i, j, k);
            const long long c = pidx(M.d, i, j, k);
            M.h[s][cur][t] = M.pn[c] - M.p0[c];
        });
        grid.sync();
    }

    // ---- boundary conditions, three ordered phases ----
    for (int ti = blockIdx.x; ti < A.bcy.n; ti += gridDim.x) {
        const int2 T = A.bcy.t[ti];
        const ens_member& M = A.mem[T.x];
        const mdx_four f{M.un, M.vn, M.wn, M.pn};
        for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
            const unsigned t = (unsigned)T.y + e;
            if (t >= (unsigned)(M.d.nx * M.d.nz)) break;
            const unsigned q = fq(t, M.fx);
            bcrb_y_col(M.d, M.bc, M.p.dy, f, (int)(t - q * M.fx.d) + 1, (int)q + 1);
        }
    }
    grid.sync();
    for (int ti = blockIdx.x; ti < A.bcx.n; ti += gridDim.x) {
        const int2 T = A.bcx.t[ti];
        const ens_member& M = A.mem[T.x];
        const mdx_four f{M.un, M.vn, M.wn, M.pn};
        for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
            const unsigned t = (unsigned)T.y + e;
            if (t >= (unsigned)(M.d.ny * M.d.nz)) break;
            const unsigned q = fq(t, M.fy);
            bcrb_x_col(M.d, M.bc, M.p.dx, f, (int)(t - q * M.fy.d) + 1, (int)q + 1);
        }
    }
    grid.sync();
    for (int ti = blockIdx.x; ti < A.bcz.n; ti += gridDim.x) {
        const int2 T = A.bcz.t[ti];
        const ens_member& M = A.mem[T.x];
        const mdx_four f{M.un, M.vn, M.wn, M.pn};
        for (int e = threadIdx.x; e < ETILE; e += blockDim.x) {
            const unsigned t = (unsigned)T.y + e;
            if (t >= (unsigned)(M.d.nx * M.d.ny)) break;
            const unsigned q = fq(t, M.fx);
            bcrb_z_col(M.d, M.bc, M.p.dz, f, (int)(t - q * M.fx.d) + 1, (int)q + 1);
        }
    }
}

// Seeded channel initial condition of one member (k_channel_ic of k_step.cu).
__global__ void k_ens_ic(mdx_dims d, double dy, uint64_t seed, double amp_u, double amp_vw,
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

void rk_coeffs(double* a, double* b, double* c) {   // src/modules/step.f90:21-23
    a[0] = 64.0 / 120.0; a[1] = 50.0 / 120.0; a[2] = 90.0 / 120.0;
    b[0] = 0.0;          b[1] = -34.0 / 120.0; b[2] = -50.0 / 120.0;
    c[0] = 64.0 / 120.0; c[1] = 16.0 / 120.0; c[2] = 40.0 / 120.0;
}

}  // namespace

struct mdx_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int n = 0;
    std::vector<mdx_member_t> members;
    mdx_solver_opts_t opts{};
    int guess_mode = MDX_GUESS_ZERO;
    std::vector<ens_member> hm;
    ens_member* dm = nullptr;
    ens_state* dst = nullptr;
    std::vector<int2> tiles[7];
    int2* dtiles[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    std::vector<int> cell_begin, half_begin;
    int* dcell_begin = nullptr;
    int* dhalf_begin = nullptr;
    int* dact = nullptr;
    double* part = nullptr;
    int threads = 256, blocks_per_sm = 0, grid = 0, variant = 0;
    bool use_graph = true, graph_ok = true;
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::vector<void*> allocs;
    std::vector<std::pair<void*, size_t>> state_arrays;   // the state a snapshot copies
    std::vector<char*> shadow;
    long long launches = 0;
    long long graph_launches = 3;
    double last_step_ms = 0.0;
    // learned warm start: one network context sized for the member with the
    // most cells (its activations fit every member), its per-member scales
    // and the flags its passes write
    mdx_ctx_t* net = nullptr;
    double* net_scal = nullptr;      // 4 per member
    int* learn_ok = nullptr;         // per member
    int gate_period = 0;             // of the loaded network's options
};

namespace {

int efail(mdx_ensemble_t* E, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (E) E->err = buf;
    return code;
}
#define ENS_CUDA(E, call)                                                                                  \
    do {                                                                                                   \
        cudaError_t e__ = (call);                                                                          \
        if (e__ != cudaSuccess)                                                                            \
            return efail((E), MDX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e__), __FILE__, \
                         __LINE__);                                                                        \
    } while (0)

template <typename T>
int ealloc(mdx_ensemble_t* E, T** p, size_t n, bool zero = true, bool state = false) {
    ENS_CUDA(E, cudaMalloc(p, sizeof(T) * std::max<size_t>(n, 1)));
    E->allocs.push_back(*p);
    if (zero) ENS_CUDA(E, cudaMemsetAsync(*p, 0, sizeof(T) * std::max<size_t>(n, 1), E->stream));
    if (state) E->state_arrays.push_back({(void*)*p, sizeof(T) * n});
    return MDX_OK;
}

void free_graph(mdx_ensemble_t* E) {
    if (E->graph) cudaGraphExecDestroy(E->graph);
    E->graph = nullptr;
}

const void* kernel_of(int variant) {
    return variant ? (const void*)k_ens_substage<2> : (const void*)k_ens_substage<1>;
}

int grid_for(mdx_ensemble_t* E, int variant, int threads, int bps, int* grid) {
    int occ = 0;
    ENS_CUDA(E, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel_of(variant), threads, 0));
    int sms = 0;
    ENS_CUDA(E, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E->device));
    if (occ < 1) return efail(E, MDX_ERR_ARG, "ensemble kernel does not fit %d threads per block", threads);
    const int b = (bps <= 0) ? occ : std::min(bps, occ);
    *grid = b * sms;
    return MDX_OK;
}

ens_args make_args(mdx_ensemble_t* E, int s, int momentum) {
    double a[3], b[3], c[3];
    rk_coeffs(a, b, c);
    ens_args A{};
    A.mem = E->dm;
    A.st = E->dst;
    A.nmem = E->n;
    ens_list* L[7] = {&A.cell, &A.half, &A.pad, &A.plane, &A.bcy, &A.bcx, &A.bcz};
    for (int q = 0; q < 7; ++q) *L[q] = ens_list{E->dtiles[q], (int)E->tiles[q].size()};
    A.cell_begin = E->dcell_begin;
    A.half_begin = E->dhalf_begin;
    A.act = E->dact;
    A.part = E->part;
    A.a = a[s];
    A.b = b[s];
    A.c = c[s];
    A.substage = s;
    A.momentum = momentum;
    A.guess_mode = momentum ? E->guess_mode : MDX_GUESS_ZERO;
    A.n_iter = E->opts.n_iter;
    A.max_iter = E->opts.max_iter;
    A.check_every = E->opts.check_every;
    A.tol = E->opts.tol;
    A.atol = E->opts.atol;
    A.mixed = E->opts.precision == MDX_PREC_MIXED && E->opts.tol > 0.0;
    A.pot = A.mixed && E->opts.inner_form == 2;
    A.inner_sor = E->opts.inner_sor;
    A.split = 0;
    A.learn_ok = E->learn_ok;
    A.gate_period = E->gate_period;
    return A;
}

int launch_substage(mdx_ensemble_t* E, int s, int momentum, int variant, int threads, int grid, int split = 0) {
    ens_args A = make_args(E, s, momentum);
    A.split = split;
    void* args[] = {&A};
    ENS_CUDA(E, cudaLaunchCooperativeKernel(kernel_of(variant), dim3(grid), dim3(threads), args, 0, E->stream));
    E->launches++;
    return MDX_OK;
}

bool learned_on(const mdx_ensemble_t* E) { return E->guess_mode == MDX_GUESS_LEARNED && E->net && E->opts.tol > 0.0; }

// The network for every member, one after another on the ensemble's stream:
// each pass reads the member's velocity after its extrapolated guess and its
// last two increments (copied by part 1), and writes its correction and a
// flag; part 2 uses them for the members that kept the extrapolated guess.
int net_pass(mdx_ensemble_t* E, int s) {
    double a[3], b[3], c[3];
    rk_coeffs(a, b, c);
    const long long l0 = E->net->launches;
    for (int m = 0; m < E->n; ++m) {
        const ens_member& M = E->hm[m];
        const int rc = mdx_unet_member_delta(E->net, M.d, M.p.dx, M.p.dy, M.p.dz, M.p.ire, M.dt * c[s], M.un, M.vn, M.wn, M.hl1,
                                             M.hl2, M.ibm ? M.mu : nullptr, M.delta, E->net_scal + 4 * m,
                                             E->learn_ok + m);
        if (rc != MDX_OK) return efail(E, rc, "member %d network pass: %s", m, mdx_last_error(E->net));
    }
    E->launches += E->net->launches - l0;
    return MDX_OK;
}

int step_eager(mdx_ensemble_t* E, int variant, int threads, int grid) {
    if (learned_on(E)) {
        for (int s = 0; s < 3; ++s) {
            MDX_TRY(launch_substage(E, s, 1, variant, threads, grid, 1));
            MDX_TRY(net_pass(E, s));
            MDX_TRY(launch_substage(E, s, 1, variant, threads, grid, 2));
        }
        return MDX_OK;
    }
    for (int s = 0; s < 3; ++s) MDX_TRY(launch_substage(E, s, 1, variant, threads, grid));
    return MDX_OK;
}

int ensure_grid(mdx_ensemble_t* E) {
    if (E->grid > 0) return MDX_OK;
    return grid_for(E, E->variant, E->threads, E->blocks_per_sm, &E->grid);
}

int read_stats(mdx_ensemble_t* E, std::vector<ens_state>& h) {
    h.resize(E->n);
    ENS_CUDA(E, cudaMemcpyAsync(h.data(), E->dst, sizeof(ens_state) * E->n, cudaMemcpyDeviceToHost, E->stream));
    ENS_CUDA(E, cudaStreamSynchronize(E->stream));
    return MDX_OK;
}

int snapshot(mdx_ensemble_t* E, bool restore) {
    if (E->shadow.empty()) {
        for (auto& a : E->state_arrays) {
            char* p = nullptr;
            ENS_CUDA(E, cudaMalloc(&p, std::max<size_t>(a.second, 1)));
            E->shadow.push_back(p);
        }
    }
    for (size_t q = 0; q < E->state_arrays.size(); ++q) {
        void* src = restore ? (void*)E->shadow[q] : E->state_arrays[q].first;
        void* dst = restore ? E->state_arrays[q].first : (void*)E->shadow[q];
        ENS_CUDA(E, cudaMemcpyAsync(dst, src, E->state_arrays[q].second, cudaMemcpyDeviceToDevice, E->stream));
    }
    return MDX_OK;
}

std::string tune_key(const mdx_ensemble_t* E) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        h ^= v;
        h *= 1099511628211ull;
    };
    for (const auto& m : E->members) {
        mix((uint64_t)m.nx);
        mix((uint64_t)m.ny);
        mix((uint64_t)m.nz);
        mix(m.amp > 0.0 ? 1 : 0);
    }
    mix((uint64_t)E->guess_mode);
    mix((uint64_t)(E->opts.tol > 0.0));
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, E->device);
    char hex[17];
    snprintf(hex, sizeof(hex), "%016llx", (unsigned long long)h);
    return std::string(prop.name) + "/" + hex;
}

// The cache is a JSON object {"<key>": {"threads": T, "blocks_per_sm": B, "low_regs": R, "ms": M}, ...}.
bool cache_lookup(const char* path, const std::string& key, int* threads, int* bps, int* low_regs) {
    if (!path) return false;
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    std::string s;
    char buf[4096];
    size_t r;
    while ((r = fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, r);
    fclose(f);
    const std::string q = "\"" + key + "\"";
    const size_t at = s.find(q);
    if (at == std::string::npos) return false;
    const size_t t = s.find("\"threads\":", at), b = s.find("\"blocks_per_sm\":", at),
                 lr = s.find("\"low_regs\":", at);
    if (t == std::string::npos || b == std::string::npos || lr == std::string::npos) return false;
    *threads = atoi(s.c_str() + t + 10);
    *bps = atoi(s.c_str() + b + 16);
    *low_regs = atoi(s.c_str() + lr + 11);
    return *threads > 0 && *threads <= MAX_THREADS && *threads % 32 == 0 && *bps > 0;
}

void cache_store(const char* path, const std::string& key, int threads, int bps, int low_regs, double ms) {
    if (!path) return;
    std::string s;
    if (FILE* f = fopen(path, "rb")) {
        char buf[4096];
        size_t r;
        while ((r = fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, r);
        fclose(f);
    }
    char entry[512];
    snprintf(entry, sizeof(entry), "\"%s\": {\"threads\": %d, \"blocks_per_sm\": %d, \"low_regs\": %d, \"ms\": %.6f}",
             key.c_str(), threads, bps, low_regs, ms);
    const size_t close = s.rfind('}');
    if (s.empty() || close == std::string::npos || s.find('{') == std::string::npos) {
        s = std::string("{\n  ") + entry + "\n}\n";
    } else {
        const bool empty = s.find('"') == std::string::npos;
        s = s.substr(0, close);
        while (!s.empty() && (s.back() == '\n' || s.back() == ' ')) s.pop_back();
        s += empty ? std::string("\n  ") + entry + "\n}\n" : std::string(",\n  ") + entry + "\n}\n";
    }
    if (FILE* f = fopen(path, "wb")) {
        fwrite(s.data(), 1, s.size(), f);
        fclose(f);
    }
}

}  // namespace

extern "C" {

void mdx_default_member(mdx_member_t* m) {
    if (!m) return;
    std::memset(m, 0, sizeof(*m));
    m->nx = 64;
    m->ny = 64;
    m->nz = 64;
    m->lx = 2.0 * 3.141592653589793;
    m->ly = 2.25;
    m->lz = 3.141592653589793;
    m->re = 3000.0;
    m->dt = 1e-3;
    m->amp = 0.05;
    m->seed = 20261203ull;
}

const char* mdx_ensemble_last_error(const mdx_ensemble_t* E) { return E ? E->err.c_str() : "null ensemble"; }

int mdx_ensemble_destroy(mdx_ensemble_t* E) {
    if (!E) return MDX_OK;
    cudaSetDevice(E->device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    free_graph(E);
    if (E->net) mdx_destroy(E->net);
    for (void* p : E->allocs) cudaFree(p);
    for (char* p : E->shadow) cudaFree(p);
    for (int q = 0; q < 7; ++q) cudaFree(E->dtiles[q]);
    cudaFree(E->dm);
    cudaFree(E->dst);
    cudaFree(E->dcell_begin);
    cudaFree(E->dhalf_begin);
    cudaFree(E->dact);
    cudaFree(E->part);
    for (auto& e : E->ev)
        if (e) cudaEventDestroy(e);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
    return MDX_OK;
}

int mdx_ensemble_create(int device, int n, const mdx_member_t* members, const mdx_solver_opts_t* opts,
                        mdx_ensemble_t** out) {
    if (!out || !members || n <= 0) return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_ensemble_create: bad arguments");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return mdx_fail(nullptr, MDX_ERR_NO_DEVICE, "mdx_ensemble_create: no CUDA device %d", device);
    mdx_solver_opts_t o;
    if (opts) o = *opts;
    else mdx_default_solver_opts(&o);
    if (o.solver != MDX_SOLVER_REDBLACK) return mdx_fail(nullptr, MDX_ERR_ARG, "the ensemble runs the red-black solver");
    if (o.precision != MDX_PREC_FP64 && o.precision != MDX_PREC_MIXED)
        return mdx_fail(nullptr, MDX_ERR_ARG, "unknown precision %d", o.precision);
    if (o.check_every < 1) o.check_every = 1;
    if (o.max_iter < 1) o.max_iter = 1;
    if (o.n_iter < 0) return mdx_fail(nullptr, MDX_ERR_ARG, "n_iter must be >= 0");
    for (int m = 0; m < n; ++m) {
        const mdx_member_t& q = members[m];
        if (q.nx < 4 || q.ny < 4 || q.nz < 4 || q.nx % 2 || q.nz % 2 || !(q.lx > 0) || !(q.ly > 2.0) || !(q.lz > 0) ||
            !(q.re > 0) || !(q.dt > 0) || q.amp < 0.0)
            return mdx_fail(nullptr, MDX_ERR_ARG, "member %d: bad grid or parameters", m);
        if ((long long)(q.nx / 2) * q.ny * q.nz >= (1LL << 31) / 2)
            return mdx_fail(nullptr, MDX_ERR_ARG, "member %d too large", m);
    }
    cudaSetDevice(device);
    mdx_ensemble_t* E = new mdx_ensemble_t();
    E->device = device;
    E->n = n;
    E->members.assign(members, members + n);
    E->opts = o;
    int rc = MDX_OK;
    auto fail = [&](int code) {
        std::string msg = E->err;
        mdx_ensemble_destroy(E);
        return mdx_fail(nullptr, code, "%s", msg.c_str());
    };
    if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete E;
        return mdx_fail(nullptr, MDX_ERR_CUDA, "stream creation failed");
    }
    E->hm.resize(n);
    std::vector<ens_state> hs(n);
    std::memset(hs.data(), 0, sizeof(ens_state) * n);
    mdx_bc_t bc;
    mdx_default_bc(&bc);
    bc.is_periodic[1] = 0;   // channel: no-slip walls, Neumann pressure (all values 0)
    for (int t = 0; t < 24; ++t) bc.bc_type[t] = 0;
    bc.bc_type[1 + 3 * (0 + 2 * 0)] = 1;
    bc.bc_type[1 + 3 * (1 + 2 * 0)] = 1;
    for (int m = 0; m < n && rc == MDX_OK; ++m) {
        const mdx_member_t& q = members[m];
        ens_member& M = E->hm[m];
        std::memset(&M, 0, sizeof(M));
        mdx_grid_t g;
        mdx_default_grid(&g);
        g.nx = q.nx; g.ny = q.ny; g.nz = q.nz;
        g.lx = q.lx; g.ly = q.ly; g.lz = q.lz;
        g.re = q.re; g.dt = q.dt;
        g.forcing_x = 2.0 / q.re; g.forcing_y = 0.0; g.forcing_z = 0.0;
        mdx_finalize_grid(&g);
        mdx_dims& d = M.d;
        d.nx = q.nx; d.ny = q.ny; d.nz = q.nz;
        d.nxp = q.nx + 2; d.nyp = q.ny + 2; d.nzp = q.nz + 2;
        d.nxh = q.nx / 2 + 1;
        d.hs = split_stride(q.nx);
        d.npad = (long long)d.nxp * d.nyp * d.nzp;
        d.nint = (long long)q.nx * q.ny * q.nz;
        d.nspec = 0;
        // the step parameters of mdx_make_params and the sweep parameters of sor_params
        mdx_step_params& p = M.p;
        p.dx = g.dx; p.dy = g.dy; p.dz = g.dz;
        const double dx2 = g.dx * g.dx, dy2 = g.dy * g.dy, dz2 = g.dz * g.dz;
        p.idx = 1.0 / g.dx; p.idy = 1.0 / g.dy; p.idz = 1.0 / g.dz;
        p.idx2 = 1.0 / dx2; p.idy2 = 1.0 / dy2; p.idz2 = 1.0 / dz2;
        p.ire = 1.0 / g.re;
        p.fx = g.forcing_x; p.fy = g.forcing_y; p.fz = g.forcing_z;
        p.nx0 = 1; p.ny0 = 2; p.nz0 = 1;
        mdx_sor_params& sp = M.sp;
        sp.dx = g.dx; sp.dy = g.dy; sp.dz = g.dz;
        sp.idx = 1.0 / g.dx; sp.idy = 1.0 / g.dy; sp.idz = 1.0 / g.dz;
        sp.idx2 = sp.idx * sp.idx; sp.idy2 = sp.idy * sp.idy; sp.idz2 = sp.idz * sp.idz;
        sp.sor = o.sor;
        M.idx = 1.0 / g.dx; M.idy = 1.0 / g.dy; M.idz = 1.0 / g.dz;
        for (int t = 0; t < 3; ++t) M.bc.per[t] = bc.is_periodic[t] ? 1 : 0;
        for (int t = 0; t < 24; ++t) { M.bc.type[t] = bc.bc_type[t]; M.bc.value[t] = bc.bc_value[t]; }
        M.dt = q.dt;
        M.fx = make_fdiv((unsigned)q.nx);
        M.fy = make_fdiv((unsigned)q.ny);
        M.fh = make_fdiv((unsigned)(q.nx / 2));
        const size_t np = (size_t)d.npad, ni = (size_t)d.nint, pl = (size_t)d.nxp * d.nyp;
        double** pads[7] = {&M.un, &M.vn, &M.wn, &M.pn, &M.us, &M.vs, &M.ws};
        for (int t = 0; t < 7 && rc == MDX_OK; ++t) rc = ealloc(E, pads[t], np, true, t < 4);
        double** ints[3] = {&M.ou, &M.ov, &M.ow};
        for (int t = 0; t < 3 && rc == MDX_OK; ++t) rc = ealloc(E, ints[t], ni, true, true);
        if (rc == MDX_OK) rc = ealloc(E, &M.p0, np);
        if (rc == MDX_OK) rc = ealloc(E, &M.guess, ni);
        for (int s = 0; s < 3 && rc == MDX_OK; ++s)
            for (int b = 0; b < 2 && rc == MDX_OK; ++b) rc = ealloc(E, &M.h[s][b], ni, true, true);
        if (o.precision == MDX_PREC_MIXED) {   // colour-split FP32 arrays, factor planes
            const size_t ns = (size_t)split_elems(d), ps = (size_t)split_plane_elems(d);
            float** f32[5] = {&M.du, &M.dv, &M.dw, &M.dp, &M.r32};
            for (int t = 0; t < 5 && rc == MDX_OK; ++t) rc = ealloc(E, f32[t], ns, true, t < 4);
            if (rc == MDX_OK) rc = ealloc(E, &M.mu32, 3 * ps, true);
            if (rc == MDX_OK) rc = ealloc(E, &M.fac32, ps, true);
        }
        if (rc == MDX_OK && q.amp > 0.0) {
            // wavy walls y0 + A sin(2 pi x / (Lx/2)) and y0 + 2 + ..., y0 = (Ly - 2)/2;
            // one z plane of each component, generated on the device (the walls
            // depend on x and y only)
            mdx_ibm_geom_t geo{};
            geo.geometry = 1;
            geo.n_wave_x = 1;
            geo.amp = q.amp;
            geo.phase = 0.0;
            geo.lambda = q.lx / 2.0;
            geo.y0 = (q.ly - 2.0) / 2.0;
            geo.height = 2.0;
            double** planes[3] = {&M.cu, &M.cv, &M.cw};
            for (int t = 0; t < 3 && rc == MDX_OK; ++t) {
                rc = ealloc(E, planes[t], pl, false);
                if (rc == MDX_OK && mdx_ibm_coeff_launch(&g, &geo, *planes[t], t == 0, t == 1, t == 2, 1, E->stream) != MDX_OK)
                    rc = efail(E, MDX_ERR_CUDA, "member %d: IBM coefficient generation failed", m);
            }
            if (rc == MDX_OK) rc = ealloc(E, &M.mu, 3 * pl);
            M.ibm = 1;
        }
    }
    if (rc != MDX_OK) return fail(rc);
    // tile lists, members back to back
    E->cell_begin.assign(n + 1, 0);
    E->half_begin.assign(n + 1, 0);
    for (int m = 0; m < n; ++m) {
        const mdx_dims& d = E->hm[m].d;
        const long long cnt[7] = {d.nint, (long long)(d.nx / 2) * d.ny * d.nz, d.npad, (long long)d.nxp * d.nyp,
                                  (long long)d.nx * d.nz, (long long)d.ny * d.nz, (long long)d.nx * d.ny};
        E->cell_begin[m] = (int)E->tiles[0].size();
        E->half_begin[m] = (int)E->tiles[1].size();
        for (int q = 0; q < 7; ++q) {
            const int step = q == 1 ? HTILE : ETILE;   // list 1: the sweep tiles
            for (long long s0 = 0; s0 < cnt[q]; s0 += step) E->tiles[q].push_back(make_int2(m, (int)s0));
        }
    }
    E->cell_begin[n] = (int)E->tiles[0].size();
    E->half_begin[n] = (int)E->tiles[1].size();
    for (int q = 0; q < 7 && rc == MDX_OK; ++q) {
        if (cudaMalloc(&E->dtiles[q], sizeof(int2) * std::max<size_t>(E->tiles[q].size(), 1)) != cudaSuccess ||
            cudaMemcpy(E->dtiles[q], E->tiles[q].data(), sizeof(int2) * E->tiles[q].size(), cudaMemcpyHostToDevice) !=
                cudaSuccess)
            rc = efail(E, MDX_ERR_CUDA, "tile list allocation failed");
    }
    if (rc == MDX_OK &&
        (cudaMalloc(&E->dcell_begin, sizeof(int) * (n + 1)) != cudaSuccess ||
         cudaMemcpy(E->dcell_begin, E->cell_begin.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMalloc(&E->dhalf_begin, sizeof(int) * (n + 1)) != cudaSuccess ||
         cudaMemcpy(E->dhalf_begin, E->half_begin.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMalloc(&E->dact, sizeof(int) * 2 * (n + 1)) != cudaSuccess ||
         cudaMemset(E->dact, 0, sizeof(int) * 2 * (n + 1)) != cudaSuccess ||
         cudaMalloc(&E->part, sizeof(double) * 3 * std::max<size_t>(E->tiles[0].size(), 1)) != cudaSuccess ||
         cudaMalloc(&E->dm, sizeof(ens_member) * n) != cudaSuccess ||
         cudaMemcpy(E->dm, E->hm.data(), sizeof(ens_member) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMalloc(&E->dst, sizeof(ens_state) * n) != cudaSuccess ||
         cudaMemcpy(E->dst, hs.data(), sizeof(ens_state) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaEventCreate(&E->ev[0]) != cudaSuccess || cudaEventCreate(&E->ev[1]) != cudaSuccess))
        rc = efail(E, MDX_ERR_CUDA, "ensemble allocation failed");
    if (rc == MDX_OK) E->state_arrays.push_back({(void*)E->dst, sizeof(ens_state) * n});
    if (rc == MDX_OK && cudaStreamSynchronize(E->stream) != cudaSuccess) rc = efail(E, MDX_ERR_CUDA, "set-up failed");
    if (rc != MDX_OK) return fail(rc);
    *out = E;
    return MDX_OK;
}

int mdx_ensemble_set_guess(mdx_ensemble_t* E, int mode) {
    if (!E) return MDX_ERR_ARG;
    if (mode != MDX_GUESS_ZERO && mode != MDX_GUESS_PREVIOUS && mode != MDX_GUESS_EXTRAPOLATED &&
        mode != MDX_GUESS_LEARNED)
        return efail(E, MDX_ERR_ARG, "ensemble guess mode %d: zero, previous, extrapolated or learned", mode);
    if (mode == MDX_GUESS_LEARNED && !E->net)
        return efail(E, MDX_ERR_STATE, "learned guess: load a network first (mdx_ensemble_unet_load)");
    if (mode == MDX_GUESS_LEARNED && !(E->opts.tol > 0.0))
        return efail(E, MDX_ERR_ARG, "learned guess: needs a residual tolerance (tol > 0)");
    E->guess_mode = mode;
    free_graph(E);
    return MDX_OK;
}

int mdx_ensemble_ic(mdx_ensemble_t* E) {
    if (!E) return MDX_ERR_ARG;
    ENS_CUDA(E, cudaSetDevice(E->device));
    MDX_TRY(ensure_grid(E));
    const double pi = 3.141592653589793;
    std::vector<double*> ycs;
    for (int m = 0; m < E->n; ++m) {
        const mdx_member_t& q = E->members[m];
        const ens_member& M = E->hm[m];
        const mdx_dims& d = M.d;
        const size_t bytes = sizeof(double) * d.npad;
        for (double* p : {M.un, M.vn, M.wn, M.pn, M.us, M.vs, M.ws}) ENS_CUDA(E, cudaMemsetAsync(p, 0, bytes, E->stream));
        for (double* p : {M.ou, M.ov, M.ow}) ENS_CUDA(E, cudaMemsetAsync(p, 0, sizeof(double) * d.nint, E->stream));
        const double y0 = (q.ly - 2.0) / 2.0, lam = q.lx / 2.0;
        std::vector<double> yc(d.nx);
        for (int i = 1; i <= d.nx; ++i) {
            const double x = (double)(i - 1) * M.p.dx;
            double v = y0 + 1.0;
            if (q.amp != 0.0) v = v + q.amp * std::sin(2.0 * pi * x / lam);
            yc[i - 1] = v;
        }
        double* dyc = nullptr;
        ENS_CUDA(E, cudaMalloc(&dyc, sizeof(double) * d.nx));
        ycs.push_back(dyc);
        ENS_CUDA(E, cudaMemcpyAsync(dyc, yc.data(), sizeof(double) * d.nx, cudaMemcpyHostToDevice, E->stream));
        k_ens_ic<<<(unsigned)((d.nint + 255) / 256), 256, 0, E->stream>>>(d, M.p.dy, q.seed, 0.1, 0.01, dyc, M.un,
                                                                           M.vn, M.wn);
        ENS_CUDA(E, cudaGetLastError());
        ENS_CUDA(E, cudaStreamSynchronize(E->stream));   // yc must outlive the copy
    }
    for (double* p : ycs) cudaFree(p);
    std::vector<ens_state> hs(E->n);
    std::memset(hs.data(), 0, sizeof(ens_state) * E->n);
    ENS_CUDA(E, cudaMemcpyAsync(E->dst, hs.data(), sizeof(ens_state) * E->n, cudaMemcpyHostToDevice, E->stream));
    MDX_TRY(launch_substage(E, 0, 0, E->variant, E->threads, E->grid));   // the t=0 projection, dt_gamma = 1
    for (int m = 0; m < E->n; ++m)
        ENS_CUDA(E, cudaMemsetAsync(E->hm[m].pn, 0, sizeof(double) * E->hm[m].d.npad, E->stream));
    std::vector<ens_state> after;
    MDX_TRY(read_stats(E, after));
    for (int m = 0; m < E->n; ++m) {
        after[m].hist_valid = 0;
        after[m].flip = 0;
        after[m].iters_total = 0;
        if (after[m].status != MDX_OK)
            return efail(E, after[m].status, "member %d: t=0 projection ended with status %d", m, after[m].status);
    }
    ENS_CUDA(E, cudaMemcpyAsync(E->dst, after.data(), sizeof(ens_state) * E->n, cudaMemcpyHostToDevice, E->stream));
    ENS_CUDA(E, cudaStreamSynchronize(E->stream));
    return MDX_OK;
}

int mdx_ensemble_unet_load(mdx_ensemble_t* E, const mdx_unet_opts_t* opts, const float* params, long long n,
                           double out_scale) {
    if (!E || !params) return MDX_ERR_ARG;
    ENS_CUDA(E, cudaSetDevice(E->device));
    ENS_CUDA(E, cudaStreamSynchronize(E->stream));
    free_graph(E);
    // the member with the most cells gives the network's grid (sizes are
    // multiples of 16, so it has the most cells at every level too)
    int big = 0;
    for (int m = 1; m < E->n; ++m)
        if (E->hm[m].d.nint > E->hm[big].d.nint) big = m;
    for (int m = 0; m < E->n; ++m) {
        const mdx_dims& d = E->hm[m].d;
        if (d.nx % 8 || d.ny % 8 || d.nz % 8)
            return efail(E, MDX_ERR_ARG, "learned guess: member %d sizes must be multiples of 8", m);
    }
    if (!E->net) {
        const mdx_member_t& q = E->members[big];
        mdx_grid_t g;
        mdx_default_grid(&g);
        g.nx = q.nx;
        g.ny = q.ny;
        g.nz = q.nz;
        g.lx = q.lx;
        g.ly = q.ly;
        g.lz = q.lz;
        g.dx = q.lx / q.nx;
        g.dy = q.ly / q.ny;
        g.dz = q.lz / q.nz;
        g.re = q.re;
        g.dt = q.dt;
        mdx_bc_t bc;
        mdx_default_bc(&bc);
        bc.is_periodic[1] = E->hm[big].bc.per[1];
        mdx_ctx_t* net = nullptr;
        int rc = mdx_create(E->device, &g, &bc, &net);
        if (rc != MDX_OK) return efail(E, rc, "learned guess: network context: %s", mdx_last_error(nullptr));
        E->net = net;
        rc = mdx_enter_field_data(net, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                  nullptr);
        if (rc == MDX_OK) rc = mdx_set_stream(net, (void*)E->stream);
        if (rc == MDX_OK) rc = mdx_unet_create(net, opts);
        if (rc != MDX_OK) return efail(E, rc, "learned guess: network: %s", mdx_last_error(net));
        MDX_TRY(ealloc(E, &E->net_scal, 4 * (size_t)E->n));
        MDX_TRY(ealloc(E, &E->learn_ok, (size_t)E->n));
        for (int m = 0; m < E->n; ++m) {
            ens_member& M = E->hm[m];
            const size_t ni = (size_t)M.d.nint;
            MDX_TRY(ealloc(E, &M.hl1, ni));
            MDX_TRY(ealloc(E, &M.hl2, ni));
            MDX_TRY(ealloc(E, &M.delta, ni));
        }
        ENS_CUDA(E, cudaMemcpy(E->dm, E->hm.data(), sizeof(ens_member) * E->n, cudaMemcpyHostToDevice));
    }
    if (opts && opts->gate_period < 0) return efail(E, MDX_ERR_ARG, "learned guess: gate_period < 0");
    E->gate_period = opts ? opts->gate_period : 0;
    int rc = mdx_unet_set_params(E->net, params, n);
    if (rc == MDX_OK) rc = mdx_unet_set_out_scale(E->net, out_scale);
    if (rc != MDX_OK) return efail(E, rc, "learned guess: parameters: %s", mdx_last_error(E->net));
    ENS_CUDA(E, cudaStreamSynchronize(E->stream));
    return MDX_OK;
}

int mdx_ensemble_unet_stats(mdx_ensemble_t* E, long long* corrections, long long* rejected, long long* gated) {
    if (!E) return MDX_ERR_ARG;
    std::vector<ens_state> h;
    MDX_TRY(read_stats(E, h));
    long long c = 0, r = 0, q = 0;
    for (const auto& S : h) {
        c += S.lr_corr;
        r += S.lr_rej;
        q += S.lr_gated;
    }
    if (corrections) *corrections = c;
    if (rejected) *rejected = r;
    if (gated) *gated = q;
    return MDX_OK;
}

int mdx_ensemble_config(mdx_ensemble_t* E, int threads, int blocks_per_sm, int low_regs) {
    if (!E) return MDX_ERR_ARG;
    const int variant = low_regs ? 1 : 0;
    if (threads < 32 || threads > MAX_THREADS || threads % 32)
        return efail(E, MDX_ERR_ARG, "threads per block must be a multiple of 32 up to %d", MAX_THREADS);
    int grid = 0;
    MDX_TRY(grid_for(E, variant, threads, blocks_per_sm, &grid));
    E->variant = variant;
    E->threads = threads;
    E->blocks_per_sm = blocks_per_sm;
    E->grid = grid;
    free_graph(E);
    return MDX_OK;
}

int mdx_ensemble_use_graph(mdx_ensemble_t* E, int on) {
    if (!E) return MDX_ERR_ARG;
    E->use_graph = on != 0;
    free_graph(E);
    return MDX_OK;
}

int mdx_ensemble_step(mdx_ensemble_t* E, int nsteps, long long* total_iters) {
    if (!E) return MDX_ERR_ARG;
    if (nsteps < 0) return efail(E, MDX_ERR_ARG, "nsteps < 0");
    ENS_CUDA(E, cudaSetDevice(E->device));
    MDX_TRY(ensure_grid(E));
    std::vector<ens_state> before;
    MDX_TRY(read_stats(E, before));
    ENS_CUDA(E, cudaEventRecord(E->ev[0], E->stream));
    for (int q = 0; q < nsteps; ++q) {
        if (E->use_graph && E->graph_ok && !E->graph) {
            cudaGraph_t g = nullptr;
            ENS_CUDA(E, cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
            const long long l0 = E->launches;
            int rc = step_eager(E, E->variant, E->threads, E->grid);
            E->graph_launches = E->launches - l0;   // kernels one replay runs
            E->launches = l0;
            cudaError_t e = cudaStreamEndCapture(E->stream, &g);
            if (rc != MDX_OK || e != cudaSuccess || !g || cudaGraphInstantiate(&E->graph, g, 0) != cudaSuccess) {
                E->graph = nullptr;
                E->graph_ok = false;   // cooperative launches not capturable here: eager
                cudaGetLastError();
            }
            if (g) cudaGraphDestroy(g);
        }
        if (E->graph) {
            ENS_CUDA(E, cudaGraphLaunch(E->graph, E->stream));
            E->launches += E->graph_launches;
        } else {
            MDX_TRY(step_eager(E, E->variant, E->threads, E->grid));
        }
    }
    ENS_CUDA(E, cudaEventRecord(E->ev[1], E->stream));
    std::vector<ens_state> after;
    MDX_TRY(read_stats(E, after));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, E->ev[0], E->ev[1]) == cudaSuccess) E->last_step_ms = nsteps ? ms / nsteps : 0.0;
    long long it = 0;
    int bad = -1;
    for (int m = 0; m < E->n; ++m) {
        it += after[m].iters_total - before[m].iters_total;
        if (after[m].status != MDX_OK && bad < 0) bad = m;
    }
    if (total_iters) *total_iters = it;
    if (bad >= 0)
        return efail(E, after[bad].status == MDX_ERR_NONFINITE ? MDX_ERR_NONFINITE : MDX_NOT_CONVERGED,
                     "member %d: last projection status %d", bad, after[bad].status);
    return MDX_OK;
}

int mdx_ensemble_member_stats(mdx_ensemble_t* E, int m, mdx_solve_stats_t* st, long long* iters_total) {
    if (!E || m < 0 || m >= E->n) return E ? efail(E, MDX_ERR_ARG, "member index") : MDX_ERR_ARG;
    std::vector<ens_state> h;
    MDX_TRY(read_stats(E, h));
    const ens_state& S = h[m];
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->iterations = S.last_iters;
        st->status = S.status;
        st->residual = S.last_residual;
        st->residual0 = S.r0;
        st->atol = S.atol;
        st->variant = E->opts.precision == MDX_PREC_MIXED && E->opts.tol > 0.0
                          ? (E->opts.inner_form == 2 ? 700 : 100) + S.outer
                          : 1;
        st->guessed = S.guessed;
    }
    if (iters_total) *iters_total = S.iters_total;
    return MDX_OK;
}

int mdx_ensemble_get(mdx_ensemble_t* E, int m, int field, double* host) {
    if (!E || !host || m < 0 || m >= E->n) return E ? efail(E, MDX_ERR_ARG, "bad argument") : MDX_ERR_ARG;
    const ens_member& M = E->hm[m];
    const double* src = field == MDX_UN ? M.un : field == MDX_VN ? M.vn : field == MDX_WN ? M.wn
                      : field == MDX_PN ? M.pn : nullptr;
    if (!src) return efail(E, MDX_ERR_ARG, "field %d: MDX_UN, MDX_VN, MDX_WN or MDX_PN", field);
    ENS_CUDA(E, cudaMemcpyAsync(host, src, sizeof(double) * M.d.npad, cudaMemcpyDeviceToHost, E->stream));
    ENS_CUDA(E, cudaStreamSynchronize(E->stream));
    return MDX_OK;
}

int mdx_ensemble_set(mdx_ensemble_t* E, int m, int field, const double* host) {
    if (!E || !host || m < 0 || m >= E->n) return E ? efail(E, MDX_ERR_ARG, "bad argument") : MDX_ERR_ARG;
    const ens_member& M = E->hm[m];
    double* dst = field == MDX_UN ? M.un : field == MDX_VN ? M.vn : field == MDX_WN ? M.wn : field == MDX_PN ? M.pn
                                                                                                              : nullptr;
    if (!dst) return efail(E, MDX_ERR_ARG, "field %d: MDX_UN, MDX_VN, MDX_WN or MDX_PN", field);
    ENS_CUDA(E, cudaMemcpyAsync(dst, host, sizeof(double) * M.d.npad, cudaMemcpyHostToDevice, E->stream));
    ENS_CUDA(E, cudaStreamSynchronize(E->stream));
    return MDX_OK;
}

int mdx_ensemble_tune(mdx_ensemble_t* E, const char* cache_path, int* threads_out, int* bps_out, int* low_regs_out,
                      double* ms_out) {
    if (!E) return MDX_ERR_ARG;
    ENS_CUDA(E, cudaSetDevice(E->device));
    const std::string key = tune_key(E);
    int t = 0, b = 0, lr = 0;
    if (cache_lookup(cache_path, key, &t, &b, &lr) && mdx_ensemble_config(E, t, b, lr) == MDX_OK) {
        if (threads_out) *threads_out = t;
        if (bps_out) *bps_out = b;
        if (low_regs_out) *low_regs_out = lr;
        if (ms_out) *ms_out = -1.0;
        return MDX_OK;
    }
    // time one step of each candidate from the same saved state
    MDX_TRY(snapshot(E, false));
    const int cand_t[3] = {128, 256, 512};
    const int cand_b[4] = {1, 2, 4, 8};
    double best = 1e300;
    int bt = E->threads, bb = E->blocks_per_sm, bv = E->variant;
    for (int v = 0; v < 2; ++v)
        for (int ti = 0; ti < 3; ++ti) {
            int occ = 0;
            ENS_CUDA(E, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel_of(v), cand_t[ti], 0));
            for (int bi = 0; bi < 4; ++bi) {
                if (cand_b[bi] > occ) continue;
                int grid = 0;
                MDX_TRY(grid_for(E, v, cand_t[ti], cand_b[bi], &grid));
                MDX_TRY(snapshot(E, true));
                ENS_CUDA(E, cudaEventRecord(E->ev[0], E->stream));
                MDX_TRY(step_eager(E, v, cand_t[ti], grid));
                ENS_CUDA(E, cudaEventRecord(E->ev[1], E->stream));
                ENS_CUDA(E, cudaEventSynchronize(E->ev[1]));
                float ms = 0.f;
                ENS_CUDA(E, cudaEventElapsedTime(&ms, E->ev[0], E->ev[1]));
                if (ms < best) {
                    best = ms;
                    bt = cand_t[ti];
                    bb = cand_b[bi];
                    bv = v;
                }
            }
        }
    MDX_TRY(snapshot(E, true));
    ENS_CUDA(E, cudaStreamSynchronize(E->stream));
    MDX_TRY(mdx_ensemble_config(E, bt, bb, bv));
    cache_store(cache_path, key, bt, bb, bv, best);
    if (threads_out) *threads_out = bt;
    if (bps_out) *bps_out = bb;
    if (low_regs_out) *low_regs_out = bv;
    if (ms_out) *ms_out = best;
    return MDX_OK;
}

int mdx_ensemble_info(mdx_ensemble_t* E, int* threads, int* grid, int* low_regs, int* graph, double* last_step_ms,
                      long long* launches) {
    if (!E) return MDX_ERR_ARG;
    MDX_TRY(ensure_grid(E));
    if (low_regs) *low_regs = E->variant;
    if (threads) *threads = E->threads;
    if (grid) *grid = E->grid;
    if (graph) *graph = E->graph ? 1 : 0;
    if (last_step_ms) *last_step_ms = E->last_step_ms;
    if (launches) *launches = E->launches;
    return MDX_OK;
}

}  // extern "C"
