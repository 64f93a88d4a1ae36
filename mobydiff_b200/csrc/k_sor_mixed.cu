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
// By default (opts.inner_form 0) step 2 carries the corrections in their
// potential form -- the accumulated phi of each cell, from which every face
// correction follows -- and step 3 forms the face corrections from it in
// FP64 (k_pot_* below).
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

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

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

// V consecutive FP32 values at p (16-byte aligned for V = 4, 8-byte for V = 2).
template <int V>
__device__ __forceinline__ void ld_vec(float (&a)[V], const float* p) {
    if constexpr (V == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        a[0] = q.x; a[1] = q.y; a[2] = q.z; a[3] = q.w;
    } else {
        const float2 q = *reinterpret_cast<const float2*>(p);
        a[0] = q.x; a[1] = q.y;
    }
}
template <int V>
__device__ __forceinline__ void ld_vec_ro(float (&a)[V], const float* __restrict__ p) {
    if constexpr (V == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(p));
        a[0] = q.x; a[1] = q.y; a[2] = q.z; a[3] = q.w;
    } else {
        const float2 q = __ldg(reinterpret_cast<const float2*>(p));
        a[0] = q.x; a[1] = q.y;
    }
}
template <int V>
__device__ __forceinline__ void st_vec(float* p, const float (&a)[V]) {
    if constexpr (V == 4) *reinterpret_cast<float4*>(p) = make_float4(a[0], a[1], a[2], a[3]);
    else *reinterpret_cast<float2*>(p) = make_float2(a[0], a[1]);
}

// One FP32 colour sweep with V consecutive cells of the swept colour per
// thread (V = 2 or 4), on the colour-split arrays.  Window w of a row is the
// positions V w .. V w + V - 1 (rows start on 16-byte boundaries).  A thread
// owns its window in the swept colour's half of row (j, k) and in the other
// half's rows (j + 1, k) and (j, k + 1) -- the lower faces of its y and z
// neighbours -- and moves each with one vector load and store, writing back
// unchanged the positions that hold no swept cell (the row's ends and its
// padding).  The x neighbours' faces u(i+1) sit one position to the right
// in rows whose swept cells have odd i (the window plus one scalar), and at
// the window's own positions in the others, except the periodic wrap of
// cell nx to position 0; they are written with scalar stores, one per cell.
// The arithmetic is sweep32_update, so the result is k_sor_sweep32's bit for
// bit.  Needs nx and nz even, and ny even when y is periodic (every neighbour
// has the other colour).
template <int PY, int V>
__global__ void __launch_bounds__(256, V == 4 ? 3 : 1)
k_sor_sweep32v(mdx_dims d, mixed_params P, int parity, int reverse, int nwin, float* __restrict__ du,
               float* __restrict__ dv, float* __restrict__ dw, float* __restrict__ dp, const float* __restrict__ r,
               const float* __restrict__ mu32, const float* __restrict__ fac32) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per_plane = (long long)nwin * d.ny;
    if (g >= per_plane * d.nz) return;
    const int kk = (int)(g / per_plane);
    const int rem = (int)(g - (long long)kk * per_plane);
    const int j = rem / nwin + 1;
    const int p0 = V * (rem - (j - 1) * nwin);
    const int k = reverse ? d.nz - kk : kk + 1;
    const int cs = 1 - parity;            // colour (i + j + k) & 1 of the swept cells
    const int eo = (cs + j + k) & 1;      // i & 1 of the swept cells of this row
    const int half = d.nx / 2;            // position of the last cell of a row
    const int jp = (PY && j == d.ny) ? 1 : j + 1;
    const int kp = (k == d.nz) ? 1 : k + 1;
    const long long H = (long long)d.hs * d.nyp * d.nzp;
    const long long own = cs * H + ((long long)k * d.nyp + j) * d.hs + p0;
    const long long oth = (1 - cs) * H + ((long long)k * d.nyp + j) * d.hs;
    const long long ojp = (1 - cs) * H + ((long long)k * d.nyp + jp) * d.hs + p0;
    const long long okp = (1 - cs) * H + ((long long)kp * d.nyp + j) * d.hs + p0;
    const int PH = d.hs * d.nyp, np = 2 * PH;
    const int hp = (eo + j) & 1;          // (i + j) & 1: the factor planes' half of the swept cells
    const int mown = hp * PH + j * d.hs + p0;
    const int mox = (1 - hp) * PH + j * d.hs;
    const int mjp = (1 - hp) * PH + jp * d.hs + p0;

    // V = 4 reads the z-invariant factor planes (L1-resident) per cell when
    // it uses them instead of holding them as vectors: 80 registers, three
    // blocks per SM instead of two
    constexpr bool SMU = V == 4;
    float u0[V], ux[V], v0[V], vy[V], w0[V], wz[V], q[V], rr[V];
    float mu_u[V], mu_ux[V], mu_v[V], mu_vy[V], mu_w[V], fc[V];
    ld_vec<V>(u0, du + own);
    ld_vec<V>(v0, dv + own);
    ld_vec<V>(w0, dw + own);
    ld_vec<V>(q, dp + own);
    ld_vec<V>(ux, du + oth + p0);
    ld_vec<V>(vy, dv + ojp);
    ld_vec<V>(wz, dw + okp);
    ld_vec_ro<V>(rr, r + own);
    if constexpr (!SMU) {
        ld_vec_ro<V>(mu_u, mu32 + mown);
        ld_vec_ro<V>(mu_v, mu32 + np + mown);
        ld_vec_ro<V>(mu_w, mu32 + 2 * np + mown);
        ld_vec_ro<V>(fc, fac32 + mown);
        ld_vec_ro<V>(mu_ux, mu32 + mox + p0);
        ld_vec_ro<V>(mu_vy, mu32 + np + mjp);
    }
    // the x-neighbour face one past the window (odd i), or the wrap target
    // position 0 of cell nx (even i)
    const int xe = eo ? p0 + V : 0;
    const bool need_xe = eo ? (p0 + V < d.hs) : (half >= p0 && half < p0 + V);
    float uxe = 0.f, muxe = 0.f;
    if (need_xe) {
        uxe = du[oth + xe];
        if constexpr (!SMU) muxe = __ldg(mu32 + mox + xe);
    }
    const bool v_lo = PY || j > 1, v_hi = PY || j < d.ny;   // wall faces v(1), v(ny+1) stay 0
#pragma unroll
    for (int e = 0; e < V; ++e) {
        const int p = p0 + e;
        const bool valid = eo ? (p < half) : (p >= 1 && p <= half);
        const bool wrap = !eo && p == half;
        const int pip = eo ? p + 1 : (wrap ? 0 : p);   // position of the x neighbour's face
        float uip, muip = 0.f;
        if (e + 1 < V) {
            uip = eo ? ux[e + 1 < V ? e + 1 : e] : (wrap ? uxe : ux[e]);
            if constexpr (!SMU) muip = eo ? mu_ux[e + 1 < V ? e + 1 : e] : (wrap ? muxe : mu_ux[e]);
        } else {
            uip = (eo || wrap) ? uxe : ux[e];
            if constexpr (!SMU) muip = (eo || wrap) ? muxe : mu_ux[e];
        }
        if (valid) {
            if constexpr (SMU)
                sweep32_update(P, rr[e], u0[e], uip, v0[e], vy[e], w0[e], wz[e], q[e], __ldg(mu32 + mown + e),
                               __ldg(mu32 + mox + pip), __ldg(mu32 + np + mown + e), __ldg(mu32 + np + mjp + e),
                               __ldg(mu32 + 2 * np + mown + e), __ldg(fac32 + mown + e), v_lo, v_hi);
            else
                sweep32_update(P, rr[e], u0[e], uip, v0[e], vy[e], w0[e], wz[e], q[e], mu_u[e], muip, mu_v[e],
                               mu_vy[e], mu_w[e], fc[e], v_lo, v_hi);
            du[oth + pip] = uip;
        }
    }
    st_vec<V>(du + own, u0);
    st_vec<V>(dv + own, v0);
    st_vec<V>(dw + own, w0);
    st_vec<V>(dp + own, q);
    st_vec<V>(dv + ojp, vy);
    st_vec<V>(dw + okp, wz);
}

// ---------------------------------------------------------------------------
// Fused red+black pass: one launch per red-black iteration of the FP32
// correction sweeps, with the result of the two colour sweeps bit for bit.
//
// A CTA owns TI x TJ columns (x, y) of cells over a chunk of TK z planes and
// marches the chunk plane by plane.  Each thread holds a pair of x-adjacent
// cells (even, odd) of one row, so in every plane one of its cells is red
// (first colour: i + j + k odd) and the other black, and the cell that is red
// in plane q is black in plane q - 1.  Step q:
//   A  publish this plane's pre-sweep face u(even) in shared memory; barrier;
//   B  red cell of plane q: phi_R from pre-sweep faces;
//   C  black cell of plane q - 1: its faces after the red sweep (pre-sweep
//      value plus the red neighbour's contribution), then phi_B; barrier;
//   D  plane q - 1's own faces and dp: the red contribution, then the black
//      one, in the two sweeps' order.
// Plane data arrive by cp.async three planes ahead into a five-plane ring.
// Halo columns (2 on the low side, 1 on the high side, in x and y) and halo
// planes recompute red and black cells of the neighbouring tiles.  Faces are
// read from x* (the pre-sweep state, never written here, so that halo reads
// never see a neighbour's results) and written to y*; dp is only read and
// written by its own CTA, in place.  Wall faces v(1), v(ny+1) (y not
// periodic) are never written; the caller keeps them 0 in both buffers.
// tests/rb32_model.py restates this kernel step by step.
// ---------------------------------------------------------------------------
template <int TI, int TJ>
struct rb32_geom {
    static constexpr int PW = TI / 2 + 2;   // pair columns (x halo 2 low, 1 high, rounded to pairs)
    static constexpr int RW = TJ + 3;       // rows (y halo 2 low, 1 high)
    static constexpr int CW = 2 * PW;
    static constexpr int NT = PW * RW;
    // plane data staged by cp.async: SLOTS planes, FIELDS values per thread
    // (u, v, v(j+1), r, dp and w(q+1) of both cells), field-major so that a
    // warp's accesses to one field are consecutive words
    static constexpr int SLOTS = 5, FIELDS = 12;
    static constexpr int slot_floats = FIELDS * NT;
};
enum { RB_U0 = 0, RB_U1, RB_V0, RB_V1, RB_VN0, RB_VN1, RB_R0, RB_R1, RB_DP0, RB_DP1, RB_W0, RB_W1 };

__device__ __forceinline__ int rb32_cx(int i, int nx) {   // unwrapped x cell -> 1..nx (0 <-> nx)
    int m = i % nx;
    if (m < 0) m += nx;
    return m == 0 ? nx : m;
}
__device__ __forceinline__ int rb32_c1(int k, int n) {    // unwrapped 1-based -> 1..n
    int m = (k - 1) % n;
    if (m < 0) m += n;
    return m + 1;
}
// 4-byte cp.async; with on == false the word is zero-filled and nothing is read
__device__ __forceinline__ void rb32_cp4(unsigned dst, const float* src, bool on) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(on ? 4 : 0) : "memory");
}

template <int PY, int TI, int TJ, int TK>
__global__ void __launch_bounds__(rb32_geom<TI, TJ>::NT)
k_rb32_fused(mdx_dims d, mixed_params P, const float* __restrict__ xu, const float* __restrict__ xv,
             const float* __restrict__ xw, float* __restrict__ yu, float* __restrict__ yv, float* __restrict__ yw,
             float* __restrict__ dp, const float* __restrict__ r, const float* __restrict__ mu32,
             const float* __restrict__ fac32) {
    using G = rb32_geom<TI, TJ>;
    constexpr int S = G::SLOTS, NT = G::NT, SF = G::slot_floats;
    extern __shared__ __align__(16) float rb32_ring[];   // [SLOTS][FIELDS][NT]
    __shared__ float U_s[2][G::RW][G::PW + 1];   // pre-sweep u(even cell), plane ring
    __shared__ float PH[2][G::RW][G::CW + 2];    // phi of both colours, plane ring; column 2 tx + c + 1
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * G::PW + tx;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int i0 = blockIdx.x * TI, j0 = 1 + blockIdx.y * TJ, k0 = 1 + blockIdx.z * TK;
    const int ie = i0 - 2 + 2 * tx;               // unwrapped even cell of the pair
    const int j = j0 - 2 + ty;
    const bool ex = PY || (j >= 1 && j <= ny);    // the row's cells exist
    const bool ex_dn = PY || j - 1 >= 1, ex_up = PY || j + 1 <= ny;
    const bool own_row = ex && ty >= 2 && ty < TJ + 2 && j <= ny;
    const int jc = PY ? rb32_c1(j, ny) : (ex ? j : 1);    // rows that load nothing point at row 1
    const int jn = PY ? rb32_c1(j + 1, ny) : (ex ? j + 1 : 1);
    const int ic0 = rb32_cx(ie, nx), ic1 = rb32_cx(ie + 1, nx), ic2 = rb32_cx(ie + 2, nx);
    // 32-bit colour-split offsets: cell (ic, row, kc) at half (ic+row+kc)&1
    const int H = d.hs * d.nyp * d.nzp, PL = d.nyp * d.hs;
    const int b0 = jc * d.hs + (ic0 >> 1), b1 = jc * d.hs + (ic1 >> 1);
    const int bn0 = jn * d.hs + (ic0 >> 1), bn1 = jn * d.hs + (ic1 >> 1);
    const int par0 = (ic0 + jc) & 1, par1 = (ic1 + jc) & 1, parn0 = (ic0 + jn) & 1, parn1 = (ic1 + jn) & 1;
    const int np = split_plane_elems(d);
    const unsigned ring0 = (unsigned)__cvta_generic_to_shared(rb32_ring) + 4u * tid;
    const float* rt = rb32_ring + tid;

    // per-column factors (z-invariant)
    float fac[2] = {0.f, 0.f}, mu_u[3] = {0.f, 0.f, 0.f}, mu_v[2] = {0.f, 0.f}, mu_vn[2] = {0.f, 0.f},
          mu_w[2] = {0.f, 0.f};
    if (ex) {
        const int q0 = pidx2(d, ic0, jc), q1 = pidx2(d, ic1, jc);
        fac[0] = __ldg(fac32 + q0);
        fac[1] = __ldg(fac32 + q1);
        mu_u[0] = __ldg(mu32 + q0);
        mu_u[1] = __ldg(mu32 + q1);
        mu_u[2] = __ldg(mu32 + pidx2(d, ic2, jc));
        mu_v[0] = __ldg(mu32 + np + q0);
        mu_v[1] = __ldg(mu32 + np + q1);
        mu_w[0] = __ldg(mu32 + 2 * np + q0);
        mu_w[1] = __ldg(mu32 + 2 * np + q1);
        mu_vn[0] = __ldg(mu32 + np + pidx2(d, ic0, jn));
        mu_vn[1] = __ldg(mu32 + np + pidx2(d, ic1, jn));
    }
    // stage plane kc (its slot at byte offset sb): u, v, v(j+1), r, dp of both
    // cells and w of plane kn = kc + 1 (periodic)
    auto issue = [&](unsigned sb, int kc, int kn) {
        const int hc = (kc & 1) ? H : 0, hn = (kn & 1) ? H : 0, hh = H - hc;   // hh: the other half at kc
        const int a0 = b0 + kc * PL + (par0 ? hh : hc), a1 = b1 + kc * PL + (par1 ? hh : hc);
        const int an0 = bn0 + kc * PL + (parn0 ? hh : hc), an1 = bn1 + kc * PL + (parn1 ? hh : hc);
        const int w0 = b0 + kn * PL + (par0 ? H - hn : hn), w1 = b1 + kn * PL + (par1 ? H - hn : hn);
        const bool vn_on = ex;   // v(j+1): the top wall face for j = ny (0 in the array)
        rb32_cp4(sb + 4u * (RB_U0 * NT), xu + a0, ex);
        rb32_cp4(sb + 4u * (RB_U1 * NT), xu + a1, ex);
        rb32_cp4(sb + 4u * (RB_V0 * NT), xv + a0, ex);
        rb32_cp4(sb + 4u * (RB_V1 * NT), xv + a1, ex);
        rb32_cp4(sb + 4u * (RB_VN0 * NT), xv + an0, vn_on);
        rb32_cp4(sb + 4u * (RB_VN1 * NT), xv + an1, vn_on);
        rb32_cp4(sb + 4u * (RB_R0 * NT), r + a0, ex);
        rb32_cp4(sb + 4u * (RB_R1 * NT), r + a1, ex);
        rb32_cp4(sb + 4u * (RB_DP0 * NT), dp + a0, own_row);
        rb32_cp4(sb + 4u * (RB_DP1 * NT), dp + a1, own_row);
        rb32_cp4(sb + 4u * (RB_W0 * NT), xw + w0, ex);
        rb32_cp4(sb + 4u * (RB_W1 * NT), xw + w1, ex);
    };
    auto knext = [&](int k) { return k == nz ? 1 : k + 1; };

    float w[2] = {0.f, 0.f}, wp[2] = {0.f, 0.f};            // w(q), w(q-1)
    float ph[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};     // phi per column at planes q, q-1, q-2
    int kq = rb32_c1(k0 - 2, nz);                            // plane q
    if (ex) {
        const int hc = (kq & 1) ? H : 0;
        w[0] = __ldg(xw + b0 + kq * PL + (par0 ? H - hc : hc));
        w[1] = __ldg(xw + b1 + kq * PL + (par1 ? H - hc : hc));
    }
    // slots: plane q in slot sq; the prologue stages planes k0-2 .. k0
    int sq = 0;
    {
        int k = kq;
        for (int t = 0; t < 3; ++t) {
            issue(ring0 + 4u * (t * SF), k, knext(k));
            asm volatile("cp.async.commit_group;\n" ::);
            k = knext(k);
        }
    }
    int k_issue = knext(knext(knext(kq)));                  // plane q + 3
    int kd = kq == 1 ? nz : kq - 1;                          // plane q - 1
    const float idx = P.idx, idy = P.idy, idz = P.idz;
    for (int q = k0 - 2; q <= k0 + TK; ++q) {
        const int h = q & 1, hp = (q - 1) & 1;
        const int sp = sq == 0 ? S - 1 : sq - 1;             // slot of plane q - 1
        const int si = sq + 3 >= S ? sq + 3 - S : sq + 3;    // slot of plane q + 3 (plane q - 2's)
        const float* cs = rt + sq * SF;
        const float* ps = rt + sp * SF;
        // stage plane q + 3; plane q is then complete
        if (q + 3 <= k0 + TK) issue(ring0 + 4u * (si * SF), k_issue, knext(k_issue));
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group 3;\n" ::: "memory");
        // A
        U_s[h][ty][tx] = cs[RB_U0 * NT];
        __syncthreads();
        const int c = ((j + q) & 1) ? 0 : 1;   // the red cell of plane q (the black cell of plane q - 1)
        // the column-c values by selection (register arrays are indexed by constants only)
        const bool c1 = c == 1;
        const float fac_c = c1 ? fac[1] : fac[0], mu_w_c = c1 ? mu_w[1] : mu_w[0];
        const float w_c = c1 ? w[1] : w[0], wp_c = c1 ? wp[1] : wp[0];
        // B: red cell of plane q
        if (ex && 2 * tx + c <= TI + 2 && ty <= TJ + 2) {
            const float ui = cs[(RB_U0 + c) * NT];
            const float uip = c1 ? U_s[h][ty][tx + 1] : cs[RB_U1 * NT];
            const float vj = cs[(RB_V0 + c) * NT], vjp = cs[(RB_VN0 + c) * NT];
            const float phi = __fmul_rn(sweep32_div(P, cs[(RB_R0 + c) * NT], ui, uip, vj, vjp, w_c, cs[(RB_W0 + c) * NT]),
                                        fac_c);
            if (c1) ph[1][0] = phi;
            else ph[0][0] = phi;
            PH[h][ty][2 * tx + c + 1] = phi;
        }
        // C reads no value B writes (its neighbours' plane q - 1 values date
        // from the last step; the red phi of plane q is its own), so no
        // barrier between them
        // C: black cell of plane q - 1, faces after the red sweep
        if (q >= k0 && ex && 2 * tx + c >= 1 && 2 * tx + c <= TI + 1 && ty >= 1 && ty <= TJ + 1) {
            const float p_left = c1 ? ph[0][1] : PH[hp][ty][2 * tx];
            const float p_right = c1 ? PH[hp][ty][2 * tx + 3] : ph[1][1];
            const float mu_ui = c1 ? mu_u[1] : mu_u[0], mu_uip = c1 ? mu_u[2] : mu_u[1];
            const float up_i = ps[(RB_U0 + c) * NT];
            const float up_ip = c1 ? U_s[hp][ty][tx + 1] : ps[RB_U1 * NT];
            const float ui = __fmaf_rn(__fmul_rn(p_left, idx), mu_ui, up_i);
            const float uip = __fmaf_rn(-__fmul_rn(p_right, idx), mu_uip, up_ip);
            float vj = ps[(RB_V0 + c) * NT];
            if (ex_dn) vj = __fmaf_rn(__fmul_rn(PH[hp][ty - 1][2 * tx + c + 1], idy), c1 ? mu_v[1] : mu_v[0], vj);
            float vjp = ps[(RB_VN0 + c) * NT];
            if (ex_up) vjp = __fmaf_rn(-__fmul_rn(PH[hp][ty + 1][2 * tx + c + 1], idy), c1 ? mu_vn[1] : mu_vn[0], vjp);
            const float ph2 = c1 ? ph[1][2] : ph[0][2], ph0 = c1 ? ph[1][0] : ph[0][0];
            const float wk = __fmaf_rn(__fmul_rn(ph2, idz), mu_w_c, wp_c);
            const float wkp = __fmaf_rn(-__fmul_rn(ph0, idz), mu_w_c, w_c);
            const float phi = __fmul_rn(sweep32_div(P, ps[(RB_R0 + c) * NT], ui, uip, vj, vjp, wk, wkp), fac_c);
            if (c1) ph[1][1] = phi;
            else ph[0][1] = phi;
            PH[hp][ty][2 * tx + c + 1] = phi;
        }
        __syncthreads();
        // D: own faces and dp of plane q - 1
        if (q >= k0 + 1 && q - 1 < k0 + TK && q - 1 <= nz && own_row) {
            const int hd = (kd & 1) ? H : 0;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int pos = 2 * tx + cc;
                if (pos < 2 || pos >= TI + 2 || ie + cc >= nx) continue;
                const bool red = ((cc + j + q - 1) & 1) == 1;
                const float phi = ph[cc][1];
                const float px = __fmul_rn(phi, idx), py = __fmul_rn(phi, idy), pz = __fmul_rn(phi, idz);
                const float pxl = __fmul_rn(cc == 1 ? ph[0][1] : PH[hp][ty][2 * tx], idx);
                const float mu = mu_u[cc];
                const float u0 = ps[(RB_U0 + cc) * NT];
                const float u2 = red ? __fmaf_rn(pxl, mu, __fmaf_rn(-px, mu, u0)) : __fmaf_rn(-px, mu, __fmaf_rn(pxl, mu, u0));
                const bool v_lo = PY || j > 1;
                const float pyd = ex_dn ? __fmul_rn(PH[hp][ty - 1][2 * tx + cc + 1], idy) : 0.f;
                const float mv = mu_v[cc];
                float v1 = ps[(RB_V0 + cc) * NT];
                if (red) {
                    if (v_lo) v1 = __fmaf_rn(-py, mv, v1);
                    if (ex_dn) v1 = __fmaf_rn(pyd, mv, v1);
                } else {
                    if (ex_dn) v1 = __fmaf_rn(pyd, mv, v1);
                    if (v_lo) v1 = __fmaf_rn(-py, mv, v1);
                }
                const float pzb = __fmul_rn(ph[cc][2], idz);
                const float mw = mu_w[cc];
                const float w2 = red ? __fmaf_rn(pzb, mw, __fmaf_rn(-pz, mw, wp[cc]))
                                     : __fmaf_rn(-pz, mw, __fmaf_rn(pzb, mw, wp[cc]));
                const int par = cc == 0 ? par0 : par1;
                const int a = (cc == 0 ? b0 : b1) + kd * PL + (par ? H - hd : hd);
                yu[a] = u2;
                yv[a] = v1;
                yw[a] = w2;
                dp[a] = __fmaf_rn(phi, P.idt, ps[(RB_DP0 + cc) * NT]);
            }
        }
        // the next plane
        wp[0] = w[0];
        wp[1] = w[1];
        w[0] = cs[RB_W0 * NT];
        w[1] = cs[RB_W1 * NT];
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            ph[cc][2] = ph[cc][1];
            ph[cc][1] = ph[cc][0];
            ph[cc][0] = 0.f;
        }
        sq = sq + 1 == S ? 0 : sq + 1;
        kd = kq;
        kq = knext(kq);
        k_issue = knext(k_issue);
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// u += du, v += dv, w += dw, p += dp over the padded arrays; corrections reset.
__global__ void k_mixed_apply(mdx_dims d, double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                              double* __restrict__ p, float* __restrict__ du, float* __restrict__ dv,
                              float* __restrict__ dw, float* __restrict__ dp) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.npad; t += (long long)gridDim.x * blockDim.x)
        mixed_apply_elem(d, t, u, v, w, p, du, dv, dw, dp);
}

// ---------------------------------------------------------------------------
// Potential form of the FP32 correction sweeps (opts.inner_form 0).
//
// Starting from zero corrections, the face updates of
// pressure_redblack.f90:117-241 leave every face at h^-1 mu (Phi(low cell) -
// Phi(high cell)), Phi being the sum of the phi a cell has taken, and dp at
// Phi/dt_gamma.  The divergence the next update of cell c needs is then
//   e(c) = r~(c) + sum over the faces f of c of a_f (Phi(c) - Phi(across f)),
//   a_f = h^-2 mu_f, 0 for a wall face (which never moves),
// and the update is Phi(c) += fac(c) e(c): the same red-black iteration in
// exact arithmetic, carried by one array instead of four.  A colour sweep
// reads Phi of the other colour and Phi and r~ of its own and writes Phi of
// its own: 8 B per cell instead of 30.
//
// Layout (pot_geom): cell (i, j, k), i in 0..nx+1, in half (i + j + k) & 1 at
// (k (ny+2) + j) hq + 3 + (i + 1) / 2.  A row of one half holds its nx/2
// interior cells at positions 4 .. nx/2 + 3 (16-byte aligned), the copy of
// cell nx at position 3 (rows of even cells) or of cell 1 at nx/2 + 4 (rows
// of odd cells); planes 0 and nz+1, and rows 0 and ny+1 when y is periodic,
// hold copies of planes nz and 1 (rows ny and 1).  A sweep writes the copies
// of the cells it updates, so no neighbour read tests for a wrap.  Corners
// are never read.  tests/pot32_model.py restates the sweep thread by thread.
// ---------------------------------------------------------------------------
struct pot_geom {
    int nx, ny, nz;
    int hq;   // row length of one half (positions)
    int rz;   // one plane of one half: hq (ny+2)
    int H;    // one half, a multiple of 64 elements
};

__host__ __device__ __forceinline__ int pot_row(const pot_geom& L, int h, int j, int k) {
    return h * L.H + (k * (L.ny + 2) + j) * L.hq;
}
__host__ __device__ __forceinline__ int pot_idx(const pot_geom& L, int i, int j, int k) {
    return pot_row(L, (i + j + k) & 1, j, k) + 3 + (i + 1) / 2;
}

pot_geom pot_make(const mdx_dims& d) {
    pot_geom L;
    L.nx = d.nx;
    L.ny = d.ny;
    L.nz = d.nz;
    L.hq = ((d.nx / 2 + 5) + 3) & ~3;
    L.rz = L.hq * (d.ny + 2);
    L.H = (int)((((long long)L.rz * (d.nz + 2)) + 63) & ~63LL);
    return L;
}

// Column table: per (i, j) {a_x of the low x face, a_y of the low y face (0
// at a wall), a_z, fac = -omega/denom}; column nx+1 repeats column 1's a_x,
// row ny+1 holds the top faces' a_y (0 at walls, row 1's when y is
// periodic).  a_f and fac are formed in FP64 (the denominator of
// pressure_redblack.f90:124-126) and rounded once.  tabu repeats the a_y of
// every column's top face, row j holding cy(i, j+1) at (i-1), rows ncu
// (nx rounded up to 4) apart, so that a row's top faces are one aligned
// vector load.
__host__ __device__ inline int pot_ncu(int nx) { return (nx + 3) & ~3; }
__global__ void k_pot_tables(pot_geom L, int py, double idx2, double idy2, double idz2, double sor,
                             const double* __restrict__ mu, int plane_mu, float4* __restrict__ tab,
                             float* __restrict__ tabu) {
    const int nxp = L.nx + 2, nyp = L.ny + 2;
    const long long np = (long long)nxp * nyp;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nxp), j = (int)(t / nxp);
        auto MU = [&](int c, int ii, int jj) { return plane_mu ? mu[c * np + ii + (long long)nxp * jj] : 1.0; };
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j >= 1 && j <= L.ny && i >= 1 && i <= L.nx) {
            const int ip = i == L.nx ? 1 : i + 1;
            const int jp = (py && j == L.ny) ? 1 : j + 1;
            const double mu_u = MU(0, i, j), mu_v = MU(1, i, j), mu_w = MU(2, i, j);
            const double denom = (mu_u + MU(0, ip, j)) * idx2 + (mu_w + mu_w) * idz2 + (mu_v + MU(1, i, jp)) * idy2;
            o.x = (float)(idx2 * mu_u);
            o.y = (py || j > 1) ? (float)(idy2 * mu_v) : 0.f;
            o.z = (float)(idz2 * mu_w);
            o.w = (float)(-sor / denom);
        } else if (j >= 1 && j <= L.ny && i == L.nx + 1) {
            o.x = (float)(idx2 * MU(0, 1, j));
        } else if (j == L.ny + 1 && i >= 1 && i <= L.nx) {
            o.y = py ? (float)(idy2 * MU(1, i, 1)) : 0.f;
        }
        tab[t] = o;
        if (j >= 1 && i >= 1 && i <= L.nx) tabu[(j - 1) * pot_ncu(L.nx) + (i - 1)] = o.y;
    }
}

// FP64 divergence of (u, v, w) per cell, stored as FP32 r~ in the potential
// layout; partial sums of r^2, max|r| and max(|u|,|v|,|w|) (the expression of
// k_mixed_residual, so the same norms).
template <int PY>
__global__ void __launch_bounds__(MDX_RED_THREADS)
k_pot_residual(mdx_dims d, pot_geom L, double idx, double idy, double idz, const double* __restrict__ u,
               const double* __restrict__ v, const double* __restrict__ w, float* __restrict__ r,
               double* __restrict__ part) {
    double s = 0.0, m = 0.0, um = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long rr = t / d.nx;
        const int j = (int)(rr % d.ny) + 1;
        const int k = (int)(rr / d.ny) + 1;
        const int ip = i == d.nx ? 1 : i + 1;
        const int jp = (PY && j == d.ny) ? 1 : j + 1;
        const int kp = k == d.nz ? 1 : k + 1;
        const long long c = pidx(d, i, j, k);
        const double dv = (__ldg(u + pidx(d, ip, j, k)) - __ldg(u + c)) * idx +
                          (__ldg(v + pidx(d, i, jp, k)) - __ldg(v + c)) * idy +
                          (__ldg(w + pidx(d, i, j, kp)) - __ldg(w + c)) * idz;
        r[pot_idx(L, i, j, k)] = (float)dv;
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

// Residual of the correction problem, e(c) of every cell, as partial sums.
__global__ void __launch_bounds__(MDX_RED_THREADS)
k_pot_corr_residual(mdx_dims d, pot_geom L, const float* __restrict__ phi, const float* __restrict__ r,
                    const float4* __restrict__ tab, double* __restrict__ part) {
    double s = 0.0, m = 0.0, z = 0.0;
    const int ncol = d.nx + 2;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long rr = t / d.nx;
        const int j = (int)(rr % d.ny) + 1;
        const int k = (int)(rr / d.ny) + 1;
        const int c = pot_idx(L, i, j, k);
        const float4 T = __ldg(tab + j * ncol + i);
        const float axr = __ldg(&tab[j * ncol + i + 1].x), ayr = __ldg(&tab[(j + 1) * ncol + i].y);
        const float e = pot_e(__ldg(r + c), __ldg(phi + c), __ldg(phi + pot_idx(L, i - 1, j, k)),
                              __ldg(phi + pot_idx(L, i + 1, j, k)), __ldg(phi + pot_idx(L, i, j - 1, k)),
                              __ldg(phi + pot_idx(L, i, j + 1, k)), __ldg(phi + pot_idx(L, i, j, k - 1)),
                              __ldg(phi + pot_idx(L, i, j, k + 1)), T.x, axr, T.y, ayr, T.z);
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

// One colour sweep of the potential form (cells of colour cs = (i+j+k)&1).
// A thread owns positions q0 .. q0+V-1 of row j (the 2V cells 2 q0 + 1 ..
// 2 q0 + 2V, both colours) and marches planes k0 .. k0+KZ-1, holding the
// other colour's values of planes k-1, k, k+1 in registers and the 2V
// columns' coefficients for the whole march.  In plane k its V swept cells
// have odd i when (cs + j + k) is odd; their x neighbours are the other
// colour's values at the same positions and one position to the left (odd)
// or right (even), that one value a scalar load.  Needs nx/2 a multiple of
// V, nz even (and ny even when y is periodic): every neighbour then has the
// other colour, so a thread reads nothing that another thread writes.
template <int PY, int V, int KZ, bool PF>
__global__ void __launch_bounds__(256)
k_pot_sweep(pot_geom L, int cs, float* __restrict__ phi, const float* __restrict__ r, const float4* __restrict__ tab) {
    const int half = L.nx / 2;
    const int q0 = V * (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    if (q0 >= half || j > L.ny) return;
    const int k0 = 1 + (int)blockIdx.z * KZ;
    const int k1 = min(k0 + KZ - 1, L.nz);
    const int ncol = L.nx + 2;
    // coefficients: column m = 0 .. 2V-1 is cell 2 q0 + 1 + m, odd cells at
    // even m (set 0), even cells at odd m (set 1)
    float axl[2][V], axr[2][V], ayl[2][V], ayr[2][V], az[2][V], fc[2][V];
    const float4* t0 = tab + j * ncol + 2 * q0 + 1;
    const float4* t1 = tab + (j + 1) * ncol + 2 * q0 + 1;
#pragma unroll
    for (int m = 0; m < 2 * V; ++m) {
        const float4 c = __ldg(t0 + m);
        const int s = m & 1, e = m >> 1;
        axl[s][e] = c.x;
        ayl[s][e] = c.y;
        az[s][e] = c.z;
        fc[s][e] = c.w;
        ayr[s][e] = __ldg(&t1[m].y);
        if (m > 0) axr[(m - 1) & 1][(m - 1) >> 1] = c.x;
    }
    axr[1][V - 1] = __ldg(&t0[2 * V].x);

    const int oh = 1 - cs;
    const int ob = pot_row(L, oh, j, 0) + 4 + q0;   // other colour, row j, plane 0, position q0
    const int sb = pot_row(L, cs, j, 0) + 4 + q0;   // swept colour
    // Every value a thread reads is either the other colour's (not written
    // by this sweep) or its own cell's before it writes it, so all reads
    // take the read-only path; with PF the loads of plane k+1 are issued
    // before plane k is computed (one plane in flight while the other is
    // used).
    struct plane_in { float zp[V], s[V], rr[V], ym[V], yp[V], xs; };
    auto load = [&](plane_in& P, int k) {
        const int ok = ob + k * L.rz, sk = sb + k * L.rz;
        ld_vec_ro<V>(P.zp, phi + ok + L.rz);
        ld_vec_ro<V>(P.s, phi + sk);
        ld_vec_ro<V>(P.rr, r + sk);
        ld_vec_ro<V>(P.ym, phi + ok - L.hq);
        ld_vec_ro<V>(P.yp, phi + ok + L.hq);
        P.xs = __ldg(phi + ok + (((cs + j + k) & 1) ? -1 : V));
    };
    float zm[V], z0[V];
    ld_vec_ro<V>(zm, phi + ob + (k0 - 1) * L.rz);
    ld_vec_ro<V>(z0, phi + ob + k0 * L.rz);
    plane_in cur, nxt;
    if (PF) load(cur, k0);
    for (int k = k0; k <= k1; ++k) {
        if (!PF) load(cur, k);
        else if (k < k1) load(nxt, k + 1);
        const int sk = sb + k * L.rz;
        const bool odd = ((cs + j + k) & 1) != 0;
        float out[V];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const float xl = odd ? (e == 0 ? cur.xs : z0[e > 0 ? e - 1 : 0]) : z0[e];
            const float xr = odd ? z0[e] : (e == V - 1 ? cur.xs : z0[e + 1 < V ? e + 1 : e]);
            const float c = cur.s[e];
            const float E = pot_e(cur.rr[e], c, xl, xr, cur.ym[e], cur.yp[e], zm[e], cur.zp[e],
                                  odd ? axl[0][e] : axl[1][e], odd ? axr[0][e] : axr[1][e],
                                  odd ? ayl[0][e] : ayl[1][e], odd ? ayr[0][e] : ayr[1][e],
                                  odd ? az[0][e] : az[1][e]);
            out[e] = __fmaf_rn(odd ? fc[0][e] : fc[1][e], E, c);
        }
        st_vec<V>(phi + sk, out);
        // copies of the updated cells
        if (odd && q0 == 0) phi[sk + half] = out[0];                  // cell nx+1 = cell 1
        if (!odd && q0 + V == half) phi[sk - q0 - 1] = out[V - 1];    // cell 0 = cell nx
        if (k == L.nz) st_vec<V>(phi + sb, out);                      // plane 0
        if (k == 1) st_vec<V>(phi + sb + (L.nz + 1) * L.rz, out);     // plane nz+1
        if (PY && j == L.ny) st_vec<V>(phi + sk - L.ny * L.hq, out);  // row 0
        if (PY && j == 1) st_vec<V>(phi + sk + L.ny * L.hq, out);     // row ny+1
#pragma unroll
        for (int e = 0; e < V; ++e) {
            zm[e] = z0[e];
            z0[e] = cur.zp[e];
        }
        if (PF && k < k1) cur = nxt;   // the last plane loads no successor
    }
}

// The same colour sweep with one warp per row (nx/2 = 32 V positions, so a
// lane owns V positions and a warp the whole row) and 8 rows per block
// (ny a multiple of 8).  The x neighbours come from the neighbouring lanes by
// shuffle, wrapping at the row's ends (x periodic); the other colour's rows
// j-1 and j+1 from a shared-memory exchange between the block's warps
// (warps 0 and 7 also load the rows just outside the block); the
// coefficients from aligned vector loads, the top faces' a_y from tabu.  The
// arithmetic is pot_e's, so the result is k_pot_sweep's bit for bit.
// V floats at p (8- or 16-byte aligned), cached in L2 only: in the
// persistent kernel Phi changes between its sweeps, so it bypasses L1.
template <int V>
__device__ __forceinline__ void ld_vec_cg(float (&a)[V], const float* p) {
    if constexpr (V == 4) {
        const float4 q = __ldcg(reinterpret_cast<const float4*>(p));
        a[0] = q.x; a[1] = q.y; a[2] = q.z; a[3] = q.w;
    } else {
        const float2 q = __ldcg(reinterpret_cast<const float2*>(p));
        a[0] = q.x; a[1] = q.y;
    }
}

// The column coefficients a lane of the warp-per-row sweeps holds: its 2V
// columns 2 q0 + 1 .. 2 q0 + 2V, odd cells at even m (set 0), even cells at
// odd m (set 1); the top faces' a_y from tabu, the next lane's first a_x by
// shuffle (lane 31: column nx+1 = column 1).
template <int V>
struct pot_coef {
    float axl[2][V], axr[2][V], ayl[2][V], ayr[2][V], az[2][V], fc[2][V];
    __device__ __forceinline__ void load(const pot_geom& L, int j, int q0, int lane, const float4* __restrict__ tab,
                                         const float* __restrict__ tabu) {
        const float4* t0 = tab + j * (L.nx + 2) + 2 * q0 + 1;
        const float* tu = tabu + j * pot_ncu(L.nx) + 2 * q0;
        float up[2 * V];
#pragma unroll
        for (int m = 0; m < 2 * V; m += 4) {
            const float4 u4 = __ldg(reinterpret_cast<const float4*>(tu + m));
            up[m] = u4.x;
            up[m + 1] = u4.y;
            up[m + 2] = u4.z;
            up[m + 3] = u4.w;
        }
#pragma unroll
        for (int m = 0; m < 2 * V; ++m) {
            const float4 c = __ldg(t0 + m);
            const int s = m & 1, e = m >> 1;
            axl[s][e] = c.x;
            ayl[s][e] = c.y;
            az[s][e] = c.z;
            fc[s][e] = c.w;
            ayr[s][e] = up[m];
            if (m > 0) axr[(m - 1) & 1][(m - 1) >> 1] = c.x;
        }
        axr[1][V - 1] = __shfl_sync(0xffffffffu, axl[0][0], (lane + 1) & 31);
    }
};

// One colour sweep of rows j0 .. j0+7 (warp w: row j0 + w), planes k0 .. k1,
// by one block of the warp-per-row kernels.  COH: Phi is read through L2
// only (it changed since the kernel started), else through the read-only
// path.
template <int PY, int V, bool COH>
__device__ __forceinline__ void pot_rows_sweep(const pot_geom& L, int cs, int j0, int k0, int k1,
                                               float* __restrict__ phi, const float* __restrict__ r,
                                               const pot_coef<V>& C, float (*ybuf)[10][32 * V]) {
    constexpr int NW = 8, RL = 32 * V;
    const int lane = threadIdx.x, w = threadIdx.y;
    const int j = j0 + w, q0 = V * lane;
    const int oh = 1 - cs;
    const int ob = pot_row(L, oh, j, 0) + 4 + q0;   // other colour, row j, plane 0, position q0
    const int sb = pot_row(L, cs, j, 0) + 4 + q0;   // swept colour
    const bool hlo = w == 0, hhi = w == NW - 1;
    const int hb = pot_row(L, oh, hlo ? j0 - 1 : j0 + NW, 0) + 4 + q0;   // the row outside the block
    auto ldp = [&](float (&a)[V], const float* p) {
        if constexpr (COH) ld_vec_cg<V>(a, p);
        else ld_vec_ro<V>(a, p);
    };
    struct plane_in { float zp[V], s[V], rr[V], h[V]; };
    auto load = [&](plane_in& P, int k) {
        ldp(P.zp, phi + ob + (k + 1) * L.rz);
        ldp(P.s, phi + sb + k * L.rz);
        ld_vec_ro<V>(P.rr, r + sb + k * L.rz);
        if (hlo || hhi) ldp(P.h, phi + hb + k * L.rz);
    };
    float zm[V], z0[V];
    ldp(zm, phi + ob + (k0 - 1) * L.rz);
    ldp(z0, phi + ob + k0 * L.rz);
    plane_in cur, nxt;
    load(cur, k0);
    for (int k = k0; k <= k1; ++k) {
        if (k < k1) load(nxt, k + 1);
        // the other colour's rows j0-1 .. j0+NW of plane k; the buffers
        // alternate with k, so one barrier per plane keeps writes of plane
        // k+1 apart from reads of plane k
        float(*yb)[RL] = ybuf[k & 1];
        st_vec<V>(&yb[w + 1][q0], z0);
        if (hlo) st_vec<V>(&yb[0][q0], cur.h);
        if (hhi) st_vec<V>(&yb[NW + 1][q0], cur.h);
        __syncthreads();
        float ym[V], yp[V];
        ld_vec<V>(ym, &yb[w][q0]);
        ld_vec<V>(yp, &yb[w + 2][q0]);
        const bool odd = ((cs + j + k) & 1) != 0;
        const float xlw = __shfl_sync(0xffffffffu, z0[V - 1], (lane + 31) & 31);   // position q0 - 1
        const float xrw = __shfl_sync(0xffffffffu, z0[0], (lane + 1) & 31);        // position q0 + V
        const int sk = sb + k * L.rz;
        float out[V];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const float xl = odd ? (e == 0 ? xlw : z0[e > 0 ? e - 1 : 0]) : z0[e];
            const float xr = odd ? z0[e] : (e == V - 1 ? xrw : z0[e + 1 < V ? e + 1 : e]);
            const float c = cur.s[e];
            const float E = pot_e(cur.rr[e], c, xl, xr, ym[e], yp[e], zm[e], cur.zp[e],
                                  odd ? C.axl[0][e] : C.axl[1][e], odd ? C.axr[0][e] : C.axr[1][e],
                                  odd ? C.ayl[0][e] : C.ayl[1][e], odd ? C.ayr[0][e] : C.ayr[1][e],
                                  odd ? C.az[0][e] : C.az[1][e]);
            out[e] = __fmaf_rn(odd ? C.fc[0][e] : C.fc[1][e], E, c);
        }
        st_vec<V>(phi + sk, out);
        // copies of the updated cells, for the residual and the FP64 update
        if (odd && lane == 0) phi[sk + RL] = out[0];                  // cell nx+1 = cell 1
        if (!odd && lane == 31) phi[sk - q0 - 1] = out[V - 1];        // cell 0 = cell nx
        if (k == L.nz) st_vec<V>(phi + sb, out);                      // plane 0
        if (k == 1) st_vec<V>(phi + sb + (L.nz + 1) * L.rz, out);     // plane nz+1
        if (PY && j == L.ny) st_vec<V>(phi + sk - L.ny * L.hq, out);  // row 0
        if (PY && j == 1) st_vec<V>(phi + sk + L.ny * L.hq, out);     // row ny+1
#pragma unroll
        for (int e = 0; e < V; ++e) {
            zm[e] = z0[e];
            z0[e] = cur.zp[e];
        }
        if (k < k1) cur = nxt;   // the last plane loads no successor
    }
}

template <int PY, int V, int KZ>
__global__ void __launch_bounds__(256)
k_pot_sweep_w(pot_geom L, int cs, float* __restrict__ phi, const float* __restrict__ r,
              const float4* __restrict__ tab, const float* __restrict__ tabu) {
    __shared__ __align__(16) float ybuf[2][10][32 * V];
    const int j0 = 1 + (int)blockIdx.x * 8;
    const int k0 = 1 + (int)blockIdx.y * KZ;
    pot_coef<V> C;
    C.load(L, j0 + (int)threadIdx.y, V * (int)threadIdx.x, threadIdx.x, tab, tabu);
    pot_rows_sweep<PY, V, false>(L, cs, j0, k0, min(k0 + KZ - 1, L.nz), phi, r, C, ybuf);
}

// The warp-per-row sweeps of `iters` red-black iterations in one cooperative
// launch: every block keeps its rows' coefficients in registers for all of
// them, and a grid-wide barrier separates the colour sweeps (every block is
// resident: the host launches this only when the grid fits the device).  z
// is cut into gridDim.y chunks of nz/gridDim.y planes, rounded.
template <int PY, int V>
__global__ void __launch_bounds__(256)
k_pot_run_w(pot_geom L, int iters, float* __restrict__ phi, const float* __restrict__ r,
            const float4* __restrict__ tab, const float* __restrict__ tabu) {
    __shared__ __align__(16) float ybuf[2][10][32 * V];
    cg::grid_group grid = cg::this_grid();
    const int j0 = 1 + (int)blockIdx.x * 8;
    const int k0 = 1 + (int)(((long long)blockIdx.y * L.nz) / gridDim.y);
    const int k1 = (int)(((long long)(blockIdx.y + 1) * L.nz) / gridDim.y);
    pot_coef<V> C;
    C.load(L, j0 + (int)threadIdx.y, V * (int)threadIdx.x, threadIdx.x, tab, tabu);
    for (int it = 0; it < iters; ++it)
        for (int cs = 1; cs >= 0; --cs) {
            pot_rows_sweep<PY, V, true>(L, cs, j0, k0, k1, phi, r, C, ybuf);
            grid.sync();
        }
}

// The warp-per-row sweep with its planes staged in shared memory: a ring of
// POT_SLOTS plane slots, each holding the other colour's rows j0-1 ..
// j0+8, the swept colour's rows j0 .. j0+7 and their r~ rows, filled by
// cp.async two planes ahead of the plane being swept.  Every neighbour value
// is then a shared-memory read (the row ends wrap, x periodic); the
// arithmetic is pot_e's, so the result is k_pot_sweep's bit for bit.
#define POT_SLOTS 5
__device__ __forceinline__ void pot_cp16(unsigned dst, const float* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void pot_cp8(unsigned dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
}
template <int PY, int V, int KZ>
__global__ void __launch_bounds__(256)
k_pot_sweep_a(pot_geom L, int cs, float* __restrict__ phi, const float* __restrict__ r,
              const float4* __restrict__ tab, const float* __restrict__ tabu) {
    constexpr int NW = 8, RL = 32 * V;
    constexpr int ROWS = 3 * NW + 2;              // other rows j0-1..j0+NW, swept rows, r~ rows
    constexpr int SLOT = ROWS * RL;               // floats per slot
    extern __shared__ __align__(16) float pring[];   // [POT_SLOTS][ROWS][RL]
    const int lane = threadIdx.x, w = threadIdx.y;
    const int j0 = 1 + (int)blockIdx.x * NW;
    const int j = j0 + w;
    const int k0 = 1 + (int)blockIdx.y * KZ;
    const int k1 = min(k0 + KZ - 1, L.nz);
    const int q0 = V * lane;
    const int ncol = L.nx + 2;
    const int oh = 1 - cs;
    // staging: warp w copies the other colour's row j (and warps 0 / NW-1
    // the rows j0-1 / j0+NW), the swept row j and its r~ row, V floats a lane
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(pring) + 4u * q0;
    const int go = pot_row(L, oh, j, 0) + 4 + q0;
    const int gs = pot_row(L, cs, j, 0) + 4 + q0;
    const bool hlo = w == 0, hhi = w == NW - 1;
    const int gh = pot_row(L, oh, hlo ? j0 - 1 : j0 + NW, 0) + 4 + q0;
    const int hrow = hlo ? 0 : NW + 1;
    auto issue = [&](int kk) {   // plane kk into its slot
        const unsigned sl = sbase + 4u * (unsigned)(((kk % POT_SLOTS) + POT_SLOTS) % POT_SLOTS) * SLOT;
        const int pk = kk * L.rz;
        if constexpr (V == 4) {
            pot_cp16(sl + 4u * (w + 1) * RL, phi + go + pk);
            pot_cp16(sl + 4u * (NW + 2 + w) * RL, phi + gs + pk);
            pot_cp16(sl + 4u * (2 * NW + 2 + w) * RL, r + gs + pk);
            if (hlo || hhi) pot_cp16(sl + 4u * hrow * RL, phi + gh + pk);
        } else {
            pot_cp8(sl + 4u * (w + 1) * RL, phi + go + pk);
            pot_cp8(sl + 4u * (NW + 2 + w) * RL, phi + gs + pk);
            pot_cp8(sl + 4u * (2 * NW + 2 + w) * RL, r + gs + pk);
            if (hlo || hhi) pot_cp8(sl + 4u * hrow * RL, phi + gh + pk);
        }
    };
    // planes k0-1 .. k0+2 in flight while the coefficients load
    for (int kk = k0 - 1; kk <= k0 + 2; ++kk) {
        if (kk <= k1 + 1) issue(kk);
        asm volatile("cp.async.commit_group;\n" ::);
    }
    float axl[2][V], axr[2][V], ayl[2][V], ayr[2][V], az[2][V], fc[2][V];
    {
        const float4* t0 = tab + j * ncol + 2 * q0 + 1;
        const float* tu = tabu + j * pot_ncu(L.nx) + 2 * q0;
        float up[2 * V];
#pragma unroll
        for (int m = 0; m < 2 * V; m += 4) {
            const float4 u4 = __ldg(reinterpret_cast<const float4*>(tu + m));
            up[m] = u4.x;
            up[m + 1] = u4.y;
            up[m + 2] = u4.z;
            up[m + 3] = u4.w;
        }
#pragma unroll
        for (int m = 0; m < 2 * V; ++m) {
            const float4 c = __ldg(t0 + m);
            const int s = m & 1, e = m >> 1;
            axl[s][e] = c.x;
            ayl[s][e] = c.y;
            az[s][e] = c.z;
            fc[s][e] = c.w;
            ayr[s][e] = up[m];
            if (m > 0) axr[(m - 1) & 1][(m - 1) >> 1] = c.x;
        }
        axr[1][V - 1] = __shfl_sync(0xffffffffu, axl[0][0], (lane + 1) & 31);
    }
    const int sb = gs;   // the swept row j, plane 0, position q0
    for (int k = k0; k <= k1; ++k) {
        // planes up to k+1 complete (only plane k+2's group may be pending)
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        // the slot of plane k+3 held plane k-2, which no warp reads any more
        if (k + 3 <= k1 + 1) issue(k + 3);
        asm volatile("cp.async.commit_group;\n" ::);
        const float* Sm = pring + ((k - 1 + POT_SLOTS) % POT_SLOTS) * SLOT;
        const float* S0 = pring + (k % POT_SLOTS) * SLOT;
        const float* Sp = pring + ((k + 1) % POT_SLOTS) * SLOT;
        float zm[V], z0[V], zp[V], ym[V], yp[V], sv[V], rr[V];
        ld_vec<V>(zm, Sm + (w + 1) * RL + q0);
        ld_vec<V>(z0, S0 + (w + 1) * RL + q0);
        ld_vec<V>(zp, Sp + (w + 1) * RL + q0);
        ld_vec<V>(ym, S0 + w * RL + q0);
        ld_vec<V>(yp, S0 + (w + 2) * RL + q0);
        ld_vec<V>(sv, S0 + (NW + 2 + w) * RL + q0);
        ld_vec<V>(rr, S0 + (2 * NW + 2 + w) * RL + q0);
        const bool odd = ((cs + j + k) & 1) != 0;
        const float xs = odd ? S0[(w + 1) * RL + ((q0 + RL - 1) & (RL - 1))] : S0[(w + 1) * RL + ((q0 + V) & (RL - 1))];
        const int sk = sb + k * L.rz;
        float out[V];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const float xl = odd ? (e == 0 ? xs : z0[e > 0 ? e - 1 : 0]) : z0[e];
            const float xr = odd ? z0[e] : (e == V - 1 ? xs : z0[e + 1 < V ? e + 1 : e]);
            const float c = sv[e];
            const float E = pot_e(rr[e], c, xl, xr, ym[e], yp[e], zm[e], zp[e], odd ? axl[0][e] : axl[1][e],
                                  odd ? axr[0][e] : axr[1][e], odd ? ayl[0][e] : ayl[1][e],
                                  odd ? ayr[0][e] : ayr[1][e], odd ? az[0][e] : az[1][e]);
            out[e] = __fmaf_rn(odd ? fc[0][e] : fc[1][e], E, c);
        }
        st_vec<V>(phi + sk, out);
        if (odd && lane == 0) phi[sk + RL] = out[0];                  // cell nx+1 = cell 1
        if (!odd && lane == 31) phi[sk - q0 - 1] = out[V - 1];        // cell 0 = cell nx
        if (k == L.nz) st_vec<V>(phi + sb, out);                      // plane 0
        if (k == 1) st_vec<V>(phi + sb + (L.nz + 1) * L.rz, out);     // plane nz+1
        if (PY && j == L.ny) st_vec<V>(phi + sk - L.ny * L.hq, out);  // row 0
        if (PY && j == 1) st_vec<V>(phi + sk + L.ny * L.hq, out);     // row ny+1
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// u, v, w, p += the corrections Phi stands for, in FP64: the low faces of
// every interior cell (u(i) += mu_u (Phi(i-1) - Phi(i))/dx, v likewise
// except a wall face v(1), w likewise) and p += Phi/dt_gamma.  Each thread
// writes its own cell's entries only.
template <int PY>
__global__ void k_pot_apply(mdx_dims d, pot_geom L, double idx, double idy, double idz, double idt,
                            const double* __restrict__ mu, int plane_mu, double* __restrict__ u,
                            double* __restrict__ v, double* __restrict__ w, double* __restrict__ p,
                            const float* __restrict__ phi) {
    const long long np = (long long)d.nxp * d.nyp;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long rr = t / d.nx;
        const int j = (int)(rr % d.ny) + 1;
        const int k = (int)(rr / d.ny) + 1;
        const long long q = i + (long long)d.nxp * j;
        const double mu_u = plane_mu ? __ldg(mu + q) : 1.0;
        const double mu_v = plane_mu ? __ldg(mu + np + q) : 1.0;
        const double mu_w = plane_mu ? __ldg(mu + 2 * np + q) : 1.0;
        const double c = (double)__ldg(phi + pot_idx(L, i, j, k));
        const long long a = pidx(d, i, j, k);
        u[a] += idx * mu_u * ((double)__ldg(phi + pot_idx(L, i - 1, j, k)) - c);
        if (PY || j > 1) v[a] += idy * mu_v * ((double)__ldg(phi + pot_idx(L, i, j - 1, k)) - c);
        w[a] += idz * mu_w * ((double)__ldg(phi + pot_idx(L, i, j, k - 1)) - c);
        p[a] += c * idt;
    }
}

bool pot_supported(const mdx_ctx_t* ctx) {
    const mdx_dims& d = ctx->d;
    if (d.nx % 4 != 0 || d.nz % 2 != 0) return false;
    if (ctx->bc.is_periodic[1] && d.ny % 2 != 0) return false;
    const pot_geom L = pot_make(d);
    return 2LL * L.H + 64 < (1LL << 31) && (long long)(d.nx + 2) * (d.ny + 2) < (1LL << 31);
}

// One allocation for Phi and r~ (zeroed: the copies and the rows a wall
// reads stay 0 until written) and the column table.
int pot_alloc(mdx_ctx_t* ctx) {
    if (ctx->pt_base) return MDX_OK;
    const pot_geom L = pot_make(ctx->d);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t arr = up(sizeof(float) * 2 * (size_t)L.H);
    const size_t tab = up(sizeof(float4) * (size_t)(ctx->d.nx + 2) * (ctx->d.ny + 2));
    const size_t tabu = up(sizeof(float) * (size_t)pot_ncu(ctx->d.nx) * (ctx->d.ny + 2));
    const size_t total = 2 * arr + tab + tabu;
    char* base = nullptr;
    MDX_CUDA(ctx, cudaMalloc(&base, total));
    MDX_CUDA(ctx, cudaMemsetAsync(base, 0, total, ctx->stream));
    ctx->pt_phi = reinterpret_cast<float*>(base);
    ctx->pt_r = reinterpret_cast<float*>(base + arr);
    ctx->pt_tab = reinterpret_cast<float4*>(base + 2 * arr);
    ctx->pt_tabu = reinterpret_cast<float*>(base + 2 * arr + tab);
    ctx->pt_base = base;
    ctx->pt_bytes = total;
    return MDX_OK;
}

// Shapes of the potential-form sweep the autotuner tries (all give the same
// bits): positions per thread V, planes per march KZ, next-plane prefetch;
// shapes 8 and 9 are the warp-per-row kernel (V = nx/64), 10-12 the
// warp-per-row kernel with its planes staged by cp.async, 13-14 the
// warp-per-row sweeps of a whole block of iterations in one cooperative
// launch (when its grid fits the device; 13: z in as many chunks as fill the
// resident blocks, 14: chunks of 16 planes).
#define POT_SHAPES 15
static const int pot_shape_v[POT_SHAPES] = {2, 2, 4, 4, 2, 4, 2, 4, 0, 0, -1, -1, -1, -2, -2};
static const int pot_shape_kz[POT_SHAPES] = {8, 16, 8, 16, 4, 4, 8, 16, 8, 16, 8, 16, 4, 8, 16};
template <int PY>
static void (*pot_run_kernel(const pot_geom& L))(pot_geom, int, float*, const float*, const float4*, const float*) {
    return L.nx / 2 == 128 ? k_pot_run_w<PY, 4> : k_pot_run_w<PY, 2>;
}
// z chunks of the cooperative run: shape 13 as many as fill the device's
// resident blocks (at most nz), shape 14 chunks of 16 planes; 0 when the
// grid does not fit
static int pot_run_chunks(const mdx_ctx_t* ctx, int shape) {
    const mdx_dims& d = ctx->d;
    const pot_geom L = pot_make(d);
    int occ = 0, sms = 0;
    const bool py = ctx->bc.is_periodic[1] != 0;
    auto fn = py ? pot_run_kernel<1>(L) : pot_run_kernel<0>(L);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const long long slots = (long long)occ * sms, rb = d.ny / 8;
    const int nch = shape == 13 ? (int)std::min<long long>(d.nz, slots / rb) : (d.nz + 15) / 16;
    return (nch >= 1 && rb * nch <= slots) ? nch : 0;
}
static bool pot_shape_ok(const mdx_ctx_t* ctx, int shape) {
    const mdx_dims& d = ctx->d;
    const int half = d.nx / 2;
    if (pot_shape_v[shape] > 0) return half % pot_shape_v[shape] == 0;
    if (!((half == 64 || half == 128) && d.ny % 8 == 0)) return false;
    if (pot_shape_v[shape] == -2) return pot_run_chunks(ctx, shape) > 0;   // the grid must be resident at once
    return true;
}
// `iters` red-black iterations of shape 13 or 14: one cooperative launch
template <int PY>
static int pot_run(mdx_ctx_t* ctx, int shape, const pot_geom& L, int iters) {
    auto fn = pot_run_kernel<PY>(L);
    const int nch = pot_run_chunks(ctx, shape);
    if (nch <= 0) return mdx_fail(ctx, MDX_ERR_CUDA, "pot run: the cooperative grid does not fit the device");
    dim3 grid(L.ny / 8, nch);
    pot_geom Lc = L;
    int it = iters;
    float* phi = ctx->pt_phi;
    const float* r = ctx->pt_r;
    const float4* tab = ctx->pt_tab;
    const float* tabu = ctx->pt_tabu;
    void* args[] = {&Lc, &it, &phi, &r, &tab, &tabu};
    mdx_event_pair p{};
    mdx_timer_begin(ctx, MDX_T_SOR_SWEEP, &p);
    MDX_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)fn, grid, dim3(32, 8), args, 0, ctx->stream));
    mdx_timer_end(ctx, &p);
    return mdx_check_launch(ctx, "pot run (cooperative)");
}
template <int PY>
static int pot_launch(mdx_ctx_t* ctx, int shape, const pot_geom& L, int cs) {
    const int V = pot_shape_v[shape], KZ = pot_shape_kz[shape];
    if (V < 0) {
        void (*afn)(pot_geom, int, float*, const float*, const float4*, const float*) = nullptr;
        const bool v4 = L.nx / 2 == 128;
        if (KZ == 8) afn = v4 ? k_pot_sweep_a<PY, 4, 8> : k_pot_sweep_a<PY, 2, 8>;
        else if (KZ == 16) afn = v4 ? k_pot_sweep_a<PY, 4, 16> : k_pot_sweep_a<PY, 2, 16>;
        else afn = v4 ? k_pot_sweep_a<PY, 4, 4> : k_pot_sweep_a<PY, 2, 4>;
        const int smem = (int)(sizeof(float) * POT_SLOTS * (3 * 8 + 2) * (L.nx / 2));
        const unsigned bit = 1u << ((v4 ? 0 : 3) + (KZ == 8 ? 0 : KZ == 16 ? 1 : 2) + 6 * PY);
        if (!(ctx->pt_attr & bit)) {
            MDX_CUDA(ctx, cudaFuncSetAttribute(afn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            ctx->pt_attr |= bit;
        }
        dim3 agrid(L.ny / 8, (L.nz + KZ - 1) / KZ);
        MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "pot sweep staged", afn, agrid, dim3(32, 8), smem, L, cs, ctx->pt_phi,
                   ctx->pt_r, ctx->pt_tab, ctx->pt_tabu);
        return MDX_OK;
    }
    if (V == 0) {
        void (*wfn)(pot_geom, int, float*, const float*, const float4*, const float*) = nullptr;
        const bool v4 = L.nx / 2 == 128;
        if (KZ == 8) wfn = v4 ? k_pot_sweep_w<PY, 4, 8> : k_pot_sweep_w<PY, 2, 8>;
        else wfn = v4 ? k_pot_sweep_w<PY, 4, 16> : k_pot_sweep_w<PY, 2, 16>;
        dim3 wgrid(L.ny / 8, (L.nz + KZ - 1) / KZ);
        MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "pot sweep rows", wfn, wgrid, dim3(32, 8), 0, L, cs, ctx->pt_phi, ctx->pt_r,
                   ctx->pt_tab, ctx->pt_tabu);
        return MDX_OK;
    }
    dim3 block(32, 8);
    dim3 grid((L.nx / 2 / V + 31) / 32, (L.ny + 7) / 8, (L.nz + KZ - 1) / KZ);
    void (*kfn)(pot_geom, int, float*, const float*, const float4*) = nullptr;
    switch (shape) {
        case 0: kfn = k_pot_sweep<PY, 2, 8, true>; break;
        case 1: kfn = k_pot_sweep<PY, 2, 16, true>; break;
        case 2: kfn = k_pot_sweep<PY, 4, 8, true>; break;
        case 3: kfn = k_pot_sweep<PY, 4, 16, true>; break;
        case 4: kfn = k_pot_sweep<PY, 2, 4, true>; break;
        case 5: kfn = k_pot_sweep<PY, 4, 4, true>; break;
        case 6: kfn = k_pot_sweep<PY, 2, 8, false>; break;
        default: kfn = k_pot_sweep<PY, 4, 16, false>; break;
    }
    MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "pot sweep", kfn, grid, block, 0, L, cs, ctx->pt_phi, ctx->pt_r, ctx->pt_tab);
    return MDX_OK;
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

// One allocation for the eight colour-split FP32 arrays (du, dv, dw, dp, r
// and the fused pass's second du, dv, dw) and the tables, each part starting
// on a 256-byte boundary, all zero (the wall faces v(1), v(ny+1) stay 0 in
// both face buffers).
int mixed_alloc(mdx_ctx_t* ctx) {
    if (ctx->mx_base) return MDX_OK;
    const size_t n = (size_t)split_elems(ctx->d), np = (size_t)split_plane_elems(ctx->d);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t arr = up(sizeof(float) * n), mu = up(sizeof(float) * 3 * np), fac = up(sizeof(float) * np);
    const size_t total = 8 * arr + mu + fac;
    char* base = nullptr;
    MDX_CUDA(ctx, cudaMalloc(&base, total));
    MDX_CUDA(ctx, cudaMemsetAsync(base, 0, total, ctx->stream));
    float** arrs[8] = {&ctx->mx_du, &ctx->mx_dv, &ctx->mx_dw, &ctx->mx_dp, &ctx->mx_r,
                       &ctx->mx_du2, &ctx->mx_dv2, &ctx->mx_dw2};
    for (int a = 0; a < 8; ++a) *arrs[a] = reinterpret_cast<float*>(base + a * arr);
    ctx->mx_mu = reinterpret_cast<float*>(base + 8 * arr);
    ctx->mx_fac = reinterpret_cast<float*>(base + 8 * arr + mu);
    ctx->mx_base = base;
    ctx->mx_bytes = total;
    return MDX_OK;
}

// Tile shapes (TI x TJ columns, TK planes) of the fused pass, tried by the
// autotuner in this order; all give the same bits.
#define RB32_SHAPES 4
template <int PY>
static int rb32_launch(mdx_ctx_t* ctx, int shape, const mixed_params& P) {
    const mdx_dims& d = ctx->d;
    auto go = [&](auto kfn, int TI, int TJ, int TK) -> int {
        const int NT = (TI / 2 + 2) * (TJ + 3);
        const size_t smem = sizeof(float) * 5 * 12 * NT;   // SLOTS x FIELDS x threads
        const unsigned bit = 1u << (shape + 4 * PY);
        if (!(ctx->rb32_attr & bit)) {
            MDX_CUDA(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            ctx->rb32_attr |= bit;
        }
        dim3 block(TI / 2 + 2, TJ + 3);
        dim3 grid((d.nx + TI - 1) / TI, (d.ny + TJ - 1) / TJ, (d.nz + TK - 1) / TK);
        MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor rb32 fused", kfn, grid, block, smem, d, P, ctx->mx_du, ctx->mx_dv,
                   ctx->mx_dw, ctx->mx_du2, ctx->mx_dv2, ctx->mx_dw2, ctx->mx_dp, ctx->mx_r, ctx->mx_mu, ctx->mx_fac);
        return MDX_OK;
    };
    switch (shape) {
        case 0: MDX_TRY(go(k_rb32_fused<PY, 64, 8, 16>, 64, 8, 16)); break;
        case 1: MDX_TRY(go(k_rb32_fused<PY, 64, 16, 16>, 64, 16, 16)); break;
        case 2: MDX_TRY(go(k_rb32_fused<PY, 32, 8, 16>, 32, 8, 16)); break;
        default: MDX_TRY(go(k_rb32_fused<PY, 64, 8, 32>, 64, 8, 32)); break;
    }
    std::swap(ctx->mx_du, ctx->mx_du2);
    std::swap(ctx->mx_dv, ctx->mx_dv2);
    std::swap(ctx->mx_dw, ctx->mx_dw2);
    return MDX_OK;
}


}  // namespace

void mdx_mixed_free(mdx_ctx_t* ctx) {
    if (ctx->mx_base) cudaFree(ctx->mx_base);
    float** arrs[10] = {&ctx->mx_du, &ctx->mx_dv, &ctx->mx_dw, &ctx->mx_dp, &ctx->mx_r, &ctx->mx_mu, &ctx->mx_fac,
                        &ctx->mx_du2, &ctx->mx_dv2, &ctx->mx_dw2};
    for (auto a : arrs) *a = nullptr;
    ctx->mx_base = nullptr;
    ctx->mx_bytes = 0;
    if (ctx->pt_base) cudaFree(ctx->pt_base);
    ctx->pt_base = nullptr;
    ctx->pt_phi = ctx->pt_r = nullptr;
    ctx->pt_tab = nullptr;
    ctx->pt_tabu = nullptr;
    ctx->pt_bytes = 0;
}

// Called after u <- u*, the FP64 IBM factors of this projection and any
// warm-start guess; r0 and umax are ||div u*|| and max|u*| before the guess,
// atol the absolute floor.
int mdx_k_projection_redblack_mixed(mdx_ctx_t* ctx, double dg, mdx_solve_stats_t* st, bool* handled, double r0,
                                    double umax, double atol) {
    *handled = false;
    if (!mixed_supported(ctx) || ctx->opts.tol <= 0.0) return MDX_OK;
    *handled = true;
    // the potential form where the grid allows it, unless the face form is asked for
    const bool pot = ctx->opts.inner_form != 1 && pot_supported(ctx);
    if (pot) MDX_TRY(pot_alloc(ctx));
    else MDX_TRY(mixed_alloc(ctx));
    const mdx_dims& d = ctx->d;
    const pot_geom L = pot_make(d);
    const mdx_grid_t& g = ctx->g;
    const mdx_solver_opts_t& o = ctx->opts;
    const int py = ctx->bc.is_periodic[1] ? 1 : 0;
    double** f = ctx->f;
    const double idx = 1.0 / g.dx, idy = 1.0 / g.dy, idz = 1.0 / g.dz;
    mixed_params P{(float)idx, (float)idy, (float)idz, (float)(1.0 / dg)};
    const int nbt = (int)std::min<long long>(((long long)d.nxp * d.nyp + 255) / 256, 1024);
    const double inner_omega = o.inner_sor > 0.0 ? o.inner_sor : o.sor;
    const int plane_mu = ctx->mu_mode == MU_PLANE ? 1 : 0;
    if (pot)
        MDX_LAUNCH(ctx, MDX_T_OTHER, "pot tables", k_pot_tables, nbt, 256, 0, L, py, idx * idx, idy * idy, idz * idz,
                   inner_omega, ctx->mu, plane_mu, ctx->pt_tab, ctx->pt_tabu);
    else
        MDX_LAUNCH(ctx, MDX_T_OTHER, "mixed tables", k_mixed_tables, nbt, 256, 0, d, py, idx * idx, idy * idy,
                   idz * idz, inner_omega, ctx->mu, plane_mu, ctx->mx_mu, ctx->mx_fac);
    MDX_TRY(mdx_reduce_init(ctx));

    auto residual = [&](double* l2, double* umax) -> int {
        if (pot && py)
            MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "pot residual", k_pot_residual<1>, ctx->red_blocks, MDX_RED_THREADS, 0, d,
                       L, idx, idy, idz, f[MDX_UN], f[MDX_VN], f[MDX_WN], ctx->pt_r, ctx->red_part);
        else if (pot)
            MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "pot residual", k_pot_residual<0>, ctx->red_blocks, MDX_RED_THREADS, 0, d,
                       L, idx, idy, idz, f[MDX_UN], f[MDX_VN], f[MDX_WN], ctx->pt_r, ctx->red_part);
        else if (py)
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
        if (pot)
            MDX_LAUNCH(ctx, MDX_T_RESIDUAL, "pot corr residual", k_pot_corr_residual, ctx->red_blocks,
                       MDX_RED_THREADS, 0, d, L, ctx->pt_phi, ctx->pt_r, ctx->pt_tab, ctx->red_part);
        else if (py)
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
    // Inner sweeps: the colour sweeps (one launch per colour) when asked
    // for; otherwise the autotuner's choice among its candidates (the fused
    // red+black pass's tile shapes, the colour sweeps, the vector colour
    // sweeps), each timed on one block of iterations of the first
    // projections (all give the same bits).
    enum { CAND_SWEEPS = RB32_SHAPES, CAND_VEC2, CAND_VEC4, CAND_NUM };
    int cands[CAND_NUM], ncand = 0;
    if (o.sor_variant == MDX_SORV_SWEEPS) {
        cands[ncand++] = CAND_SWEEPS;
    } else if (o.sor_variant == MDX_SORV_FUSED8 || o.sor_variant == MDX_SORV_FUSED16) {
        for (int c = 0; c < RB32_SHAPES; ++c) cands[ncand++] = c;
    } else if (o.sor_variant == MDX_SORV_SPLIT || o.sor_variant == MDX_SORV_SPLITV) {
        cands[ncand++] = CAND_VEC2;
        cands[ncand++] = CAND_VEC4;
    } else {
        for (int c = 0; c < CAND_NUM; ++c) cands[ncand++] = c;
    }
    if (ncand > 1 && !ctx->tune_ev[0]) {
        MDX_CUDA(ctx, cudaEventCreate(&ctx->tune_ev[0]));
        MDX_CUDA(ctx, cudaEventCreate(&ctx->tune_ev[1]));
    }
    int used_kind = 1;   // 1 colour sweeps, 3 fused pass, 5 vector colour sweeps
    auto colour_sweeps = [&](int iters) -> int {
        const int na = d.nx / 2;
        dim3 block(32, 4, 2);
        dim3 grid((na + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
        for (int it = 0; it < iters; ++it)
            for (int parity = 0; parity < 2; ++parity) {
                auto kfn = py ? k_sor_sweep32<1> : k_sor_sweep32<0>;
                MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep fp32", kfn, grid, block, 0, d, P, parity, parity,
                           ctx->mx_du, ctx->mx_dv, ctx->mx_dw, ctx->mx_dp, ctx->mx_r, ctx->mx_mu, ctx->mx_fac);
            }
        return MDX_OK;
    };
    auto vector_sweeps = [&](int iters, int V) -> int {
        const int nwin = (d.nx / 2 + V) / V;   // windows covering positions 0 .. nx/2
        const long long nthr = (long long)nwin * d.ny * d.nz;
        const int nb = (int)((nthr + 255) / 256);
        auto kfn = V == 4 ? (py ? k_sor_sweep32v<1, 4> : k_sor_sweep32v<0, 4>)
                          : (py ? k_sor_sweep32v<1, 2> : k_sor_sweep32v<0, 2>);
        for (int it = 0; it < iters; ++it)
            for (int parity = 0; parity < 2; ++parity)
                MDX_LAUNCH(ctx, MDX_T_SOR_SWEEP, "sor sweep fp32 vec", kfn, nb, 256, 0, d, P, parity, parity, nwin,
                           ctx->mx_du, ctx->mx_dv, ctx->mx_dw, ctx->mx_dp, ctx->mx_r, ctx->mx_mu, ctx->mx_fac);
        return MDX_OK;
    };
    // the potential form's sweeps: the autotuner's choice among its shapes,
    // each timed on one block of iterations of the first projections (all
    // give the same bits)
    int pcands[POT_SHAPES], npc = 0;
    if (pot && o.sor_variant >= 1 && o.sor_variant <= POT_SHAPES && pot_shape_ok(ctx, o.sor_variant - 1))
        pcands[npc++] = o.sor_variant - 1;   // one shape asked for
    else if (pot)
        for (int c = 0; c < POT_SHAPES; ++c)
            if (pot_shape_ok(ctx, c)) pcands[npc++] = c;
    if (pot && npc > 1 && !ctx->tune_ev[0]) {
        MDX_CUDA(ctx, cudaEventCreate(&ctx->tune_ev[0]));
        MDX_CUDA(ctx, cudaEventCreate(&ctx->tune_ev[1]));
    }
    auto pot_sweeps = [&](int iters) -> int {
        mdx_event_pair run{};
        int cand = ctx->pt_tuned - 1;
        const bool tuning = cand < 0;
        int slot = 0;
        if (tuning) {
            while (slot < npc - 1 && ctx->pt_tune_ms[pcands[slot]] > 0.0) ++slot;
            cand = pcands[slot];
            if (npc > 1) MDX_CUDA(ctx, cudaEventRecord(ctx->tune_ev[0], ctx->stream));
        }
        mdx_sweep_run_begin(ctx, &run);
        if (pot_shape_v[cand] == -2 && iters > 0)
            MDX_TRY(py ? pot_run<1>(ctx, cand, L, iters) : pot_run<0>(ctx, cand, L, iters));
        else
            for (int it = 0; it < iters; ++it)
                for (int cs = 1; cs >= 0; --cs)   // first colour i+j+k odd, as the face form
                    MDX_TRY(py ? pot_launch<1>(ctx, cand, L, cs) : pot_launch<0>(ctx, cand, L, cs));
        mdx_sweep_run_end(ctx, &run, 2LL * iters);
        used_kind = 7;
        if (tuning && npc == 1) {
            ctx->pt_tuned = cand + 1;
        } else if (tuning) {
            MDX_CUDA(ctx, cudaEventRecord(ctx->tune_ev[1], ctx->stream));
            MDX_CUDA(ctx, cudaEventSynchronize(ctx->tune_ev[1]));
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, ctx->tune_ev[0], ctx->tune_ev[1]) == cudaSuccess && iters > 0)
                ctx->pt_tune_ms[cand] = ms > 0.f ? ms / iters : 1e-9;
            if (slot == npc - 1 && ctx->pt_tune_ms[cand] > 0.0) {
                int best = pcands[0];
                for (int t = 1; t < npc; ++t)
                    if (ctx->pt_tune_ms[pcands[t]] < ctx->pt_tune_ms[best]) best = pcands[t];
                ctx->pt_tuned = best + 1;
            }
        }
        return MDX_OK;
    };
    auto sweeps = [&](int iters) -> int {
        if (pot) return pot_sweeps(iters);
        mdx_event_pair run{};
        int cand = cands[0];
        bool tuning = false;
        int slot = 0;
        if (ncand > 1) {
            cand = ctx->rb32_tuned - 1;
            tuning = cand < 0;
            if (tuning) {
                while (slot < ncand - 1 && ctx->rb32_tune_ms[cands[slot]] > 0.0) ++slot;
                cand = cands[slot];
                MDX_CUDA(ctx, cudaEventRecord(ctx->tune_ev[0], ctx->stream));
            }
        }
        mdx_sweep_run_begin(ctx, &run);
        if (cand < RB32_SHAPES) {
            for (int it = 0; it < iters; ++it) MDX_TRY(py ? rb32_launch<1>(ctx, cand, P) : rb32_launch<0>(ctx, cand, P));
            used_kind = 3;
        } else if (cand == CAND_SWEEPS) {
            MDX_TRY(colour_sweeps(iters));
            used_kind = 1;
        } else {
            MDX_TRY(vector_sweeps(iters, cand == CAND_VEC4 ? 4 : 2));
            used_kind = 5;
        }
        mdx_sweep_run_end(ctx, &run);
        if (tuning) {
            MDX_CUDA(ctx, cudaEventRecord(ctx->tune_ev[1], ctx->stream));
            MDX_CUDA(ctx, cudaEventSynchronize(ctx->tune_ev[1]));
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, ctx->tune_ev[0], ctx->tune_ev[1]) == cudaSuccess && iters > 0)
                ctx->rb32_tune_ms[cand] = ms > 0.f ? ms / iters : 1e-9;
            if (slot == ncand - 1 && ctx->rb32_tune_ms[cand] > 0.0) {
                int best = cands[0];
                for (int t = 1; t < ncand; ++t)
                    if (ctx->rb32_tune_ms[cands[t]] < ctx->rb32_tune_ms[best]) best = cands[t];
                ctx->rb32_tuned = best + 1;
            }
        }
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
            if (pot) {
                const int nb = (int)std::min<long long>((d.nint + 255) / 256, 8192);
                auto kfn = py ? k_pot_apply<1> : k_pot_apply<0>;
                MDX_LAUNCH(ctx, MDX_T_OTHER, "pot apply", kfn, nb, 256, 0, d, L, idx, idy, idz, 1.0 / dg, ctx->mu,
                           plane_mu, f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], ctx->pt_phi);
                MDX_CUDA(ctx, cudaMemsetAsync(ctx->pt_phi, 0, sizeof(float) * 2 * (size_t)L.H, ctx->stream));
            } else {
                const long long n = d.npad;
                MDX_LAUNCH(ctx, MDX_T_OTHER, "mixed apply", k_mixed_apply,
                           (int)std::min<long long>((n + 255) / 256, 8192), 256, 0, d, f[MDX_UN], f[MDX_VN],
                           f[MDX_WN], f[MDX_PN], ctx->mx_du, ctx->mx_dv, ctx->mx_dw, ctx->mx_dp);
            }
            MDX_TRY(residual(&r, nullptr));
            if (!std::isfinite(r)) { s.status = MDX_ERR_NONFINITE; break; }
            if (r <= target) { s.status = MDX_OK; break; }
        }
        s.residual = r / r0;
    }
    s.iterations = it;
    // mixed path: 100 + outer FP64 corrections with the colour sweeps, 300 +
    // outer with the fused red+black pass, 500 + outer with the vector
    // colour sweeps, 700 + outer with the potential form
    s.variant = 100 * used_kind + outer;
    ctx->last = s;
    if (st) *st = s;
    return MDX_OK;
}
