// k_fft.cu -- FFT pressure path: divergence, batched 2-D real FFT over the
// periodic x-z planes, Thomas solve in y, inverse FFT and the projection.
// Reference: src/modules/pressure_solver.f90:77-173,
// src/modules/pressure/pressure_fft.f90:20-148 and the FFTW/cuFFT backends
// (pressure_backend_fftw.f90:22-93, pressure_backend_cufft.f90:29-122).
//
// Data flow per projection (HBM passes):
//   k_div_fftx   us,vs,ws -> spec        divergence/dt_gamma of one x row
//                                        (build_fft_rhs) and its real FFT in
//                                        shared memory
//   k_fftz<fwd>  spec -> spec            complex FFT along z per (kx, y)
//   k_thomas     spec -> spec            tridiagonal solve along y per mode
//   k_fftz<inv>  spec -> spec
//   k_ifftx      spec -> phi             inverse real FFT of one row, *1/(nx nz)
//   k_correct    us,vs,ws,phi,pn -> un,vn,wn,pn
//
// Where nx/2 and nz are 32 P (P = 1, 2, 4, 8, 16) each line is one warp's
// four-step transform: a P-point DFT in registers and a 32-point DFT across
// the lanes by shuffles (k_div_fftx_w, k_fftz_w, k_ifftx_w).  Other lengths
// use shared-memory Stockham transforms (the formulation of Govindaraju et
// al., "High performance discrete Fourier transforms on graphics
// processors", SC 2008) with radices 4, 2, 3, 5, 7.  The real transform of
// length nx is a complex transform of length nx/2 on packed even/odd samples
// plus the standard split step.  Twiddles are tables built on the host with
// long-double cosl/sinl.
//
// Parity: the divergence, Thomas and correction arithmetic follow the
// reference order with -fmad=false; the FFT differs from FFTW in operation
// order only, so FFT-path fields agree to rounding.
#include "mdx_internal.cuh"

#include <algorithm>
#include <cmath>
#include <type_traits>

// ---------------------------------------------------------------------------
// Plans and twiddles (host)
// ---------------------------------------------------------------------------
void mdx_fft_make_plan(int n, mdx_fft_plan* p, bool* ok) {
    p->n = n;
    p->nstages = 0;
    int m = n;
    *ok = true;
    for (int r : {4, 2, 3, 5, 7}) {
        while (m % r == 0) {
            if (p->nstages >= MDX_MAX_STAGES) { *ok = false; return; }
            p->radix[p->nstages++] = r;
            m /= r;
        }
    }
    if (m != 1) *ok = false;
    // one radix-2 stage is cheaper at the end than between radix-4 stages
    // only in bank terms; keep the order 4..4,2,3,5,7.
}

void mdx_fft_twiddles(int n, std::vector<double2>& tw) {
    tw.resize(n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < n; ++t) {
        const long double a = two_pi * (long double)t / (long double)n;
        tw[t] = make_double2((double)cosl(a), (double)(-sinl(a)));
    }
}

// ---------------------------------------------------------------------------
// Device complex helpers
// ---------------------------------------------------------------------------
// Complex types of the FP64 path (double2) and of the FP32 inner solve of
// the mixed-precision path (float2); one code for both.
template <typename C2> struct cx;
template <> struct cx<double2> {
    typedef double R;
    __device__ __forceinline__ static double2 mk(double a, double b) { return make_double2(a, b); }
};
template <> struct cx<float2> {
    typedef float R;
    __device__ __forceinline__ static float2 mk(float a, float b) { return make_float2(a, b); }
};
template <typename C2> __device__ __forceinline__ C2 cadd(C2 a, C2 b) { return cx<C2>::mk(a.x + b.x, a.y + b.y); }
template <typename C2> __device__ __forceinline__ C2 csub(C2 a, C2 b) { return cx<C2>::mk(a.x - b.x, a.y - b.y); }
template <typename C2> __device__ __forceinline__ C2 cmul(C2 a, C2 b) {
    return cx<C2>::mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C2> __device__ __forceinline__ C2 cconj(C2 a) { return cx<C2>::mk(a.x, -a.y); }
// a * (-i) and a * (+i)
template <typename C2> __device__ __forceinline__ C2 cmul_mi(C2 a) { return cx<C2>::mk(a.y, -a.x); }
template <typename C2> __device__ __forceinline__ C2 cmul_pi(C2 a) { return cx<C2>::mk(-a.y, a.x); }
// complex product with fused multiply-adds (the transforms only; the
// divergence, Thomas and correction arithmetic keep separate rounding)
__device__ __forceinline__ double fma_r(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_r(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <typename C2> __device__ __forceinline__ C2 cmul_f(C2 a, C2 b) {
    return cx<C2>::mk(fma_r(a.x, b.x, -(a.y * b.y)), fma_r(a.x, b.y, a.y * b.x));
}

// Twiddle exp(-+2 pi i t / n) from the forward table (conjugated for INV).
template <bool INV, typename C2>
__device__ __forceinline__ C2 twid(const C2* __restrict__ tw, int t) {
    C2 w = __ldg(tw + t);
    if (INV) w.y = -w.y;
    return w;
}

// Radix-r DFT in registers.  For r = 3, 5, 7 the roots come from the table:
// W_r^m = tw[m * (n/r) * tws].
template <bool INV, typename C2>
__device__ __forceinline__ void dft_r(C2* a, int r, const C2* __restrict__ tw, int root_step) {
    if (r == 2) {
        const C2 x0 = a[0], x1 = a[1];
        a[0] = cadd(x0, x1);
        a[1] = csub(x0, x1);
    } else if (r == 4) {
        const C2 x0 = a[0], x1 = a[1], x2 = a[2], x3 = a[3];
        const C2 s02 = cadd(x0, x2), d02 = csub(x0, x2);
        const C2 s13 = cadd(x1, x3), d13 = csub(x1, x3);
        const C2 rd13 = INV ? cmul_pi(d13) : cmul_mi(d13);
        a[0] = cadd(s02, s13);
        a[1] = cadd(d02, rd13);
        a[2] = csub(s02, s13);
        a[3] = csub(d02, rd13);
    } else {
        C2 b[7];
        for (int p = 0; p < r; ++p) {
            C2 acc = a[0];
            for (int q = 1; q < r; ++q) acc = cadd(acc, cmul(a[q], twid<INV>(tw, ((p * q) % r) * root_step)));
            b[p] = acc;
        }
        for (int p = 0; p < r; ++p) a[p] = b[p];
    }
}

// In-place (ping-pong) Stockham FFT of `nlines` lines of length n held in
// shared memory at A[line*ls + t]; all threads of the block participate.
// `tw` is a table of exp(-2 pi i t / N) with N = n * tws.  Returns the
// buffer holding the result (A or B).
template <bool INV, typename C2>
__device__ C2* smem_fft(C2* A, C2* B, int n, int nlines, int ls, const mdx_fft_plan& pl, const C2* __restrict__ tw,
                        int tws) {
    int Ns = 1;
    for (int s = 0; s < pl.nstages; ++s) {
        const int r = pl.radix[s];
        const int nr = n / r;
        const int total = nlines * nr;
        const int tstep = (n / (Ns * r)) * tws;
        const int root_step = nr * tws;
        for (int t = threadIdx.x; t < total; t += blockDim.x) {
            const int line = t / nr;
            const int jb = t - line * nr;
            const int k = jb % Ns;
            const C2* src = A + line * ls;
            C2 a[7];
            for (int q = 0; q < r; ++q) a[q] = src[jb + q * nr];
            if (Ns > 1)
                for (int q = 1; q < r; ++q) a[q] = cmul(a[q], twid<INV>(tw, q * k * tstep));
            dft_r<INV>(a, r, tw, root_step);
            C2* dst = B + line * ls;
            const int base = (jb / Ns) * Ns * r + k;
            for (int p = 0; p < r; ++p) dst[base + p * Ns] = a[p];
        }
        __syncthreads();
        C2* t = A; A = B; B = t;
        Ns *= r;
    }
    return A;
}

// ---------------------------------------------------------------------------
// Divergence (build_fft_rhs, pressure_solver.f90:102-111) + forward real FFT
// along x of each (k, j) row.  Rows are numbered r = (k-1) + nz*(j-1), the
// order of plane_hat(nxh, nz, ny).  R rows per block, M = nx/2.
// ---------------------------------------------------------------------------
template <typename C2>
__global__ void __launch_bounds__(256)
k_div_fftx(mdx_dims d, int R, double dx, double dy, double dz, mdx_dscal dgs, const double* __restrict__ us,
           const double* __restrict__ vs, const double* __restrict__ ws, C2* __restrict__ spec,
           mdx_fft_plan pl, const C2* __restrict__ twx) {
    const double dt_gamma = dgs.get();
    typedef typename cx<C2>::R RT;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    C2* sm = reinterpret_cast<C2*>(sm_raw);
    const int M = d.nx / 2;
    C2* A = sm;
    C2* B = sm + R * M;
    const int nrows = d.nz * d.ny;
    const int row0 = blockIdx.x * R;
    for (int t = threadIdx.x; t < R * M; t += blockDim.x) {
        const int rl = t / M, n = t - rl * M;
        const int row = row0 + rl;
        C2 z = cx<C2>::mk(0, 0);
        if (row < nrows) {
            const int k = row % d.nz + 1, j = row / d.nz + 1;
            double x[2];
            for (int e = 0; e < 2; ++e) {
                const int i = 2 * n + 1 + e;
                const long long c = pidx(d, i, j, k);
                x[e] = ((__ldg(us + c + 1) - __ldg(us + c)) / dx + (__ldg(vs + c + d.nxp) - __ldg(vs + c)) / dy +
                        (__ldg(ws + c + (long long)d.nxp * d.nyp) - __ldg(ws + c)) / dz) / dt_gamma;
            }
            z = cx<C2>::mk((RT)x[0], (RT)x[1]);
        }
        A[rl * M + n] = z;
    }
    __syncthreads();
    C2* Z = smem_fft<false>(A, B, M, R, M, pl, twx, 2);
    // split step: X_k = E_k + W^k O_k, E = (Z_k + conj Z_{M-k})/2, O = -i/2 (Z_k - conj Z_{M-k})
    const int nxh = M + 1;
    for (int t = threadIdx.x; t < R * nxh; t += blockDim.x) {
        const int rl = t / nxh, kx = t - rl * nxh;
        const int row = row0 + rl;
        if (row >= nrows) continue;
        const C2 zk = Z[rl * M + (kx == M ? 0 : kx)];
        const C2 zc = cconj(Z[rl * M + (kx == 0 ? 0 : M - kx)]);
        const RT h = (RT)0.5;
        const C2 e = cx<C2>::mk(h * (zk.x + zc.x), h * (zk.y + zc.y));
        const C2 o = cmul_mi(cx<C2>::mk(h * (zk.x - zc.x), h * (zk.y - zc.y)));
        const C2 X = cadd(e, cmul(__ldg(twx + kx), o));
        spec[(long long)row * nxh + kx] = X;
    }
}

// ---------------------------------------------------------------------------
// Complex FFT along z of spec(kx, :, j) for a tile of TX kx values per block.
// ---------------------------------------------------------------------------
template <bool INV, typename C2>
__global__ void __launch_bounds__(256)
k_fftz(mdx_dims d, int TX, C2* __restrict__ spec, mdx_fft_plan pl, const C2* __restrict__ twz) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    C2* sm = reinterpret_cast<C2*>(sm_raw);
    const int nz = d.nz, nxh = d.nxh, ls = nz + 1;
    C2* A = sm;
    C2* B = sm + TX * ls;
    const int ntiles = (nxh + TX - 1) / TX;
    const int j = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x - j * ntiles) * TX;
    C2* base = spec + (long long)j * nz * nxh;
    for (int t = threadIdx.x; t < TX * nz; t += blockDim.x) {
        const int c = t % TX, kz = t / TX;
        const int kx = kx0 + c;
        A[c * ls + kz] = (kx < nxh) ? base[(long long)kz * nxh + kx] : cx<C2>::mk(0, 0);
    }
    __syncthreads();
    C2* Z = smem_fft<INV>(A, B, nz, TX, ls, pl, twz, 1);
    for (int t = threadIdx.x; t < TX * nz; t += blockDim.x) {
        const int c = t % TX, kz = t / TX;
        const int kx = kx0 + c;
        if (kx < nxh) base[(long long)kz * nxh + kx] = Z[c * ls + kz];
    }
}

// ---------------------------------------------------------------------------
// Thomas tables, init_tridiag_coefficients (pressure_fft.f90:46-94): for each
// (kx, kz <= nz/2) the reciprocal pivots dinv_j and c'_j.  kz and nz-kz have
// bitwise-equal modified wavenumbers (sin is odd), so one table serves both.
// ---------------------------------------------------------------------------
__global__ void k_thomas_tables(int nxh, int nzh, int ny, double dyi2, const double* __restrict__ kxp,
                                const double* __restrict__ kzp, double* __restrict__ dinv, double* __restrict__ cp) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nxh * nzh) return;
    const int kx = m % nxh, kz = m / nxh;
    const long long plane = (long long)nxh * nzh;
    const double k_tot = kxp[kx] + kzp[kz];
    double cprev;
    if (kx == 0 && kz == 0) {
        dinv[m] = 1.0;
        cp[m] = 0.0;
        cprev = 0.0;
    } else {
        const double b = -dyi2 - k_tot, c = dyi2;
        const double di = 1.0 / b;
        dinv[m] = di;
        cprev = c * di;
        cp[m] = cprev;
    }
    const double a = dyi2;
    for (int jj = 2; jj <= ny; ++jj) {
        double b, c;
        if (jj < ny) { b = -2.0 * dyi2 - k_tot; c = dyi2; }
        else { b = -dyi2 - k_tot; c = 0.0; }
        const double denom = b - a * cprev;
        const double di = 1.0 / denom;
        const double cc = (jj < ny) ? c * di : 0.0;
        dinv[(jj - 1) * plane + m] = di;
        cp[(jj - 1) * plane + m] = cc;
        cprev = cc;
    }
}

// solve_tridiagonal_y, pressure_fft.f90:102-148: one thread per (kx, kz);
// the forward sweep stores dp in place, the back substitution overwrites it
// with the solution.  SKIP0: the (0, 0) mode is left to an FP64 solve and
// zeroed here (the mixed-precision path).
template <typename C2, bool SKIP0>
__global__ void __launch_bounds__(128)
k_thomas(mdx_dims d, typename cx<C2>::R dyi2, C2* __restrict__ spec, const typename cx<C2>::R* __restrict__ dinv,
         const typename cx<C2>::R* __restrict__ cp) {
    typedef typename cx<C2>::R RT;
    const int nxh = d.nxh, nz = d.nz, ny = d.ny, nzh = d.nz / 2 + 1;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nxh * nz) return;
    const int kx = m % nxh, kz = m / nxh;
    const int kzt = (kz <= nz / 2) ? kz : nz - kz;
    const int mt = kx + nxh * kzt;
    const long long tplane = (long long)nxh * nzh;
    const long long splane = (long long)nxh * nz;
    C2* col = spec + m;
    if (SKIP0 && kx == 0 && kz == 0) {
        for (int jj = 1; jj <= ny; ++jj) col[(jj - 1) * splane] = cx<C2>::mk(0, 0);
        return;
    }
    const RT a = dyi2;
    C2 dp;
    if (kx == 0 && kz == 0) {
        dp = cx<C2>::mk(0, 0);
    } else {
        const C2 r = col[0];
        const RT di = __ldg(dinv + mt);
        dp = cx<C2>::mk(r.x * di, r.y * di);
    }
    col[0] = dp;
    // The recurrences are serial in y, their operands are not: each block of
    // TU rows is loaded before it is used, so one thread keeps TU row loads in
    // flight (same arithmetic in the same order).
    constexpr int TU = 8;
    int jj = 2;
    for (; jj + TU - 1 <= ny; jj += TU) {
        C2 r[TU];
        RT di[TU];
#pragma unroll
        for (int u = 0; u < TU; ++u) {
            r[u] = col[(jj - 1 + u) * splane];
            di[u] = __ldg(dinv + (jj - 1 + u) * tplane + mt);
        }
#pragma unroll
        for (int u = 0; u < TU; ++u) {
            dp = cx<C2>::mk((r[u].x - a * dp.x) * di[u], (r[u].y - a * dp.y) * di[u]);
            col[(jj - 1 + u) * splane] = dp;
        }
    }
    for (; jj <= ny; ++jj) {
        const C2 r = col[(jj - 1) * splane];
        const RT di = __ldg(dinv + (jj - 1) * tplane + mt);
        dp = cx<C2>::mk((r.x - a * dp.x) * di, (r.y - a * dp.y) * di);
        col[(jj - 1) * splane] = dp;
    }
    C2 nxt = dp;  // plane_hat(ny) = dp(ny)
    jj = ny - 1;
    for (; jj - TU + 1 >= 1; jj -= TU) {
        C2 dj[TU];
        RT c[TU];
#pragma unroll
        for (int u = 0; u < TU; ++u) {
            dj[u] = col[(jj - 1 - u) * splane];
            c[u] = __ldg(cp + (jj - 1 - u) * tplane + mt);
        }
#pragma unroll
        for (int u = 0; u < TU; ++u) {
            nxt = cx<C2>::mk(dj[u].x - c[u] * nxt.x, dj[u].y - c[u] * nxt.y);
            col[(jj - 1 - u) * splane] = nxt;
        }
    }
    for (; jj >= 1; --jj) {
        const C2 dj = col[(jj - 1) * splane];
        const RT c = __ldg(cp + (jj - 1) * tplane + mt);
        nxt = cx<C2>::mk(dj.x - c * nxt.x, dj.y - c * nxt.y);
        col[(jj - 1) * splane] = nxt;
    }
}

// ---------------------------------------------------------------------------
// Inverse real FFT along x of each row (c2r contract: imaginary parts of the
// kx = 0 and kx = nx/2 bins are ignored), scaled by 1/(nx*nz) as
// scale_pressure_correction_* (pressure_backend_fftw.f90:80-93).
// ---------------------------------------------------------------------------
template <typename C2>
__global__ void __launch_bounds__(256)
k_ifftx(mdx_dims d, int R, typename cx<C2>::R scale, const C2* __restrict__ spec, typename cx<C2>::R* __restrict__ phi,
        mdx_fft_plan pl, const C2* __restrict__ twx) {
    typedef typename cx<C2>::R RT;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    C2* sm = reinterpret_cast<C2*>(sm_raw);
    const int M = d.nx / 2, nxh = M + 1;
    C2* A = sm;
    C2* B = sm + R * M;
    const int nrows = d.nz * d.ny;
    const int row0 = blockIdx.x * R;
    // Z'_k = (X_k + conj X_{M-k}) + i W^{-k} (X_k - conj X_{M-k}),  k < M
    for (int t = threadIdx.x; t < R * M; t += blockDim.x) {
        const int rl = t / M, k = t - rl * M;
        const int row = row0 + rl;
        C2 z = cx<C2>::mk(0, 0);
        if (row < nrows) {
            const C2* X = spec + (long long)row * nxh;
            C2 xk = X[k], xm = X[M - k];
            if (k == 0) { xk.y = 0; xm.y = 0; }   // kx = 0 and kx = M bins are real
            const C2 xc = cconj(xm);
            const C2 e = cadd(xk, xc);
            const C2 o = cmul(csub(xk, xc), cconj(__ldg(twx + k)));
            z = cadd(e, cmul_pi(o));
        }
        A[rl * M + k] = z;
    }
    __syncthreads();
    C2* Z = smem_fft<true>(A, B, M, R, M, pl, twx, 2);
    for (int t = threadIdx.x; t < R * M; t += blockDim.x) {
        const int rl = t / M, n = t - rl * M;
        const int row = row0 + rl;
        if (row >= nrows) continue;
        const C2 z = Z[rl * M + n];
        RT* out = phi + (long long)row * d.nx;
        out[2 * n] = z.x * scale;
        out[2 * n + 1] = z.y * scale;
    }
}

// ---------------------------------------------------------------------------
// Warp-shuffle transforms of length N = 32 P, P = 1, 2, 4, 8, 16: one warp
// per line, no block barrier inside a transform.  The length splits as
// N = P x 32: lane l holds x[l + 32 m] (m < P), takes the P-point DFT over m
// in registers, multiplies by W_N^(l p), and the 32-point DFT across the
// lanes runs for each p as five radix-2 decimation-in-frequency stages whose
// partner values come from __shfl_xor_sync:
//   X[p + P q] = sum_l W_32^(l q) W_N^(l p) sum_m x[l + 32 m] W_P^(m p).
// Lane l ends holding X[wout(l, q)] in v[q].  Roots come from the same
// long-double twiddle tables as the Stockham transforms: W_N^t = tw[t tws].
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int wlog2(int p) { return p <= 1 ? 0 : 1 + wlog2(p / 2); }
// reversal of the low `bits` (<= 4) bits of x
__host__ __device__ __forceinline__ constexpr int wbrev(int x, int bits) {
    return (((x & 1) << 3) | ((x & 2) << 1) | ((x & 4) >> 1) | ((x & 8) >> 3)) >> (4 - bits);
}

template <bool INV, int P, typename C2>
__device__ __forceinline__ void warp_fft(C2 (&v)[P], int lane, const C2* __restrict__ tw, int tws) {
    constexpr int N = 32 * P;
    constexpr int LP = wlog2(P);
    // P-point DIF in registers; v[i] then holds Y[brev(i)]
#pragma unroll
    for (int s = 0; s < LP; ++s) {
        const int h = P >> (s + 1);
#pragma unroll
        for (int b = 0; b < P; b += 2 * h) {
#pragma unroll
            for (int r = 0; r < h; ++r) {
                const C2 a0 = v[b + r], a1 = v[b + r + h];
                const C2 dd = csub(a0, a1);
                v[b + r] = cadd(a0, a1);
                if (r == 0) v[b + r + h] = dd;
                else if (2 * r == h) v[b + r + h] = INV ? cmul_pi(dd) : cmul_mi(dd);   // W_4^1 = -i
                else v[b + r + h] = cmul_f(dd, twid<INV>(tw, r * (N / (2 * h)) * tws));
            }
        }
    }
    C2 y[P];
#pragma unroll
    for (int i = 0; i < P; ++i) y[wbrev(i, LP)] = v[i];
#pragma unroll
    for (int p = 1; p < P; ++p) y[p] = cmul_f(y[p], twid<INV>(tw, lane * p * tws));
    // 32-point DIF across the lanes; the roots of the last two stages are
    // 1 and W_4 = -i, applied without a multiply.  For P >= 2 each stage
    // trades the lane bit h for register bit 0: a lane keeps the elements
    // whose register bit 0 equals its lane bit h, sends the other half to its
    // partner, and computes both outputs of the butterflies it holds, so a
    // stage moves P/2 elements per lane instead of P (wout gives where each
    // register ends up).
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int h = 16 >> s;
        const bool up = (lane & h) != 0;
        C2 w = cx<C2>::mk(1, 0);
        if (h > 2) w = twid<INV>(tw, (lane & (h - 1)) * (N / (2 * h)) * tws);   // W_2h^(l mod h)
        const bool rot = (h == 2) && (lane & 1);
        if (P == 1) {
            C2 o;
            o.x = __shfl_xor_sync(0xffffffffu, y[0].x, h);
            o.y = __shfl_xor_sync(0xffffffffu, y[0].y, h);
            if (!up) {
                y[0] = cadd(y[0], o);
            } else {
                const C2 dd = csub(o, y[0]);
                if (h > 2) y[0] = cmul_f(dd, w);
                else if (rot) y[0] = INV ? cmul_pi(dd) : cmul_mi(dd);
                else y[0] = dd;
            }
        } else {
#pragma unroll
            for (int p0 = 0; p0 < P; p0 += 2) {
                const C2 keep = up ? y[p0 + 1] : y[p0];
                const C2 send = up ? y[p0] : y[p0 + 1];
                C2 o;
                o.x = __shfl_xor_sync(0xffffffffu, send.x, h);
                o.y = __shfl_xor_sync(0xffffffffu, send.y, h);
                const C2 lo = up ? o : keep;     // the element of the lower lane of the pair
                const C2 hi = up ? keep : o;
                y[p0] = cadd(lo, hi);
                const C2 dd = csub(lo, hi);
                if (h > 2) y[p0 + 1] = cmul_f(dd, w);
                else if (rot) y[p0 + 1] = INV ? cmul_pi(dd) : cmul_mi(dd);
                else y[p0 + 1] = dd;
            }
        }
    }
#pragma unroll
    for (int p = 0; p < P; ++p) v[p] = y[p];
}

// Shared-memory swizzle of element k of a line: the natural-order reads
// (k = l + 32 m) and the transform's writes (k = wout(l, q)) of a warp both
// spread over all bank groups of G = 128 / sizeof(C2) elements (checked for
// every P and both element sizes in tests/test_fft_warp_model.py).
template <int P, typename C2> __device__ __forceinline__ int wsw(int k) {
    constexpr int G = 128 / (int)sizeof(C2);
    return P == 1 ? 0 : (k / P) & (G - 1);
}
template <int P, typename C2> __device__ __forceinline__ int wline(int k) { return k ^ wsw<P, C2>(k); }
// z tiles: G columns per z row; column c of row kz at kz*G + (c ^ wcol(kz))
template <int P, typename C2> __device__ __forceinline__ int wcol(int kz) {
    constexpr int G = 128 / (int)sizeof(C2);
    return (kz ^ wsw<P, C2>(kz)) & (G - 1);
}
__device__ __forceinline__ int brev5(int l) { return (int)(__brev((unsigned)l) >> 27); }
// Index of the transform output that warp_fft leaves in register q of lane
// l.  With the bit trades of the lane stages, the conceptual lane c is
// (q bit 0, l bits 0..3) and the conceptual register p is (l bit 4,
// q bits 1..); the output is X[p + P brev5(c)].
template <int P> __device__ __forceinline__ int wout(int lane, int q) {
    if (P == 1) return brev5(lane);
    const int p = (q & ~1) | (lane >> 4);
    const int cl = (q & 1) | ((lane & 15) << 1);
    return p + P * brev5(cl);
}
// one complex element global -> shared, asynchronous (cp.async; 16 bytes
// bypass L1, 8 bytes through it)
template <typename C2> __device__ __forceinline__ void cp_async_elem(C2* dst, const C2* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (sizeof(C2) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

// build_fft_rhs + forward real FFT along x, one warp per (k, j) row; M = nx/2 = 32 P.
template <int P, typename C2>
__global__ void __launch_bounds__(256, P >= 16 ? 2 : 4)
k_div_fftx_w(mdx_dims d, double dx, double dy, double dz, mdx_dscal dgs, const double* __restrict__ us,
             const double* __restrict__ vs, const double* __restrict__ ws, C2* __restrict__ spec,
             const C2* __restrict__ twx) {
    const double dt_gamma = dgs.get();
    typedef typename cx<C2>::R RT;
    constexpr int M = 32 * P;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    C2* buf = reinterpret_cast<C2*>(sm_raw) + warp * M;
    const int row = blockIdx.x * 8 + warp;
    if (row >= d.nz * d.ny) return;
    const int k = row % d.nz + 1, j = row / d.nz + 1;
    const long long plane = (long long)d.nxp * d.nyp;
    C2 v[P];
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int n = lane + 32 * m;
        double x[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const long long c = pidx(d, 2 * n + 1 + e, j, k);
            x[e] = ((__ldg(us + c + 1) - __ldg(us + c)) / dx + (__ldg(vs + c + d.nxp) - __ldg(vs + c)) / dy +
                    (__ldg(ws + c + plane) - __ldg(ws + c)) / dz) / dt_gamma;
        }
        v[m] = cx<C2>::mk((RT)x[0], (RT)x[1]);
    }
    warp_fft<false, P>(v, lane, twx, 2);
#pragma unroll
    for (int p = 0; p < P; ++p) buf[wline<P, C2>(wout<P>(lane, p))] = v[p];
    __syncwarp();
    // split step: X_k = E_k + W^k O_k, E = (Z_k + conj Z_{M-k})/2, O = -i/2 (Z_k - conj Z_{M-k})
    C2* X = spec + (long long)row * d.nxh;
    const RT h = (RT)0.5;
#pragma unroll
    for (int m = 0; m <= P; ++m) {
        const int kx = lane + 32 * m;
        if (m == P && lane != 0) break;
        const C2 zk = buf[wline<P, C2>(kx & (M - 1))];
        const C2 zc = cconj(buf[wline<P, C2>((M - kx) & (M - 1))]);
        const C2 e = cx<C2>::mk(h * (zk.x + zc.x), h * (zk.y + zc.y));
        const C2 o = cmul_mi(cx<C2>::mk(h * (zk.x - zc.x), h * (zk.y - zc.y)));
        X[kx] = cadd(e, cmul_f(__ldg(twx + kx), o));
    }
}

// Complex FFT along z of spec(kx, :, j), nz = 32 P: a block stages TX = G
// consecutive kx columns of one j (one 128-byte row segment per kz: 8 FP64
// or 16 FP32 complex values) through shared memory; one warp per column.
template <typename C2> __host__ __device__ constexpr int ztile_w() { return 128 / (int)sizeof(C2); }
template <bool INV, int P, typename C2>
__global__ void __launch_bounds__(32 * ztile_w<C2>(), P >= 16 ? 1 : (sizeof(C2) == 16 ? 4 : 2))
k_fftz_w(mdx_dims d, C2* __restrict__ spec, const C2* __restrict__ twz) {
    constexpr int NZ = 32 * P, TX = ztile_w<C2>();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    C2* S = reinterpret_cast<C2*>(sm_raw);
    const int nxh = d.nxh;
    const int ntiles = (nxh + TX - 1) / TX;
    const int j = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x - j * ntiles) * TX;
    C2* base = spec + (long long)j * NZ * nxh + kx0;
    const int ncol = min(TX, nxh - kx0);
    // the whole tile in flight at once: asynchronous copies into the
    // swizzled layout (columns >= ncol are neither read nor transformed)
#pragma unroll
    for (int e = 0; e < P; ++e) {
        const int t = threadIdx.x + e * 32 * TX;
        const int c = t % TX, kz = t / TX;
        if (c < ncol) cp_async_elem(&S[kz * TX + (c ^ wcol<P, C2>(kz))], base + (long long)kz * nxh + c);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
    if (c < ncol) {
        C2 v[P];
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const int kz = lane + 32 * m;
            v[m] = S[kz * TX + (c ^ wcol<P, C2>(kz))];
        }
        warp_fft<INV, P>(v, lane, twz, 1);
        __syncwarp();
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int kz = wout<P>(lane, p);
            S[kz * TX + (c ^ wcol<P, C2>(kz))] = v[p];
        }
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < P; ++e) {
        const int t = threadIdx.x + e * 32 * TX;
        const int c = t % TX, kz = t / TX;
        if (c < ncol) base[(long long)kz * nxh + c] = S[kz * TX + (c ^ wcol<P, C2>(kz))];
    }
}

// Inverse real FFT along x (c2r contract) scaled by 1/(nx nz), one warp per row.
template <int P, typename C2>
__global__ void __launch_bounds__(256)
k_ifftx_w(mdx_dims d, typename cx<C2>::R scale, const C2* __restrict__ spec, typename cx<C2>::R* __restrict__ phi,
          const C2* __restrict__ twx) {
    constexpr int M = 32 * P;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    C2* buf = reinterpret_cast<C2*>(sm_raw) + warp * M;
    const int row = blockIdx.x * 8 + warp;
    if (row >= d.nz * d.ny) return;
    const C2* X = spec + (long long)row * d.nxh;
    // Z'_k = (X_k + conj X_{M-k}) + i W^{-k} (X_k - conj X_{M-k}),  k < M
    C2 v[P];
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int kk = lane + 32 * m;
        C2 xk = X[kk], xm = X[M - kk];
        if (kk == 0) { xk.y = 0; xm.y = 0; }   // kx = 0 and kx = M bins are real
        const C2 xc = cconj(xm);
        const C2 e = cadd(xk, xc);
        const C2 o = cmul_f(csub(xk, xc), cconj(__ldg(twx + kk)));
        v[m] = cadd(e, cmul_pi(o));
    }
    warp_fft<true, P>(v, lane, twx, 2);
#pragma unroll
    for (int p = 0; p < P; ++p) buf[wline<P, C2>(wout<P>(lane, p))] = v[p];
    __syncwarp();
    C2* out = reinterpret_cast<C2*>(phi + (long long)row * d.nx);
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int n = lane + 32 * m;
        const C2 z = buf[wline<P, C2>(n)];
        out[n] = cx<C2>::mk(z.x * scale, z.y * scale);
    }
}

// ---------------------------------------------------------------------------
// apply_fft_pressure_correction, pressure_solver.f90:150-169.
// ---------------------------------------------------------------------------
template <bool IBM>
__global__ void __launch_bounds__(256)
k_correct(mdx_dims d, double dx, double dy, double dz, mdx_dscal dgs, const double* __restrict__ phi,
          const double* __restrict__ us, const double* __restrict__ vs, const double* __restrict__ ws,
          double* __restrict__ un, double* __restrict__ vn, double* __restrict__ wn, double* __restrict__ pn,
          const double* __restrict__ cu, const double* __restrict__ cv, const double* __restrict__ cw) {
    const double dt_gamma = dgs.get();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > d.nx || j > d.ny || k > d.nz) return;
    int im = i - 1, km = k - 1;
    if (im < 1) im = d.nx;
    if (km < 1) km = d.nz;
    const long long c = pidx(d, i, j, k);
    const double r = __ldg(phi + ridx(d, i, k, j));
    double u = (__ldg(us + c) - dt_gamma * (r - __ldg(phi + ridx(d, im, k, j))) / dx);
    double w = (__ldg(ws + c) - dt_gamma * (r - __ldg(phi + ridx(d, i, km, j))) / dz);
    if (IBM) {
        u = u / (1.0 + dt_gamma * __ldg(cu + c));
        w = w / (1.0 + dt_gamma * __ldg(cw + c));
    } else {
        u = u / 1.0;
        w = w / 1.0;
    }
    un[c] = u;
    wn[c] = w;
    pn[c] = pn[c] + r;
    if (j >= 2) {
        double v = (__ldg(vs + c) - dt_gamma * (r - __ldg(phi + ridx(d, i, k, j - 1))) / dy);
        if (IBM) v = v / (1.0 + dt_gamma * __ldg(cv + c));
        vn[c] = v;
    }
}

// Forward real FFT along x of each row of rhs(nx, nz, ny): rows r =
// (k-1) + nz*(j-1) of nx reals -> nx/2+1 complex in plane_hat order.
__global__ void __launch_bounds__(256)
k_fftx_r2c(mdx_dims d, int R, const double* __restrict__ rhs, double2* __restrict__ spec, mdx_fft_plan pl,
           const double2* __restrict__ twx) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = reinterpret_cast<double2*>(sm_raw);
    const int M = d.nx / 2;
    double2* A = sm;
    double2* B = sm + R * M;
    const int nrows = d.nz * d.ny;
    const int row0 = blockIdx.x * R;
    for (int t = threadIdx.x; t < R * M; t += blockDim.x) {
        const int rl = t / M, n = t - rl * M;
        const int row = row0 + rl;
        A[rl * M + n] = (row < nrows) ? make_double2(__ldg(rhs + (long long)row * d.nx + 2 * n),
                                                     __ldg(rhs + (long long)row * d.nx + 2 * n + 1))
                                      : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2* Z = smem_fft<false>(A, B, M, R, M, pl, twx, 2);
    const int nxh = M + 1;
    for (int t = threadIdx.x; t < R * nxh; t += blockDim.x) {
        const int rl = t / nxh, kx = t - rl * nxh;
        const int row = row0 + rl;
        if (row >= nrows) continue;
        const double2 zk = Z[rl * M + (kx == M ? 0 : kx)];
        const double2 zc = cconj(Z[rl * M + (kx == 0 ? 0 : M - kx)]);
        const double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
        const double2 o = cmul_mi(make_double2(0.5 * (zk.x - zc.x), 0.5 * (zk.y - zc.y)));
        spec[(long long)row * nxh + kx] = cadd(e, cmul(__ldg(twx + kx), o));
    }
}

// ---------------------------------------------------------------------------
// Walls in x or z on the FFT path.  With a wall (pressure Neumann) in x, the
// red-black method keeps the wall faces u(1), u(nx+1) at their boundary
// values and makes every cell divergence-free: the correction solves the
// pressure equation with a Neumann condition at both x faces.  That problem
// of length nx is the periodic one of length 2 nx on the even extension
// (mirror the right-hand side about each wall): the extension's solution is
// even, its ghost cells equal the cells they mirror, and the modified
// wavenumbers 4/dx^2 sin^2(pi k / 2nx) of length 2 nx are the cosine
// transform's eigenvalues.  So the periodic transforms solve it exactly on
// the extended grid dfft; the correction then leaves the wall faces alone.
// ---------------------------------------------------------------------------

// rhs(i,k,j) = div(u*)/dt_gamma on the physical grid, the faces as the
// boundary routine left them (build_fft_rhs's expression,
// pressure_solver.f90:77-115).
__global__ void k_div_rhs(mdx_dims d, double dx, double dy, double dz, mdx_dscal dgs, const double* __restrict__ us,
                          const double* __restrict__ vs, const double* __restrict__ ws, double* __restrict__ rhs) {
    const double dt_gamma = dgs.get();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > d.nx || j > d.ny || k > d.nz) return;
    const long long c = pidx(d, i, j, k);
    rhs[ridx(d, i, k, j)] = ((__ldg(us + c + 1) - __ldg(us + c)) / dx + (__ldg(vs + c + d.nxp) - __ldg(vs + c)) / dy +
                             (__ldg(ws + c + (long long)d.nxp * d.nyp) - __ldg(ws + c)) / dz) / dt_gamma;
}

// The extension: cell I of the solve grid is cell I (I <= n) or its mirror
// 2n + 1 - I of the physical grid in a direction with walls.
__global__ void k_extend(mdx_dims d, mdx_dims e, const double* __restrict__ rhs, double* __restrict__ ext) {
    const long long n = (long long)e.nx * e.nz * e.ny;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int I = (int)(t % e.nx) + 1;
        const long long r = t / e.nx;
        const int K = (int)(r % e.nz) + 1;
        const int j = (int)(r / e.nz) + 1;
        const int i = I <= d.nx ? I : 2 * d.nx + 1 - I;
        const int k = K <= d.nz ? K : 2 * d.nz + 1 - K;
        ext[t] = __ldg(rhs + ridx(d, i, k, j));
    }
}

// phi of the physical cells: the first nx x nz block of each plane.
__global__ void k_restrict(mdx_dims d, mdx_dims e, const double* __restrict__ ext, double* __restrict__ phi) {
    const long long n = d.nint;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long r = t / d.nx;
        const int k = (int)(r % d.nz) + 1;
        const int j = (int)(r / d.nz) + 1;
        phi[t] = __ldg(ext + ridx(e, i, k, j));
    }
}

// apply_fft_pressure_correction (pressure_solver.f90:117-173) with walls in
// x (WX) or z (WZ): a wall face u(1) / w(1) keeps its boundary value (no
// correction), as the red-black sweeps leave it; other faces as k_correct.
template <bool IBM, bool WX, bool WZ>
__global__ void __launch_bounds__(256)
k_correct_walls(mdx_dims d, double dx, double dy, double dz, mdx_dscal dgs, const double* __restrict__ phi,
                const double* __restrict__ us, const double* __restrict__ vs, const double* __restrict__ ws,
                double* __restrict__ un, double* __restrict__ vn, double* __restrict__ wn, double* __restrict__ pn,
                const double* __restrict__ cu, const double* __restrict__ cv, const double* __restrict__ cw) {
    const double dt_gamma = dgs.get();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > d.nx || j > d.ny || k > d.nz) return;
    int im = i - 1, km = k - 1;
    if (im < 1) im = d.nx;
    if (km < 1) km = d.nz;
    const long long c = pidx(d, i, j, k);
    const double r = __ldg(phi + ridx(d, i, k, j));
    if (WX && i == 1) {
        un[c] = __ldg(us + c);
    } else {
        double u = (__ldg(us + c) - dt_gamma * (r - __ldg(phi + ridx(d, im, k, j))) / dx);
        if (IBM) u = u / (1.0 + dt_gamma * __ldg(cu + c));
        un[c] = u;
    }
    if (WZ && k == 1) {
        wn[c] = __ldg(ws + c);
    } else {
        double w = (__ldg(ws + c) - dt_gamma * (r - __ldg(phi + ridx(d, i, km, j))) / dz);
        if (IBM) w = w / (1.0 + dt_gamma * __ldg(cw + c));
        wn[c] = w;
    }
    pn[c] = pn[c] + r;
    if (j >= 2) {
        double v = (__ldg(vs + c) - dt_gamma * (r - __ldg(phi + ridx(d, i, k, j - 1))) / dy);
        if (IBM) v = v / (1.0 + dt_gamma * __ldg(cv + c));
        vn[c] = v;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int rows_per_block(int M) { return M >= 1024 ? 1 : 1024 / M; }
static int ztile(int nz) {
    int tx = 2048 / (nz + 1);
    if (tx > 32) tx = 32;
    if (tx < 1) tx = 1;
    return tx;
}

// Warp-shuffle transform lengths: 32 P with P = 1, 2, 4, 8, 16 (0: none).
static int warp_p(int n) {
    if (n % 32 != 0) return 0;
    const int p = n / 32;
    return (p == 1 || p == 2 || p == 4 || p == 8 || p == 16) ? p : 0;
}
template <typename F> static int with_p(int p, F&& f) {
    switch (p) {
        case 1: return f(std::integral_constant<int, 1>());
        case 2: return f(std::integral_constant<int, 2>());
        case 4: return f(std::integral_constant<int, 4>());
        case 8: return f(std::integral_constant<int, 8>());
        case 16: return f(std::integral_constant<int, 16>());
    }
    return MDX_ERR_ARG;
}
static int fft_px(const mdx_ctx_t* ctx) { return ctx->opts.fft_kernel == 0 ? warp_p(ctx->d.nx / 2) : 0; }
static int fft_pz(const mdx_ctx_t* ctx) { return ctx->opts.fft_kernel == 0 ? warp_p(ctx->d.nz) : 0; }

template <typename C2> static int fft_warp_attrs(mdx_ctx_t* ctx) {
    const int px = warp_p(ctx->d.nx / 2), pz = warp_p(ctx->d.nz);
    if (px)
        MDX_TRY(with_p(px, [&](auto pc) -> int {
            constexpr int P = decltype(pc)::value;
            const int sm = 8 * 32 * P * (int)sizeof(C2);
            MDX_CUDA(ctx, cudaFuncSetAttribute(k_div_fftx_w<P, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            MDX_CUDA(ctx, cudaFuncSetAttribute(k_ifftx_w<P, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            return MDX_OK;
        }));
    if (pz)
        MDX_TRY(with_p(pz, [&](auto pc) -> int {
            constexpr int P = decltype(pc)::value;
            const int sm = 32 * P * 128;
            MDX_CUDA(ctx, cudaFuncSetAttribute(k_fftz_w<false, P, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            MDX_CUDA(ctx, cudaFuncSetAttribute(k_fftz_w<true, P, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            return MDX_OK;
        }));
    return MDX_OK;
}

// The three transform passes of a projection, warp-shuffle where the length
// allows and opts.fft_kernel is 0, shared-memory Stockham otherwise.
template <typename C2>
static int launch_div_fftx(mdx_ctx_t* ctx, const char* what, mdx_dscal dg, C2* spec, const C2* twx) {
    const mdx_dims& d = ctx->d;
    const mdx_grid_t& g = ctx->g;
    double** f = ctx->f;
    const int nrows = d.nz * d.ny;
    if (const int px = fft_px(ctx))
        return with_p(px, [&](auto pc) -> int {
            constexpr int P = decltype(pc)::value;
            auto kern = k_div_fftx_w<P, C2>;
            MDX_LAUNCH(ctx, MDX_T_FFT_FWD, what, kern, (nrows + 7) / 8, 256, 8 * 32 * P * sizeof(C2), d, g.dx, g.dy,
                       g.dz, dg, f[MDX_US], f[MDX_VS], f[MDX_WS], spec, twx);
            return MDX_OK;
        });
    const int M = d.nx / 2, R = rows_per_block(M);
    auto kern = k_div_fftx<C2>;
    MDX_LAUNCH(ctx, MDX_T_FFT_FWD, what, kern, (nrows + R - 1) / R, 256, sizeof(C2) * 2 * R * M, d, R, g.dx, g.dy,
               g.dz, dg, f[MDX_US], f[MDX_VS], f[MDX_WS], spec, ctx->plan_xh, twx);
    return MDX_OK;
}

template <bool INV, typename C2>
static int launch_fftz(mdx_ctx_t* ctx, const char* what, C2* spec, const C2* twz) {
    const mdx_dims& d = ctx->d;
    const int cls = INV ? MDX_T_FFT_INV : MDX_T_FFT_FWD;
    if (const int pz = fft_pz(ctx))
        return with_p(pz, [&](auto pc) -> int {
            constexpr int P = decltype(pc)::value;
            auto kern = k_fftz_w<INV, P, C2>;
            constexpr int TX = ztile_w<C2>();
            MDX_LAUNCH(ctx, cls, what, kern, ((d.nxh + TX - 1) / TX) * d.ny, 32 * TX, 32 * P * 128, d, spec, twz);
            return MDX_OK;
        });
    const int TX = ztile(d.nz);
    auto kern = k_fftz<INV, C2>;
    MDX_LAUNCH(ctx, cls, what, kern, ((d.nxh + TX - 1) / TX) * d.ny, 256, sizeof(C2) * 2 * TX * (d.nz + 1), d, TX,
               spec, ctx->plan_z, twz);
    return MDX_OK;
}

template <typename C2>
static int launch_ifftx(mdx_ctx_t* ctx, const char* what, typename cx<C2>::R scale, const C2* spec,
                        typename cx<C2>::R* phi, const C2* twx) {
    const mdx_dims& d = ctx->d;
    const int nrows = d.nz * d.ny;
    if (const int px = fft_px(ctx))
        return with_p(px, [&](auto pc) -> int {
            constexpr int P = decltype(pc)::value;
            auto kern = k_ifftx_w<P, C2>;
            MDX_LAUNCH(ctx, MDX_T_FFT_INV, what, kern, (nrows + 7) / 8, 256, 8 * 32 * P * sizeof(C2), d, scale, spec,
                       phi, twx);
            return MDX_OK;
        });
    const int M = d.nx / 2, R = rows_per_block(M);
    auto kern = k_ifftx<C2>;
    MDX_LAUNCH(ctx, MDX_T_FFT_INV, what, kern, (nrows + R - 1) / R, 256, sizeof(C2) * 2 * R * M, d, R, scale, spec,
               phi, ctx->plan_xh, twx);
    return MDX_OK;
}

// Walls in x or z: the pressure boundary condition must be Neumann (type 1,
// value 0) on both faces of that direction, and y must have walls with
// Neumann pressure (the Thomas solve).  Returns MDX_OK and sets the flags.
static int fft_wall_setup(mdx_ctx_t* ctx) {
    const mdx_bc_t& b = ctx->bc;
    ctx->fft_ext_x = b.is_periodic[0] ? 0 : 1;
    ctx->fft_ext_z = b.is_periodic[2] ? 0 : 1;
    if (!ctx->fft_ext_x && !ctx->fft_ext_z) return MDX_OK;
    auto neumann_p = [&](int dir) {
        return b.bc_type[bci(dir, 0, 0)] == 1 && b.bc_value[bci(dir, 0, 0)] == 0.0 && b.bc_type[bci(dir, 1, 0)] == 1 &&
               b.bc_value[bci(dir, 1, 0)] == 0.0;
    };
    for (int dir : {1, 3})
        if (!b.is_periodic[dir - 1] && !neumann_p(dir))
            return mdx_fail(ctx, MDX_ERR_ARG,
                            "FFT solver: a non-periodic %c direction needs Neumann pressure (type 1, value 0) on both "
                            "faces (the red-black solver takes other pressure conditions)", dir == 1 ? 'x' : 'z');
    if (b.is_periodic[1] || !neumann_p(2))
        return mdx_fail(ctx, MDX_ERR_ARG, "FFT solver with walls in x or z: y needs walls with Neumann pressure");
    if (ctx->opts.precision == MDX_PREC_MIXED)
        return mdx_fail(ctx, MDX_ERR_ARG, "FFT solver: mixed precision needs periodic x and z");
    return MDX_OK;
}

int mdx_fft_init(mdx_ctx_t* ctx) {
    const mdx_dims& d = ctx->d;
    if (d.nx % 2 != 0)
        return mdx_fail(ctx, MDX_ERR_ARG, "FFT solver: nx must be even (nx=%d)", d.nx);
    MDX_TRY(fft_wall_setup(ctx));
    // the solve grid: twice the length in a direction with walls
    mdx_dims e = d;
    e.nx = ctx->fft_ext_x ? 2 * d.nx : d.nx;
    e.nz = ctx->fft_ext_z ? 2 * d.nz : d.nz;
    e.nxp = e.nx + 2;
    e.nzp = e.nz + 2;
    e.nxh = e.nx / 2 + 1;
    e.npad = (long long)e.nxp * e.nyp * e.nzp;
    e.nint = (long long)e.nx * e.ny * e.nz;
    e.nspec = (long long)e.nxh * e.nz * e.ny;
    e.hs = split_stride(e.nx);
    ctx->dfft = e;
    const mdx_dims& D = e;
    bool ok1 = false, ok2 = false;
    mdx_fft_make_plan(D.nx / 2, &ctx->plan_xh, &ok1);
    mdx_fft_make_plan(D.nz, &ctx->plan_z, &ok2);
    if (!ok1 || !ok2)
        return mdx_fail(ctx, MDX_ERR_ARG, "FFT solver: nx/2=%d and nz=%d (solve grid) must factor into 2,3,5,7",
                        D.nx / 2, D.nz);
    if (D.nx / 2 > 4096 || D.nz > 4096)
        return mdx_fail(ctx, MDX_ERR_ARG, "FFT solver: nx/2 and nz of the solve grid must be <= 4096");
    std::vector<double2> tx, tz;
    mdx_fft_twiddles(D.nx, tx);
    mdx_fft_twiddles(D.nz, tz);
    MDX_CUDA(ctx, cudaMalloc(&ctx->tw_x, sizeof(double2) * D.nx));
    MDX_CUDA(ctx, cudaMalloc(&ctx->tw_z, sizeof(double2) * D.nz));
    MDX_CUDA(ctx, cudaMemcpy(ctx->tw_x, tx.data(), sizeof(double2) * D.nx, cudaMemcpyHostToDevice));
    MDX_CUDA(ctx, cudaMemcpy(ctx->tw_z, tz.data(), sizeof(double2) * D.nz, cudaMemcpyHostToDevice));
    MDX_CUDA(ctx, cudaMalloc(&ctx->spec, sizeof(double2) * D.nspec));
    if (!ctx->f[MDX_PHI]) {
        MDX_CUDA(ctx, cudaMalloc(&ctx->f[MDX_PHI], sizeof(double) * d.nint));
        MDX_CUDA(ctx, cudaMemset(ctx->f[MDX_PHI], 0, sizeof(double) * d.nint));
    }
    if (ctx->fft_ext_x || ctx->fft_ext_z) MDX_CUDA(ctx, cudaMalloc(&ctx->phi_ext, sizeof(double) * D.nint));

    // Modified wavenumbers on the host with libm sin, pressure_fft.f90:53,61
    // (of the solve grid's lengths).
    const double pi = 3.141592653589793;
    const int nzh = D.nz / 2 + 1;
    std::vector<double> kxp(D.nxh), kzp(D.nz);
    for (int ikx = 1; ikx <= D.nxh; ++ikx) {
        const int kx = ikx - 1;
        const double s = std::sin(pi * (double)kx / (double)D.nx);
        kxp[ikx - 1] = (4.0 / (ctx->g.dx * ctx->g.dx)) * (s * s);
    }
    for (int ikz = 1; ikz <= D.nz; ++ikz) {
        const int kz = (ikz <= D.nz / 2 + 1) ? ikz - 1 : ikz - D.nz - 1;
        const double s = std::sin(pi * (double)kz / (double)D.nz);
        kzp[ikz - 1] = (4.0 / (ctx->g.dz * ctx->g.dz)) * (s * s);
    }
    double *dkx = nullptr, *dkz = nullptr;
    MDX_CUDA(ctx, cudaMalloc(&dkx, sizeof(double) * D.nxh));
    MDX_CUDA(ctx, cudaMalloc(&dkz, sizeof(double) * D.nz));
    MDX_CUDA(ctx, cudaMemcpy(dkx, kxp.data(), sizeof(double) * D.nxh, cudaMemcpyHostToDevice));
    MDX_CUDA(ctx, cudaMemcpy(dkz, kzp.data(), sizeof(double) * D.nz, cudaMemcpyHostToDevice));
    const long long tsize = (long long)D.ny * D.nxh * nzh;
    MDX_CUDA(ctx, cudaMalloc(&ctx->thomas_dinv, sizeof(double) * tsize));
    MDX_CUDA(ctx, cudaMalloc(&ctx->thomas_cp, sizeof(double) * tsize));
    const double dyi2 = 1.0 / (ctx->g.dy * ctx->g.dy);
    const int nm = D.nxh * nzh;
    k_thomas_tables<<<(nm + 127) / 128, 128, 0, ctx->stream>>>(D.nxh, nzh, D.ny, dyi2, dkx, dkz, ctx->thomas_dinv,
                                                              ctx->thomas_cp);
    int rc = mdx_check_launch(ctx, "thomas tables");
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(dkx);
    cudaFree(dkz);
    if (rc != MDX_OK) return rc;

    const int M = D.nx / 2;
    const size_t smx = sizeof(double2) * 2 * rows_per_block(M) * M;
    const size_t smz = sizeof(double2) * 2 * ztile(D.nz) * (D.nz + 1);
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_div_fftx<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_fftx_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_ifftx<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_fftz<false, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_fftz<true, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
    if (!ctx->fft_ext_x && !ctx->fft_ext_z) MDX_TRY(fft_warp_attrs<double2>(ctx));
    return MDX_OK;
}

void mdx_fft_free(mdx_ctx_t* ctx) {
    cudaFree(ctx->spec32); ctx->spec32 = nullptr;
    cudaFree(ctx->tw_x32); ctx->tw_x32 = nullptr;
    cudaFree(ctx->tw_z32); ctx->tw_z32 = nullptr;
    cudaFree(ctx->phi32); ctx->phi32 = nullptr;
    cudaFree(ctx->dinv32); ctx->dinv32 = nullptr;
    cudaFree(ctx->cp32); ctx->cp32 = nullptr;
    cudaFree(ctx->rhs0); ctx->rhs0 = nullptr;
    cudaFree(ctx->phi0); ctx->phi0 = nullptr;
    cudaFree(ctx->spec); ctx->spec = nullptr;
    cudaFree(ctx->tw_x); ctx->tw_x = nullptr;
    cudaFree(ctx->tw_z); ctx->tw_z = nullptr;
    cudaFree(ctx->thomas_dinv); ctx->thomas_dinv = nullptr;
    cudaFree(ctx->thomas_cp); ctx->thomas_cp = nullptr;
    cudaFree(ctx->phi_ext); ctx->phi_ext = nullptr;
    ctx->fft_ext_x = ctx->fft_ext_z = 0;
}

// The projection with walls in x or z: divergence on the physical grid,
// its even extension, the Stockham transforms, Thomas and the inverse on the
// solve grid, the physical block of phi, the correction.
static int projection_fft_walls(mdx_ctx_t* ctx, mdx_dscal dg) {
    const mdx_dims& d = ctx->d;
    const mdx_dims& e = ctx->dfft;
    const mdx_grid_t& g = ctx->g;
    double** f = ctx->f;
    dim3 block(32, 4, 2);
    dim3 grid((d.nx + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
    MDX_LAUNCH(ctx, MDX_T_FFT_FWD, "div rhs", k_div_rhs, grid, block, 0, d, g.dx, g.dy, g.dz, dg, f[MDX_US], f[MDX_VS],
               f[MDX_WS], f[MDX_PHI]);
    const int nb = (int)std::min<long long>((e.nint + 255) / 256, 8192);
    MDX_LAUNCH(ctx, MDX_T_FFT_FWD, "extend rhs", k_extend, nb, 256, 0, d, e, f[MDX_PHI], ctx->phi_ext);
    const int M = e.nx / 2, R = rows_per_block(M), nrows = e.nz * e.ny;
    const size_t smx = sizeof(double2) * 2 * R * M;
    MDX_LAUNCH(ctx, MDX_T_FFT_FWD, "fft x (extended)", k_fftx_r2c, (nrows + R - 1) / R, 256, smx, e, R, ctx->phi_ext,
               ctx->spec, ctx->plan_xh, ctx->tw_x);
    const int TX = ztile(e.nz);
    const size_t smz = sizeof(double2) * 2 * TX * (e.nz + 1);
    const int zblocks = ((e.nxh + TX - 1) / TX) * e.ny;
    MDX_LAUNCH(ctx, MDX_T_FFT_FWD, "fft z (extended)", (k_fftz<false, double2>), zblocks, 256, smz, e, TX, ctx->spec,
               ctx->plan_z, ctx->tw_z);
    const int nm = e.nxh * e.nz;
    MDX_LAUNCH(ctx, MDX_T_THOMAS, "thomas (extended)", (k_thomas<double2, false>), (nm + 127) / 128, 128, 0, e,
               1.0 / (g.dy * g.dy), ctx->spec, ctx->thomas_dinv, ctx->thomas_cp);
    MDX_LAUNCH(ctx, MDX_T_FFT_INV, "ifft z (extended)", (k_fftz<true, double2>), zblocks, 256, smz, e, TX, ctx->spec,
               ctx->plan_z, ctx->tw_z);
    MDX_LAUNCH(ctx, MDX_T_FFT_INV, "ifft x (extended)", k_ifftx<double2>, (nrows + R - 1) / R, 256, smx, e, R,
               1.0 / (double)((long long)e.nx * e.nz), ctx->spec, ctx->phi_ext, ctx->plan_xh, ctx->tw_x);
    const int nbd = (int)std::min<long long>((d.nint + 255) / 256, 8192);
    MDX_LAUNCH(ctx, MDX_T_FFT_INV, "restrict phi", k_restrict, nbd, 256, 0, d, e, ctx->phi_ext, f[MDX_PHI]);
    // u <- u* on the whole padded arrays first, as the red-black projection
    // starts (pressure_redblack.f90:63-84): the edges and corners of the
    // ghost layers, which the face rules of apply_bc_redblack do not set and
    // the predictor's diagonal neighbours read, then hold u*'s values there
    const size_t bytes = sizeof(double) * (size_t)d.npad;
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_UN], f[MDX_US], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_VN], f[MDX_VS], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_WN], f[MDX_WS], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    auto go = [&](auto kern) -> int {
        MDX_LAUNCH(ctx, MDX_T_CORRECT, "correction (walls)", kern, grid, block, 0, d, g.dx, g.dy, g.dz, dg, f[MDX_PHI],
                   f[MDX_US], f[MDX_VS], f[MDX_WS], f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN], f[MDX_COEF_U],
                   f[MDX_COEF_V], f[MDX_COEF_W]);
        return MDX_OK;
    };
    const bool ibm = !ctx->ibm_zero, wx = ctx->fft_ext_x, wz = ctx->fft_ext_z;
    if (ibm) {
        if (wx && wz) return go(k_correct_walls<true, true, true>);
        if (wx) return go(k_correct_walls<true, true, false>);
        return go(k_correct_walls<true, false, true>);
    }
    if (wx && wz) return go(k_correct_walls<false, true, true>);
    if (wx) return go(k_correct_walls<false, true, false>);
    return go(k_correct_walls<false, false, true>);
}

// pressure_projection of the FFT builds, pressure_solver.f90:58-61.
int mdx_k_projection_fft(mdx_ctx_t* ctx, mdx_dscal dg) {
    if (!ctx->spec) return mdx_fail(ctx, MDX_ERR_STATE, "FFT solver workspace missing (its set-up failed)");
    if (ctx->fft_ext_x || ctx->fft_ext_z) return projection_fft_walls(ctx, dg);
    if (ctx->opts.precision == MDX_PREC_MIXED) {
        if (dg.p) return mdx_fail(ctx, MDX_ERR_STATE, "device-resident dt needs the FP64 FFT path");
        return mdx_k_projection_fft_mixed(ctx, dg.v);
    }
    const mdx_dims& d = ctx->d;
    const mdx_grid_t& g = ctx->g;
    double** f = ctx->f;
    auto kth = k_thomas<double2, false>;
    MDX_TRY(launch_div_fftx<double2>(ctx, "div+fft x", dg, ctx->spec, ctx->tw_x));
    MDX_TRY((launch_fftz<false, double2>(ctx, "fft z", ctx->spec, ctx->tw_z)));
    const int nm = d.nxh * d.nz;
    MDX_LAUNCH(ctx, MDX_T_THOMAS, "thomas", kth, (nm + 127) / 128, 128, 0, d, 1.0 / (g.dy * g.dy), ctx->spec,
               ctx->thomas_dinv, ctx->thomas_cp);
    MDX_TRY((launch_fftz<true, double2>(ctx, "ifft z", ctx->spec, ctx->tw_z)));
    const double scale = 1.0 / (double)(d.nx * d.nz);
    MDX_TRY(launch_ifftx<double2>(ctx, "ifft x", scale, ctx->spec, f[MDX_PHI], ctx->tw_x));
    dim3 block(32, 4, 2);
    dim3 grid((d.nx + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
    if (ctx->ibm_zero)
        MDX_LAUNCH(ctx, MDX_T_CORRECT, "correction", k_correct<false>, grid, block, 0, d, g.dx, g.dy, g.dz, dg,
                   f[MDX_PHI], f[MDX_US], f[MDX_VS], f[MDX_WS], f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN],
                   f[MDX_COEF_U], f[MDX_COEF_V], f[MDX_COEF_W]);
    else
        MDX_LAUNCH(ctx, MDX_T_CORRECT, "correction", k_correct<true>, grid, block, 0, d, g.dx, g.dy, g.dz, dg,
                   f[MDX_PHI], f[MDX_US], f[MDX_VS], f[MDX_WS], f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN],
                   f[MDX_COEF_U], f[MDX_COEF_V], f[MDX_COEF_W]);
    return MDX_OK;
}

// ---------------------------------------------------------------------------
// Mixed precision on the FFT path: the x-z FFTs and the Thomas solves run in
// FP32 inside FP64 defect correction.  Each pass takes the FP64 divergence of
// the current velocity (k_div_fftx computes it in FP64 and hands FP32 to the
// transform), solves for the FP32 correction phi, and corrects u, v, w and p
// in FP64.  The zero-wavenumber mode -- the near-singular Neumann problem in y
// pinned at j = 1 -- stays FP64: its right-hand side is the FP64 plane sum of
// the divergence, its Thomas solve uses the FP64 tables, and its solution is
// added to phi in FP64.  Without IBM the FFT-path correction makes the
// discrete divergence exactly L(phi_exact - phi) / dt_gamma, so the next pass
// solves the defect; passes repeat until ||div u|| <= max(tol ||div u*||,
// atol), the red-black path's stop rule.
// ---------------------------------------------------------------------------

// FP64 plane sums of the divergence/dt_gamma (the (0,0) Fourier coefficient of
// each y plane), one block per plane, fixed order.
__global__ void __launch_bounds__(256)
k_zero_rhs(mdx_dims d, double dx, double dy, double dz, double dt_gamma, const double* __restrict__ us,
           const double* __restrict__ vs, const double* __restrict__ ws, double* __restrict__ rhs0) {
    const int j = blockIdx.x + 1;
    double s = 0.0;
    for (int t = threadIdx.x; t < d.nx * d.nz; t += blockDim.x) {
        const int i = t % d.nx + 1, k = t / d.nx + 1;
        const long long c = pidx(d, i, j, k);
        s += ((__ldg(us + c + 1) - __ldg(us + c)) / dx + (__ldg(vs + c + d.nxp) - __ldg(vs + c)) / dy +
              (__ldg(ws + c + (long long)d.nxp * d.nyp) - __ldg(ws + c)) / dz) / dt_gamma;
    }
    __shared__ double sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) rhs0[j - 1] = sh[0];
}

// The (0, 0) column of k_thomas in FP64, scaled by 1/(nx nz) like the inverse
// transform: phi0[j] is that mode's contribution to phi on plane j.
__global__ void k_zero_solve(int ny, long long tplane, double dyi2, double scale, const double* __restrict__ dinv,
                             const double* __restrict__ cp, const double* __restrict__ rhs0, double* __restrict__ phi0) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double a = dyi2;
    double dp = 0.0;   // the pinned row j = 1
    phi0[0] = dp;
    for (int jj = 2; jj <= ny; ++jj) {
        dp = (rhs0[jj - 1] - a * dp) * dinv[(jj - 1) * tplane];
        phi0[jj - 1] = dp;
    }
    double nxt = dp;
    phi0[ny - 1] = nxt * scale;
    for (int jj = ny - 1; jj >= 1; --jj) {
        nxt = phi0[jj - 1] - cp[(jj - 1) * tplane] * nxt;
        phi0[jj - 1] = nxt;
    }
    for (int jj = 1; jj < ny; ++jj) phi0[jj - 1] *= scale;
}

__global__ void k_to_float(long long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        b[t] = (float)a[t];
}

// apply_fft_pressure_correction with phi = FP32 correction + FP64 zero mode.
template <bool IBM>
__global__ void __launch_bounds__(256)
k_correct_mixed(mdx_dims d, double dx, double dy, double dz, double dt_gamma, const float* __restrict__ phi,
                const double* __restrict__ phi0, const double* __restrict__ us, const double* __restrict__ vs,
                const double* __restrict__ ws, double* __restrict__ un, double* __restrict__ vn,
                double* __restrict__ wn, double* __restrict__ pn, const double* __restrict__ cu,
                const double* __restrict__ cv, const double* __restrict__ cw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > d.nx || j > d.ny || k > d.nz) return;
    int im = i - 1, km = k - 1;
    if (im < 1) im = d.nx;
    if (km < 1) km = d.nz;
    const long long c = pidx(d, i, j, k);
    const double p0 = __ldg(phi0 + j - 1);
    const double r = (double)__ldg(phi + ridx(d, i, k, j)) + p0;
    double u = __ldg(us + c) - dt_gamma * (r - ((double)__ldg(phi + ridx(d, im, k, j)) + p0)) / dx;
    double w = __ldg(ws + c) - dt_gamma * (r - ((double)__ldg(phi + ridx(d, i, km, j)) + p0)) / dz;
    if (IBM) {
        u = u / (1.0 + dt_gamma * __ldg(cu + c));
        w = w / (1.0 + dt_gamma * __ldg(cw + c));
    }
    un[c] = u;
    wn[c] = w;
    pn[c] = pn[c] + r;
    if (j >= 2) {
        const double rm = (double)__ldg(phi + ridx(d, i, k, j - 1)) + __ldg(phi0 + j - 2);
        double v = __ldg(vs + c) - dt_gamma * (r - rm) / dy;
        if (IBM) v = v / (1.0 + dt_gamma * __ldg(cv + c));
        vn[c] = v;
    }
}

static int fft_mixed_alloc(mdx_ctx_t* ctx) {
    if (ctx->spec32) return MDX_OK;
    const mdx_dims& d = ctx->d;
    const int nzh = d.nz / 2 + 1;
    const long long tsize = (long long)d.ny * d.nxh * nzh;
    MDX_CUDA(ctx, cudaMalloc(&ctx->spec32, sizeof(float2) * d.nspec));
    MDX_CUDA(ctx, cudaMalloc(&ctx->phi32, sizeof(float) * d.nint));
    MDX_CUDA(ctx, cudaMalloc(&ctx->dinv32, sizeof(float) * tsize));
    MDX_CUDA(ctx, cudaMalloc(&ctx->cp32, sizeof(float) * tsize));
    MDX_CUDA(ctx, cudaMalloc(&ctx->rhs0, sizeof(double) * d.ny));
    MDX_CUDA(ctx, cudaMalloc(&ctx->phi0, sizeof(double) * d.ny));
    std::vector<double2> tx, tz;
    mdx_fft_twiddles(d.nx, tx);
    mdx_fft_twiddles(d.nz, tz);
    std::vector<float2> fx(d.nx), fz(d.nz);
    for (int t = 0; t < d.nx; ++t) fx[t] = make_float2((float)tx[t].x, (float)tx[t].y);
    for (int t = 0; t < d.nz; ++t) fz[t] = make_float2((float)tz[t].x, (float)tz[t].y);
    MDX_CUDA(ctx, cudaMalloc(&ctx->tw_x32, sizeof(float2) * d.nx));
    MDX_CUDA(ctx, cudaMalloc(&ctx->tw_z32, sizeof(float2) * d.nz));
    MDX_CUDA(ctx, cudaMemcpy(ctx->tw_x32, fx.data(), sizeof(float2) * d.nx, cudaMemcpyHostToDevice));
    MDX_CUDA(ctx, cudaMemcpy(ctx->tw_z32, fz.data(), sizeof(float2) * d.nz, cudaMemcpyHostToDevice));
    const int nb = (int)std::min<long long>((tsize + 255) / 256, 4096);
    MDX_LAUNCH(ctx, MDX_T_OTHER, "thomas tables fp32", k_to_float, nb, 256, 0, tsize, ctx->thomas_dinv, ctx->dinv32);
    MDX_LAUNCH(ctx, MDX_T_OTHER, "thomas tables fp32", k_to_float, nb, 256, 0, tsize, ctx->thomas_cp, ctx->cp32);
    const int M = d.nx / 2;
    const size_t smx = sizeof(float2) * 2 * rows_per_block(M) * M;
    const size_t smz = sizeof(float2) * 2 * ztile(d.nz) * (d.nz + 1);
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_div_fftx<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_ifftx<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_fftz<false, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_fftz<true, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
    MDX_TRY(fft_warp_attrs<float2>(ctx));
    return MDX_OK;
}

int mdx_k_projection_fft_mixed(mdx_ctx_t* ctx, double dg) {
    MDX_TRY(fft_mixed_alloc(ctx));
    const mdx_dims& d = ctx->d;
    const mdx_grid_t& g = ctx->g;
    const mdx_solver_opts_t& o = ctx->opts;
    double** f = ctx->f;
    const int nm = d.nxh * d.nz;
    const double dyi2 = 1.0 / (g.dy * g.dy);
    const double scale = 1.0 / (double)(d.nx * d.nz);
    const long long tplane = (long long)d.nxh * (d.nz / 2 + 1);
    const size_t pad = sizeof(double) * d.npad;
    auto kth = k_thomas<float2, true>;
    auto kcor = ctx->ibm_zero ? k_correct_mixed<false> : k_correct_mixed<true>;
    dim3 block(32, 4, 2);
    dim3 grid((d.nx + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
    // the stop rule of the red-black path, on ||div u*|| before the first pass
    double r0 = 0.0, linf = 0.0, umax = 0.0;
    MDX_TRY(mdx_k_div_norms(ctx, f[MDX_US], f[MDX_VS], f[MDX_WS], &r0, &linf, &umax));
    const double tol = o.tol > 0.0 ? o.tol : 1e-10;
    const double atol = (o.atol < 0.0) ? mdx_div_floor(ctx, umax) : o.atol;
    const double target = std::max(tol * r0, atol);
    mdx_solve_stats_t st{};
    st.residual0 = r0;
    st.atol = atol;
    st.status = MDX_NOT_CONVERGED;
    double r = r0;
    int pass = 0;
    const int max_pass = 8;
    while (pass < max_pass) {
        if (pass > 0) {   // the corrected state becomes the next pass's u*
            MDX_TRY(mdx_k_apply_bc(ctx));
            MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_US], f[MDX_UN], pad, cudaMemcpyDeviceToDevice, ctx->stream));
            MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_VS], f[MDX_VN], pad, cudaMemcpyDeviceToDevice, ctx->stream));
            MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_WS], f[MDX_WN], pad, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        MDX_TRY(launch_div_fftx<float2>(ctx, "div+fft x fp32", dg, ctx->spec32, ctx->tw_x32));
        MDX_LAUNCH(ctx, MDX_T_FFT_FWD, "zero mode rhs", k_zero_rhs, d.ny, 256, 0, d, g.dx, g.dy, g.dz, dg, f[MDX_US],
                   f[MDX_VS], f[MDX_WS], ctx->rhs0);
        MDX_TRY((launch_fftz<false, float2>(ctx, "fft z fp32", ctx->spec32, ctx->tw_z32)));
        MDX_LAUNCH(ctx, MDX_T_THOMAS, "thomas fp32", kth, (nm + 127) / 128, 128, 0, d, (float)dyi2, ctx->spec32,
                   ctx->dinv32, ctx->cp32);
        MDX_LAUNCH(ctx, MDX_T_THOMAS, "zero mode fp64", k_zero_solve, 1, 32, 0, d.ny, tplane, dyi2, scale,
                   ctx->thomas_dinv, ctx->thomas_cp, ctx->rhs0, ctx->phi0);
        MDX_TRY((launch_fftz<true, float2>(ctx, "ifft z fp32", ctx->spec32, ctx->tw_z32)));
        MDX_TRY(launch_ifftx<float2>(ctx, "ifft x fp32", (float)scale, ctx->spec32, ctx->phi32, ctx->tw_x32));
        MDX_LAUNCH(ctx, MDX_T_CORRECT, "correction mixed", kcor, grid, block, 0, d, g.dx, g.dy, g.dz, dg, ctx->phi32,
                   ctx->phi0, f[MDX_US], f[MDX_VS], f[MDX_WS], f[MDX_UN], f[MDX_VN], f[MDX_WN], f[MDX_PN],
                   f[MDX_COEF_U], f[MDX_COEF_V], f[MDX_COEF_W]);
        ++pass;
        MDX_TRY(mdx_k_div_norms(ctx, f[MDX_UN], f[MDX_VN], f[MDX_WN], &r, &linf));
        if (!std::isfinite(r)) { st.status = MDX_ERR_NONFINITE; break; }
        if (r <= target) { st.status = MDX_OK; break; }
    }
    st.iterations = pass;
    st.residual = r0 > 0.0 ? r / r0 : 0.0;
    st.variant = 200 + pass;   // FFT mixed path: 200 + FP64 passes
    ctx->last = st;
    return MDX_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free FFT pressure solve.
//
// mdx_solve_pressure_fft_noalloc runs the same kernels as the context path
// (x real FFT, z FFT, Thomas solve in y, inverse FFTs, 1/(nx*nz) scale) on
// device arrays the caller owns, with every intermediate array (spectrum,
// Thomas tables, twiddles, modified wavenumbers) placed in the file-scope
// array below instead of memory from cudaMalloc.  It exists for callers that
// cannot allocate device memory through the CUDA runtime themselves, such as
// an OpenMP-offload Fortran program whose device arrays belong to the OpenMP
// runtime (the reference hands cuFFT such arrays through use_device_addr).
//
// The array is MDX_NOALLOC_SCRATCH_BYTES per device and lives as long as the
// library is loaded.  Its device address is looked up (cudaGetSymbolAddress)
// on a device's first call, and again on every later call made outside a
// stream capture, so the first call on a device should come before any
// stream capture.  All calls share the array and it keeps the last call's
// contents; every call rewrites all of it that it reads (tables, twiddles
// and wavenumbers are rebuilt on the device each call), so nothing needs
// clearing.  Calls that overlap on the GPU (two streams, or two host
// threads) race on the array.
// ---------------------------------------------------------------------------
#include <mutex>

#define MDX_NOALLOC_SCRATCH_BYTES (8u << 20)
#define MDX_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char mdx_noalloc_scratch[MDX_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[MDX_NOALLOC_MAX_DEVICES] = {nullptr};

static size_t noalloc_align(size_t b) { return (b + 255) & ~(size_t)255; }

// The allocation-free solve's trigonometric tables: twiddles
// W_n^t = exp(-2 pi i t / n) of the x (n = nx) and z (n = nz) transforms,
// and the modified wavenumbers 4/h^2 sin^2(pi k / n) with k = ikx - 1 for
// x and the signed kz for z (pressure_fft.f90:53,61).
__global__ void k_noalloc_trig(int nx, int nz, int nxh, double dx, double dz, double2* __restrict__ twx,
                               double2* __restrict__ twz, double* __restrict__ kxp, double* __restrict__ kzp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double s, c;
    if (t < nx) {
        sincospi(2.0 * (double)t / (double)nx, &s, &c);
        twx[t] = make_double2(c, -s);
    }
    if (t < nz) {
        sincospi(2.0 * (double)t / (double)nz, &s, &c);
        twz[t] = make_double2(c, -s);
        const int kz = (t + 1 <= nz / 2 + 1) ? t : t - nz;
        const double q = sinpi((double)kz / (double)nz);
        kzp[t] = (4.0 / (dz * dz)) * (q * q);
    }
    if (t < nxh) {
        const double q = sinpi((double)t / (double)nx);
        kxp[t] = (4.0 / (dx * dx)) * (q * q);
    }
}

extern "C" int mdx_solve_pressure_fft_noalloc(const double* rhs, double* phi, int nx, int ny, int nz, double dx,
                                              double dy, double dz, void* stream) {
    if (!rhs || !phi) return mdx_fail(nullptr, MDX_ERR_ARG, "noalloc solve: null rhs or phi");
    if (nx < 2 || ny < 2 || nz < 2 || nx % 2 != 0)
        return mdx_fail(nullptr, MDX_ERR_ARG, "noalloc solve: need even nx >= 2, ny >= 2, nz >= 2 (got %d %d %d)", nx,
                        ny, nz);
    if (!(dx > 0.0 && dy > 0.0 && dz > 0.0)) return mdx_fail(nullptr, MDX_ERR_ARG, "noalloc solve: dx, dy, dz must be > 0");
    mdx_fft_plan plx, plz;
    bool ok1 = false, ok2 = false;
    mdx_fft_make_plan(nx / 2, &plx, &ok1);
    mdx_fft_make_plan(nz, &plz, &ok2);
    if (!ok1 || !ok2 || nx / 2 > 4096 || nz > 4096)
        return mdx_fail(nullptr, MDX_ERR_ARG, "noalloc solve: nx/2=%d and nz=%d must factor into 2,3,5,7 (<= 4096)",
                        nx / 2, nz);
    mdx_dims d{};
    d.nx = nx; d.ny = ny; d.nz = nz;
    d.nxp = nx + 2; d.nyp = ny + 2; d.nzp = nz + 2;
    d.nxh = nx / 2 + 1;
    d.nint = (long long)nx * ny * nz;
    d.nspec = (long long)d.nxh * nz * ny;
    const int nzh = nz / 2 + 1;
    // scratch layout: spectrum | dinv | c' | twiddles x | twiddles z | kx^2 | kz^2
    const size_t b_spec = noalloc_align(sizeof(double2) * (size_t)d.nspec);
    const size_t b_tab = noalloc_align(sizeof(double) * (size_t)ny * d.nxh * nzh);
    const size_t b_twx = noalloc_align(sizeof(double2) * (size_t)nx);
    const size_t b_twz = noalloc_align(sizeof(double2) * (size_t)nz);
    const size_t b_kx = noalloc_align(sizeof(double) * (size_t)d.nxh);
    const size_t b_kz = noalloc_align(sizeof(double) * (size_t)nz);
    const size_t need = b_spec + 2 * b_tab + b_twx + b_twz + b_kx + b_kz;
    if (need > MDX_NOALLOC_SCRATCH_BYTES)
        return mdx_fail(nullptr, MDX_ERR_ARG,
                        "noalloc solve: grid %dx%dx%d needs %zu bytes of scratch, the static array holds %u",
                        nx, ny, nz, need, (unsigned)MDX_NOALLOC_SCRATCH_BYTES);

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mdx_fail(nullptr, MDX_ERR_NO_DEVICE, "noalloc solve: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= MDX_NOALLOC_MAX_DEVICES) return mdx_fail(nullptr, MDX_ERR_ARG, "noalloc solve: device %d", dev);
    cudaStream_t st = (cudaStream_t)stream;
    // The array's device address belongs to the context current now.  Outside
    // a stream capture it is looked up on every call, so that a context made
    // current since the last call (a device reset, or a runtime that brings
    // its own context) gets its own address; during a capture the lookup is
    // not made (it may load the module, which a capture forbids) and the
    // address from the last call on this device outside a capture is used.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        (void)cudaGetLastError();
        cap = cudaStreamCaptureStatusActive;
    }
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (cap == cudaStreamCaptureStatusNone) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, mdx_noalloc_scratch);
            if (e != cudaSuccess)
                return mdx_fail(nullptr, MDX_ERR_CUDA, "noalloc solve: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            g_noalloc_addr[dev] = p;
        } else if (!g_noalloc_addr[dev]) {
            return mdx_fail(nullptr, MDX_ERR_STATE,
                            "noalloc solve: first call on device %d made during a stream capture; call once before", dev);
        }
        base = (unsigned char*)g_noalloc_addr[dev];
    }
    double2* spec = (double2*)base;
    double* dinv = (double*)(base + b_spec);
    double* cp = (double*)(base + b_spec + b_tab);
    double2* twx = (double2*)(base + b_spec + 2 * b_tab);
    double2* twz = (double2*)(base + b_spec + 2 * b_tab + b_twx);
    double* kxp = (double*)(base + b_spec + 2 * b_tab + b_twx + b_twz);
    double* kzp = (double*)(base + b_spec + 2 * b_tab + b_twx + b_twz + b_kx);

    // Twiddles and modified wavenumbers (pressure_fft.f90:53,61) are built on
    // the device in the scratch, so the call copies nothing from the host.
    {
        const int nmax = std::max(nx, nz);
        k_noalloc_trig<<<(nmax + 255) / 256, 256, 0, st>>>(nx, nz, d.nxh, dx, dz, twx, twz, kxp, kzp);
    }

    const double dyi2 = 1.0 / (dy * dy);
    const int nm = d.nxh * nzh;
    k_thomas_tables<<<(nm + 127) / 128, 128, 0, st>>>(d.nxh, nzh, ny, dyi2, kxp, kzp, dinv, cp);
    const int M = nx / 2;
    const int R = rows_per_block(M);
    const int nrows = nz * ny;
    const size_t smx = sizeof(double2) * 2 * R * M;
    const int xblocks = (nrows + R - 1) / R;
    const int TX = ztile(nz);
    const size_t smz = sizeof(double2) * 2 * TX * (nz + 1);
    const int zblocks = ((d.nxh + TX - 1) / TX) * ny;
    const cudaError_t a1 = cudaFuncSetAttribute(k_fftx_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx);
    const cudaError_t a2 = cudaFuncSetAttribute(k_ifftx<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx);
    const cudaError_t a3 =
        cudaFuncSetAttribute(k_fftz<false, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz);
    const cudaError_t a4 =
        cudaFuncSetAttribute(k_fftz<true, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz);
    if (a1 != cudaSuccess || a2 != cudaSuccess || a3 != cudaSuccess || a4 != cudaSuccess)
        return mdx_fail(nullptr, MDX_ERR_CUDA, "noalloc solve: cudaFuncSetAttribute failed");
    k_fftx_r2c<<<xblocks, 256, smx, st>>>(d, R, rhs, spec, plx, twx);
    k_fftz<false, double2><<<zblocks, 256, smz, st>>>(d, TX, spec, plz, twz);
    k_thomas<double2, false><<<(d.nxh * nz + 127) / 128, 128, 0, st>>>(d, dyi2, spec, dinv, cp);
    k_fftz<true, double2><<<zblocks, 256, smz, st>>>(d, TX, spec, plz, twz);
    k_ifftx<double2><<<xblocks, 256, smx, st>>>(d, R, 1.0 / (double)(nx * nz), spec, phi, plx, twx);
    e = cudaGetLastError();
    if (e != cudaSuccess) return mdx_fail(nullptr, MDX_ERR_CUDA, "noalloc solve: launch: %s", cudaGetErrorString(e));
    return MDX_OK;
}
