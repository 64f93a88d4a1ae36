// mdx_oracle.cpp -- CPU FP64 restatement of the mobydiff RK3 time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
// mobydiff_b200/: only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg load it.  The product never links or calls it.
//
// Parity status: UNPINNED.  The reference (Fortran 2008 + FFTW3 + HDF5) has
// no tests, golden vectors or fixtures, and no Fortran compiler, FFTW or HDF5
// exists in this image, so the reference binary cannot be run here.  This
// restatement follows the reference source line by line (citations below,
// paths relative to the mobydiff project root) and is strengthened by:
//   * its FFT checked against numpy's pocketfft (tests/golden/fft_*.npz),
//   * analytic known-answer tests of the discrete operators (tests/).
//
// Floating point: compiled with -O2 -ffp-contract=off and no -march, which is
// what gfortran -O2 produces on x86-64 for the reference (SSE2, no FMA), and
// every expression keeps the reference's Fortran evaluation order so results
// are bit-for-bit those of the reference arithmetic.  The FFT is our own
// (FFTW is absent), so FFT-path results agree to rounding, not bitwise.
//
// Layout: padded arrays (0:nx+1, 0:ny+1, 0:nz+1) in Fortran order,
// element (i,j,k) at i + (nx+2)*(j + (ny+2)*k); oldrhs arrays (1:nx,1:ny,1:nz)
// unpadded; FFT workspace rhs(nx,nz,ny) and plane_hat(nxh,nz,ny) with
// nxh = nx/2+1, as src/modules/pressure_workspace.f90:10-22.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <map>
#include <mutex>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

extern "C" {

// Mirror of grid_type (src/modules/init.f90:5-12), only what the step uses.
typedef struct {
    int nx, ny, nz;
    double lx, ly, lz;
    double dx, dy, dz;
    double re;
    double forcing_x, forcing_y, forcing_z;
} or_grid;

// Mirror of boundary_type (src/modules/boundary.f90:6-10).  bc_type and
// bc_value use the Fortran memory order of bcType(1:3,0:1,0:3):
// index (dir-1) + 3*(side + 2*var), dir x/y/z = 1..3, side min/max = 0/1,
// var p/u/v/w = 0..3.
typedef struct {
    int periodic[3];
    int bc_type[24];
    double bc_value[24];
} or_bc;

// The field_type arrays (src/modules/init.f90:14-19) plus IBM coefficients
// (src/modules/ibm.f90:32).
typedef struct {
    double *un, *us, *vn, *vs, *wn, *ws, *pn;
    double *oldrhsu, *oldrhsv, *oldrhsw;
    const double *coef_u, *coef_v, *coef_w;
} or_fields;

}  // extern "C"

namespace {

inline size_t P(const or_grid* g, int i, int j, int k) {
    return (size_t)i + (size_t)(g->nx + 2) * ((size_t)j + (size_t)(g->ny + 2) * (size_t)k);
}
inline size_t Q(const or_grid* g, int i, int j, int k) {  // (1:nx,1:ny,1:nz)
    return (size_t)(i - 1) + (size_t)g->nx * ((size_t)(j - 1) + (size_t)g->ny * (size_t)(k - 1));
}
inline int BCI(int dir, int side, int var) { return (dir - 1) + 3 * (side + 2 * var); }

// ---------------------------------------------------------------------------
// FFT: recursive mixed-radix decimation-in-time Cooley-Tukey with twiddles
// evaluated in long double.  Independent of the CUDA implementation (which is
// a shared-memory Stockham formulation).  Stands in for FFTW3 (not vendored,
// not installed; README.md:11 asks for fftw >= 3.1).
// ---------------------------------------------------------------------------
struct Plan1D {
    int n;
    std::vector<int> fac;
    std::vector<cd> tw;  // exp(-2*pi*i*t/n)
};

Plan1D make_plan(int n) {
    Plan1D p;
    p.n = n;
    int m = n;
    for (int r : {4, 2, 3, 5, 7}) {
        while (m % r == 0) { p.fac.push_back(r); m /= r; }
    }
    for (int r = 11; m > 1; r += 2) {
        while (m % r == 0) { p.fac.push_back(r); m /= r; }
    }
    p.tw.resize(n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < n; ++t) {
        long double a = two_pi * (long double)t / (long double)n;
        p.tw[t] = cd((double)cosl(a), (double)(-sinl(a)));
    }
    return p;
}

std::mutex g_plan_mu;
std::map<int, Plan1D*> g_plans;
const Plan1D& plan_for(int n) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find(n);
    if (it != g_plans.end()) return *it->second;
    Plan1D* p = new Plan1D(make_plan(n));
    g_plans[n] = p;
    return *p;
}

// out[0..n) = DFT of in[0], in[s], in[2s], ... ; sign -1 forward, +1 inverse.
void fft_rec(const cd* in, cd* out, int n, int s, const int* fac, const Plan1D& P0, int tws, int sign) {
    if (n == 1) { out[0] = in[0]; return; }
    int r = fac[0];
    int m = n / r;
    for (int q = 0; q < r; ++q) fft_rec(in + (size_t)q * s, out + (size_t)q * m, m, s * r, fac + 1, P0, tws * r, sign);
    std::vector<cd> yv(r), tv(r);
    cd* y = yv.data();
    cd* tmp = tv.data();
    for (int k = 0; k < m; ++k) {
        for (int q = 0; q < r; ++q) {
            int t = (int)(((long long)q * k * tws) % P0.n);
            cd w = P0.tw[t];
            if (sign > 0) w = std::conj(w);
            y[q] = out[(size_t)q * m + k] * w;
        }
        for (int pp = 0; pp < r; ++pp) {
            cd acc(0.0, 0.0);
            for (int q = 0; q < r; ++q) {
                int t = (int)(((long long)((q * pp) % r) * (P0.n / r)) % P0.n);
                cd w = P0.tw[t];
                if (sign > 0) w = std::conj(w);
                acc += y[q] * w;
            }
            tmp[pp] = acc;
        }
        for (int pp = 0; pp < r; ++pp) out[(size_t)pp * m + k] = tmp[pp];
    }
}

void fft1d(cd* data, int n, int sign, cd* work) {
    const Plan1D& p = plan_for(n);
    fft_rec(data, work, n, 1, p.fac.data(), p, 1, sign);
    std::memcpy(data, work, sizeof(cd) * n);
}

// Batched 2-D real-to-complex transform over [nz][nx] per y plane, FFTW
// forward sign, unnormalised: the plan of
// src/modules/pressure/pressure_backend_fftw.f90:22-49 (rank 2, dims
// [nz,nx], batch ny, idist nx*nz, odist nxh*nz).
void fft2_r2c(const or_grid* g, const double* rhs, cd* hat) {
    const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1;
    #pragma omp parallel
    {
        std::vector<cd> row(std::max(nx, nz)), work(std::max(nx, nz));
        #pragma omp for schedule(static)
        for (int j = 0; j < ny; ++j) {
            const double* src = rhs + (size_t)j * nx * nz;
            cd* dst = hat + (size_t)j * nxh * nz;
            for (int k = 0; k < nz; ++k) {
                for (int i = 0; i < nx; ++i) row[i] = cd(src[(size_t)k * nx + i], 0.0);
                fft1d(row.data(), nx, -1, work.data());
                for (int i = 0; i < nxh; ++i) dst[(size_t)k * nxh + i] = row[i];
            }
            for (int i = 0; i < nxh; ++i) {
                for (int k = 0; k < nz; ++k) row[k] = dst[(size_t)k * nxh + i];
                fft1d(row.data(), nz, -1, work.data());
                for (int k = 0; k < nz; ++k) dst[(size_t)k * nxh + i] = row[k];
            }
        }
    }
}

// Inverse (complex-to-real, unnormalised).  The c2r contract: the Hermitian
// extension of each x row is inverted, imaginary parts of the kx=0 and (even
// nx) kx=nx/2 bins are ignored.  `hat` is consumed.
void fft2_c2r(const or_grid* g, cd* hat, double* rhs) {
    const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1;
    #pragma omp parallel
    {
        std::vector<cd> row(std::max(nx, nz)), work(std::max(nx, nz));
        #pragma omp for schedule(static)
        for (int j = 0; j < ny; ++j) {
            double* dst = rhs + (size_t)j * nx * nz;
            cd* src = hat + (size_t)j * nxh * nz;
            for (int i = 0; i < nxh; ++i) {
                for (int k = 0; k < nz; ++k) row[k] = src[(size_t)k * nxh + i];
                fft1d(row.data(), nz, +1, work.data());
                for (int k = 0; k < nz; ++k) src[(size_t)k * nxh + i] = row[k];
            }
            for (int k = 0; k < nz; ++k) {
                for (int i = 0; i < nxh; ++i) row[i] = src[(size_t)k * nxh + i];
                row[0] = cd(row[0].real(), 0.0);
                if (nx % 2 == 0) row[nx / 2] = cd(row[nx / 2].real(), 0.0);
                for (int i = nxh; i < nx; ++i) row[i] = std::conj(row[nx - i]);
                fft1d(row.data(), nx, +1, work.data());
                for (int i = 0; i < nx; ++i) dst[(size_t)k * nx + i] = row[i].real();
            }
        }
    }
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// RK3 coefficients, src/modules/step.f90:21-23.
// ---------------------------------------------------------------------------
void or_rk_coeffs(double* alpha, double* beta, double* gamma) {
    alpha[0] = 64.0 / 120.0; alpha[1] = 50.0 / 120.0; alpha[2] = 90.0 / 120.0;
    beta[0] = 0.0;           beta[1] = -34.0 / 120.0; beta[2] = -50.0 / 120.0;
    gamma[0] = 64.0 / 120.0; gamma[1] = 16.0 / 120.0; gamma[2] = 40.0 / 120.0;
}

// ---------------------------------------------------------------------------
// Predictor, src/modules/step.f90:27-207 (momentum).
// ---------------------------------------------------------------------------
void or_momentum(const or_grid* g, const or_bc* bc, or_fields* f,
                 double dt_alpha, double dt_beta, double dt_gamma) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dx = g->dx, dy = g->dy, dz = g->dz;
    const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
    const double re = g->re;
    const double idx = 1.0 / dx, idy = 1.0 / dy, idz = 1.0 / dz;
    const double idx2 = 1.0 / dx2, idy2 = 1.0 / dy2, idz2 = 1.0 / dz2;
    const double ire = 1.0 / re;
    const double forcing_x = g->forcing_x, forcing_y = g->forcing_y, forcing_z = g->forcing_z;
    int nx0 = 2; if (bc->periodic[0]) nx0 -= 1;   // step.f90:71-73
    int ny0 = 2; if (bc->periodic[1]) ny0 -= 1;
    int nz0 = 2; if (bc->periodic[2]) nz0 -= 1;
    const double *un = f->un, *vn = f->vn, *wn = f->wn, *pn = f->pn;
    double *us = f->us, *vs = f->vs, *ws = f->ws;

    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k) {
        for (int j = 1; j <= ny; ++j) {
            for (int i = 1; i <= nx; ++i) {
                const int ip = i + 1, im = i - 1, jp = j + 1, jm = j - 1, kp = k + 1, km = k - 1;
                if (i >= nx0) {  // step.f90:106-136
                    double s;
                    s = un[P(g, ip, j, k)] + un[P(g, i, j, k)];
                    double uu_p = 0.25 * (s * s);
                    s = un[P(g, i, j, k)] + un[P(g, im, j, k)];
                    double uu_m = 0.25 * (s * s);
                    double uv_p = 0.25 * (un[P(g, i, jp, k)] + un[P(g, i, j, k)]) * (vn[P(g, i, jp, k)] + vn[P(g, im, jp, k)]);
                    double uv_m = 0.25 * (un[P(g, i, j, k)] + un[P(g, i, jm, k)]) * (vn[P(g, i, j, k)] + vn[P(g, im, j, k)]);
                    double uw_p = 0.25 * (un[P(g, i, j, k)] + un[P(g, i, j, kp)]) * (wn[P(g, i, j, kp)] + wn[P(g, im, j, kp)]);
                    double uw_m = 0.25 * (un[P(g, i, j, k)] + un[P(g, i, j, km)]) * (wn[P(g, i, j, k)] + wn[P(g, im, j, k)]);
                    double diff_ux = (un[P(g, im, j, k)] - 2.0 * un[P(g, i, j, k)] + un[P(g, ip, j, k)]) * idx2;
                    double diff_uy = (un[P(g, i, jm, k)] - 2.0 * un[P(g, i, j, k)] + un[P(g, i, jp, k)]) * idy2;
                    double diff_uz = (un[P(g, i, j, km)] - 2.0 * un[P(g, i, j, k)] + un[P(g, i, j, kp)]) * idz2;
                    double dpx = (pn[P(g, i, j, k)] - pn[P(g, im, j, k)]) * idx;
                    double rhsu = -((uu_p - uu_m) * idx) - (uv_p - uv_m) * idy - (uw_p - uw_m) * idz
                                  + forcing_x + ire * (diff_ux + diff_uy + diff_uz);
                    double v = un[P(g, i, j, k)] + dt_alpha * rhsu + dt_beta * f->oldrhsu[Q(g, i, j, k)] - dt_gamma * dpx;
                    double mu_u = 1.0 / (1.0 + dt_gamma * f->coef_u[P(g, i, j, k)]);
                    us[P(g, i, j, k)] = v * mu_u;
                    f->oldrhsu[Q(g, i, j, k)] = rhsu;
                }
                if (j >= ny0) {  // step.f90:138-168
                    double s;
                    double vu_p = 0.25 * (vn[P(g, i, j, k)] + vn[P(g, ip, j, k)]) * (un[P(g, ip, j, k)] + un[P(g, ip, jm, k)]);
                    double vu_m = 0.25 * (vn[P(g, i, j, k)] + vn[P(g, im, j, k)]) * (un[P(g, i, j, k)] + un[P(g, i, jm, k)]);
                    s = vn[P(g, i, j, k)] + vn[P(g, i, jp, k)];
                    double vv_p = 0.25 * (s * s);
                    s = vn[P(g, i, j, k)] + vn[P(g, i, jm, k)];
                    double vv_m = 0.25 * (s * s);
                    double vw_p = 0.25 * (vn[P(g, i, j, kp)] + vn[P(g, i, j, k)]) * (wn[P(g, i, j, kp)] + wn[P(g, i, jm, kp)]);
                    double vw_m = 0.25 * (vn[P(g, i, j, km)] + vn[P(g, i, j, k)]) * (wn[P(g, i, j, k)] + wn[P(g, i, jm, k)]);
                    double diff_vx = (vn[P(g, im, j, k)] - 2.0 * vn[P(g, i, j, k)] + vn[P(g, ip, j, k)]) * idx2;
                    double diff_vy = (vn[P(g, i, jm, k)] - 2.0 * vn[P(g, i, j, k)] + vn[P(g, i, jp, k)]) * idy2;
                    double diff_vz = (vn[P(g, i, j, km)] - 2.0 * vn[P(g, i, j, k)] + vn[P(g, i, j, kp)]) * idz2;
                    double dpy = (pn[P(g, i, j, k)] - pn[P(g, i, jm, k)]) * idy;
                    double rhsv = -((vu_p - vu_m) * idx) - (vv_p - vv_m) * idy - (vw_p - vw_m) * idz
                                  + forcing_y + ire * (diff_vx + diff_vy + diff_vz);
                    double v = vn[P(g, i, j, k)] + dt_alpha * rhsv + dt_beta * f->oldrhsv[Q(g, i, j, k)] - dt_gamma * dpy;
                    double mu_v = 1.0 / (1.0 + dt_gamma * f->coef_v[P(g, i, j, k)]);
                    vs[P(g, i, j, k)] = v * mu_v;
                    f->oldrhsv[Q(g, i, j, k)] = rhsv;
                }
                if (k >= nz0) {  // step.f90:170-200
                    double s;
                    double wu_p = 0.25 * (wn[P(g, i, j, k)] + wn[P(g, ip, j, k)]) * (un[P(g, ip, j, k)] + un[P(g, ip, j, km)]);
                    double wu_m = 0.25 * (wn[P(g, i, j, k)] + wn[P(g, im, j, k)]) * (un[P(g, i, j, k)] + un[P(g, i, j, km)]);
                    s = wn[P(g, i, j, k)] + wn[P(g, i, j, kp)];
                    double ww_p = 0.25 * (s * s);
                    s = wn[P(g, i, j, k)] + wn[P(g, i, j, km)];
                    double ww_m = 0.25 * (s * s);
                    double wv_p = 0.25 * (wn[P(g, i, j, k)] + wn[P(g, i, jp, k)]) * (vn[P(g, i, jp, k)] + vn[P(g, i, jp, km)]);
                    double wv_m = 0.25 * (wn[P(g, i, j, k)] + wn[P(g, i, jm, k)]) * (vn[P(g, i, j, k)] + vn[P(g, i, j, km)]);
                    double diff_wx = (wn[P(g, im, j, k)] - 2.0 * wn[P(g, i, j, k)] + wn[P(g, ip, j, k)]) * idx2;
                    double diff_wy = (wn[P(g, i, jm, k)] - 2.0 * wn[P(g, i, j, k)] + wn[P(g, i, jp, k)]) * idy2;
                    double diff_wz = (wn[P(g, i, j, km)] - 2.0 * wn[P(g, i, j, k)] + wn[P(g, i, j, kp)]) * idz2;
                    double dpz = (pn[P(g, i, j, k)] - pn[P(g, i, j, km)]) * idz;
                    // step.f90:186-191: the y flux comes before the z flux in the w equation
                    double rhsw = -((wu_p - wu_m) * idx) - (wv_p - wv_m) * idy - (ww_p - ww_m) * idz
                                  + forcing_z + ire * (diff_wx + diff_wy + diff_wz);
                    double v = wn[P(g, i, j, k)] + dt_alpha * rhsw + dt_beta * f->oldrhsw[Q(g, i, j, k)] - dt_gamma * dpz;
                    double mu_w = 1.0 / (1.0 + dt_gamma * f->coef_w[P(g, i, j, k)]);
                    ws[P(g, i, j, k)] = v * mu_w;
                    f->oldrhsw[Q(g, i, j, k)] = rhsw;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// CFL, src/modules/step.f90:210-258 (max over the padded arrays).
// ---------------------------------------------------------------------------
double or_get_cfl(const or_grid* g, const or_fields* f) {
    const size_t n = (size_t)(g->nx + 2) * (g->ny + 2) * (g->nz + 2);
    double c = 0.0;
    for (size_t t = 0; t < n; ++t) c = std::max(c, std::fabs(f->un[t] / g->dx));
    for (size_t t = 0; t < n; ++t) c = std::max(c, std::fabs(f->vn[t] / g->dy));
    for (size_t t = 0; t < n; ++t) c = std::max(c, std::fabs(f->wn[t] / g->dz));
    return c;
}

// ---------------------------------------------------------------------------
// apply_bc for the FFT builds, src/modules/boundary.f90:23-170 (the
// #ifndef USE_REDBLACK branches).  Walls in y, periodic x and z, applied to
// the n and * arrays; three phases in the reference order.
// ---------------------------------------------------------------------------
void or_apply_bc(const or_grid* g, or_fields* f) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    double *un = f->un, *vn = f->vn, *wn = f->wn, *us = f->us, *vs = f->vs, *ws = f->ws, *pn = f->pn;
    for (int i = 0; i <= nx + 1; ++i) {          // boundary.f90:48-67
        for (int k = 0; k <= nz + 1; ++k) {
            un[P(g, i, ny + 1, k)] = -un[P(g, i, ny, k)];
            vn[P(g, i, ny + 1, k)] = 0.0;
            wn[P(g, i, ny + 1, k)] = -wn[P(g, i, ny, k)];
            un[P(g, i, 0, k)] = -un[P(g, i, 1, k)];
            vn[P(g, i, 1, k)] = 0.0;
            wn[P(g, i, 0, k)] = -wn[P(g, i, 1, k)];
            us[P(g, i, ny + 1, k)] = -us[P(g, i, ny, k)];
            vs[P(g, i, ny + 1, k)] = 0.0;
            ws[P(g, i, ny + 1, k)] = -ws[P(g, i, ny, k)];
            us[P(g, i, 0, k)] = -us[P(g, i, 1, k)];
            vs[P(g, i, 1, k)] = 0.0;
            ws[P(g, i, 0, k)] = -ws[P(g, i, 1, k)];
        }
    }
    for (int j = 0; j <= ny + 1; ++j) {          // boundary.f90:87-117
        for (int k = 0; k <= nz + 1; ++k) {
            un[P(g, 0, j, k)] = un[P(g, nx, j, k)];
            wn[P(g, 0, j, k)] = wn[P(g, nx, j, k)];
            un[P(g, nx + 1, j, k)] = un[P(g, 1, j, k)];
            wn[P(g, nx + 1, j, k)] = wn[P(g, 1, j, k)];
            us[P(g, 0, j, k)] = us[P(g, nx, j, k)];
            ws[P(g, 0, j, k)] = ws[P(g, nx, j, k)];
            us[P(g, nx + 1, j, k)] = us[P(g, 1, j, k)];
            ws[P(g, nx + 1, j, k)] = ws[P(g, 1, j, k)];
            if (j >= 1) {
                vn[P(g, 0, j, k)] = vn[P(g, nx, j, k)];
                vn[P(g, nx + 1, j, k)] = vn[P(g, 1, j, k)];
                vs[P(g, 0, j, k)] = vs[P(g, nx, j, k)];
                vs[P(g, nx + 1, j, k)] = vs[P(g, 1, j, k)];
            }
            if (j >= 1 && j <= ny) {
                pn[P(g, 0, j, k)] = pn[P(g, nx, j, k)];
                pn[P(g, nx + 1, j, k)] = pn[P(g, 1, j, k)];
            }
        }
    }
    for (int i = 0; i <= nx + 1; ++i) {          // boundary.f90:137-168
        for (int j = 0; j <= ny + 1; ++j) {
            un[P(g, i, j, 0)] = un[P(g, i, j, nz)];
            wn[P(g, i, j, 0)] = wn[P(g, i, j, nz)];
            un[P(g, i, j, nz + 1)] = un[P(g, i, j, 1)];
            wn[P(g, i, j, nz + 1)] = wn[P(g, i, j, 1)];
            us[P(g, i, j, 0)] = us[P(g, i, j, nz)];
            ws[P(g, i, j, 0)] = ws[P(g, i, j, nz)];
            us[P(g, i, j, nz + 1)] = us[P(g, i, j, 1)];
            ws[P(g, i, j, nz + 1)] = ws[P(g, i, j, 1)];
            if (j >= 1) {
                vn[P(g, i, j, 0)] = vn[P(g, i, j, nz)];
                vn[P(g, i, j, nz + 1)] = vn[P(g, i, j, 1)];
                vs[P(g, i, j, 0)] = vs[P(g, i, j, nz)];
                vs[P(g, i, j, nz + 1)] = vs[P(g, i, j, 1)];
            }
            if (j >= 1 && j <= ny) {
                pn[P(g, i, j, 0)] = pn[P(g, i, j, nz)];
                pn[P(g, i, j, nz + 1)] = pn[P(g, i, j, 1)];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// apply_bc_redblack, src/modules/boundary.f90:173-368: general per-face
// Dirichlet/Neumann/periodic on un,vn,wn,pn, in the reference's sequential
// face order (bottom, top, left, right, front, back).
// ---------------------------------------------------------------------------
void or_apply_bc_redblack(const or_grid* g, const or_bc* bc, or_fields* f) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dx = g->dx, dy = g->dy, dz = g->dz;
    double *un = f->un, *vn = f->vn, *wn = f->wn, *pn = f->pn;
    const int* T = bc->bc_type;
    const double* V = bc->bc_value;
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) {   // bottom, :207-232
        if (bc->periodic[1]) {
            un[P(g, i, 0, k)] = un[P(g, i, ny, k)];
            vn[P(g, i, 0, k)] = vn[P(g, i, ny, k)];
            wn[P(g, i, 0, k)] = wn[P(g, i, ny, k)];
            pn[P(g, i, 0, k)] = pn[P(g, i, ny, k)];
        } else {
            if (T[BCI(2, 0, 1)] == 0) un[P(g, i, 0, k)] = 2 * V[BCI(2, 0, 1)] - un[P(g, i, 1, k)];
            else un[P(g, i, 0, k)] = un[P(g, i, 1, k)] - V[BCI(2, 0, 1)] * dy;
            if (T[BCI(2, 0, 2)] == 0) vn[P(g, i, 1, k)] = V[BCI(2, 0, 2)];
            else vn[P(g, i, 1, k)] = vn[P(g, i, 2, k)] - V[BCI(2, 0, 2)] * dy;
            if (T[BCI(2, 0, 3)] == 0) wn[P(g, i, 0, k)] = 2 * V[BCI(2, 0, 3)] - wn[P(g, i, 1, k)];
            else wn[P(g, i, 0, k)] = wn[P(g, i, 1, k)] - V[BCI(2, 0, 3)] * dy;
        }
    }
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) {   // top, :233-258
        if (bc->periodic[1]) {
            un[P(g, i, ny + 1, k)] = un[P(g, i, 1, k)];
            vn[P(g, i, ny + 1, k)] = vn[P(g, i, 1, k)];
            wn[P(g, i, ny + 1, k)] = wn[P(g, i, 1, k)];
            pn[P(g, i, ny + 1, k)] = pn[P(g, i, 1, k)];
        } else {
            if (T[BCI(2, 1, 1)] == 0) un[P(g, i, ny + 1, k)] = 2 * V[BCI(2, 1, 1)] - un[P(g, i, ny, k)];
            else un[P(g, i, ny + 1, k)] = un[P(g, i, ny, k)] + V[BCI(2, 1, 1)] * dy;
            if (T[BCI(2, 1, 2)] == 0) vn[P(g, i, ny + 1, k)] = V[BCI(2, 1, 2)];
            else vn[P(g, i, ny + 1, k)] = vn[P(g, i, ny, k)] + V[BCI(2, 1, 2)] * dy;
            if (T[BCI(2, 1, 3)] == 0) wn[P(g, i, ny + 1, k)] = 2 * V[BCI(2, 1, 3)] - wn[P(g, i, ny, k)];
            else wn[P(g, i, ny + 1, k)] = wn[P(g, i, ny, k)] + V[BCI(2, 1, 3)] * dy;
        }
    }
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) {   // left, :259-284
        if (bc->periodic[0]) {
            un[P(g, 0, j, k)] = un[P(g, nx, j, k)];
            vn[P(g, 0, j, k)] = vn[P(g, nx, j, k)];
            wn[P(g, 0, j, k)] = wn[P(g, nx, j, k)];
            pn[P(g, 0, j, k)] = pn[P(g, nx, j, k)];
        } else {
            if (T[BCI(1, 0, 1)] == 0) un[P(g, 1, j, k)] = V[BCI(1, 0, 1)];
            else un[P(g, 1, j, k)] = un[P(g, 2, j, k)] - V[BCI(1, 0, 1)] * dx;
            if (T[BCI(1, 0, 2)] == 0) vn[P(g, 0, j, k)] = 2 * V[BCI(1, 0, 2)] - vn[P(g, 1, j, k)];
            else vn[P(g, 0, j, k)] = vn[P(g, 1, j, k)] - V[BCI(1, 0, 2)] * dx;
            if (T[BCI(1, 0, 3)] == 0) wn[P(g, 0, j, k)] = 2 * V[BCI(1, 0, 3)] - wn[P(g, 1, j, k)];
            else wn[P(g, 0, j, k)] = wn[P(g, 1, j, k)] - V[BCI(1, 0, 3)] * dx;
        }
    }
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) {   // right, :285-310
        if (bc->periodic[0]) {
            un[P(g, nx + 1, j, k)] = un[P(g, 1, j, k)];
            vn[P(g, nx + 1, j, k)] = vn[P(g, 1, j, k)];
            wn[P(g, nx + 1, j, k)] = wn[P(g, 1, j, k)];
            pn[P(g, nx + 1, j, k)] = pn[P(g, 1, j, k)];
        } else {
            if (T[BCI(1, 1, 1)] == 0) un[P(g, nx + 1, j, k)] = V[BCI(1, 1, 1)];
            else un[P(g, nx + 1, j, k)] = un[P(g, nx, j, k)] + V[BCI(1, 1, 1)] * dx;
            if (T[BCI(1, 1, 2)] == 0) vn[P(g, nx + 1, j, k)] = 2 * V[BCI(1, 1, 2)] - vn[P(g, nx, j, k)];
            else vn[P(g, nx + 1, j, k)] = vn[P(g, nx, j, k)] + V[BCI(1, 1, 2)] * dx;
            if (T[BCI(1, 1, 3)] == 0) wn[P(g, nx + 1, j, k)] = 2 * V[BCI(1, 1, 3)] - wn[P(g, nx, j, k)];
            else wn[P(g, nx + 1, j, k)] = wn[P(g, nx, j, k)] + V[BCI(1, 1, 3)] * dx;
        }
    }
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {   // front, :311-337
        if (bc->periodic[2]) {
            un[P(g, i, j, 0)] = un[P(g, i, j, nz)];
            vn[P(g, i, j, 0)] = vn[P(g, i, j, nz)];
            wn[P(g, i, j, 0)] = wn[P(g, i, j, nz)];
            pn[P(g, i, j, 0)] = pn[P(g, i, j, nz)];
        } else {
            if (T[BCI(3, 0, 1)] == 0) un[P(g, i, j, 0)] = 2 * V[BCI(3, 0, 1)] - un[P(g, i, j, 1)];
            else un[P(g, i, j, 0)] = un[P(g, i, j, 1)] - V[BCI(3, 0, 1)] * dz;
            if (T[BCI(3, 0, 2)] == 0) vn[P(g, i, j, 0)] = 2 * V[BCI(3, 0, 2)] - vn[P(g, i, j, 1)];
            else vn[P(g, i, j, 0)] = vn[P(g, i, j, 1)] - V[BCI(3, 0, 2)] * dz;
            if (T[BCI(3, 0, 3)] == 0) wn[P(g, i, j, 1)] = V[BCI(3, 0, 3)];
            else wn[P(g, i, j, 1)] = wn[P(g, i, j, 2)] - V[BCI(3, 0, 3)] * dz;
        }
    }
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {   // back, :338-364
        if (bc->periodic[2]) {
            un[P(g, i, j, nz + 1)] = un[P(g, i, j, 1)];
            vn[P(g, i, j, nz + 1)] = vn[P(g, i, j, 1)];
            wn[P(g, i, j, nz + 1)] = wn[P(g, i, j, 1)];
            pn[P(g, i, j, nz + 1)] = pn[P(g, i, j, 1)];
        } else {
            if (T[BCI(3, 1, 1)] == 0) un[P(g, i, j, nz + 1)] = 2 * V[BCI(3, 1, 1)] - un[P(g, i, j, nz)];
            else un[P(g, i, j, nz + 1)] = un[P(g, i, j, nz)] + V[BCI(3, 1, 1)] * dz;
            if (T[BCI(3, 1, 2)] == 0) vn[P(g, i, j, nz + 1)] = 2 * V[BCI(3, 1, 2)] - vn[P(g, i, j, nz)];
            else vn[P(g, i, j, nz + 1)] = vn[P(g, i, j, nz)] + V[BCI(3, 1, 2)] * dz;
            if (T[BCI(3, 1, 3)] == 0) wn[P(g, i, j, nz + 1)] = V[BCI(3, 1, 3)];
            else wn[P(g, i, j, nz + 1)] = wn[P(g, i, j, nz)] + V[BCI(3, 1, 3)] * dz;
        }
    }
}

// ---------------------------------------------------------------------------
// FFT pressure path.
// ---------------------------------------------------------------------------

// build_fft_rhs, src/modules/pressure_solver.f90:77-115.
void or_build_fft_rhs(const or_grid* g, const or_fields* f, double dt_gamma, double* rhs) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dx = g->dx, dy = g->dy, dz = g->dz;
    #pragma omp parallel for schedule(static)
    for (int j = 1; j <= ny; ++j)
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i)
                rhs[(size_t)(i - 1) + (size_t)nx * ((size_t)(k - 1) + (size_t)nz * (j - 1))] =
                    ((f->us[P(g, i + 1, j, k)] - f->us[P(g, i, j, k)]) / dx
                     + (f->vs[P(g, i, j + 1, k)] - f->vs[P(g, i, j, k)]) / dy
                     + (f->ws[P(g, i, j, k + 1)] - f->ws[P(g, i, j, k)]) / dz) / dt_gamma;
}

// Modified wavenumbers, src/modules/pressure/pressure_fft.f90:53,61.
static void modified_wavenumbers(const or_grid* g, std::vector<double>& kxp, std::vector<double>& kzp) {
    const double pi = 3.141592653589793;
    const int nx = g->nx, nz = g->nz, nxh = nx / 2 + 1;
    kxp.resize(nxh);
    kzp.resize(nz);
    for (int ikx = 1; ikx <= nxh; ++ikx) {
        int kx = ikx - 1;
        double s = std::sin(pi * (double)kx / (double)nx);
        kxp[ikx - 1] = (4.0 / (g->dx * g->dx)) * (s * s);
    }
    for (int ikz = 1; ikz <= nz; ++ikz) {
        int kz = (ikz <= nz / 2 + 1) ? ikz - 1 : ikz - nz - 1;
        double s = std::sin(pi * (double)kz / (double)nz);
        kzp[ikz - 1] = (4.0 / (g->dz * g->dz)) * (s * s);
    }
}

// Thomas coefficients (src/modules/pressure/pressure_fft.f90:46-94) and the
// per-mode forward/back substitution (:102-148).  The complex coefficients of
// the reference have zero imaginary part, so the complex arithmetic reduces
// exactly to the same real operations on the real and imaginary parts.
void or_solve_tridiagonal_y(const or_grid* g, cd* hat) {
    const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1;
    const double dyi2 = 1.0 / (g->dy * g->dy);
    std::vector<double> kxp, kzp;
    modified_wavenumbers(g, kxp, kzp);
    #pragma omp parallel
    {
        std::vector<double> cp(ny), dinv(ny);
        std::vector<cd> dp(ny);
        #pragma omp for schedule(static) collapse(2)
        for (int ikz = 1; ikz <= nz; ++ikz) {
            for (int ikx = 1; ikx <= nxh; ++ikx) {
                const double k_tot = kxp[ikx - 1] + kzp[ikz - 1];
                const bool zero_mode = (ikx == 1 && ikz == 1);
                if (zero_mode) { dinv[0] = 1.0; cp[0] = 0.0; }
                else {
                    double b = -dyi2 - k_tot, c = dyi2;
                    dinv[0] = 1.0 / b;
                    cp[0] = c * dinv[0];
                }
                const double a = dyi2;
                for (int jj = 2; jj <= ny; ++jj) {
                    double b, c;
                    if (jj < ny) { b = -2.0 * dyi2 - k_tot; c = dyi2; }
                    else { b = -dyi2 - k_tot; c = 0.0; }
                    double denom = b - a * cp[jj - 2];
                    dinv[jj - 1] = 1.0 / denom;
                    cp[jj - 1] = (jj < ny) ? c * dinv[jj - 1] : 0.0;
                }
                auto H = [&](int jj) -> cd& {
                    return hat[(size_t)(ikx - 1) + (size_t)nxh * ((size_t)(ikz - 1) + (size_t)nz * (jj - 1))];
                };
                if (zero_mode) dp[0] = cd(0.0, 0.0);
                else { cd r = H(1); dp[0] = cd(r.real() * dinv[0], r.imag() * dinv[0]); }
                for (int jj = 2; jj <= ny; ++jj) {
                    cd r = H(jj);
                    double re = (r.real() - a * dp[jj - 2].real()) * dinv[jj - 1];
                    double im = (r.imag() - a * dp[jj - 2].imag()) * dinv[jj - 1];
                    dp[jj - 1] = cd(re, im);
                }
                H(ny) = dp[ny - 1];
                for (int jj = ny - 1; jj >= 1; --jj) {
                    cd nxt = H(jj + 1);
                    H(jj) = cd(dp[jj - 1].real() - cp[jj - 1] * nxt.real(), dp[jj - 1].imag() - cp[jj - 1] * nxt.imag());
                }
            }
        }
    }
}

// apply_fft_pressure_correction, src/modules/pressure_solver.f90:117-173.
void or_fft_correction(const or_grid* g, or_fields* f, double dt_gamma, const double* rhs) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dx = g->dx, dy = g->dy, dz = g->dz;
    auto R = [&](int i, int k, int j) { return rhs[(size_t)(i - 1) + (size_t)nx * ((size_t)(k - 1) + (size_t)nz * (j - 1))]; };
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                int im = i - 1, km = k - 1;
                if (im < 1) im = nx;
                if (km < 1) km = nz;
                f->un[P(g, i, j, k)] = (f->us[P(g, i, j, k)] - dt_gamma * (R(i, k, j) - R(im, k, j)) / dx)
                                       / (1.0 + dt_gamma * f->coef_u[P(g, i, j, k)]);
                f->wn[P(g, i, j, k)] = (f->ws[P(g, i, j, k)] - dt_gamma * (R(i, k, j) - R(i, km, j)) / dz)
                                       / (1.0 + dt_gamma * f->coef_w[P(g, i, j, k)]);
                f->pn[P(g, i, j, k)] = f->pn[P(g, i, j, k)] + R(i, k, j);
                if (j >= 2)
                    f->vn[P(g, i, j, k)] = (f->vs[P(g, i, j, k)] - dt_gamma * (R(i, k, j) - R(i, k, j - 1)) / dy)
                                           / (1.0 + dt_gamma * f->coef_v[P(g, i, j, k)]);
            }
}

// Poisson solve of the FFTW backend, src/modules/pressure/pressure_backend_fftw.f90:51-93:
// forward r2c, tridiagonal in y, backward c2r, scale by 1/(nx*nz).  `rhs` in,
// phi out (same array).
void or_solve_pressure_fft(const or_grid* g, double* rhs) {
    const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1;
    std::vector<cd> hat((size_t)nxh * nz * ny);
    fft2_r2c(g, rhs, hat.data());
    or_solve_tridiagonal_y(g, hat.data());
    fft2_c2r(g, hat.data(), rhs);
    const double scale = 1.0 / (double)(nx * nz);
    const size_t n = (size_t)nx * ny * nz;
    for (size_t t = 0; t < n; ++t) rhs[t] = rhs[t] * scale;
}

// Exposed FFT pieces for the known-answer tests.
void or_fft2_r2c(const or_grid* g, const double* rhs, double* hat_interleaved) {
    fft2_r2c(g, rhs, reinterpret_cast<cd*>(hat_interleaved));
}
void or_fft2_c2r(const or_grid* g, double* hat_interleaved, double* rhs) {
    fft2_c2r(g, reinterpret_cast<cd*>(hat_interleaved), rhs);
}

// pressure_projection for the FFT builds, src/modules/pressure_solver.f90:48-63.
// `phi_out` (nx*nz*ny, may be null) receives the pressure correction.
void or_pressure_projection_fft(const or_grid* g, or_fields* f, double dt_gamma, double* phi_out) {
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    std::vector<double> rhs(n);
    or_build_fft_rhs(g, f, dt_gamma, rhs.data());
    or_solve_pressure_fft(g, rhs.data());
    or_fft_correction(g, f, dt_gamma, rhs.data());
    if (phi_out) std::memcpy(phi_out, rhs.data(), n * sizeof(double));
}

// ---------------------------------------------------------------------------
// Red-black SOR, src/modules/pressure/pressure_redblack.f90:27-254.
// ---------------------------------------------------------------------------

// One colour sweep (:89-245).  Same-colour cells share no face, so the cell
// order inside a sweep does not change the result; `parallel` selects an
// OpenMP loop over k for the timed baseline.
static void sor_sweep(const or_grid* g, const or_bc* bc, or_fields* f, double dt_gamma, double sor, int parity, bool parallel) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double dx = g->dx, dy = g->dy, dz = g->dz;
    const int nActive = nx / 2;
    const double idx = 1.0 / dx, idy = 1.0 / dy, idz = 1.0 / dz;
    const double idx2 = idx * idx, idy2 = idy * idy, idz2 = idz * idz;
    const double idt = 1.0 / dt_gamma;
    const int* T = bc->bc_type;
    const double* V = bc->bc_value;
    const int perx = bc->periodic[0], pery = bc->periodic[1], perz = bc->periodic[2];
    double *un = f->un, *vn = f->vn, *wn = f->wn, *pn = f->pn;
    const double *cu = f->coef_u, *cv = f->coef_v, *cw = f->coef_w;
    #pragma omp parallel for schedule(static) if (parallel)
    for (int k = 1; k <= nz; ++k) {
        for (int j = 1; j <= ny; ++j) {
            for (int ni = 1; ni <= nActive; ++ni) {
                int jp = j + 1;
                if (pery && jp > ny) jp = 1;
                int kp = k + 1;
                if (perz && kp > nz) kp = 1;
                const int iLo = 1 + ((j + k + parity) % 2);
                const int i = iLo + 2 * (ni - 1);
                int ip = i + 1;
                if (perx && ip > nx) ip = 1;
                const double mu_u_i = 1.0 / (1.0 + dt_gamma * cu[P(g, i, j, k)]);
                const double mu_u_ip = 1.0 / (1.0 + dt_gamma * cu[P(g, ip, j, k)]);
                const double mu_v_j = 1.0 / (1.0 + dt_gamma * cv[P(g, i, j, k)]);
                const double mu_v_jp = 1.0 / (1.0 + dt_gamma * cv[P(g, i, jp, k)]);
                const double mu_w_k = 1.0 / (1.0 + dt_gamma * cw[P(g, i, j, k)]);
                const double mu_w_kp = 1.0 / (1.0 + dt_gamma * cw[P(g, i, j, kp)]);
                const double denom = (mu_u_i + mu_u_ip) * idx2 + (mu_w_k + mu_w_kp) * idz2 + (mu_v_j + mu_v_jp) * idy2;
                if (!perx) {  // :128-144
                    if (i < 2) {
                        if (T[BCI(1, 0, 1)] == 0) un[P(g, i, j, k)] = V[BCI(1, 0, 1)];
                        else un[P(g, i, j, k)] = un[P(g, ip, j, k)] - V[BCI(1, 0, 1)] * dx;
                    }
                    if (i >= nx) {
                        if (T[BCI(1, 1, 1)] == 0) un[P(g, ip, j, k)] = V[BCI(1, 1, 1)];
                        else un[P(g, ip, j, k)] = un[P(g, nx, j, k)] + V[BCI(1, 1, 1)] * dx;
                    }
                }
                if (!pery) {  // :146-162
                    if (j < 2) {
                        if (T[BCI(2, 0, 2)] == 0) vn[P(g, i, j, k)] = V[BCI(2, 0, 2)];
                        else vn[P(g, i, j, k)] = vn[P(g, i, jp, k)] - V[BCI(2, 0, 2)] * dy;
                    }
                    if (j >= ny) {
                        if (T[BCI(2, 1, 2)] == 0) vn[P(g, i, jp, k)] = V[BCI(2, 1, 2)];
                        else vn[P(g, i, jp, k)] = vn[P(g, i, j, k)] + V[BCI(2, 1, 2)] * dy;
                    }
                }
                if (!perz) {  // :164-180
                    if (k < 2) {
                        if (T[BCI(3, 0, 3)] == 0) wn[P(g, i, j, k)] = V[BCI(3, 0, 3)];
                        else wn[P(g, i, j, k)] = wn[P(g, i, j, kp)] - V[BCI(3, 0, 3)] * dz;
                    }
                    if (k >= nz) {
                        if (T[BCI(3, 1, 3)] == 0) wn[P(g, i, j, kp)] = V[BCI(3, 1, 3)];
                        else wn[P(g, i, j, kp)] = wn[P(g, i, j, k)] + V[BCI(3, 1, 3)] * dz;
                    }
                }
                // :183-186
                const double phi = ((un[P(g, ip, j, k)] - un[P(g, i, j, k)]) * idx
                                    + (vn[P(g, i, jp, k)] - vn[P(g, i, j, k)]) * idy
                                    + (wn[P(g, i, j, kp)] - wn[P(g, i, j, k)]) * idz) * (-sor / denom);
                pn[P(g, i, j, k)] = pn[P(g, i, j, k)] + phi * idt;
                // :190-241
                un[P(g, i, j, k)] = un[P(g, i, j, k)] - phi * idx * mu_u_i;
                if (!perx && i == 1) {
                    if (T[BCI(1, 0, 0)] == 0) un[P(g, i, j, k)] = un[P(g, i, j, k)] + V[BCI(1, 0, 0)] * idx * mu_u_i;
                    else un[P(g, i, j, k)] = un[P(g, i, j, k)] + (phi * idx - V[BCI(1, 0, 0)]) * mu_u_i;
                }
                un[P(g, ip, j, k)] = un[P(g, ip, j, k)] + phi * idx * mu_u_ip;
                if (!perx && i == nx) {
                    if (T[BCI(1, 1, 0)] == 0) un[P(g, ip, j, k)] = un[P(g, ip, j, k)] - V[BCI(1, 1, 0)] * idx * mu_u_ip;
                    else un[P(g, ip, j, k)] = un[P(g, ip, j, k)] + (V[BCI(1, 1, 0)] - phi * idx) * mu_u_ip;
                }
                vn[P(g, i, j, k)] = vn[P(g, i, j, k)] - phi * idy * mu_v_j;
                if (!pery && j == 1) {
                    if (T[BCI(2, 0, 0)] == 0) vn[P(g, i, j, k)] = vn[P(g, i, j, k)] + V[BCI(2, 0, 0)] * idy * mu_v_j;
                    else vn[P(g, i, j, k)] = vn[P(g, i, j, k)] + (phi * idy - V[BCI(2, 0, 0)]) * mu_v_j;
                }
                vn[P(g, i, jp, k)] = vn[P(g, i, jp, k)] + phi * idy * mu_v_jp;
                if (!pery && j == ny) {
                    if (T[BCI(2, 1, 0)] == 0) vn[P(g, i, jp, k)] = vn[P(g, i, jp, k)] - V[BCI(2, 1, 0)] * idy * mu_v_jp;
                    else vn[P(g, i, jp, k)] = vn[P(g, i, jp, k)] + (V[BCI(2, 1, 0)] - phi * idy) * mu_v_jp;
                }
                wn[P(g, i, j, k)] = wn[P(g, i, j, k)] - phi * idz * mu_w_k;
                if (!perz && k == 1) {
                    if (T[BCI(3, 0, 0)] == 0) wn[P(g, i, j, k)] = wn[P(g, i, j, k)] + V[BCI(3, 0, 0)] * idz * mu_w_k;
                    else wn[P(g, i, j, k)] = wn[P(g, i, j, k)] + (phi * idz - V[BCI(3, 0, 0)]) * mu_w_k;
                }
                wn[P(g, i, j, kp)] = wn[P(g, i, j, kp)] + phi * idz * mu_w_kp;
                if (!perz && k == nz) {
                    // :237 -- the Dirichlet branch has no mu factor in the reference
                    if (T[BCI(3, 1, 0)] == 0) wn[P(g, i, j, kp)] = wn[P(g, i, j, kp)] - V[BCI(3, 1, 0)] * idz;
                    else wn[P(g, i, j, kp)] = wn[P(g, i, j, kp)] + (V[BCI(3, 1, 0)] - phi * idz) * mu_w_kp;
                }
            }
        }
    }
}

// Discrete divergence with the sweep's neighbour rule, L2 norm and max-abs
// over the nx*ny*nz cells, and max(|u|,|v|,|w|) over the same cells.
// Summed per k plane then over planes so the result does not depend on the
// thread count.
void or_divergence_norms3(const or_grid* g, const or_bc* bc, const or_fields* f, double* l2, double* linf,
                          double* umax) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double idx = 1.0 / g->dx, idy = 1.0 / g->dy, idz = 1.0 / g->dz;
    std::vector<double> ps(nz), pm(nz), pu(nz);
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k) {
        double s = 0.0, m = 0.0, um = 0.0;
        int kp = k + 1;
        if (bc->periodic[2] && kp > nz) kp = 1;
        for (int j = 1; j <= ny; ++j) {
            int jp = j + 1;
            if (bc->periodic[1] && jp > ny) jp = 1;
            for (int i = 1; i <= nx; ++i) {
                int ip = i + 1;
                if (bc->periodic[0] && ip > nx) ip = 1;
                double d = (f->un[P(g, ip, j, k)] - f->un[P(g, i, j, k)]) * idx
                         + (f->vn[P(g, i, jp, k)] - f->vn[P(g, i, j, k)]) * idy
                         + (f->wn[P(g, i, j, kp)] - f->wn[P(g, i, j, k)]) * idz;
                s += d * d;
                m = std::max(m, std::fabs(d));
                um = std::max(um, std::max(std::fabs(f->un[P(g, i, j, k)]),
                                           std::max(std::fabs(f->vn[P(g, i, j, k)]), std::fabs(f->wn[P(g, i, j, k)]))));
            }
        }
        ps[k - 1] = s;
        pm[k - 1] = m;
        pu[k - 1] = um;
    }
    double s = 0.0, m = 0.0, um = 0.0;
    for (int k = 0; k < nz; ++k) { s += ps[k]; m = std::max(m, pm[k]); um = std::max(um, pu[k]); }
    *l2 = std::sqrt(s);
    *linf = m;
    if (umax) *umax = um;
}

void or_divergence_norms(const or_grid* g, const or_bc* bc, const or_fields* f, double* l2, double* linf) {
    or_divergence_norms3(g, bc, f, l2, linf, nullptr);
}

// pressure_projection_redblack (:27-254): copy u* into u over the padded
// arrays (:63-84), then colour sweeps.  tol <= 0 reproduces the reference's
// fixed nIter.  tol > 0 is the residual-driven extension: after every
// `check_every` full iterations the divergence L2 norm r is compared with
// max(tol * r0, atol), r0 its value on u*; atol < 0 selects the round-off
// floor eps*sqrt(ncells)*max|u*|*(1/dx+1/dy+1/dz).  Stops on convergence or
// after max_iter iterations.  Returns 0 on convergence / fixed count, 1 if
// max_iter was reached, 2 on a non-finite residual.
int or_pressure_projection_redblack(const or_grid* g, const or_bc* bc, or_fields* f, double dt_gamma,
                                    int niter, double sor, double tol, double atol, int max_iter, int check_every,
                                    int parallel, int* iters_out, double* res_out) {
    const size_t n = (size_t)(g->nx + 2) * (g->ny + 2) * (g->nz + 2);
    for (size_t t = 0; t < n; ++t) { f->un[t] = f->us[t]; f->vn[t] = f->vs[t]; f->wn[t] = f->ws[t]; }
    int status = 0;
    int it = 0;
    double r0 = 0.0, r = 0.0, linf = 0.0, umax = 0.0;
    if (tol <= 0.0) {
        for (it = 0; it < niter; ++it) {
            sor_sweep(g, bc, f, dt_gamma, sor, 0, parallel != 0);
            sor_sweep(g, bc, f, dt_gamma, sor, 1, parallel != 0);
        }
    } else {
        or_divergence_norms3(g, bc, f, &r0, &linf, &umax);
        const double eps = 2.220446049250313e-16;
        if (atol < 0.0) atol = eps * std::sqrt((double)((size_t)g->nx * g->ny * g->nz)) * umax *
                               (1.0 / g->dx + 1.0 / g->dy + 1.0 / g->dz);
        const double target = std::max(tol * r0, atol);
        r = r0;
        if (!std::isfinite(r0) || !std::isfinite(umax)) {
            if (iters_out) *iters_out = 0;
            if (res_out) *res_out = 0.0;
            return 2;
        }
        if (r0 <= target) {
            if (iters_out) *iters_out = 0;
            if (res_out) *res_out = (r0 > 0.0) ? 1.0 : 0.0;
            return 0;
        }
        status = 1;
        while (it < max_iter) {
            int m = std::min(check_every, max_iter - it);
            for (int q = 0; q < m; ++q) {
                sor_sweep(g, bc, f, dt_gamma, sor, 0, parallel != 0);
                sor_sweep(g, bc, f, dt_gamma, sor, 1, parallel != 0);
            }
            it += m;
            or_divergence_norms(g, bc, f, &r, &linf);
            if (!std::isfinite(r)) { status = 2; break; }
            if (r <= target) { status = 0; break; }
        }
    }
    if (iters_out) *iters_out = it;
    if (res_out) *res_out = (r0 > 0.0) ? r / r0 : 0.0;
    return status;
}

// One colour sweep exposed for the sweep-level parity tests.
void or_sor_sweep(const or_grid* g, const or_bc* bc, or_fields* f, double dt_gamma, double sor, int parity) {
    sor_sweep(g, bc, f, dt_gamma, sor, parity, false);
}

// ---------------------------------------------------------------------------
// IBM coefficients, src/modules/ibm.f90:84-187 (set_ibm_coeff with
// USE_IBM_SECONDORDER, the CMake default, CMakeLists.txt:11).
// geometry 0: the reference's lower-wall sinusoid (ibm.f90:45-50,94-97);
// geometry 1: the wavy channel of the configs, fluid between
//   y_lo(x) = y0 + amp*sin(2*pi*x/lambda + phase) and y_lo(x) + height.
// ---------------------------------------------------------------------------
typedef struct {
    int geometry;
    int n_wave_x;
    double amp, phase, lambda, y0, height;
} or_ibm;

static bool is_in_body(const double* x, const or_ibm* ib, const or_grid* g) {
    const double pi = 3.141592653589793;
    if (ib->geometry == 0) {
        double y_body = ib->amp * 0.5 * (1.0 + std::sin(2.0 * pi * (double)ib->n_wave_x * x[0] / g->lx + ib->phase)) + 2 * g->dy;
        return x[1] < y_body;
    }
    double y_lo = ib->y0 + ib->amp * std::sin(2.0 * pi * x[0] / ib->lambda + ib->phase);
    double y_hi = y_lo + ib->height;
    return x[1] < y_lo || x[1] > y_hi;
}

// NORM2 with the scaled-sum algorithm of the Fortran runtime; for the
// axis-aligned differences used here it returns |d| exactly.
static double norm2_3(const double* v) {
    double scale = 0.0, ssq = 1.0;
    for (int t = 0; t < 3; ++t) {
        if (v[t] != 0.0) {
            double a = std::fabs(v[t]);
            if (scale < a) { double q = scale / a; ssq = 1.0 + ssq * (q * q); scale = a; }
            else { double q = a / scale; ssq = ssq + q * q; }
        }
    }
    return scale * std::sqrt(ssq);
}

static void bisection(const double* xAin, double* xB, const or_ibm* ib, const or_grid* g) {  // ibm.f90:101-130
    double xa[3] = {xAin[0], xAin[1], xAin[2]};
    double xb[3] = {xB[0], xB[1], xB[2]};
    double xm[3] = {0, 0, 0};
    for (int it = 1; it <= 200; ++it) {
        for (int t = 0; t < 3; ++t) xm[t] = 0.5 * (xa[t] + xb[t]);
        double d[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
        if (norm2_3(d) < 1.0e-10) break;
        bool la = is_in_body(xa, ib, g);
        bool lm = is_in_body(xm, ib, g);
        if (lm == la) { for (int t = 0; t < 3; ++t) xa[t] = xm[t]; }
        else { for (int t = 0; t < 3; ++t) xb[t] = xm[t]; }
    }
    for (int t = 0; t < 3; ++t) xB[t] = xm[t];
}

void or_set_ibm_coeff(const or_grid* g, const or_ibm* ib, double* coeff, int dix, int diy, int diz) {
    const int ni = g->nx + 2, nj = g->ny + 2, nk = g->nz + 2;
    static const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    #pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 1; iz <= nk; ++iz)
        for (int iy = 1; iy <= nj; ++iy)
            for (int ix = 1; ix <= ni; ++ix) {
                double c = 0.0;
                double xA[3];
                xA[0] = ((double)ix - (double)dix * 0.5 - 1.5) * g->dx;
                xA[1] = ((double)iy - (double)diy * 0.5 - 1.5) * g->dy;
                xA[2] = ((double)iz - (double)diz * 0.5 - 1.5) * g->dz;
                if (is_in_body(xA, ib, g)) {
                    c = 1.0e30;
                } else {
                    for (int n = 0; n < 6; ++n) {
                        double xB[3];
                        xB[0] = ((double)(ix + nb[n][0]) - (double)dix * 0.5 - 1.5) * g->dx;
                        xB[1] = ((double)(iy + nb[n][1]) - (double)diy * 0.5 - 1.5) * g->dy;
                        xB[2] = ((double)(iz + nb[n][2]) - (double)diz * 0.5 - 1.5) * g->dz;
                        double dd[3] = {xB[0] - xA[0], xB[1] - xA[1], xB[2] - xA[2]};
                        double d0 = norm2_3(dd);
                        if (is_in_body(xB, ib, g)) {
                            bisection(xA, xB, ib, g);
                            double de[3] = {xB[0] - xA[0], xB[1] - xA[1], xB[2] - xA[2]};
                            double d = norm2_3(de);
                            c = c + ((d0 - d) / d) / (d0 * d0);
                        }
                    }
                }
                coeff[(size_t)(ix - 1) + (size_t)ni * ((size_t)(iy - 1) + (size_t)nj * (iz - 1))] = c;
            }
    const size_t n = (size_t)ni * nj * nk;
    for (size_t t = 0; t < n; ++t) coeff[t] = coeff[t] / g->re;  // ibm.f90:186
}

// ---------------------------------------------------------------------------
// Seeded channel initial condition (new: the reference zero-initialises,
// src/modules/init.f90:67-70).  Counter-based SplitMix64: the 64-bit finaliser
// of Steele, Lea & Flood (2014) applied to seed + golden * (field<<40 | index).
// u = max(0, 1 - (y - yc)^2) + U(-amp_u, amp_u) at the u faces, v and w
// U(-amp_vw, amp_vw); yc = y0 + 1 (+ wall wave for the wavy channel, if
// wave_amp != 0).  Interior cells only; ghosts and p are zero.
// ---------------------------------------------------------------------------
static inline uint64_t ic_hash(uint64_t seed, uint64_t field, uint64_t lin) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * ((field << 40) | lin);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline double ic_uniform(uint64_t seed, uint64_t field, uint64_t lin, double amp) {
    double u01 = (double)(ic_hash(seed, field, lin) >> 11) * (1.0 / 9007199254740992.0);
    return amp * (2.0 * u01 - 1.0);
}

void or_channel_ic(const or_grid* g, uint64_t seed, double amp_u, double amp_vw, double y0,
                   double wave_amp, double wave_lambda, double* un, double* vn, double* wn) {
    const double pi = 3.141592653589793;
    for (int k = 1; k <= g->nz; ++k)
        for (int j = 1; j <= g->ny; ++j)
            for (int i = 1; i <= g->nx; ++i) {
                const size_t t = P(g, i, j, k);
                const double x = (double)(i - 1) * g->dx;
                const double y = ((double)j - 0.5) * g->dy;
                double yc = y0 + 1.0;
                if (wave_amp != 0.0) yc = yc + wave_amp * std::sin(2.0 * pi * x / wave_lambda);
                const double e = y - yc;
                double base = 1.0 - e * e;
                if (base < 0.0) base = 0.0;
                un[t] = base + ic_uniform(seed, 0, t, amp_u);
                vn[t] = (j == 1) ? 0.0 : ic_uniform(seed, 1, t, amp_vw);
                wn[t] = ic_uniform(seed, 2, t, amp_vw);
            }
}

// ---------------------------------------------------------------------------
// Driver: nsteps RK3 steps, src/main.f90:66-90 (fixed dt, no output).
// solver 0: FFT path (apply_bc before and after the projection);
// solver 1: red-black (no apply_bc after the predictor; apply_bc_redblack
// after the projection).  Returns the worst SOR status.
// ---------------------------------------------------------------------------
int or_run(const or_grid* g, const or_bc* bc, or_fields* f, double dt, int nsteps, int solver,
           int niter, double sor, double tol, double atol, int max_iter, int check_every, int parallel,
           int* total_iters) {
    double a[3], b[3], c[3];
    or_rk_coeffs(a, b, c);
    int worst = 0, tot = 0;
    for (int step = 1; step <= nsteps; ++step) {
        for (int s = 0; s < 3; ++s) {
            const double dt_alpha = dt * a[s], dt_beta = dt * b[s], dt_gamma = dt * c[s];
            or_momentum(g, bc, f, dt_alpha, dt_beta, dt_gamma);
            if (solver == 0) {
                or_apply_bc(g, f);
                or_pressure_projection_fft(g, f, dt_gamma, nullptr);
                or_apply_bc(g, f);
            } else {
                int it = 0;
                double res = 0.0;
                int st = or_pressure_projection_redblack(g, bc, f, dt_gamma, niter, sor, tol, atol, max_iter, check_every,
                                                         parallel, &it, &res);
                tot += it;
                if (st > worst) worst = st;
                or_apply_bc_redblack(g, bc, f);
            }
        }
    }
    if (total_iters) *total_iters = tot;
    return worst;
}

void or_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
