// k_ibm.cu -- IBM coefficients generated on the device: set_ibm_coeff,
// src/modules/ibm.f90:133-187 (USE_IBM_SECONDORDER, the CMake default), with
// isInBody (:84-99) and the bisection (:101-130).
//
// One thread per padded cell.  A solid cell gets SOLID = 1e30 (:20, :165); a
// fluid cell sums, over its six neighbours that lie in the body, ((d0-d)/d)/d0^2
// with d0 the neighbour distance and d the distance to the wall found by
// bisection (tolerance 1e-10, at most 200 halvings, :21-22); everything is
// divided by Re (:186).  This file is compiled with -fmad=false and keeps the
// host restatement's expression order (host_config.cpp, mdx_set_ibm_coeff), and
// sqrt and division are correctly rounded on both, so the two agree bit for
// bit wherever the host's and the device's sin agree; sin may differ in the
// last bit, which can only move a bisection decision for a point within one
// rounding of the wall.
//
// The wall geometries depend on x and y only, so the coefficients of every z
// plane are equal; the context keeps its z-invariant fast path.
#include "mdx_internal.cuh"

#include <algorithm>

namespace {

struct ibm_dev {
    int geometry, n_wave_x;
    double amp, phase, lambda, y0, height;
    double dx, dy, dz, lx, re;
};

__device__ bool in_body(const double* x, const ibm_dev& b) {   // ibm.f90:84-99, and the wavy channel
    const double pi = 3.141592653589793;
    if (b.geometry == 0) {
        const double y_body = b.amp * 0.5 * (1.0 + sin(2.0 * pi * (double)b.n_wave_x * x[0] / b.lx + b.phase)) + 2 * b.dy;
        return x[1] < y_body;
    }
    const double y_lo = b.y0 + b.amp * sin(2.0 * pi * x[0] / b.lambda + b.phase);
    return x[1] < y_lo || x[1] > y_lo + b.height;
}

// Euclidean norm by the scaled sum of squares (the Fortran NORM2 method).
__device__ double norm2(const double* v) {
    double scale = 0.0, ssq = 1.0;
    for (int t = 0; t < 3; ++t) {
        if (v[t] == 0.0) continue;
        const double a = fabs(v[t]);
        if (scale < a) {
            const double q = scale / a;
            ssq = 1.0 + ssq * (q * q);
            scale = a;
        } else {
            const double q = a / scale;
            ssq = ssq + q * q;
        }
    }
    return scale * sqrt(ssq);
}

__device__ void bisect(const double* xa_in, double* xb_io, const ibm_dev& b) {   // ibm.f90:101-130
    double xa[3] = {xa_in[0], xa_in[1], xa_in[2]};
    double xb[3] = {xb_io[0], xb_io[1], xb_io[2]};
    double xm[3] = {0.0, 0.0, 0.0};
    for (int it = 0; it < 200; ++it) {
        for (int t = 0; t < 3; ++t) xm[t] = 0.5 * (xa[t] + xb[t]);
        const double dd[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
        if (norm2(dd) < 1.0e-10) break;
        const bool la = in_body(xa, b), lm = in_body(xm, b);
        double* dst = (lm == la) ? xa : xb;
        for (int t = 0; t < 3; ++t) dst[t] = xm[t];
    }
    for (int t = 0; t < 3; ++t) xb_io[t] = xm[t];
}

__device__ void coord(const ibm_dev& b, int dix, int diy, int diz, int ix, int iy, int iz, double* x) {   // :161-163
    x[0] = ((double)ix - (double)dix * 0.5 - 1.5) * b.dx;
    x[1] = ((double)iy - (double)diy * 0.5 - 1.5) * b.dy;
    x[2] = ((double)iz - (double)diz * 0.5 - 1.5) * b.dz;
}

// Coefficient of padded cell (ix, iy, iz), 1-based as in the reference loops.
__device__ double coeff_cell(const ibm_dev& b, int dix, int diy, int diz, int ix, int iy, int iz) {
    double xa[3];
    coord(b, dix, diy, diz, ix, iy, iz, xa);
    if (in_body(xa, b)) return 1.0e30;   // SOLID
    const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    double c = 0.0;
    for (int n = 0; n < 6; ++n) {
        double xb[3];
        coord(b, dix, diy, diz, ix + nb[n][0], iy + nb[n][1], iz + nb[n][2], xb);
        const double d0v[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
        const double d0 = norm2(d0v);
        if (in_body(xb, b)) {
            bisect(xa, xb, b);
            const double dv[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
            const double d = norm2(dv);
            c = c + ((d0 - d) / d) / (d0 * d0);
        }
    }
    return c;
}

// The first `planes` z planes (all nz+2 for a padded array, 1 for a plane) of
// component (dix, diy, diz), Fortran order.
__global__ void k_ibm_coeff(ibm_dev b, int ni, int nj, int planes, int dix, int diy, int diz,
                            double* __restrict__ coeff) {
    const long long n = (long long)ni * nj * planes;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(t % ni) + 1;
        const long long r = t / ni;
        const int iy = (int)(r % nj) + 1;
        const int iz = (int)(r / nj) + 1;
        coeff[t] = coeff_cell(b, dix, diy, diz, ix, iy, iz) / b.re;   // :186
    }
}

ibm_dev make_dev(const mdx_grid_t* g, const mdx_ibm_geom_t* geom) {
    ibm_dev b;
    b.geometry = geom->geometry;
    b.n_wave_x = geom->n_wave_x;
    b.amp = geom->amp; b.phase = geom->phase; b.lambda = geom->lambda; b.y0 = geom->y0; b.height = geom->height;
    b.dx = g->dx; b.dy = g->dy; b.dz = g->dz; b.lx = g->lx; b.re = g->re;
    return b;
}

int check_geom(const mdx_grid_t* g, const mdx_ibm_geom_t* geom) {
    if (!g || !geom) return MDX_ERR_ARG;
    if (geom->geometry != 0 && geom->geometry != 1) return MDX_ERR_ARG;
    if (geom->geometry == 1 && !(geom->lambda != 0.0)) return MDX_ERR_ARG;
    if (g->nx < 1 || g->ny < 1 || g->nz < 1) return MDX_ERR_ARG;
    return MDX_OK;
}

}  // namespace

// Device planes or padded arrays of one component, for callers inside the
// library (the ensemble builds its members' z-invariant planes with it).
int mdx_ibm_coeff_launch(const mdx_grid_t* g, const mdx_ibm_geom_t* geom, double* d_coeff, int dix, int diy, int diz,
                         int planes, cudaStream_t stream) {
    const int rc = check_geom(g, geom);
    if (rc != MDX_OK) return rc;
    const int ni = g->nx + 2, nj = g->ny + 2;
    const long long n = (long long)ni * nj * planes;
    const int nb = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    k_ibm_coeff<<<nb, 256, 0, stream>>>(make_dev(g, geom), ni, nj, planes, dix, diy, diz, d_coeff);
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

extern "C" int mdx_set_ibm_coeff_device(const mdx_grid_t* g, const mdx_ibm_geom_t* geom, double* d_coeff, int dix,
                                        int diy, int diz, void* stream) {
    if (!d_coeff) return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_set_ibm_coeff_device: null coefficient array");
    const int rc = mdx_ibm_coeff_launch(g, geom, d_coeff, dix, diy, diz, g ? g->nz + 2 : 0, (cudaStream_t)stream);
    if (rc == MDX_ERR_ARG) return mdx_fail(nullptr, rc, "mdx_set_ibm_coeff_device: bad grid or geometry");
    if (rc != MDX_OK) return mdx_fail(nullptr, rc, "mdx_set_ibm_coeff_device: launch failed");
    return MDX_OK;
}
