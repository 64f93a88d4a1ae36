// mdx_main.cpp -- host driver of libmobyb200, the C++ counterpart of the
// reference's program main (src/main.f90:10-120): read input.ini, set up
// fields, pressure solver and IBM, run the RK3 loop through the C ABI with
// the same call order, CFL/adaptive dt and VTK output, and print the same
// progress and timing lines.
//
//   mdx_main [input.ini]
//
// In the reference the driver stays Fortran and binds the same C entry
// points through iso_c_binding; this program exists because no Fortran
// compiler is available here, and it is the end-to-end user of the library.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mobydiff_b200.h"

static void die(mdx_ctx_t* ctx, int rc, const char* what) {
    std::fprintf(stderr, "error: %s failed (%d): %s\n", what, rc, mdx_last_error(ctx));
    std::exit(1);
}
#define CHECK(ctx, call)                       \
    do {                                       \
        int rc__ = (call);                     \
        if (rc__ != MDX_OK) die(ctx, rc__, #call); \
    } while (0)

static bool output_is_due(int step, int interval) {   // io.f90:31-39
    return interval > 0 && step % interval == 0;
}

// Legacy-ASCII VTK of cell-centred velocity, io.f90:168-259 (same header
// lines and ES20.12 number format).
// write_field, src/modules/io.f90:105-137: "<prefix>_<step>.h5" through the
// reference's own entry point, with the driver's grid and time.
static int write_field(mdx_ctx_t* ctx, const mdx_grid_t& g, int step, const char* prefix) {
    char name[600];
    std::snprintf(name, sizeof(name), "%s_%d.h5", prefix, step);
    std::printf(" current time step: %12d   field filename: %s\n", step, name);
    const size_t n = (size_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
    std::vector<double> h(4 * n);
    int rc = mdx_update_host(ctx, h.data(), h.data() + n, h.data() + 2 * n, h.data() + 3 * n);
    if (rc != MDX_OK) return rc;
    if (fdm_h5_write_field(name, g.nx, g.ny, g.nz, g.lx, g.ly, g.lz, g.dx, g.dy, g.dz, g.re, g.dt, g.t_current,
                           h.data(), h.data() + n, h.data() + 2 * n, h.data() + 3 * n) != 0) {
        std::printf(" error: could not write HDF5 field file: %s\n", name);
        return MDX_ERR_IO;
    }
    return MDX_OK;
}

// One value under the Fortran edit descriptor ES20.12 (io.f90:237-257):
// 12 digits after the point, exponent E+dd, and for a three-digit exponent
// the form +ddd without the letter E; right-justified in 20 characters.
static void put_es20_12(FILE* fp, double x) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.12E", x);
    char* e = std::strchr(b, 'E');
    if (e && std::strlen(e + 2) > 2) std::memmove(e, e + 1, std::strlen(e + 1) + 1);   // E+123 -> +123
    std::fprintf(fp, "%20s", b);
}

static int write_vtk(mdx_ctx_t* ctx, const mdx_grid_t& g, int step, const char* prefix) {
    char name[512];
    std::snprintf(name, sizeof(name), "%s_%d.vtk", prefix, step);
    std::printf(" current time step: %12d    filename: %s   cfl: %23.15E\n", step, name, g.cfl * g.dt);
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    std::vector<double> uc(n), vc(n), wc(n);
    int rc = mdx_center_vel(ctx, uc.data(), vc.data(), wc.data());
    if (rc != MDX_OK) return rc;
    FILE* fp = std::fopen(name, "w");
    if (!fp) return MDX_ERR_IO;
    std::fprintf(fp, "# vtk DataFile Version 3.0\n3D velocity field\nASCII\nDATASET STRUCTURED_POINTS\n");
    std::fprintf(fp, "DIMENSIONS %d %d %d\n", g.nx + 1, g.ny + 1, g.nz + 1);
    std::fprintf(fp, "ORIGIN ");
    for (double x : {0.0, 0.0, 0.0}) put_es20_12(fp, x);
    std::fprintf(fp, "\nSPACING ");
    for (double x : {g.dx, g.dy, g.dz}) put_es20_12(fp, x);
    std::fprintf(fp, "\nFIELD FieldData 1\nTIME 1 1 double\n");
    put_es20_12(fp, g.t_current);
    std::fprintf(fp, "\nCELL_DATA %zu\nVECTORS U double\n", n);
    for (size_t t = 0; t < n; ++t) {
        put_es20_12(fp, uc[t]);
        put_es20_12(fp, vc[t]);
        put_es20_12(fp, wc[t]);
        std::fputc('\n', fp);
    }
    std::fclose(fp);
    return MDX_OK;
}

int main(int argc, char** argv) {
    const char* input = (argc > 1 && argv[1][0]) ? argv[1] : "input.ini";
    mdx_grid_t g;
    mdx_bc_t bc;
    mdx_solver_opts_t opts;
    mdx_run_config_t run;

    std::printf(" initialising grid...\n");
    mdx_default_grid(&g);
    std::printf(" initialising BCs...\n");
    mdx_default_bc(&bc);
    mdx_default_solver_opts(&opts);
    CHECK(nullptr, mdx_read_runtime_config(input, &g, &bc, &opts, &run));
    int ndev = 0;
    if (mdx_device_count(&ndev) != MDX_OK) die(nullptr, MDX_ERR_NO_DEVICE, "mdx_device_count");
    std::printf(" CUDA devices available: %d\n", ndev);

    std::printf(" initialising fields...\n");
    mdx_ctx_t* ctx = nullptr;
    CHECK(nullptr, mdx_create(0, &g, &bc, &ctx));
    CHECK(ctx, mdx_enter_field_data(ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                    nullptr, nullptr));   // init_field: everything zero

    std::printf(" initialising pressure solver...\n");
    CHECK(ctx, mdx_init_pressure_solver(ctx, &opts));
    if (run.guess != MDX_GUESS_ZERO) CHECK(ctx, mdx_set_pressure_guess(ctx, run.guess, 1));

    std::printf(" initialising IBM...\n");
    const size_t npad = (size_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
    std::vector<double> cu, cv, cw;
    double y0 = run.ibm_y0 < 0.0 ? (g.ly - run.ibm_height) / 2.0 : run.ibm_y0;
    double lam = run.ibm_lambda > 0.0 ? run.ibm_lambda : g.lx / 2.0;
    if (run.ibm >= 0) {
        mdx_ibm_geom_t geom;
        std::memset(&geom, 0, sizeof(geom));
        geom.geometry = run.ibm;
        geom.n_wave_x = 1;
        if (run.ibm == 0) {
            geom.amp = 5 * g.dy;   // ibm.f90:45-50
        } else {
            geom.amp = run.ibm_amp;
            geom.lambda = lam;
            geom.y0 = y0;
            geom.height = run.ibm_height;
        }
        cu.resize(npad);
        cv.resize(npad);
        cw.resize(npad);
        CHECK(nullptr, mdx_set_ibm_coeff(&g, &geom, cu.data(), 1, 0, 0));
        CHECK(nullptr, mdx_set_ibm_coeff(&g, &geom, cv.data(), 0, 1, 0));
        CHECK(nullptr, mdx_set_ibm_coeff(&g, &geom, cw.data(), 0, 0, 1));
        CHECK(ctx, mdx_enter_ibm_data(ctx, cu.data(), cv.data(), cw.data()));
    }
    if (run.ic == 1) {
        mdx_solve_stats_t st;
        const double wave = (run.ibm == 1) ? run.ibm_amp : 0.0;
        const double ic_y0 = (run.ibm == 1) ? y0 : (g.ly - 2.0) / 2.0;
        CHECK(ctx, mdx_channel_ic(ctx, run.seed, 0.1, 0.01, ic_y0, wave, lam, &st));
    }

    std::printf(" main loop starting...\n");
    std::fflush(stdout);
    auto t0 = std::chrono::steady_clock::now();
    long long total_iters = 0;
    // src/main.f90:66-106.  The steps up to the next output run in one
    // mdx_step_adaptive call: t += dt, the three substages, then with
    // cflmax > 0 the CFL and dt = min(cflmax/cfl, dtmax) after every step
    // (on the FFT path inside the step's CUDA graph, on the device).
    auto next_due = [](int i, int interval) { return interval > 0 ? ((i + interval - 1) / interval) * interval : 0; };
    for (int i = 1; i <= g.nsteps;) {
        int last = g.nsteps;
        if (run.output_interval > 0) last = std::min(last, next_due(i, run.output_interval));
        if (run.field_interval > 0) last = std::min(last, next_due(i, run.field_interval));
        long long it = 0;
        CHECK(ctx, mdx_step_adaptive(ctx, last - i + 1, g.cflmax, g.dtmax, &it));
        total_iters += it;
        CHECK(ctx, mdx_get_time(ctx, &g.dt, &g.t_current, &g.cfl));
        i = last;
        // main.f90:92-93: the CFL is also computed when output is due
        if (!(g.cflmax > 0.0) && output_is_due(i, run.output_interval)) CHECK(ctx, mdx_get_cfl(ctx, &g.cfl));
        if (run.output_interval > 0 && output_is_due(i, run.output_interval))
            CHECK(ctx, write_vtk(ctx, g, i, run.output_prefix));
        if (run.field_interval > 0 && output_is_due(i, run.field_interval))   // io.f90:95-137
            CHECK(ctx, write_field(ctx, g, i, run.field_prefix));
        ++i;
    }
    double dummy = 0.0;
    CHECK(ctx, mdx_divergence_norms(ctx, &dummy, &dummy));   // drains the stream
    auto t1 = std::chrono::steady_clock::now();
    const double loop_seconds = std::chrono::duration<double>(t1 - t0).count();
    std::printf(" main loop ended...\n");
    std::printf("timing: nsteps %d loop_seconds %16.8E seconds_per_step %16.8E\n", g.nsteps, loop_seconds,
                loop_seconds / (double)g.nsteps);
    if (opts.solver == MDX_SOLVER_REDBLACK) std::printf("red-black iterations: %lld\n", total_iters);
    mdx_destroy_pressure_solver(ctx);
    mdx_exit_ibm_data(ctx);
    mdx_exit_field_data(ctx);
    mdx_destroy(ctx);
    return 0;
}
