/*
 * mobydiff_b200.h -- C ABI of libmobyb200.so, the sm_100a implementation of
 * the mobydiff RK3 time step.
 *
 * The entry points replace the OpenMP-offload bodies of the reference's
 * Fortran modules one for one.  Each declaration names the reference
 * interface it stands in for (paths relative to the mobydiff project root).
 * A Fortran caller binds them with iso_c_binding (the bind(C) interfaces are
 * in mobydiff_b200/fortran/mdx_bindings.f90); the driver, the INI reader, I/O
 * and IBM geometry set-up stay on the host.
 *
 * Conventions
 *   - Every call returns an int status: MDX_OK (0) or one of MDX_ERR_*;
 *     mdx_last_error() gives the message of the last failure on a context.
 *   - Field arrays are the reference's host arrays, unchanged: padded
 *     (0:nx+1,0:ny+1,0:nz+1) in Fortran order, element (i,j,k) at
 *     i + (nx+2)*(j + (ny+2)*k); oldrhs* are (1:nx,1:ny,1:nz).
 *     src/modules/init.f90:14-19, src/modules/field_hdf5.c:4-7.
 *   - Device mirrors are owned by the context (allocated in
 *     mdx_enter_field_data, freed in mdx_exit_field_data), like OpenMP
 *     `target enter/exit data` in src/modules/gpu_runtime.f90:22-48.
 *   - One CUDA stream per context; calls are stream-ordered and return without
 *     a host synchronisation except where they hand results to the host
 *     (updates to the host, CFL, projection statistics).
 *   - Single host thread per context.
 */
#ifndef MOBYDIFF_B200_H
#define MOBYDIFF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MDX_OK                0
#define MDX_ERR_ARG           1   /* invalid argument / unsupported size      */
#define MDX_ERR_CUDA          2   /* a CUDA runtime call failed               */
#define MDX_ERR_NO_DEVICE     3   /* no usable CUDA device                    */
#define MDX_ERR_STATE         4   /* call out of order (e.g. no field data)   */
#define MDX_NOT_CONVERGED     5   /* SOR hit max_iter before the tolerance    */
#define MDX_ERR_NONFINITE     6   /* NaN/Inf detected in a residual or field  */
#define MDX_ERR_IO            7   /* file could not be read / parsed          */
#define MDX_ERR_TIMEOUT       8   /* a bounded device wait gave up            */

/* ---- pressure solvers / precisions ------------------------------------ */
#define MDX_SOLVER_FFT        0   /* batched x-z real FFT + Thomas in y      */
#define MDX_SOLVER_REDBLACK   1   /* red-black SOR                            */
#define MDX_PREC_FP64         0
#define MDX_PREC_MIXED        1   /* FP32 inner solve in FP64 defect correction */

/* ---- field identifiers for mdx_copy_field ----------------------------- */
enum {
    MDX_UN = 0, MDX_US, MDX_VN, MDX_VS, MDX_WN, MDX_WS, MDX_PN,
    MDX_OLDRHSU, MDX_OLDRHSV, MDX_OLDRHSW,
    MDX_COEF_U, MDX_COEF_V, MDX_COEF_W,
    MDX_PHI,          /* last pressure correction, rhs(nx,nz,ny) layout (FFT path) */
    MDX_NUM_FIELDS
};

/* grid_type, src/modules/init.f90:5-12 (same components, same order). */
typedef struct {
    int nx, ny, nz;
    int nsteps;
    double lx, ly, lz;
    double dx, dy, dz;
    double re, dt, t_final, t_current, cfl, cflmax, dtmax;
    double forcing_x, forcing_y, forcing_z;
} mdx_grid_t;

/* boundary_type, src/modules/boundary.f90:6-10.  bc_type / bc_value keep the
 * Fortran memory order of bcType(1:3,0:1,0:3): index (dir-1)+3*(side+2*var),
 * dir x/y/z = 1..3, side min/max = 0/1, var p/u/v/w = 0..3; 0 Dirichlet,
 * 1 Neumann. */
typedef struct {
    int is_periodic[3];
    int bc_type[24];
    double bc_value[24];
} mdx_bc_t;

/* pressure_solver_type knobs (src/modules/pressure_workspace.f90:7-8) plus the
 * [b200] input.ini section.  mdx_default_solver_opts() fills the reference
 * defaults (FFT, nIter 3, sor 1.5, fixed iteration count). */
typedef struct {
    int solver;        /* MDX_SOLVER_*                                        */
    int n_iter;        /* red-black: sweeps per projection when tol <= 0      */
    double sor;        /* red-black over-relaxation factor                    */
    double tol;        /* red-black: stop when ||div u||2 <= tol*||div u*||2; <= 0: fixed n_iter */
    int max_iter;      /* red-black: iteration cap when tol > 0               */
    int check_every;   /* red-black: iterations between residual checks       */
    int precision;     /* MDX_PREC_*                                          */
    int sor_variant;   /* red-black kernels (bit-identical results): 0 auto -- the
                          first projection times each variant on one residual-check
                          block of its own iterations and keeps the fastest; 1 one
                          launch per colour; 2 fused red+black pass, 32x8 tiles;
                          3 fused pass, 32x16 tiles; 4 one launch per colour on
                          colour-split copies of u, v, w, p made once per projection;
                          5 the same with two cells per thread and 16-byte accesses
                          (2-5: periodic x and z, IBM factors 1 or z-invariant).
                          FP32 sweeps of the mixed precision: 1 one launch per colour,
                          one cell per thread; 2 or 3 the fused red+black pass (one
                          launch per iteration) in the fastest of four tile shapes; 4 or
                          5 one launch per colour with 2 or 4 cells per thread, the faster;
                          0 the fastest of all seven, each timed on one block of the
                          first iterations (all give the same bits).  In the potential
                          form (inner_form 0 or 2): 1-15 pin one shape of its sweep
                          kernels, 0 the fastest of those the grid allows (all give the
                          same bits) */
    int sor_kz;        /* z planes per block of the fused pass (0: default 16) */
    int check_mode;    /* red-black, tol > 0: 0 (default) residual checks at multiples of check_every,
                          up to 8 blocks apart while the residual falls at a steady rate that
                          puts the target more than twice as far; 1: every check_every
                          iterations (the stop is then the first multiple of check_every that
                          meets the target) */
    int fft_kernel;    /* FFT path: 0 (default) warp-shuffle transforms where nx/2 and nz are
                          32, 64, 128, 256 or 512 (shared-memory Stockham otherwise); 1 always
                          the shared-memory Stockham transforms */
    int inner_form;    /* mixed-precision red-black: what the FP32 correction sweeps carry.
                          0 (default): the potential form -- the accumulated phi of each
                          cell alone, swept with the 7-point stencil that the face updates
                          of pressure_redblack.f90:117-241 amount to (the same iteration in
                          exact arithmetic; 8 B per cell per colour sweep instead of 30),
                          where nx is a multiple of 4, the face form otherwise; the ensemble
                          keeps the face form; 1: the face form (corrections du, dv, dw, dp
                          updated face by face, kernels chosen by sor_variant); 2: the
                          potential form in the ensemble's persistent kernel as well */
    int reserved_i[2];
    double atol;       /* red-black: absolute floor of ||div u||2, also accepted as converged.
                          < 0 (default): the FP64 round-off level of the divergence,
                          eps*sqrt(nx*ny*nz)*max|u*|*(1/dx+1/dy+1/dz); 0: none */
    double inner_sor;  /* mixed precision: over-relaxation of the FP32 correction sweeps
                          (the outer FP64 test is unchanged); <= 0 (default): sor */
    double reserved_d[6];
} mdx_solver_opts_t;

/* Statistics of the last pressure projection. */
typedef struct {
    int iterations;     /* red-black iterations (red+black = 1); 0 for FFT   */
    int status;         /* MDX_OK / MDX_NOT_CONVERGED / MDX_ERR_NONFINITE    */
    double residual;    /* final ||div u||2 / ||div u*||2 (red-black)        */
    double residual0;   /* ||div u*||2                                       */
    double atol;        /* absolute floor used (red-black)                   */
    int variant;        /* red-black kernel variant of the last iterations;
                           100 + n: mixed precision with n FP64 corrections
                           (300 + n with the fused FP32 pass, 500 + n with the
                           FP32 sweeps of 2 or 4 cells per thread, 700 + n with
                           the potential form, opts.inner_form);
                           200 + n: FFT path in mixed precision, n FP64 passes
                           (iterations = n as well) */
    int guessed;        /* 1 when a warm-start guess was applied             */
} mdx_solve_stats_t;

/* Warm starts of the red-black projection (no counterpart in the reference,
 * which starts every projection from phi = 0). */
#define MDX_GUESS_ZERO        0   /* the reference's start                          */
#define MDX_GUESS_PREVIOUS    1   /* increment of the same RK substage, previous step */
#define MDX_GUESS_LEARNED     2   /* extrapolated increment plus the U-Net's correction
                                     predicted from the divergence it leaves           */
#define MDX_GUESS_EXTRAPOLATED 3  /* 2*dp(n-1) - dp(n-2) of the same RK substage      */

/* Per-kernel-class device time, filled when timing is on (mdx_set_timing).
 * MDX_T_SOR_BLOCK is not a kernel class: it is the device time of each run of
 * back-to-back red-black sweep launches between two residual checks, every
 * run timed, with `launches` the sweep launches inside the timed runs. */
enum {
    MDX_T_MOMENTUM = 0, MDX_T_BC, MDX_T_FFT_FWD, MDX_T_THOMAS, MDX_T_FFT_INV,
    MDX_T_CORRECT, MDX_T_SOR_SWEEP, MDX_T_RESIDUAL, MDX_T_OTHER, MDX_T_SOR_BLOCK, MDX_T_NUM
};
typedef struct {
    double ms[MDX_T_NUM];
    long long launches[MDX_T_NUM];
} mdx_timing_t;

typedef struct mdx_ctx mdx_ctx_t;

/* ---- library / device ------------------------------------------------- */

/* Library version string. */
const char* mdx_version(void);

/* Replaces init_openmp_offload, src/modules/gpu_runtime.f90:11-20: reports
 * the number of CUDA devices (0 when none; returns MDX_ERR_NO_DEVICE then). */
int mdx_device_count(int* count);

/* Message of the last failed call on ctx (or of the last failed
 * context-less call when ctx is NULL). */
const char* mdx_last_error(const mdx_ctx_t* ctx);

/* Fill the reference defaults: mdx_grid_t from init_grid
 * (src/modules/init.f90:23-44), mdx_bc_t from init_bc
 * (src/modules/boundary.f90:14-20), solver options from
 * pressure_workspace.f90:7-8 with the FFT solver. */
void mdx_default_grid(mdx_grid_t* g);
void mdx_default_bc(mdx_bc_t* bc);
void mdx_default_solver_opts(mdx_solver_opts_t* o);

/* finalize_grid, src/modules/init.f90:38-44: dx,dy,dz and t_final. */
void mdx_finalize_grid(mdx_grid_t* g);

/* ---- host-side helpers (no device needed) ------------------------------ */

/* read_runtime_config, src/modules/config.f90:10-75, with the same
 * sections, keys, aliases, comment rules and warnings; plus the [b200]
 * section (solver, tol, omega, max_iter, check_every, precision, seed, ...).
 * A missing file keeps the defaults (config.f90:33-45) and returns MDX_OK.
 * Outputs may be NULL. */
typedef struct {
    int output_interval;
    int field_interval;
    char output_prefix[256];
    char field_prefix[256];
    /* [b200] section */
    int ic;              /* 0 = zero fields (reference), 1 = seeded channel IC */
    uint64_t seed;
    int ibm;             /* -1 none, 0 reference bump (ibm.f90:45-50), 1 wavy channel */
    double ibm_amp, ibm_lambda, ibm_y0, ibm_height;
    int warnings;        /* number of warnings printed */
    int guess;           /* red-black warm start: MDX_GUESS_ZERO / _PREVIOUS / _EXTRAPOLATED */
} mdx_run_config_t;
int mdx_read_runtime_config(const char* path, mdx_grid_t* g, mdx_bc_t* bc, mdx_solver_opts_t* opts,
                            mdx_run_config_t* run);

/* set_ibm_coeff with USE_IBM_SECONDORDER, src/modules/ibm.f90:133-187, on the
 * host (the reference computes the coefficients on the host once).
 * geometry 0: the reference's lower-wall sinusoid with amp (ibm.f90:84-99);
 * geometry 1: wavy channel, fluid for y_lo(x) < y < y_lo(x)+height with
 * y_lo(x) = y0 + amp*sin(2*pi*x/lambda + phase).
 * coeff: padded array; dix/diy/diz select the u/v/w staggering. */
typedef struct {
    int geometry;
    int n_wave_x;
    double amp, phase, lambda, y0, height;
} mdx_ibm_geom_t;
/* ---- field files (HDF5), src/modules/field_hdf5.c ------------------------
 * The reference's two C entry points under their own names and signatures
 * (field_hdf5.c:149-204, bound by io.f90:7-24), written without libhdf5:
 * root attributes nx, ny, nz (int32) and lx, ly, lz, dx, dy, dz, re, dt,
 * t_current (float64), datasets un, vn, wn, pn (float64, dims
 * (nx+2, ny+2, nz+2), C order).  Host arrays in the padded Fortran layout.
 * Return 0 on success, 1 on any failure, as the reference does. */
int fdm_h5_write_field(const char* filename, int nx, int ny, int nz, double lx, double ly, double lz, double dx,
                       double dy, double dz, double re, double dt, double t_current, const double* un,
                       const double* vn, const double* wn, const double* pn);
int fdm_h5_read_field(const char* filename, int nx, int ny, int nz, double* un, double* vn, double* wn, double* pn);
/* The scalar root attributes of a field file (no counterpart in the
 * reference, whose read_field reads the datasets only): dims = nx, ny, nz;
 * vals = lx, ly, lz, dx, dy, dz, re, dt, t_current.  MDX_ERR_IO on failure. */
int mdx_h5_read_header(const char* filename, int* dims, double* vals);
/* Why the last fdm_h5_read_field / mdx_h5_read_header call failed. */
const char* mdx_h5_last_error(void);

int mdx_set_ibm_coeff(const mdx_grid_t* g, const mdx_ibm_geom_t* geom, double* coeff, int dix, int diy, int diz);
/* The same coefficients computed on the device into d_coeff (a padded
 * (nx+2)(ny+2)(nz+2) device array), stream-ordered on `stream` (a
 * cudaStream_t, NULL for the default stream).  Same arithmetic as the host
 * routine; the device sin may round differently from the host's in the last
 * bit, which can move a bisected wall distance only for a point within one
 * rounding of the wall.  No counterpart in the reference (its
 * set_ibm_coeff is a host loop, src/modules/ibm.f90:133-187). */
int mdx_set_ibm_coeff_device(const mdx_grid_t* g, const mdx_ibm_geom_t* geom, double* d_coeff, int dix, int diy,
                             int diz, void* stream);

/* ---- context ---------------------------------------------------------- */

/* Create a context on `device` for grid g and boundary set bc. */
int mdx_create(int device, const mdx_grid_t* g, const mdx_bc_t* bc, mdx_ctx_t** out);
int mdx_destroy(mdx_ctx_t* ctx);

/* Replace the boundary set of a context.  The reference passes bc to
 * momentum / pressure_projection / apply_bc_redblack on every call
 * (src/modules/step.f90:27, pressure_solver.f90:48, boundary.f90:173) while
 * enter_field_data gets none (gpu_runtime.f90:22), so a Fortran shim creates
 * the context with init_bc defaults and updates it here when bc changes. */
int mdx_set_bc(mdx_ctx_t* ctx, const mdx_bc_t* bc);

/* Re and body force (grid_type re, forcing_x/y/z, src/modules/init.f90:14-19)
 * of an existing context, for running several flows on one context (the
 * reference sets them once from input.ini).  IBM coefficients carry 1/Re:
 * re-enter them after a change. */
int mdx_set_flow(mdx_ctx_t* ctx, double re, double fx, double fy, double fz);

/* Use an external CUDA stream (cudaStream_t) instead of the context's own;
 * NULL restores the context stream. */
int mdx_set_stream(mdx_ctx_t* ctx, void* stream);
int mdx_get_stream(mdx_ctx_t* ctx, void** stream);

/* enter_field_data / exit_field_data, src/modules/gpu_runtime.f90:22-48:
 * allocate the 10 device mirrors and copy the host arrays in; free them.
 * Any host pointer may be NULL, which zero-fills that mirror. */
int mdx_enter_field_data(mdx_ctx_t* ctx,
                         const double* un, const double* us, const double* oldrhsu,
                         const double* vn, const double* vs, const double* oldrhsv,
                         const double* wn, const double* ws, const double* oldrhsw,
                         const double* pn);
int mdx_exit_field_data(mdx_ctx_t* ctx);

/* `!$omp target update from/to` of un,vn,wn,pn around output and restart,
 * src/modules/io.f90:123-128 and :160-165.  update_host synchronises. */
int mdx_update_host(mdx_ctx_t* ctx, double* un, double* vn, double* wn, double* pn);
int mdx_update_device(mdx_ctx_t* ctx, const double* un, const double* vn, const double* wn, const double* pn);

/* Copy any one array between host and device (direction 0: device->host,
 * synchronising; 1: host->device).  MDX_PHI is device->host only. */
int mdx_copy_field(mdx_ctx_t* ctx, int field, double* host, int direction);

/* enter_ibm_data / exit_ibm_data, src/modules/ibm.f90:57-81.  NULL
 * coefficients mean "no body" (all zero).  exit restores zero coefficients. */
int mdx_enter_ibm_data(mdx_ctx_t* ctx, const double* coef_u, const double* coef_v, const double* coef_w);
/* write_field / read_field, src/modules/io.f90:105-166: the device mirrors
 * of un, vn, wn, pn to the host and into a field file with the context's
 * grid and t_current; or a field file into the mirrors (synchronising). */
int mdx_write_field_h5(mdx_ctx_t* ctx, const char* filename);
int mdx_read_field_h5(mdx_ctx_t* ctx, const char* filename);
/* The reference's IBM setup, src/main.f90:58-61 -- set_ibm_coeff for u, v, w
 * (ibm.f90:133-187) then enter_ibm_data -- in one call, the coefficients
 * generated on the device (mdx_set_ibm_coeff_device) straight into the
 * context's mirrors: no host arrays, no copies. */
int mdx_enter_ibm_geometry(mdx_ctx_t* ctx, const mdx_ibm_geom_t* geom);
int mdx_exit_ibm_data(mdx_ctx_t* ctx);

/* ---- time step ---------------------------------------------------------- */

/* momentum, src/modules/step.f90:27-207 (predictor of u*,v*,w*, RHS store). */
int mdx_momentum(mdx_ctx_t* ctx, double dt_alpha, double dt_beta, double dt_gamma);

/* apply_bc, src/modules/boundary.f90:23-170 (FFT builds: y walls, periodic
 * x/z on the n and * arrays), and apply_bc_redblack, :173-368. */
int mdx_apply_bc(mdx_ctx_t* ctx);
int mdx_apply_bc_redblack(mdx_ctx_t* ctx);

/* init_pressure_solver / destroy_pressure_solver,
 * src/modules/pressure_solver.f90:35-46,65-74 (plans, Thomas tables,
 * workspace; the red-black even-size check of pressure_redblack.f90:16-18). */
int mdx_init_pressure_solver(mdx_ctx_t* ctx, const mdx_solver_opts_t* opts);
int mdx_destroy_pressure_solver(mdx_ctx_t* ctx);

/* pressure_projection, src/modules/pressure_solver.f90:48-63.  stats may be
 * NULL; with stats or a residual tolerance the call synchronises. */
int mdx_pressure_projection(mdx_ctx_t* ctx, double dt_gamma, mdx_solve_stats_t* stats);

/* Statistics of the last pressure projection (including those run inside
 * mdx_step). */
int mdx_last_solve_stats(const mdx_ctx_t* ctx, mdx_solve_stats_t* stats);

/* Warm start of the red-black projection: mode MDX_GUESS_*; record != 0
 * keeps the pressure increment of every projection (p_after - p_before, per
 * RK substage, projections numbered in call order, three per step) even
 * without a guess.  The guess is applied as the sweeps apply phi and the
 * projection still runs to its tolerance relative to ||div u*||; a guess
 * that does not lower ||div u|| below ||div u*|| is undone (with tol > 0).
 * Needs periodic x and z and y periodic or Neumann-pressure walls
 * (otherwise no guess is applied).  The t=0 projection of mdx_channel_ic
 * resets the history. */
int mdx_set_pressure_guess(mdx_ctx_t* ctx, int mode, int record);

/* Copy the recorded increment of RK substage s (0..2) to host (nx,ny,nz)
 * cells, x fastest (synchronises); MDX_ERR_STATE if none was recorded. */
int mdx_get_increment(mdx_ctx_t* ctx, int substage, double* host);

/* Save (restore = 0) or restore (restore != 0) the warm-start history --
 * the recorded increments and the projection count -- in a device-side copy,
 * so that steps can be replayed from a saved u, v, w, p with the same
 * guesses.  No counterpart in the reference. */
int mdx_warm_checkpoint(mdx_ctx_t* ctx, int restore);

/* ---- batched ensemble (no counterpart in the reference) -----------------
 * Many independent wavy-wall channels of different sizes advanced together:
 * one persistent cooperative launch per RK3 substage for all members
 * (momentum, red-black projection to each member's own tolerance, boundary
 * conditions), the three launches of a step captured in a CUDA graph.
 * Every member: periodic x and z, no-slip walls in y with Neumann
 * pressure, walls y0 + A sin(2 pi x/(Lx/2)) and y0 + 2 + ... imposed by the
 * IBM of mdx_set_ibm_coeff (geometry 1) when A > 0 (y0 = (Ly-2)/2), forcing
 * 2/Re in x, FP64 red-black sweeps.  With a fixed iteration count (tol <= 0)
 * each member's fields are bit-for-bit the single-context path's. */
typedef struct {
    int nx, ny, nz;        /* even nx and nz                                   */
    double lx, ly, lz;     /* ly > 2                                           */
    double re, dt;
    double amp;            /* wall amplitude A (0: no IBM)                     */
    uint64_t seed;         /* initial condition (mdx_channel_ic's)             */
    int reserved_i[4];
    double reserved_d[4];
} mdx_member_t;

typedef struct mdx_ensemble mdx_ensemble_t;

void mdx_default_member(mdx_member_t* m);
/* opts: MDX_SOLVER_REDBLACK, MDX_PREC_FP64; n_iter / tol / max_iter /
 * check_every / atol / sor as for a context. */
int mdx_ensemble_create(int device, int n, const mdx_member_t* members, const mdx_solver_opts_t* opts,
                        mdx_ensemble_t** out);
int mdx_ensemble_destroy(mdx_ensemble_t* ens);
const char* mdx_ensemble_last_error(const mdx_ensemble_t* ens);
/* MDX_GUESS_ZERO, MDX_GUESS_PREVIOUS, MDX_GUESS_EXTRAPOLATED, or
 * MDX_GUESS_LEARNED once a network is loaded (mdx_ensemble_unet_load) and
 * tol > 0. */
int mdx_ensemble_set_guess(mdx_ensemble_t* ens, int mode);
/* Seeded channel initial condition of every member, projected at t = 0
 * (dt_gamma = 1), then p = 0 (mdx_channel_ic with y0 = (Ly-2)/2, the
 * member's amplitude and lambda = Lx/2, noise amplitudes 0.1 and 0.01). */
int mdx_ensemble_ic(mdx_ensemble_t* ens);
/* nsteps RK3 steps of every member; *total_iters = red-black iterations of
 * all members (synchronises).  MDX_NOT_CONVERGED / MDX_ERR_NONFINITE when a
 * member's projection ended so. */
int mdx_ensemble_step(mdx_ensemble_t* ens, int nsteps, long long* total_iters);
int mdx_ensemble_member_stats(mdx_ensemble_t* ens, int member, mdx_solve_stats_t* last, long long* iters_total);
/* Padded field MDX_UN, MDX_VN, MDX_WN or MDX_PN of a member. */
int mdx_ensemble_get(mdx_ensemble_t* ens, int member, int field, double* host);
int mdx_ensemble_set(mdx_ensemble_t* ens, int member, int field, const double* host);
/* Launch shape of the persistent kernel: threads per block (multiple of
 * 32, <= 512), blocks per SM (0: as many as fit) and the register variant
 * (low_regs != 0: 64 registers per thread, twice the resident warps). */
int mdx_ensemble_config(mdx_ensemble_t* ens, int threads, int blocks_per_sm, int low_regs);
/* Time one step of each candidate launch shape from the same saved state and
 * keep the fastest; the choice is cached in the JSON file cache_path (may be
 * NULL) under a key of the member sizes, the mode and the device name
 * (*ms = -1 when it came from the cache). */
int mdx_ensemble_tune(mdx_ensemble_t* ens, const char* cache_path, int* threads, int* blocks_per_sm, int* low_regs,
                      double* ms);
int mdx_ensemble_use_graph(mdx_ensemble_t* ens, int on);
int mdx_ensemble_info(mdx_ensemble_t* ens, int* threads, int* grid, int* low_regs, int* graph, double* last_step_ms,
                      long long* launches);

/* ---- learned warm start (no counterpart in the reference) ----------------
 * A 4-level 3-D U-Net on the cells of the grid (channels-last BF16
 * activations and weights, FP32 accumulation on the tensor cores).  With
 * mode MDX_GUESS_LEARNED, once the extrapolated increment has been applied,
 * the net maps four per-cell inputs
 *     div u left by the extrapolated guess / its RMS,
 *     dp(n-1) / RMS(dp(n-1)),  dp(n-2) / RMS(dp(n-1)),  IBM factor mu of the cell
 * to a correction of the increment, out * out_scale * RMS(div) * h2 / dt_gamma
 * with h2 = 1/(1/dx^2+1/dy^2+1/dz^2).  A correction that does not lower
 * ||div u|| is undone; the sweeps then run to the usual tolerance.
 * The net is trained on the device (Adam, FP32 master weights) on
 * snapshots the projection records: inputs as above and the target
 * (dp_converged - dp_extrapolated) * dt_gamma / (RMS(div) * h2).
 * Needs nx, ny, nz multiples of 8 and the warm-start boundary conditions. */
typedef struct {
    int channels0;          /* channels at full resolution: 16                  */
    int channels;           /* channels of the three coarser levels: 16 or 32   */
    int extra_bottleneck;   /* extra 3x3x3 convolutions at the coarsest level, 0..8 */
    int capacity;           /* snapshots kept on the device for training        */
    double slope;           /* leaky-ReLU slope, (0, 1]; 1 makes the net linear */
    uint64_t seed;          /* weight initialisation                            */
    int conv_kernel;        /* 0 (default): forward convolutions and data gradients on levels whose
                               nx is a multiple of 128 run on tcgen05 (tensor-memory accumulators),
                               the rest on mma.sync; 1: mma.sync everywhere                  */
    int step_rule;          /* 0 (default): apply the correction as predicted, keep it when it lowers
                               ||div u||; 1: apply alpha x the correction with alpha the step that
                               minimises the energy norm of the pressure error along it,
                               alpha = -<delta, d0> / <delta, d1 - d0> (d0, d1 the divergence before
                               and after the correction), kept when alpha > 0               */
    int gate_period;        /* 0 (default): correct every projection that has a two-step history;
                               P > 0: per RK substage, apply the correction or not by the red-black
                               iterations each choice took (exponential averages, weight 1/2):
                               the first projection without it, the next with it, then the
                               cheaper one, with the other re-tried every P-th projection  */
    int reserved_i[5];
    double reserved_d[8];
} mdx_unet_opts_t;

typedef struct {
    long long corrections;  /* learned corrections applied                      */
    long long rejected;     /* corrections undone (did not lower ||div u||)     */
    long long snapshots;    /* snapshots recorded since creation                */
    int stored;             /* snapshots held now (<= capacity)                 */
    int trained;            /* weights trained or set                           */
    double out_scale;       /* output scale of the net                          */
    double last_gain;       /* ||div|| after the extrapolated guess / after the correction */
    double infer_ms;        /* device time of the last correction               */
    double train_ms;        /* device time of the last mdx_unet_train call      */
    long long tc_convs;     /* convolution launches on tcgen05 since creation   */
    double last_step;       /* step_rule 1: the last step length alpha           */
    long long gated;        /* projections the gate left to the extrapolated guess */
    double reserved_d[3];
} mdx_unet_stats_t;

void mdx_default_unet_opts(mdx_unet_opts_t* opts);

/* Learned warm start in the ensemble (no counterpart in the reference): the
 * trained parameters and output scale of a network with options `opts`
 * (from a context: mdx_unet_get_params / mdx_unet_get_out_scale; the net is
 * fully convolutional, so one trained on any grid applies to every member;
 * member sizes must be multiples of 8).  With MDX_GUESS_LEARNED each
 * substage runs as two cooperative launches with the network between them:
 * the first applies the members' extrapolated increments, the network then
 * runs for every member in turn on its own grid (one network sized for the
 * member with the most cells; scales and the zero-mean projection on the
 * device, no host read, so the step stays one CUDA graph), and the second
 * applies each correction, keeps it where it lowers ||div u|| (else back to
 * the extrapolated increment) and sweeps to the tolerance. */
int mdx_ensemble_unet_load(mdx_ensemble_t* ens, const mdx_unet_opts_t* opts, const float* params, long long n,
                           double out_scale);
/* Learned corrections kept and undone, and projections the gate left to
 * the extrapolated guess (opts->gate_period > 0 at mdx_ensemble_unet_load:
 * per member and RK substage, as for a context), over all members since
 * creation (synchronises; each pointer may be NULL). */
int mdx_ensemble_unet_stats(mdx_ensemble_t* ens, long long* corrections, long long* rejected, long long* gated);
int mdx_unet_create(mdx_ctx_t* ctx, const mdx_unet_opts_t* opts);
int mdx_unet_destroy(mdx_ctx_t* ctx);
/* Record a snapshot in every converged projection that had an extrapolated
 * guess (guess mode MDX_GUESS_EXTRAPOLATED or MDX_GUESS_LEARNED); the oldest
 * is overwritten once `capacity` are held. */
int mdx_unet_record(mdx_ctx_t* ctx, int on);
/* `iters` Adam steps (one snapshot each, in a seeded random order) at
 * learning rate lr; the mean-square loss of the first and the last step. */
int mdx_unet_train(mdx_ctx_t* ctx, int iters, double lr, double* loss_first, double* loss_last);
/* Parameters, FP32, in this order per 3x3x3 convolution: W[tap][cout][cin]
 * (tap = 9*(dz+1) + 3*(dy+1) + (dx+1)), bias[cout]; then the 1x1 head
 * w[channels0], b.  Convolutions in the order enc0a, enc0b, enc1a, enc1b,
 * enc2a, enc2b, enc3a, enc3b, the extra bottleneck ones, dec2, dec1, dec0. */
long long mdx_unet_param_count(const mdx_ctx_t* ctx);
int mdx_unet_get_params(mdx_ctx_t* ctx, float* host, long long n);
int mdx_unet_set_params(mdx_ctx_t* ctx, const float* host, long long n);   /* marks the net trained */
int mdx_unet_get_out_scale(mdx_ctx_t* ctx, double* scale);
int mdx_unet_set_out_scale(mdx_ctx_t* ctx, double scale);
/* One forward and backward pass on host inputs in [5][ncells] (the
 * normalised divergence, the last two increments, the IBM factor and the
 * viscous-number channel) and target [ncells] (cells x fastest): loss = mean((out - target)^2), its gradient
 * with respect to every parameter (param_count floats) and the output
 * [ncells].  No update; used to check the kernels against a CPU network. */
int mdx_unet_loss_grad(mdx_ctx_t* ctx, const float* in, const float* target, double* loss, float* grad, float* out);
int mdx_unet_stats(mdx_ctx_t* ctx, mdx_unet_stats_t* stats);

/* get_cfl, src/modules/step.f90:210-258 (synchronises). */
int mdx_get_cfl(mdx_ctx_t* ctx, double* cfl);

/* center_vel, src/modules/io.f90:184-222: cell-centred velocities
 * (1:nx,1:ny,1:nz) copied to the host (synchronises). */
int mdx_center_vel(mdx_ctx_t* ctx, double* uc, double* vc, double* wc);

/* `nsteps` whole RK3 steps with fixed dt, src/main.f90:66-90 (substage
 * order momentum -> apply_bc -> pressure_projection -> apply_bc, or the
 * red-black variant).  Adds nsteps*dt to g.t_current.  The FFT path is
 * replayed from a CUDA graph.  total_iters (may be NULL) returns the summed
 * red-black iterations. */
int mdx_step(mdx_ctx_t* ctx, int nsteps, long long* total_iters);

/* `nsteps` RK3 steps with the reference's adaptive dt, src/main.f90:66-97:
 * t += dt, the three substages, then cfl = get_cfl and, when cflmax > 0
 * and cfl > 0, dt = min(cflmax/cfl, dtmax).  cflmax <= 0: mdx_step (fixed
 * dt, no CFL).  On the FP64 FFT path every step is one CUDA graph in which
 * the kernels read dt from device memory and the CFL reduction and the dt
 * update run on the device; dt, t_current and cfl come back to the host
 * once, after the last step.  On the other paths the CFL is read after
 * every step.  g.dt, g.t_current, g.cfl, g.cflmax and g.dtmax are updated
 * (mdx_get_time).  total_iters as mdx_step (0 on the FFT path). */
int mdx_step_adaptive(mdx_ctx_t* ctx, int nsteps, double cflmax, double dtmax, long long* total_iters);

/* The context's dt, t_current and the last CFL number (each may be NULL). */
int mdx_get_time(mdx_ctx_t* ctx, double* dt, double* t_current, double* cfl);

/* Set the dt mdx_step and mdx_step_adaptive start from (> 0, finite). */
int mdx_set_dt(mdx_ctx_t* ctx, double dt);

/* Seeded channel initial condition + projection at t=0 (new; the reference
 * zero-initialises, src/modules/init.f90:67-70): u = max(0,1-(y-yc(x))^2) +
 * U(-amp_u,amp_u), v,w = U(-amp_vw,amp_vw) (counter-based SplitMix64 on
 * seed, field and padded index), yc(x) = y0 + 1 + wave_amp*sin(2*pi*x/
 * wave_lambda); then apply_bc, pressure_projection with dt_gamma = 1 and p=0.
 * Requires field data and an initialised pressure solver. */
int mdx_channel_ic(mdx_ctx_t* ctx, uint64_t seed, double amp_u, double amp_vw, double y0,
                   double wave_amp, double wave_lambda, mdx_solve_stats_t* stats);

/* Device divergence norms of (un,vn,wn) with the red-black neighbour rule
 * (synchronises). */
int mdx_divergence_norms(mdx_ctx_t* ctx, double* l2, double* linf);

/* Per-kernel-class device timing with CUDA events on the context stream.
 * on = 1: every 8th launch of a class is bracketed by an event pair, and
 * every run of back-to-back sweeps (MDX_T_SOR_BLOCK) as well; on = 2: only
 * the sweep runs, so that no event sits between two sweeps.  get_timing
 * reports the launches of each class since set_timing and their total time
 * estimated as launches x the sampled mean; MDX_T_SOR_BLOCK is the measured
 * total of the runs (synchronises). */
int mdx_set_timing(mdx_ctx_t* ctx, int on);
int mdx_get_timing(mdx_ctx_t* ctx, mdx_timing_t* out);

/* Number of kernel launches issued by the library on this context so far. */
long long mdx_launch_count(const mdx_ctx_t* ctx);

/* ---- allocation-free pressure solve --------------------------------------- */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory through the CUDA runtime -- e.g. an OpenMP-offload Fortran program
 * whose device arrays belong to the OpenMP runtime and are handed over with
 * use_device_addr -- this solves the FFT-path pressure equation on device
 * arrays the caller owns, without a context and without allocating.
 *
 * rhs, phi: device arrays in the rhs(nx,nz,ny) order (x fastest, then z,
 * then y); phi = the FFT + Thomas solution scaled by 1/(nx*nz), the result
 * of the context path (pressure_backend_*.f90 solve_pressure_*).  phi may
 * equal rhs.  The call is enqueued on `stream` (cudaStream_t, NULL = legacy
 * default stream) and returns without synchronising.
 *
 * Every intermediate (spectrum, Thomas tables, twiddles, wavenumbers) lives in
 * one static device array of 8 MiB per device, which the library holds until
 * the process exits; grids needing more (e.g. above about 64 x 64 x 128) are
 * rejected with MDX_ERR_ARG before any device work.  The array's address is
 * looked up on the first call on each device (and again on later calls made
 * outside a stream capture, so that a newly current context gets its own), so
 * make that first call before any stream capture.  The tables, twiddles and
 * wavenumbers are built on the device by every call; nothing is copied from
 * host memory.  All calls share the array and it keeps the last call's
 * contents; calls that overlap on the GPU (different streams or threads) race
 * on it.  Requires even nx; nx/2 and nz must factor into 2, 3, 5, 7. */
int mdx_solve_pressure_fft_noalloc(const double* rhs, double* phi, int nx, int ny, int nz, double dx, double dy,
                                   double dz, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MOBYDIFF_B200_H */
