// mdx_internal.cuh -- context, device layout and shared helpers of libmobyb200.
#pragma once

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mobydiff_b200.h"

// Device layout.  Every field keeps the reference's host layout so that the
// drop-in copies are flat memcpys: padded (0:nx+1,0:ny+1,0:nz+1) Fortran
// order, x fastest.  The FFT workspace keeps the reference's orders too:
// phi / rhs (nx,nz,ny) real and the spectrum (nxh,nz,ny) complex
// (src/modules/pressure_workspace.f90:10-22).
struct mdx_dims {
    int nx, ny, nz;
    int nxp, nyp, nzp;   // nx+2, ny+2, nz+2
    int nxh;             // nx/2+1
    long long npad;      // (nx+2)(ny+2)(nz+2)
    long long nint;      // nx*ny*nz
    long long nspec;     // nxh*nz*ny
    int hs;              // row length of the colour-split layout, (nx+2)/2 rounded up to a multiple of 4
};

// Rows of the colour-split layout start on 16-byte boundaries (FP32), so
// that a colour sweep can move four consecutive cells with one vector access.
__host__ __device__ inline int split_stride(int nx) { return ((nx + 2) / 2 + 3) & ~3; }

__host__ __device__ inline long long pidx(const mdx_dims& d, int i, int j, int k) {
    return (long long)i + (long long)d.nxp * ((long long)j + (long long)d.nyp * (long long)k);
}
__host__ __device__ inline long long qidx(const mdx_dims& d, int i, int j, int k) {  // (1:nx,1:ny,1:nz)
    return (long long)(i - 1) + (long long)d.nx * ((long long)(j - 1) + (long long)d.ny * (long long)(k - 1));
}
__host__ __device__ inline long long ridx(const mdx_dims& d, int i, int k, int j) {  // rhs(i,k,j), 1-based
    return (long long)(i - 1) + (long long)d.nx * ((long long)(k - 1) + (long long)d.nz * (long long)(j - 1));
}

// Colour-split layout (the mixed path's FP32 arrays, the FP64 sweeps' working
// copies, the ensemble's FP32 arrays): element (i, j, k) of the padded grid
// lives in half (i + j + k) & 1 at (k (ny+2) + j) hs + i/2, hs >= (nx+2)/2,
// so the cells of one colour in a row -- and the faces they own or share --
// are consecutive: every access of a colour sweep is unit-stride.  A face
// belongs to the cell on its high side (u(i) to cell i).  nx is even, so
// (nx+2)/2 is whole; positions (nx+2)/2 .. hs-1 of a row are padding that
// holds no element.
__host__ __device__ __forceinline__ long long cidx(const mdx_dims& d, int i, int j, int k) {
    return ((i + j + k) & 1) * ((long long)d.hs * d.nyp * d.nzp) + ((long long)k * d.nyp + j) * d.hs + (i >> 1);
}
__host__ __device__ inline long long split_elems(const mdx_dims& d) { return 2LL * d.hs * d.nyp * d.nzp; }
// (i, j) planes of the IBM factors and sweep factors, split the same way by
// (i + j) & 1: for one colour and one z plane all rows of the cells' factors
// lie in one half.  A plane of one component holds split_plane_elems values.
__host__ __device__ __forceinline__ int pidx2(const mdx_dims& d, int i, int j) {
    return ((i + j) & 1) * (d.hs * d.nyp) + j * d.hs + (i >> 1);
}
__host__ __device__ inline int split_plane_elems(const mdx_dims& d) { return 2 * d.hs * d.nyp; }


// Red-black kernel variants (opts.sor_variant; k_sor.cu, k_sor_mixed.cu).
enum {
    MDX_SORV_AUTO = 0, MDX_SORV_SWEEPS = 1, MDX_SORV_FUSED8 = 2, MDX_SORV_FUSED16 = 3, MDX_SORV_SPLIT = 4,
    MDX_SORV_SPLITV = 5, MDX_SORV_NUM = 6
};

// A step scalar (dt times an RK coefficient) handed to a kernel either by
// value or, on the adaptive-dt path, as the address of the device's dt and
// the coefficient, so that a CUDA graph replays the step with the dt the
// device computed after the step before.  get() is the one FP64 multiply
// dt * coefficient that the host does otherwise.
struct mdx_dscal {
    double v = 0.0;
    const double* p = nullptr;
    double m = 0.0;
    mdx_dscal() = default;
    __host__ __device__ mdx_dscal(double x) : v(x) {}
    __host__ __device__ mdx_dscal(const double* dt, double coef) : p(dt), m(coef) {}
    __device__ __forceinline__ double get() const { return p ? *p * m : v; }
};

// Scalars of one time step, passed by value to kernels.
struct mdx_step_params {
    double dx, dy, dz;
    double idx, idy, idz, idx2, idy2, idz2, ire;
    double fx, fy, fz;
    int nx0, ny0, nz0;
};

struct mdx_bc_dev {
    int per[3];
    int type[24];
    double value[24];
};
__host__ __device__ inline int bci(int dir, int side, int var) { return (dir - 1) + 3 * (side + 2 * var); }

// FFT plan for one length: radix list and twiddle table exp(-2 pi i t/n).
#define MDX_MAX_STAGES 16
struct mdx_fft_plan {
    int n;
    int nstages;
    int radix[MDX_MAX_STAGES];
};

struct mdx_event_pair { cudaEvent_t a, b; int cls; long long n; };   // n: launches inside the pair

struct mdx_ctx {
    int device = 0;
    mdx_grid_t g{};
    mdx_bc_t bc{};
    mdx_bc_dev bcd{};
    mdx_solver_opts_t opts{};
    mdx_dims d{};
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;

    bool fields = false;
    bool solver = false;
    double* f[MDX_NUM_FIELDS] = {nullptr};   // device mirrors (MDX_PHI -> phi)
    bool ibm_zero = true;                    // all IBM coefficients zero
    bool coef_zinv = false;                  // coefficients equal on every z plane
    double* sor_alt[4] = {nullptr};          // second u,v,w,p state of the fused red-black pass
    double* split_f[4] = {nullptr};          // colour-split copies of u,v,w,p (split sweeps)
    double* split_tab = nullptr;             // their column factors: mu_u, mu_v, mu_w, fac planes (pidx2)
    bool split_norms = false;                // divergence norms read colour-split arrays
    bool fused_attr = false;
    // mixed-precision red-black: FP32 corrections, FP32 residual, IBM tables,
    // carved from one allocation (mx_du is its base) of mx_bytes
    float *mx_du = nullptr, *mx_dv = nullptr, *mx_dw = nullptr, *mx_dp = nullptr, *mx_r = nullptr;
    float *mx_mu = nullptr, *mx_fac = nullptr;
    // the fused red+black pass reads faces from mx_du/dv/dw and writes the
    // second buffers, then the pointers swap
    float *mx_du2 = nullptr, *mx_dv2 = nullptr, *mx_dw2 = nullptr;
    void* mx_base = nullptr;
    size_t mx_bytes = 0;
    int rb32_tuned = 0;                      // FP32 inner sweeps: candidate + 1 chosen by the autotuner (0: not yet;
                                             // candidates: the fused pass's 4 tile shapes, the colour sweeps, the
                                             // vector colour sweeps with 2 and 4 cells per thread)
    unsigned rb32_attr = 0;                  // fused FP32 pass: shared-memory attribute set, bit per kernel
    double rb32_tune_ms[8] = {0.0};          // time per iteration per candidate
    // potential form of the FP32 sweeps (opts.inner_form 0): phi and r~ in
    // their own colour-split layout (k_sor_mixed.cu pot_geom) and one float4
    // table per (i, j) column, carved from one allocation of pt_bytes
    float *pt_phi = nullptr, *pt_r = nullptr;
    float4* pt_tab = nullptr;
    float* pt_tabu = nullptr;                // the columns' top-face a_y, one row per y row
    void* pt_base = nullptr;
    size_t pt_bytes = 0;
    int pt_tuned = 0;                        // candidate + 1 chosen by the autotuner (0: not yet)
    unsigned pt_attr = 0;                    // staged sweeps: shared-memory attribute set, bit per kernel
    double pt_tune_ms[16] = {0.0};            // time per iteration per candidate
    // warm starts: increments of the last projection of each RK substage
    int guess_mode = 0;                      // MDX_GUESS_*
    bool record_increments = false;
    double* dp_hist[3] = {nullptr, nullptr, nullptr};   // (nx,ny,nz) cells, previous step
    double* dp_hist2[3] = {nullptr, nullptr, nullptr};  // the step before
    double* p_before = nullptr;              // padded p at the start of the projection
    double* guess = nullptr;                 // increment guess of the current projection
    int hist_valid = 0;                      // bit s: dp_hist[s] holds an increment; bit 3+s: dp_hist2[s]
    double* ckpt = nullptr;                  // saved dp_hist, dp_hist2 (mdx_warm_checkpoint)
    int ckpt_valid = -1;                     // hist_valid at the save, -1: none
    long long ckpt_count = 0;
    long long proj_count = 0;                // projections since the t=0 projection
    void* unet = nullptr;                    // learned warm start (k_unet.cu)
    int sor_tuned = 0;                       // red-black kernel variant chosen by the autotuner (0: not yet)
    double sor_tune_ms[8] = {0.0};           // time per iteration of a timed residual-check block, per variant
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};
    double* mu = nullptr;                    // red-black IBM factors 1/(1+dt_gamma*coef)
    long long mu_elems = 0;
    int mu_mode = 0;

    // FFT workspace
    double2* spec = nullptr;                 // (nxh, nz, ny)
    double* thomas_dinv = nullptr;           // (ny, nxh, nz/2+1)
    double* thomas_cp = nullptr;             // (ny, nxh, nz/2+1)
    double2* tw_x = nullptr;                 // exp(-2 pi i t/nx), t < nx
    double2* tw_z = nullptr;                 // exp(-2 pi i t/nz), t < nz
    mdx_fft_plan plan_xh{};                  // complex length nx/2 (packed real transform)
    mdx_fft_plan plan_z{};                   // complex length nz
    // FFT path with walls in x or z (pressure Neumann there): the pressure
    // equation is solved on the even extension of the grid in those
    // directions, periodic of twice the length; the workspace above is then
    // sized for dfft instead of d
    int fft_ext_x = 0, fft_ext_z = 0;
    mdx_dims dfft{};                         // the solve grid (d itself without walls in x and z)
    double* phi_ext = nullptr;               // right-hand side, then phi, on dfft in rhs(i,k,j) order
    // mixed-precision FFT path: FP32 spectrum, correction, twiddles, Thomas
    // tables; FP64 zero-wavenumber right-hand side and solution per y
    float2 *spec32 = nullptr, *tw_x32 = nullptr, *tw_z32 = nullptr;
    float *phi32 = nullptr, *dinv32 = nullptr, *cp32 = nullptr;
    double *rhs0 = nullptr, *phi0 = nullptr;

    // reductions
    double* red_part = nullptr;              // per-block partials (2 per block)
    int red_blocks = 0;
    double* red_out = nullptr;               // device result [2]
    double* red_host = nullptr;              // pinned host result [2]

    mdx_solve_stats_t last{};

    // CUDA graph of one FFT-path RK3 step
    cudaGraphExec_t step_graph = nullptr;
    double graph_dt = 0.0;
    long long graph_launches = 0;
    // adaptive-dt FFT step: {dt, t_current, cfl} on the device, read by the
    // step's kernels and updated by its last kernel; the graph of one step
    // and the cflmax / dtmax it was captured with
    double* dt_dev = nullptr;
    cudaGraphExec_t adapt_graph = nullptr;
    double adapt_cflmax = 0.0, adapt_dtmax = 0.0;
    long long adapt_launches = 0;

    // timing: 0 off, 1 sampled launches + sweep runs, 2 sweep runs only
    int timing = 0;
    std::vector<mdx_event_pair> ev_pending;
    std::vector<cudaEvent_t> ev_free;
    mdx_timing_t tim{};                      // sums over the sampled launches
    long long tim_issued[MDX_T_NUM] = {0};   // launches per class since set_timing(1)
    long long launches = 0;
    bool capturing = false;
};

// Iterations until the next residual check of a red-black solve.  Once the
// residual falls at a steady geometric rate -- the rates of the last two
// check intervals agree within 25 % -- that rate predicts the iterations left
// to the target, and the next check comes after half of them, in whole
// check_every blocks (1 to 8).  Checks far from the target are sparse, the
// last ones check_every apart, and every check lands on a multiple of
// check_every.  While the rate changes (the first sweeps, or a plateau of the
// over-relaxed iteration) and in mode 1, every block is checked.
struct mdx_check_schedule {
    int every = 1, mode = 0;
    int last_it = 0;
    double last_r = 0.0, rate = 0.0;   // natural-log decrease per iteration of the last interval
    void start(int check_every, int check_mode, double r) {
        every = check_every > 0 ? check_every : 1;
        mode = check_mode;
        last_it = 0;
        last_r = r;
        rate = 0.0;
    }
    int next(int it, double r, double target) {
        const double rt = (it > last_it && r > 0.0 && last_r > r) ? std::log(last_r / r) / (double)(it - last_it) : 0.0;
        const bool steady = rt > 0.0 && rate > 0.0 && std::fabs(rt - rate) <= 0.25 * rt;
        rate = rt;
        last_it = it;
        last_r = r;
        if (mode == 1 || !steady || !(r > target) || !(target > 0.0)) return every;
        const double left = std::log(r / target) / rt;
        const double blocks = std::floor(0.5 * left / (double)every);
        return every * (int)std::min(8.0, std::max(1.0, blocks));
    }
};

// ---- error helpers -------------------------------------------------------
int mdx_fail(mdx_ctx_t* ctx, int code, const char* fmt, ...);
#define MDX_CUDA(ctx, call)                                                                   \
    do {                                                                                      \
        cudaError_t e__ = (call);                                                             \
        if (e__ != cudaSuccess)                                                               \
            return mdx_fail((ctx), MDX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                            cudaGetErrorString(e__), __FILE__, __LINE__);                     \
    } while (0)
#define MDX_TRY(expr)                         \
    do {                                      \
        int r__ = (expr);                     \
        if (r__ != MDX_OK) return r__;        \
    } while (0)

// ---- launch bookkeeping ----------------------------------------------------
void mdx_timer_begin(mdx_ctx_t* ctx, int cls, mdx_event_pair* p);
void mdx_timer_end(mdx_ctx_t* ctx, mdx_event_pair* p);
// A run of back-to-back sweep launches between two residual checks, timed
// whole (MDX_T_SOR_BLOCK) whenever timing is on; `end` counts the launches
// issued since `begin`.
void mdx_sweep_run_begin(mdx_ctx_t* ctx, mdx_event_pair* p);
// sweeps >= 0: the colour sweeps the run made, when one launch makes several
// (the cooperative potential-form runs); otherwise the launches are counted
void mdx_sweep_run_end(mdx_ctx_t* ctx, mdx_event_pair* p, long long sweeps = -1);
int mdx_check_launch(mdx_ctx_t* ctx, const char* what);

// Launch wrapper: times the launch when timing is on and checks the launch.
#define MDX_LAUNCH(ctx, cls, what, kernel, grid, block, smem, ...)                     \
    do {                                                                               \
        mdx_event_pair p__{};                                                          \
        mdx_timer_begin((ctx), (cls), &p__);                                           \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);               \
        mdx_timer_end((ctx), &p__);                                                    \
        MDX_TRY(mdx_check_launch((ctx), (what)));                                      \
    } while (0)

// ---- per-module entry points (internal) --------------------------------------
mdx_step_params mdx_make_params(const mdx_ctx_t* ctx);
int mdx_k_momentum(mdx_ctx_t* ctx, mdx_dscal da, mdx_dscal db, mdx_dscal dg);
int mdx_k_apply_bc(mdx_ctx_t* ctx);
int mdx_k_apply_bc_redblack(mdx_ctx_t* ctx);
int mdx_fft_init(mdx_ctx_t* ctx);
void mdx_fft_free(mdx_ctx_t* ctx);
int mdx_k_projection_fft(mdx_ctx_t* ctx, mdx_dscal dg);
int mdx_k_projection_fft_mixed(mdx_ctx_t* ctx, double dg);
int mdx_k_projection_redblack(mdx_ctx_t* ctx, double dg, mdx_solve_stats_t* st);
int mdx_k_div_norms(mdx_ctx_t* ctx, const double* u, const double* v, const double* w, double* l2, double* linf,
                    double* umax = nullptr);
// Round-off floor of ||div u||_2: eps*sqrt(ncells)*umax*(1/dx+1/dy+1/dz).
double mdx_div_floor(const mdx_ctx_t* ctx, double umax);
int mdx_reduce_partials(mdx_ctx_t* ctx, double* sum, double* max1, double* max2);
#define MDX_RED_THREADS 256
int mdx_k_projection_redblack_mixed(mdx_ctx_t* ctx, double dg, mdx_solve_stats_t* st, bool* handled, double r0,
                                    double umax, double atol);
void mdx_mixed_free(mdx_ctx_t* ctx);
int mdx_ibm_coeff_launch(const mdx_grid_t* g, const mdx_ibm_geom_t* geom, double* d_coeff, int dix, int diy, int diz,
                         int planes, cudaStream_t stream);
// warm starts (k_warm.cu, k_unet.cu)
bool mdx_guess_supported(const mdx_ctx_t* ctx);
int mdx_warm_alloc(mdx_ctx_t* ctx);
void mdx_warm_free(mdx_ctx_t* ctx);
int mdx_warm_begin(mdx_ctx_t* ctx);
int mdx_warm_end(mdx_ctx_t* ctx, bool converged, int iterations);
int mdx_apply_guess(mdx_ctx_t* ctx, const double* gs, double dg);
int mdx_undo_guess(mdx_ctx_t* ctx);
int mdx_make_guess(mdx_ctx_t* ctx, bool* made);
// Make and apply this projection's guess; *rg = ||div u|| after it (r0 when
// none was kept or tol <= 0).
int mdx_guess_apply(mdx_ctx_t* ctx, double dg, double r0, bool* guessed, double* rg);
// learned correction of an applied extrapolated guess and snapshot capture (k_unet.cu)
int mdx_unet_correct(mdx_ctx_t* ctx, double dg, double* rg);
int mdx_unet_finish(mdx_ctx_t* ctx, bool converged, int iterations);
// The learned correction for another grid (an ensemble member), no host read
// (k_unet.cu): delta and its flag *ok on the device.
int mdx_unet_member_delta(mdx_ctx_t* nc, const mdx_dims& dm, double dx, double dy, double dz, double ire, double dg,
                          const double* un, const double* vn, const double* wn, const double* dp1, const double* dp2,
                          const double* mu_planes, double* delta, double* scal, int* ok);
void mdx_unet_free(mdx_ctx_t* ctx);
int mdx_k_div_norms_async(mdx_ctx_t* ctx, const double* u, const double* v, const double* w);
int mdx_k_cfl(mdx_ctx_t* ctx, double* cfl);
int mdx_k_dt_update(mdx_ctx_t* ctx, double* s, double cflmax, double dtmax);
int mdx_k_center_vel(mdx_ctx_t* ctx, double* uc, double* vc, double* wc);
int mdx_k_channel_ic(mdx_ctx_t* ctx, uint64_t seed, double amp_u, double amp_vw, const double* yc_host);
int mdx_k_fill(mdx_ctx_t* ctx, double* p, long long n, double v);
int mdx_reduce_init(mdx_ctx_t* ctx);

// Host-side modules.
void mdx_rk_coeffs(double* a, double* b, double* c);
void mdx_fft_make_plan(int n, mdx_fft_plan* p, bool* ok);
void mdx_fft_twiddles(int n, std::vector<double2>& tw);
