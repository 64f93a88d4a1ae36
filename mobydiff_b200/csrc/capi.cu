// capi.cu -- the extern "C" entry points of libmobyb200.so (declared in
// include/mobydiff_b200.h): context and device-mirror management, the
// reference-facing time-step calls, the CUDA-graph replay of whole RK3
// steps, and per-kernel-class event timing.
#include "mdx_internal.cuh"

#include <cmath>
#include <cstring>
#include <mutex>

static thread_local std::string g_err;   // last error of context-less calls

int mdx_fail(mdx_ctx_t* ctx, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    else g_err = buf;
    return code;
}

int mdx_check_launch(mdx_ctx_t* ctx, const char* what) {
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mdx_fail(ctx, MDX_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
    return MDX_OK;
}

// ---- timing ------------------------------------------------------------------
static cudaEvent_t ev_get(mdx_ctx_t* ctx) {
    if (!ctx->ev_free.empty()) {
        cudaEvent_t e = ctx->ev_free.back();
        ctx->ev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Fold completed event pairs into the per-class sums; with `wait` the stream
// is drained first so that every pending pair completes.
static void timing_resolve(mdx_ctx_t* ctx, bool wait) {
    if (ctx->ev_pending.empty()) return;
    if (wait) cudaStreamSynchronize(ctx->stream);
    size_t keep = 0;
    for (size_t q = 0; q < ctx->ev_pending.size(); ++q) {
        mdx_event_pair& p = ctx->ev_pending[q];
        if (!wait && cudaEventQuery(p.b) != cudaSuccess) {
            ctx->ev_pending[keep++] = p;
            continue;
        }
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            ctx->tim.ms[p.cls] += ms;
            ctx->tim.launches[p.cls] += p.n;
        }
        ctx->ev_free.push_back(p.a);
        ctx->ev_free.push_back(p.b);
    }
    ctx->ev_pending.resize(keep);
}

// Every MDX_TIMING_STRIDE-th launch of a class is bracketed by events, so
// that timing a long run costs little host time; get_timing scales the
// sampled mean to all launches of the class.
#define MDX_TIMING_STRIDE 8

void mdx_timer_begin(mdx_ctx_t* ctx, int cls, mdx_event_pair* p) {
    p->a = p->b = nullptr;
    p->cls = cls;
    p->n = 1;
    if (ctx->timing != 1 || ctx->capturing) return;
    if ((ctx->tim_issued[cls]++) % MDX_TIMING_STRIDE != 0) return;
    if (ctx->ev_pending.size() >= 4096) timing_resolve(ctx, false);
    if (ctx->ev_pending.size() >= 16384) timing_resolve(ctx, true);
    p->a = ev_get(ctx);
    p->b = ev_get(ctx);
    cudaEventRecord(p->a, ctx->stream);
}

void mdx_timer_end(mdx_ctx_t* ctx, mdx_event_pair* p) {
    if (!p->a) return;
    cudaEventRecord(p->b, ctx->stream);
    ctx->ev_pending.push_back(*p);
}

void mdx_sweep_run_begin(mdx_ctx_t* ctx, mdx_event_pair* p) {
    p->a = p->b = nullptr;
    p->cls = MDX_T_SOR_BLOCK;
    p->n = ctx->launches;
    if (!ctx->timing || ctx->capturing) return;
    if (ctx->ev_pending.size() >= 4096) timing_resolve(ctx, false);
    if (ctx->ev_pending.size() >= 16384) timing_resolve(ctx, true);
    p->a = ev_get(ctx);
    p->b = ev_get(ctx);
    cudaEventRecord(p->a, ctx->stream);
}

void mdx_sweep_run_end(mdx_ctx_t* ctx, mdx_event_pair* p, long long sweeps) {
    if (!p->a) return;
    cudaEventRecord(p->b, ctx->stream);
    p->n = sweeps >= 0 ? sweeps : ctx->launches - p->n;
    ctx->ev_pending.push_back(*p);
}

// ---- helpers -------------------------------------------------------------------
void mdx_rk_coeffs(double* a, double* b, double* c) {   // src/modules/step.f90:21-23
    a[0] = 64.0 / 120.0; a[1] = 50.0 / 120.0; a[2] = 90.0 / 120.0;
    b[0] = 0.0;          b[1] = -34.0 / 120.0; b[2] = -50.0 / 120.0;
    c[0] = 64.0 / 120.0; c[1] = 16.0 / 120.0; c[2] = 40.0 / 120.0;
}

static int need_fields(mdx_ctx_t* ctx) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (!ctx->fields) return mdx_fail(ctx, MDX_ERR_STATE, "field data not entered (call mdx_enter_field_data)");
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    return MDX_OK;
}

static int need_solver(mdx_ctx_t* ctx) {
    MDX_TRY(need_fields(ctx));
    if (!ctx->solver) return mdx_fail(ctx, MDX_ERR_STATE, "pressure solver not initialised (call mdx_init_pressure_solver)");
    return MDX_OK;
}

static size_t field_elems(const mdx_ctx_t* ctx, int f) {
    if (f == MDX_OLDRHSU || f == MDX_OLDRHSV || f == MDX_OLDRHSW || f == MDX_PHI) return (size_t)ctx->d.nint;
    return (size_t)ctx->d.npad;
}

static void release_graph(mdx_ctx_t* ctx) {
    if (ctx->step_graph) cudaGraphExecDestroy(ctx->step_graph);
    ctx->step_graph = nullptr;
    if (ctx->adapt_graph) cudaGraphExecDestroy(ctx->adapt_graph);
    ctx->adapt_graph = nullptr;
}

extern "C" {

const char* mdx_version(void) { return "mobydiff_b200 0.1 (sm_100a)"; }

const char* mdx_last_error(const mdx_ctx_t* ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

int mdx_device_count(int* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) n = 0;
    if (count) *count = n;
    if (n <= 0) return mdx_fail(nullptr, MDX_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    return MDX_OK;
}

void mdx_finalize_grid(mdx_grid_t* g) {   // src/modules/init.f90:38-44
    g->dx = g->lx / (double)g->nx;
    g->dy = g->ly / (double)g->ny;
    g->dz = g->lz / (double)g->nz;
    g->t_final = g->dt * (double)g->nsteps;
}

void mdx_default_grid(mdx_grid_t* g) {   // src/modules/init.f90:23-36
    std::memset(g, 0, sizeof(*g));
    g->nx = 200; g->ny = 200; g->nz = 200;
    g->nsteps = 10000;
    g->lx = 1.0; g->ly = 1.0; g->lz = 1.0;
    g->re = 100.0;
    g->forcing_x = 1.0; g->forcing_y = 0.0; g->forcing_z = 0.0;
    g->dt = 1.0e-4;
    g->cflmax = 0.0;
    g->dtmax = 1.0e-3;
    g->t_current = 0.0;
    g->cfl = 0.0;
    mdx_finalize_grid(g);
}

void mdx_default_bc(mdx_bc_t* bc) {   // src/modules/boundary.f90:14-20
    std::memset(bc, 0, sizeof(*bc));
    bc->is_periodic[0] = bc->is_periodic[1] = bc->is_periodic[2] = 1;
}

void mdx_default_solver_opts(mdx_solver_opts_t* o) {   // src/modules/pressure_workspace.f90:7-8
    std::memset(o, 0, sizeof(*o));
    o->solver = MDX_SOLVER_FFT;
    o->n_iter = 3;
    o->sor = 1.5;
    o->tol = 0.0;
    o->max_iter = 100000;
    o->check_every = 10;
    o->precision = MDX_PREC_FP64;
    o->atol = -1.0;
    o->inner_sor = 0.0;
}

int mdx_create(int device, const mdx_grid_t* g, const mdx_bc_t* bc, mdx_ctx_t** out) {
    if (!g || !bc || !out) return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_create: null argument");
    *out = nullptr;
    if (g->nx < 2 || g->ny < 2 || g->nz < 2)
        return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_create: nx, ny, nz must be >= 2 (got %d %d %d)", g->nx, g->ny, g->nz);
    const long long npad = (long long)(g->nx + 2) * (g->ny + 2) * (g->nz + 2);
    if (npad >= (1LL << 40)) return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_create: grid too large");
    if (!(g->dx > 0.0 && g->dy > 0.0 && g->dz > 0.0 && g->re > 0.0))
        return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_create: dx, dy, dz and re must be positive (call mdx_finalize_grid)");
    int n = 0;
    if (mdx_device_count(&n) != MDX_OK) return MDX_ERR_NO_DEVICE;
    if (device < 0 || device >= n) return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_create: device %d of %d", device, n);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return mdx_fail(nullptr, MDX_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    mdx_ctx_t* ctx = new mdx_ctx_t();
    ctx->device = device;
    ctx->g = *g;
    ctx->bc = *bc;
    for (int t = 0; t < 3; ++t) ctx->bcd.per[t] = bc->is_periodic[t] ? 1 : 0;
    for (int t = 0; t < 24; ++t) { ctx->bcd.type[t] = bc->bc_type[t]; ctx->bcd.value[t] = bc->bc_value[t]; }
    mdx_default_solver_opts(&ctx->opts);
    mdx_dims& d = ctx->d;
    d.nx = g->nx; d.ny = g->ny; d.nz = g->nz;
    d.nxp = g->nx + 2; d.nyp = g->ny + 2; d.nzp = g->nz + 2;
    d.nxh = g->nx / 2 + 1;
    d.hs = split_stride(g->nx);
    d.npad = npad;
    d.nint = (long long)g->nx * g->ny * g->nz;
    d.nspec = (long long)d.nxh * g->nz * g->ny;
    e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return mdx_fail(nullptr, MDX_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return MDX_OK;
}

int mdx_destroy_pressure_solver(mdx_ctx_t* ctx) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_graph(ctx);
    mdx_fft_free(ctx);
    cudaFree(ctx->f[MDX_PHI]);
    ctx->f[MDX_PHI] = nullptr;
    cudaFree(ctx->mu);
    ctx->mu = nullptr;
    ctx->mu_elems = 0;
    for (int t = 0; t < 4; ++t) {
        cudaFree(ctx->split_f[t]);
        ctx->split_f[t] = nullptr;
    }
    cudaFree(ctx->split_tab);
    ctx->split_tab = nullptr;
    ctx->split_norms = false;
    mdx_mixed_free(ctx);
    mdx_warm_free(ctx);
    ctx->solver = false;
    return MDX_OK;
}

int mdx_exit_field_data(mdx_ctx_t* ctx) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_graph(ctx);
    for (int f = 0; f < MDX_PHI; ++f) {
        cudaFree(ctx->f[f]);
        ctx->f[f] = nullptr;
    }
    for (int t = 0; t < 4; ++t) {   // the fused red-black pass swaps these with the field mirrors
        cudaFree(ctx->sor_alt[t]);
        ctx->sor_alt[t] = nullptr;
    }
    mdx_warm_free(ctx);
    mdx_unet_free(ctx);
    ctx->fields = false;
    return MDX_OK;
}

int mdx_destroy(mdx_ctx_t* ctx) {
    if (!ctx) return MDX_OK;
    cudaSetDevice(ctx->device);
    mdx_destroy_pressure_solver(ctx);
    mdx_exit_field_data(ctx);
    cudaFree(ctx->red_part);
    cudaFree(ctx->red_out);
    cudaFreeHost(ctx->red_host);
    cudaFree(ctx->dt_dev);
    for (int t = 0; t < 2; ++t)
        if (ctx->tune_ev[t]) cudaEventDestroy(ctx->tune_ev[t]);
    for (auto& p : ctx->ev_pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : ctx->ev_free) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return MDX_OK;
}

// Re and the body force of an existing context (the reference reads them
// once from input.ini; a training pipeline recording several flows on one
// context changes them between runs).  IBM coefficients, which carry 1/Re,
// are the caller's to re-enter.
int mdx_set_flow(mdx_ctx_t* ctx, double re, double fx, double fy, double fz) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (!(re > 0.0) || !std::isfinite(re) || !std::isfinite(fx) || !std::isfinite(fy) || !std::isfinite(fz))
        return mdx_fail(ctx, MDX_ERR_ARG, "mdx_set_flow: Re must be positive and the forces finite");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_graph(ctx);
    ctx->g.re = re;
    ctx->g.forcing_x = fx;
    ctx->g.forcing_y = fy;
    ctx->g.forcing_z = fz;
    return MDX_OK;
}

int mdx_set_bc(mdx_ctx_t* ctx, const mdx_bc_t* bc) {
    if (!ctx || !bc) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_set_bc: null argument");
    if (ctx->solver && ctx->opts.solver == MDX_SOLVER_REDBLACK && bc->is_periodic[1] && ctx->d.ny % 2 != 0)
        return mdx_fail(ctx, MDX_ERR_ARG, "red-black pressure solver with periodic y requires even ny");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_graph(ctx);
    ctx->bc = *bc;
    for (int t = 0; t < 3; ++t) ctx->bcd.per[t] = bc->is_periodic[t] ? 1 : 0;
    for (int t = 0; t < 24; ++t) { ctx->bcd.type[t] = bc->bc_type[t]; ctx->bcd.value[t] = bc->bc_value[t]; }
    ctx->sor_tuned = 0;
    for (int t = 0; t < 8; ++t) ctx->sor_tune_ms[t] = 0.0;
    ctx->rb32_tuned = 0;
    for (int t = 0; t < 8; ++t) ctx->rb32_tune_ms[t] = 0.0;
    ctx->pt_tuned = 0;
    for (int t = 0; t < 16; ++t) ctx->pt_tune_ms[t] = 0.0;
    // FFT solver: walls in x or z change the solve grid (and need Neumann
    // pressure there); rebuild its workspace for the new conditions
    if (ctx->solver && ctx->opts.solver == MDX_SOLVER_FFT &&
        (ctx->fft_ext_x || ctx->fft_ext_z || !bc->is_periodic[0] || !bc->is_periodic[2])) {
        mdx_fft_free(ctx);
        MDX_TRY(mdx_fft_init(ctx));
    }
    return MDX_OK;
}

int mdx_set_stream(mdx_ctx_t* ctx, void* stream) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_graph(ctx);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return MDX_OK;
}

int mdx_get_stream(mdx_ctx_t* ctx, void** stream) {
    if (!ctx || !stream) return mdx_fail(ctx, MDX_ERR_ARG, "null argument");
    *stream = (void*)ctx->stream;
    return MDX_OK;
}

int mdx_enter_field_data(mdx_ctx_t* ctx, const double* un, const double* us, const double* oldrhsu,
                         const double* vn, const double* vs, const double* oldrhsv, const double* wn,
                         const double* ws, const double* oldrhsw, const double* pn) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->fields) MDX_TRY(mdx_exit_field_data(ctx));
    const double* src[MDX_PHI] = {un, us, vn, vs, wn, ws, pn, oldrhsu, oldrhsv, oldrhsw, nullptr, nullptr, nullptr};
    for (int f = 0; f < MDX_PHI; ++f) {
        const size_t bytes = sizeof(double) * field_elems(ctx, f);
        cudaError_t e = cudaMalloc(&ctx->f[f], bytes);
        if (e != cudaSuccess) {
            mdx_exit_field_data(ctx);
            return mdx_fail(ctx, MDX_ERR_CUDA, "cudaMalloc of field %d (%zu bytes): %s", f, bytes, cudaGetErrorString(e));
        }
        if (src[f]) MDX_CUDA(ctx, cudaMemcpyAsync(ctx->f[f], src[f], bytes, cudaMemcpyHostToDevice, ctx->stream));
        else MDX_CUDA(ctx, cudaMemsetAsync(ctx->f[f], 0, bytes, ctx->stream));
    }
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->ibm_zero = true;
    ctx->fields = true;
    return MDX_OK;
}

int mdx_update_host(mdx_ctx_t* ctx, double* un, double* vn, double* wn, double* pn) {
    MDX_TRY(need_fields(ctx));
    double* dst[4] = {un, vn, wn, pn};
    const int ids[4] = {MDX_UN, MDX_VN, MDX_WN, MDX_PN};
    for (int t = 0; t < 4; ++t)
        if (dst[t])
            MDX_CUDA(ctx, cudaMemcpyAsync(dst[t], ctx->f[ids[t]], sizeof(double) * ctx->d.npad, cudaMemcpyDeviceToHost,
                                          ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MDX_OK;
}

int mdx_update_device(mdx_ctx_t* ctx, const double* un, const double* vn, const double* wn, const double* pn) {
    MDX_TRY(need_fields(ctx));
    const double* src[4] = {un, vn, wn, pn};
    const int ids[4] = {MDX_UN, MDX_VN, MDX_WN, MDX_PN};
    for (int t = 0; t < 4; ++t)
        if (src[t])
            MDX_CUDA(ctx, cudaMemcpyAsync(ctx->f[ids[t]], src[t], sizeof(double) * ctx->d.npad, cudaMemcpyHostToDevice,
                                          ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MDX_OK;
}

int mdx_copy_field(mdx_ctx_t* ctx, int field, double* host, int direction) {
    MDX_TRY(need_fields(ctx));
    if (field < 0 || field >= MDX_NUM_FIELDS || !host) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_copy_field: bad field/pointer");
    if (field == MDX_PHI && (direction != 0 || !ctx->f[MDX_PHI]))
        return mdx_fail(ctx, MDX_ERR_ARG, "mdx_copy_field: phi is device->host only and needs the FFT solver");
    const size_t bytes = sizeof(double) * field_elems(ctx, field);
    if (direction == 0) {
        MDX_CUDA(ctx, cudaMemcpyAsync(host, ctx->f[field], bytes, cudaMemcpyDeviceToHost, ctx->stream));
        MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    } else {
        MDX_CUDA(ctx, cudaMemcpyAsync(ctx->f[field], host, bytes, cudaMemcpyHostToDevice, ctx->stream));
        MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (field >= MDX_COEF_U && field <= MDX_COEF_W) {
            ctx->ibm_zero = false;
            ctx->coef_zinv = false;
        }
    }
    return MDX_OK;
}

int mdx_enter_ibm_data(mdx_ctx_t* ctx, const double* cu, const double* cv, const double* cw) {
    MDX_TRY(need_fields(ctx));
    release_graph(ctx);
    const double* src[3] = {cu, cv, cw};
    bool any = false, zinv = true;
    const size_t n = (size_t)ctx->d.npad;
    const size_t plane = (size_t)ctx->d.nxp * ctx->d.nyp;
    for (int t = 0; t < 3; ++t) {
        double* dst = ctx->f[MDX_COEF_U + t];
        if (src[t]) {
            for (size_t q = 0; q < n && !any; ++q) any = (src[t][q] != 0.0);
            // geometry that depends on x and y only gives equal z planes
            for (size_t q = plane; q < n && zinv; ++q) zinv = (src[t][q] == src[t][q % plane]);
            MDX_CUDA(ctx, cudaMemcpyAsync(dst, src[t], sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
        } else {
            MDX_CUDA(ctx, cudaMemsetAsync(dst, 0, sizeof(double) * n, ctx->stream));
        }
    }
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->ibm_zero = !any;
    ctx->coef_zinv = zinv;
    return MDX_OK;
}

// write_field (io.f90:105-137): device mirrors -> host -> field file.
int mdx_write_field_h5(mdx_ctx_t* ctx, const char* filename) {
    MDX_TRY(need_fields(ctx));
    if (!filename) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_write_field_h5: null file name");
    const size_t n = (size_t)ctx->d.npad;
    std::vector<double> h(4 * n);
    const int ids[4] = {MDX_UN, MDX_VN, MDX_WN, MDX_PN};
    for (int t = 0; t < 4; ++t)
        MDX_CUDA(ctx, cudaMemcpyAsync(h.data() + t * n, ctx->f[ids[t]], sizeof(double) * n, cudaMemcpyDeviceToHost,
                                      ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const mdx_grid_t& g = ctx->g;
    if (fdm_h5_write_field(filename, g.nx, g.ny, g.nz, g.lx, g.ly, g.lz, g.dx, g.dy, g.dz, g.re, g.dt, g.t_current,
                           h.data(), h.data() + n, h.data() + 2 * n, h.data() + 3 * n) != 0)
        return mdx_fail(ctx, MDX_ERR_IO, "could not write HDF5 field file: %s", filename);
    return MDX_OK;
}

// read_field (io.f90:139-166): field file -> host -> device mirrors.
int mdx_read_field_h5(mdx_ctx_t* ctx, const char* filename) {
    MDX_TRY(need_fields(ctx));
    if (!filename) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_read_field_h5: null file name");
    const size_t n = (size_t)ctx->d.npad;
    std::vector<double> h(4 * n);
    const mdx_grid_t& g = ctx->g;
    if (fdm_h5_read_field(filename, g.nx, g.ny, g.nz, h.data(), h.data() + n, h.data() + 2 * n, h.data() + 3 * n) != 0)
        return mdx_fail(ctx, MDX_ERR_IO, "could not read HDF5 field file: %s", mdx_h5_last_error());
    const int ids[4] = {MDX_UN, MDX_VN, MDX_WN, MDX_PN};
    for (int t = 0; t < 4; ++t)
        MDX_CUDA(ctx, cudaMemcpyAsync(ctx->f[ids[t]], h.data() + t * n, sizeof(double) * n, cudaMemcpyHostToDevice,
                                      ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MDX_OK;
}

// set_ibm_coeff for u, v, w then enter_ibm_data (src/main.f90:58-61), with
// the coefficients generated on the device straight into the mirrors.
int mdx_enter_ibm_geometry(mdx_ctx_t* ctx, const mdx_ibm_geom_t* geom) {
    MDX_TRY(need_fields(ctx));
    if (!geom) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_enter_ibm_geometry: null geometry");
    release_graph(ctx);
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    for (int t = 0; t < 3; ++t) {
        const int rc = mdx_ibm_coeff_launch(&ctx->g, geom, ctx->f[MDX_COEF_U + t], t == 0, t == 1, t == 2,
                                            ctx->d.nzp, ctx->stream);
        if (rc != MDX_OK) return mdx_fail(ctx, rc, "mdx_enter_ibm_geometry: bad geometry or launch failure");
        ctx->launches++;
    }
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->ibm_zero = false;   // a body is present (SOLID cells at least)
    ctx->coef_zinv = true;   // the walls depend on x and y only
    return MDX_OK;
}

int mdx_exit_ibm_data(mdx_ctx_t* ctx) {
    MDX_TRY(need_fields(ctx));
    release_graph(ctx);
    for (int t = 0; t < 3; ++t)
        MDX_CUDA(ctx, cudaMemsetAsync(ctx->f[MDX_COEF_U + t], 0, sizeof(double) * ctx->d.npad, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->ibm_zero = true;
    return MDX_OK;
}

int mdx_momentum(mdx_ctx_t* ctx, double dt_alpha, double dt_beta, double dt_gamma) {
    MDX_TRY(need_fields(ctx));
    return mdx_k_momentum(ctx, dt_alpha, dt_beta, dt_gamma);
}

int mdx_apply_bc(mdx_ctx_t* ctx) {
    MDX_TRY(need_fields(ctx));
    return mdx_k_apply_bc(ctx);
}

int mdx_apply_bc_redblack(mdx_ctx_t* ctx) {
    MDX_TRY(need_fields(ctx));
    return mdx_k_apply_bc_redblack(ctx);
}

int mdx_init_pressure_solver(mdx_ctx_t* ctx, const mdx_solver_opts_t* opts) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->solver) MDX_TRY(mdx_destroy_pressure_solver(ctx));
    mdx_solver_opts_t o;
    if (opts) o = *opts;
    else mdx_default_solver_opts(&o);
    if (o.solver != MDX_SOLVER_FFT && o.solver != MDX_SOLVER_REDBLACK)
        return mdx_fail(ctx, MDX_ERR_ARG, "unknown solver %d", o.solver);
    if (o.precision != MDX_PREC_FP64 && o.precision != MDX_PREC_MIXED)
        return mdx_fail(ctx, MDX_ERR_ARG, "unknown precision %d", o.precision);
    if (o.inner_form < 0 || o.inner_form > 2)
        return mdx_fail(ctx, MDX_ERR_ARG, "inner_form must be 0, 1 or 2, got %d", o.inner_form);
    if (o.check_every < 1) o.check_every = 1;
    if (o.max_iter < 1) o.max_iter = 1;
    if (o.n_iter < 0) return mdx_fail(ctx, MDX_ERR_ARG, "n_iter must be >= 0");
    ctx->opts = o;
    ctx->sor_tuned = 0;
    for (int t = 0; t < 8; ++t) ctx->sor_tune_ms[t] = 0.0;
    ctx->rb32_tuned = 0;
    for (int t = 0; t < 8; ++t) ctx->rb32_tune_ms[t] = 0.0;
    ctx->pt_tuned = 0;
    for (int t = 0; t < 16; ++t) ctx->pt_tune_ms[t] = 0.0;
    MDX_TRY(mdx_reduce_init(ctx));
    if (o.solver == MDX_SOLVER_REDBLACK) {
        // src/modules/pressure/pressure_redblack.f90:16-18
        if (ctx->d.nx % 2 != 0 || ctx->d.nz % 2 != 0)
            return mdx_fail(ctx, MDX_ERR_ARG, "red-black pressure solver requires even nx and nz for periodic coloring");
        // a periodic y wrap joins cells of one colour when ny is odd; the
        // parallel sweep would then race where the reference loop is ordered
        if (ctx->bc.is_periodic[1] && ctx->d.ny % 2 != 0)
            return mdx_fail(ctx, MDX_ERR_ARG, "red-black pressure solver with periodic y requires even ny");
    } else {
        MDX_TRY(mdx_fft_init(ctx));
    }
    ctx->solver = true;
    return MDX_OK;
}

int mdx_pressure_projection(mdx_ctx_t* ctx, double dt_gamma, mdx_solve_stats_t* stats) {
    MDX_TRY(need_solver(ctx));
    if (!(dt_gamma != 0.0)) return mdx_fail(ctx, MDX_ERR_ARG, "dt_gamma must be non-zero");
    if (ctx->opts.solver == MDX_SOLVER_FFT) {
        MDX_TRY(mdx_k_projection_fft(ctx, dt_gamma));
        if (ctx->opts.precision != MDX_PREC_MIXED) {
            mdx_solve_stats_t s{};
            ctx->last = s;
        }
        if (stats) {
            MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            *stats = ctx->last;
        }
        if (ctx->last.status == MDX_ERR_NONFINITE)
            return mdx_fail(ctx, MDX_ERR_NONFINITE, "non-finite divergence in the FFT defect correction");
        if (ctx->last.status == MDX_NOT_CONVERGED)
            return mdx_fail(ctx, MDX_NOT_CONVERGED, "FFT defect correction not converged after %d passes",
                            ctx->last.iterations);
        return MDX_OK;
    }
    mdx_solve_stats_t s{};
    MDX_TRY(mdx_k_projection_redblack(ctx, dt_gamma, &s));
    if (stats) *stats = s;
    if (s.status == MDX_ERR_NONFINITE) return mdx_fail(ctx, MDX_ERR_NONFINITE, "non-finite divergence in the red-black solve");
    if (s.status == MDX_NOT_CONVERGED)
        return mdx_fail(ctx, MDX_NOT_CONVERGED, "red-black solve not converged after %d iterations (residual %.3e)",
                        s.iterations, s.residual);
    return MDX_OK;
}

int mdx_last_solve_stats(const mdx_ctx_t* ctx, mdx_solve_stats_t* stats) {
    if (!ctx || !stats) return mdx_fail(nullptr, MDX_ERR_ARG, "mdx_last_solve_stats: null argument");
    *stats = ctx->last;
    return MDX_OK;
}

int mdx_get_cfl(mdx_ctx_t* ctx, double* cfl) {
    MDX_TRY(need_fields(ctx));
    if (!cfl) return mdx_fail(ctx, MDX_ERR_ARG, "null cfl");
    MDX_TRY(mdx_k_cfl(ctx, cfl));
    ctx->g.cfl = *cfl;
    return MDX_OK;
}

int mdx_center_vel(mdx_ctx_t* ctx, double* uc, double* vc, double* wc) {
    MDX_TRY(need_fields(ctx));
    return mdx_k_center_vel(ctx, uc, vc, wc);
}

int mdx_divergence_norms(mdx_ctx_t* ctx, double* l2, double* linf) {
    MDX_TRY(need_fields(ctx));
    double a = 0.0, b = 0.0;
    MDX_TRY(mdx_k_div_norms(ctx, ctx->f[MDX_UN], ctx->f[MDX_VN], ctx->f[MDX_WN], &a, &b));
    if (l2) *l2 = a;
    if (linf) *linf = b;
    return MDX_OK;
}

// One RK3 substage sequence, src/main.f90:69-89.
// One RK3 step with dt; with dtp (the FP64 FFT path only) the kernels read
// dt from the device instead.
static int rk_step_eager(mdx_ctx_t* ctx, double dt, long long* iters, const double* dtp = nullptr) {
    double a[3], b[3], c[3];
    mdx_rk_coeffs(a, b, c);
    for (int s = 0; s < 3; ++s) {
        const double da = dt * a[s], db = dt * b[s], dg = dt * c[s];
        if (dtp) {
            MDX_TRY(mdx_k_momentum(ctx, mdx_dscal(dtp, a[s]), mdx_dscal(dtp, b[s]), mdx_dscal(dtp, c[s])));
            MDX_TRY(mdx_k_apply_bc(ctx));
            MDX_TRY(mdx_k_projection_fft(ctx, mdx_dscal(dtp, c[s])));
            MDX_TRY(mdx_k_apply_bc(ctx));
            continue;
        }
        MDX_TRY(mdx_k_momentum(ctx, da, db, dg));
        if (ctx->opts.solver == MDX_SOLVER_FFT) {
            MDX_TRY(mdx_k_apply_bc(ctx));
            MDX_TRY(mdx_k_projection_fft(ctx, dg));
            if (ctx->opts.precision == MDX_PREC_MIXED) {
                if (iters) *iters += ctx->last.iterations;
                if (ctx->last.status != MDX_OK)
                    return mdx_fail(ctx, ctx->last.status, "FFT defect correction ended with status %d",
                                    ctx->last.status);
            }
            MDX_TRY(mdx_k_apply_bc(ctx));
        } else {
            mdx_solve_stats_t st{};
            MDX_TRY(mdx_k_projection_redblack(ctx, dg, &st));
            if (iters) *iters += st.iterations;
            if (st.status == MDX_ERR_NONFINITE)
                return mdx_fail(ctx, MDX_ERR_NONFINITE, "non-finite divergence in the red-black solve");
            if (st.status == MDX_NOT_CONVERGED)
                return mdx_fail(ctx, MDX_NOT_CONVERGED, "red-black solve not converged after %d iterations", st.iterations);
            MDX_TRY(mdx_k_apply_bc_redblack(ctx));
        }
    }
    return MDX_OK;
}

static int capture_fft_step(mdx_ctx_t* ctx, double dt) {
    release_graph(ctx);
    cudaGraph_t graph = nullptr;
    MDX_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->capturing = true;
    const long long before = ctx->launches;
    int rc = rk_step_eager(ctx, dt, nullptr);
    ctx->graph_launches = ctx->launches - before;   // kernels per replay
    ctx->launches = before;                         // capture launches nothing
    ctx->capturing = false;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc != MDX_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (e != cudaSuccess) return mdx_fail(ctx, MDX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ctx->step_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { ctx->step_graph = nullptr; return mdx_fail(ctx, MDX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    ctx->graph_dt = dt;
    return MDX_OK;
}

// One adaptive-dt step as a CUDA graph: the RK3 substages reading dt from
// ctx->dt_dev, then get_cfl's reduction and the dt update on the device.
static int capture_adaptive_step(mdx_ctx_t* ctx, double cflmax, double dtmax) {
    release_graph(ctx);
    cudaGraph_t graph = nullptr;
    MDX_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->capturing = true;
    const long long before = ctx->launches;
    int rc = rk_step_eager(ctx, 0.0, nullptr, ctx->dt_dev);
    if (rc == MDX_OK) rc = mdx_k_dt_update(ctx, ctx->dt_dev, cflmax, dtmax);
    ctx->adapt_launches = ctx->launches - before;
    ctx->launches = before;
    ctx->capturing = false;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc != MDX_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (e != cudaSuccess) return mdx_fail(ctx, MDX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ctx->adapt_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { ctx->adapt_graph = nullptr; return mdx_fail(ctx, MDX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    ctx->adapt_cflmax = cflmax;
    ctx->adapt_dtmax = dtmax;
    return MDX_OK;
}

int mdx_step_adaptive(mdx_ctx_t* ctx, int nsteps, double cflmax, double dtmax, long long* total_iters) {
    MDX_TRY(need_solver(ctx));
    if (nsteps < 0) return mdx_fail(ctx, MDX_ERR_ARG, "nsteps < 0");
    if (!std::isfinite(cflmax) || !std::isfinite(dtmax) || (cflmax > 0.0 && !(dtmax > 0.0)))
        return mdx_fail(ctx, MDX_ERR_ARG, "cflmax and dtmax must be finite, dtmax > 0 when cflmax > 0");
    ctx->g.cflmax = cflmax;
    ctx->g.dtmax = dtmax;
    if (!(cflmax > 0.0)) return mdx_step(ctx, nsteps, total_iters);   // fixed dt, no CFL (main.f90:92-97)
    long long iters = 0;
    const bool use_graph = ctx->opts.solver == MDX_SOLVER_FFT && ctx->opts.precision == MDX_PREC_FP64 && !ctx->timing;
    if (!use_graph) {
        for (int n = 0; n < nsteps; ++n) {
            const double dt = ctx->g.dt;
            ctx->g.t_current = ctx->g.t_current + dt;
            MDX_TRY(rk_step_eager(ctx, dt, &iters));
            double cfl = 0.0;
            MDX_TRY(mdx_k_cfl(ctx, &cfl));
            ctx->g.cfl = cfl;
            if (cfl > 0.0) ctx->g.dt = std::fmin(cflmax / cfl, dtmax);
        }
        if (total_iters) *total_iters = iters;
        return MDX_OK;
    }
    if (!ctx->dt_dev) MDX_CUDA(ctx, cudaMalloc(&ctx->dt_dev, 4 * sizeof(double)));
    if (!ctx->adapt_graph || ctx->adapt_cflmax != cflmax || ctx->adapt_dtmax != dtmax)
        MDX_TRY(capture_adaptive_step(ctx, cflmax, dtmax));
    double* hs = ctx->red_host;   // pinned, 3 doubles: {dt, t, cfl} in and out
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    hs[0] = ctx->g.dt;
    hs[1] = ctx->g.t_current;
    hs[2] = ctx->g.cfl;
    MDX_CUDA(ctx, cudaMemcpyAsync(ctx->dt_dev, hs, 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    for (int n = 0; n < nsteps; ++n) {
        MDX_CUDA(ctx, cudaGraphLaunch(ctx->adapt_graph, ctx->stream));
        ctx->launches += ctx->adapt_launches;
    }
    MDX_CUDA(ctx, cudaMemcpyAsync(hs, ctx->dt_dev, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->g.dt = hs[0];
    ctx->g.t_current = hs[1];
    ctx->g.cfl = hs[2];
    if (total_iters) *total_iters = 0;
    return MDX_OK;
}

int mdx_get_time(mdx_ctx_t* ctx, double* dt, double* t_current, double* cfl) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (dt) *dt = ctx->g.dt;
    if (t_current) *t_current = ctx->g.t_current;
    if (cfl) *cfl = ctx->g.cfl;
    return MDX_OK;
}

int mdx_set_dt(mdx_ctx_t* ctx, double dt) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (!(dt > 0.0) || !std::isfinite(dt)) return mdx_fail(ctx, MDX_ERR_ARG, "dt must be positive and finite");
    ctx->g.dt = dt;
    return MDX_OK;
}

int mdx_step(mdx_ctx_t* ctx, int nsteps, long long* total_iters) {
    MDX_TRY(need_solver(ctx));
    if (nsteps < 0) return mdx_fail(ctx, MDX_ERR_ARG, "nsteps < 0");
    long long iters = 0;
    const double dt = ctx->g.dt;
    // the mixed FFT path decides its passes on the host: no graph
    const bool use_graph = ctx->opts.solver == MDX_SOLVER_FFT && ctx->opts.precision == MDX_PREC_FP64 && !ctx->timing;
    if (use_graph && (!ctx->step_graph || ctx->graph_dt != dt)) MDX_TRY(capture_fft_step(ctx, dt));
    for (int n = 0; n < nsteps; ++n) {
        ctx->g.t_current = ctx->g.t_current + dt;   // src/main.f90:67
        if (use_graph) {
            MDX_CUDA(ctx, cudaGraphLaunch(ctx->step_graph, ctx->stream));
            ctx->launches += ctx->graph_launches;
        } else {
            MDX_TRY(rk_step_eager(ctx, dt, &iters));
        }
    }
    if (total_iters) *total_iters = iters;
    return MDX_OK;
}

int mdx_channel_ic(mdx_ctx_t* ctx, uint64_t seed, double amp_u, double amp_vw, double y0, double wave_amp,
                   double wave_lambda, mdx_solve_stats_t* stats) {
    MDX_TRY(need_solver(ctx));
    const mdx_dims& d = ctx->d;
    std::vector<double> yc(d.nx);
    const double pi = 3.141592653589793;
    for (int i = 1; i <= d.nx; ++i) {
        const double x = (double)(i - 1) * ctx->g.dx;
        double v = y0 + 1.0;
        if (wave_amp != 0.0) v = v + wave_amp * std::sin(2.0 * pi * x / wave_lambda);
        yc[i - 1] = v;
    }
    const size_t bytes = sizeof(double) * d.npad;
    double** f = ctx->f;
    for (int t : {MDX_UN, MDX_VN, MDX_WN, MDX_PN, MDX_US, MDX_VS, MDX_WS})
        MDX_CUDA(ctx, cudaMemsetAsync(f[t], 0, bytes, ctx->stream));
    for (int t : {MDX_OLDRHSU, MDX_OLDRHSV, MDX_OLDRHSW})
        MDX_CUDA(ctx, cudaMemsetAsync(f[t], 0, sizeof(double) * d.nint, ctx->stream));
    MDX_TRY(mdx_k_channel_ic(ctx, seed, amp_u, amp_vw, yc.data()));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_US], f[MDX_UN], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_VS], f[MDX_VN], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(f[MDX_WS], f[MDX_WN], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    mdx_solve_stats_t s{};
    // the t=0 projection takes no guess and starts the increment history afresh
    const int guess_mode = ctx->guess_mode;
    const bool record = ctx->record_increments;
    ctx->guess_mode = MDX_GUESS_ZERO;
    ctx->record_increments = false;
    int rc = MDX_OK;
    if (ctx->opts.solver == MDX_SOLVER_FFT) {
        rc = mdx_k_apply_bc(ctx);
        if (rc == MDX_OK) rc = mdx_k_projection_fft(ctx, 1.0);
        if (rc == MDX_OK) rc = mdx_k_apply_bc(ctx);
    } else {
        rc = mdx_k_projection_redblack(ctx, 1.0, &s);
        if (rc == MDX_OK) rc = mdx_k_apply_bc_redblack(ctx);
    }
    ctx->guess_mode = guess_mode;
    ctx->record_increments = record;
    ctx->proj_count = 0;
    ctx->hist_valid = 0;
    MDX_TRY(rc);
    MDX_CUDA(ctx, cudaMemsetAsync(f[MDX_PN], 0, bytes, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (stats) *stats = s;
    if (s.status == MDX_ERR_NONFINITE) return mdx_fail(ctx, MDX_ERR_NONFINITE, "non-finite divergence in the t=0 projection");
    if (s.status == MDX_NOT_CONVERGED) return mdx_fail(ctx, MDX_NOT_CONVERGED, "t=0 projection not converged");
    return MDX_OK;
}

int mdx_set_timing(mdx_ctx_t* ctx, int on) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    timing_resolve(ctx, true);
    std::memset(&ctx->tim, 0, sizeof(ctx->tim));
    std::memset(ctx->tim_issued, 0, sizeof(ctx->tim_issued));
    if (on < 0 || on > 2) return mdx_fail(ctx, MDX_ERR_ARG, "timing mode %d (0 off, 1 sampled launches, 2 sweep runs)", on);
    ctx->timing = on;
    return MDX_OK;
}

int mdx_get_timing(mdx_ctx_t* ctx, mdx_timing_t* out) {
    if (!ctx || !out) return mdx_fail(ctx, MDX_ERR_ARG, "null argument");
    timing_resolve(ctx, true);
    // scale the sampled launches' mean to every launch of the class
    for (int c = 0; c < MDX_T_NUM; ++c) {
        if (c == MDX_T_SOR_BLOCK) {   // every run timed: the measured total
            out->launches[c] = ctx->tim.launches[c];
            out->ms[c] = ctx->tim.ms[c];
            continue;
        }
        const long long timed = ctx->tim.launches[c];
        out->launches[c] = ctx->tim_issued[c];
        out->ms[c] = timed > 0 ? ctx->tim.ms[c] * (double)ctx->tim_issued[c] / (double)timed : 0.0;
    }
    return MDX_OK;
}

long long mdx_launch_count(const mdx_ctx_t* ctx) { return ctx ? ctx->launches : 0; }

}  // extern "C"
