// host_config.cpp -- host-side set-up that the reference performs on the CPU
// once per run: the input.ini reader (src/modules/config.f90) and the IBM
// coefficient generator (src/modules/ibm.f90).  Neither touches the device.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/mobydiff_b200.h"

namespace {

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}
std::string rtrim(const std::string& s) {
    size_t e = s.find_last_not_of(' ');
    return e == std::string::npos ? std::string() : s.substr(0, e + 1);
}
std::string ltrim(const std::string& s) {   // Fortran adjustl moves leading blanks only
    size_t b = s.find_first_not_of(' ');
    return b == std::string::npos ? std::string() : s.substr(b);
}

// clean_string, config.f90:415-431: trim, adjustl, strip one pair of
// matching surrounding quotes.
std::string clean_string(const std::string& v) {
    std::string t = rtrim(ltrim(v));
    if (t.size() >= 2 && ((t.front() == '"' && t.back() == '"') || (t.front() == '\'' && t.back() == '\'')))
        return t.substr(1, t.size() - 2);
    return t;
}

// First item of a Fortran list-directed read: separators are blanks,
// commas, slashes (and tabs).
std::string first_item(const std::string& v) {
    size_t b = v.find_first_not_of(" \t");
    if (b == std::string::npos) return std::string();
    size_t e = v.find_first_of(" \t,/", b);
    return v.substr(b, e == std::string::npos ? std::string::npos : e - b);
}

bool parse_int(const std::string& v, int* out) {
    std::string t = first_item(v);
    if (t.empty()) return false;
    size_t p = 0;
    if (t[p] == '+' || t[p] == '-') ++p;
    if (p >= t.size()) return false;
    for (size_t q = p; q < t.size(); ++q)
        if (!std::isdigit((unsigned char)t[q])) return false;
    errno = 0;
    long long x = std::strtoll(t.c_str(), nullptr, 10);
    if (errno != 0 || x > 2147483647LL || x < -2147483648LL) return false;
    *out = (int)x;
    return true;
}

// Fortran real input: digits with optional point and an exponent letter
// e/E/d/D/q/Q.
bool parse_real(const std::string& v, double* out) {
    std::string t = first_item(v);
    if (t.empty()) return false;
    std::string c;
    bool digit = false;
    for (char ch : t) {
        if (ch == 'd' || ch == 'D' || ch == 'q' || ch == 'Q') ch = 'e';
        if (std::isdigit((unsigned char)ch)) digit = true;
        c.push_back(ch);
    }
    if (!digit) return false;
    char* end = nullptr;
    errno = 0;
    double x = std::strtod(c.c_str(), &end);
    if (end == c.c_str() || *end != '\0' || errno == ERANGE) return false;
    *out = x;
    return true;
}

struct Reader {
    mdx_grid_t* g;
    mdx_bc_t* bc;
    mdx_solver_opts_t* o;
    mdx_run_config_t* run;
    bool nsteps_seen = false, t_final_seen = false;
    int warnings = 0;

    void warn(const char* msg, int line) {
        std::printf(" warning: %s on input line %d\n", msg, line);
        std::fflush(stdout);
        ++warnings;
    }
    void rd_int(const std::string& v, int* t, int line) {
        int x;
        if (parse_int(v, &x)) *t = x;
        else warn("could not parse integer", line);
    }
    void rd_real(const std::string& v, double* t, int line) {
        double x;
        if (parse_real(v, &x)) *t = x;
        else warn("could not parse real value", line);
    }
    void rd_bool(const std::string& v, int* t, int line) {   // config.f90:279-295
        std::string s = lower(clean_string(v));
        if (s == "true" || s == "t" || s == ".true." || s == "yes" || s == "y" || s == "1" || s == "periodic") *t = 1;
        else if (s == "false" || s == "f" || s == ".false." || s == "no" || s == "n" || s == "0" ||
                 s == "nonperiodic" || s == "non-periodic") *t = 0;
        else warn("could not parse logical value", line);
    }
    void rd_bc_type(const std::string& v, int* t, int line) {   // config.f90:297-319
        std::string s = lower(clean_string(v));
        if (s == "dirichlet" || s == "d" || s == "fixed" || s == "value" || s == "0") { *t = 0; return; }
        if (s == "neumann" || s == "n" || s == "gradient" || s == "normal_gradient" || s == "1") { *t = 1; return; }
        int x;
        if (parse_int(s, &x) && (x == 0 || x == 1)) *t = x;
        else warn("boundary type must be dirichlet/0 or neumann/1", line);
    }

    static int dir_index(const std::string& s) {   // config.f90:234-247
        if (s == "x" || s == "i" || s == "streamwise") return 1;
        if (s == "y" || s == "j" || s == "wallnormal" || s == "wall_normal") return 2;
        if (s == "z" || s == "k" || s == "spanwise") return 3;
        return 0;
    }
    static int side_index(const std::string& s) {   // :249-260
        if (s == "min" || s == "lo" || s == "low" || s == "lower" || s == "left" || s == "bottom" || s == "front") return 0;
        if (s == "max" || s == "hi" || s == "high" || s == "upper" || s == "right" || s == "top" || s == "back") return 1;
        return -1;
    }
    static int var_index(const std::string& s) {   // :262-277
        if (s == "p" || s == "pressure") return 0;
        if (s == "u" || s == "un") return 1;
        if (s == "v" || s == "vn") return 2;
        if (s == "w" || s == "wn") return 3;
        return -1;
    }

    void boundary(const std::string& key, const std::string& value, int line) {   // :172-203
        if (key == "periodic_x" || key == "x_periodic" || key == "isperiodic_x" || key == "x_is_periodic")
            return rd_bool(value, &bc->is_periodic[0], line);
        if (key == "periodic_y" || key == "y_periodic" || key == "isperiodic_y" || key == "y_is_periodic")
            return rd_bool(value, &bc->is_periodic[1], line);
        if (key == "periodic_z" || key == "z_periodic" || key == "isperiodic_z" || key == "z_is_periodic")
            return rd_bool(value, &bc->is_periodic[2], line);
        // parse_boundary_key, :205-232: <dir>_<side>_<var>_<field>
        int dir = 0, side = -1, var = -1;
        std::string field;
        size_t p1 = key.find('_');
        if (p1 != std::string::npos && p1 >= 1) {
            size_t p2 = key.find('_', p1 + 1);
            if (p2 != std::string::npos && p2 >= p1 + 2) {
                size_t p3 = key.find('_', p2 + 1);
                if (p3 != std::string::npos && p3 >= p2 + 2) {
                    dir = dir_index(key.substr(0, p1));
                    side = side_index(key.substr(p1 + 1, p2 - p1 - 1));
                    var = var_index(key.substr(p2 + 1, p3 - p2 - 1));
                    field = rtrim(key.substr(p3 + 1));
                }
            }
        }
        if (dir == 0 || side < 0 || var < 0) {
            std::printf(" warning: unknown boundary key on input line %d: %s\n", line, key.c_str());
            std::fflush(stdout);
            ++warnings;
            return;
        }
        const int idx = (dir - 1) + 3 * (side + 2 * var);
        if (field == "type") rd_bc_type(value, &bc->bc_type[idx], line);
        else if (field == "value") rd_real(value, &bc->bc_value[idx], line);
        else warn("boundary key must end in _type or _value", line);
    }

    void b200(const std::string& key, const std::string& value, int line) {
        const std::string v = lower(clean_string(value));
        if (key == "solver") {
            if (v == "fft" || v == "0") o->solver = MDX_SOLVER_FFT;
            else if (v == "redblack" || v == "red-black" || v == "sor" || v == "1") o->solver = MDX_SOLVER_REDBLACK;
            else warn("b200 solver must be fft or redblack", line);
        } else if (key == "tol" || key == "tolerance") {
            rd_real(value, &o->tol, line);
        } else if (key == "omega" || key == "sor") {
            rd_real(value, &o->sor, line);
        } else if (key == "inner_omega" || key == "inner_sor") {
            rd_real(value, &o->inner_sor, line);
        } else if (key == "check_mode" || key == "residual_checks") {
            if (v == "adaptive" || v == "0") o->check_mode = 0;
            else if (v == "fixed" || v == "every" || v == "1") o->check_mode = 1;
            else warn("b200 residual_checks must be adaptive or fixed", line);
        } else if (key == "fft_kernel") {
            if (v == "warp" || v == "0") o->fft_kernel = 0;
            else if (v == "stockham" || v == "1") o->fft_kernel = 1;
            else warn("b200 fft_kernel must be warp or stockham", line);
        } else if (key == "inner_form") {
            if (v == "potential" || v == "0") o->inner_form = 0;
            else if (v == "faces" || v == "1") o->inner_form = 1;
            else if (v == "potential_all" || v == "2") o->inner_form = 2;
            else warn("b200 inner_form must be potential, faces or potential_all", line);
        } else if (key == "max_iter") {
            rd_int(value, &o->max_iter, line);
        } else if (key == "check_every") {
            rd_int(value, &o->check_every, line);
        } else if (key == "precision") {
            if (v == "fp64" || v == "double" || v == "0") o->precision = MDX_PREC_FP64;
            else if (v == "mixed" || v == "1") o->precision = MDX_PREC_MIXED;
            else warn("b200 precision must be fp64 or mixed", line);
        } else if (run && (key == "guess" || key == "warm_start")) {
            if (v == "zero" || v == "0") run->guess = MDX_GUESS_ZERO;
            else if (v == "previous" || v == "1") run->guess = MDX_GUESS_PREVIOUS;
            else if (v == "extrapolated" || v == "3") run->guess = MDX_GUESS_EXTRAPOLATED;
            else warn("b200 guess must be zero, previous or extrapolated", line);
        } else if (run && key == "ic") {
            if (v == "zero" || v == "0") run->ic = 0;
            else if (v == "channel" || v == "1") run->ic = 1;
            else warn("b200 ic must be zero or channel", line);
        } else if (run && key == "seed") {
            std::string t = first_item(value);
            char* end = nullptr;
            unsigned long long s = std::strtoull(t.c_str(), &end, 10);
            if (t.empty() || *end != '\0') warn("could not parse integer", line);
            else run->seed = (uint64_t)s;
        } else if (run && key == "ibm") {
            if (v == "none" || v == "off" || v == "-1") run->ibm = -1;
            else if (v == "reference" || v == "bump" || v == "0") run->ibm = 0;
            else if (v == "wavy" || v == "wavy_channel" || v == "1") run->ibm = 1;
            else warn("b200 ibm must be none, reference or wavy", line);
        } else if (run && key == "ibm_amp") {
            rd_real(value, &run->ibm_amp, line);
        } else if (run && key == "ibm_lambda") {
            rd_real(value, &run->ibm_lambda, line);
        } else if (run && key == "ibm_y0") {
            rd_real(value, &run->ibm_y0, line);
        } else if (run && key == "ibm_height") {
            rd_real(value, &run->ibm_height, line);
        }
    }

    void apply(const std::string& section, const std::string& key_in, const std::string& value, int line) {
        const std::string sec = lower(rtrim(section));
        const std::string key = lower(rtrim(key_in));
        if (sec == "grid") {   // config.f90:100-114
            if (key == "nx") rd_int(value, &g->nx, line);
            else if (key == "ny") rd_int(value, &g->ny, line);
            else if (key == "nz") rd_int(value, &g->nz, line);
            else if (key == "lx") rd_real(value, &g->lx, line);
            else if (key == "ly") rd_real(value, &g->ly, line);
            else if (key == "lz") rd_real(value, &g->lz, line);
        } else if (sec == "flow") {   // :115-125
            if (key == "re") rd_real(value, &g->re, line);
            else if (key == "forcing_x" || key == "force_x" || key == "body_force_x" || key == "meanpx") rd_real(value, &g->forcing_x, line);
            else if (key == "forcing_y" || key == "force_y" || key == "body_force_y" || key == "meanpy") rd_real(value, &g->forcing_y, line);
            else if (key == "forcing_z" || key == "force_z" || key == "body_force_z" || key == "meanpz") rd_real(value, &g->forcing_z, line);
        } else if (sec == "time") {   // :126-140
            if (key == "dt") rd_real(value, &g->dt, line);
            else if (key == "nsteps" || key == "steps") { rd_int(value, &g->nsteps, line); nsteps_seen = true; }
            else if (key == "t_final") { rd_real(value, &g->t_final, line); t_final_seen = true; }
            else if (key == "cflmax") rd_real(value, &g->cflmax, line);
            else if (key == "dtmax") rd_real(value, &g->dtmax, line);
        } else if (sec == "output") {   // :141-151
            if (!run) return;
            if (key == "interval" || key == "output_interval") rd_int(value, &run->output_interval, line);
            else if (key == "prefix") std::snprintf(run->output_prefix, sizeof(run->output_prefix), "%s", clean_string(value).c_str());
            else if (key == "field_interval" || key == "hdf5_interval" || key == "h5_interval") rd_int(value, &run->field_interval, line);
            else if (key == "field_prefix" || key == "hdf5_prefix" || key == "h5_prefix")
                std::snprintf(run->field_prefix, sizeof(run->field_prefix), "%s", clean_string(value).c_str());
        } else if (sec == "pressure") {   // :152-166 (the red-black knobs)
            if (key == "niter" || key == "n_iter" || key == "iterations") {
                int n = o->n_iter;
                rd_int(value, &n, line);
                if (n > 0) o->n_iter = n;
                else warn("pressure nIter must be positive", line);
            } else if (key == "sor" || key == "omega") {
                rd_real(value, &o->sor, line);
            }
        } else if (sec == "boundary") {
            boundary(key, value, line);
        } else if (sec == "b200") {
            b200(key, value, line);
        }
        // other sections are ignored, as in the reference (no case default)
    }
};

}  // namespace

extern "C" int mdx_read_runtime_config(const char* path, mdx_grid_t* g, mdx_bc_t* bc, mdx_solver_opts_t* opts,
                                       mdx_run_config_t* run) {
    mdx_grid_t gd;
    mdx_bc_t bd;
    mdx_solver_opts_t od;
    if (!g) { mdx_default_grid(&gd); g = &gd; }
    if (!bc) { mdx_default_bc(&bd); bc = &bd; }
    if (!opts) { mdx_default_solver_opts(&od); opts = &od; }
    if (run) {   // config.f90:25-28 and the [b200] defaults
        std::memset(run, 0, sizeof(*run));
        run->output_interval = 1;
        run->field_interval = 0;
        std::snprintf(run->output_prefix, sizeof(run->output_prefix), "data");
        std::snprintf(run->field_prefix, sizeof(run->field_prefix), "field");
        run->ic = 0;
        run->seed = 20261203ULL;
        run->ibm = 0;          // the reference always applies its IBM bump (src/main.f90:57-61)
        run->ibm_amp = 0.05;
        run->ibm_lambda = 0.0; // 0: lx/2
        run->ibm_y0 = -1.0;    // <0: centre a channel of ibm_height in ly
        run->ibm_height = 2.0;
    }
    if (!path) return MDX_ERR_ARG;
    FILE* fp = std::fopen(path, "r");
    if (!fp) {   // config.f90:33-45
        std::printf(" input file not found; using defaults: %s\n", path);
        std::fflush(stdout);
        mdx_finalize_grid(g);
        return MDX_OK;
    }
    Reader r{g, bc, opts, run};
    std::string section;
    char buf[4096];
    int line_no = 0;
    while (std::fgets(buf, sizeof(buf), fp)) {
        ++line_no;
        std::string line(buf);
        while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
        if (line.size() > 512) line.resize(512);   // character(len=512) :: line
        // strip_comment, :358-369
        size_t cut = line.find_first_of(";#");
        if (cut != std::string::npos) line.resize(cut);
        line = ltrim(line);
        if (rtrim(line).empty()) continue;
        if (line[0] == '[') {   // parse_section, :321-330
            size_t last = line.find(']');
            if (last != std::string::npos && last + 1 > 2) section = lower(rtrim(line.substr(1, last - 1)));
            continue;
        }
        // split_key_value, :332-356
        std::string key, value;
        size_t eq = line.find('=');
        if (eq != std::string::npos) {
            key = ltrim(line.substr(0, eq));
            value = ltrim(line.substr(eq + 1));
        } else {
            size_t sep = line.find_first_of(" \t");
            if (sep != std::string::npos) {
                key = ltrim(line.substr(0, sep));
                value = ltrim(line.substr(sep + 1));
            } else {
                key = line;
            }
        }
        key = rtrim(key);
        value = rtrim(value);
        if (key.empty()) continue;
        r.apply(section, key, value, line_no);
    }
    std::fclose(fp);
    if (r.t_final_seen && !r.nsteps_seen) {   // :71-73
        double q = std::ceil(g->t_final / g->dt);
        g->nsteps = std::max(1, (int)q);
    }
    mdx_finalize_grid(g);
    if (run) run->warnings = r.warnings;
    return MDX_OK;
}

// ---------------------------------------------------------------------------
// IBM coefficients, src/modules/ibm.f90:84-187 (set_ibm_coeff with
// USE_IBM_SECONDORDER, the CMake default).
// ---------------------------------------------------------------------------
namespace {

bool in_body(const double* x, const mdx_ibm_geom_t* ib, const mdx_grid_t* g) {
    const double pi = 3.141592653589793;
    if (ib->geometry == 0) {   // ibm.f90:94-97
        const double y_body =
            ib->amp * 0.5 * (1.0 + std::sin(2.0 * pi * (double)ib->n_wave_x * x[0] / g->lx + ib->phase)) + 2 * g->dy;
        return x[1] < y_body;
    }
    const double y_lo = ib->y0 + ib->amp * std::sin(2.0 * pi * x[0] / ib->lambda + ib->phase);
    return x[1] < y_lo || x[1] > y_lo + ib->height;
}

// Euclidean norm by the scaled sum of squares (the Fortran NORM2 method).
double norm2(const double* v) {
    double scale = 0.0, ssq = 1.0;
    for (int t = 0; t < 3; ++t) {
        if (v[t] == 0.0) continue;
        const double a = std::fabs(v[t]);
        if (scale < a) {
            const double q = scale / a;
            ssq = 1.0 + ssq * (q * q);
            scale = a;
        } else {
            const double q = a / scale;
            ssq = ssq + q * q;
        }
    }
    return scale * std::sqrt(ssq);
}

void bisect(const double* xa_in, double* xb_io, const mdx_ibm_geom_t* ib, const mdx_grid_t* g) {   // ibm.f90:101-130
    double xa[3] = {xa_in[0], xa_in[1], xa_in[2]};
    double xb[3] = {xb_io[0], xb_io[1], xb_io[2]};
    double xm[3] = {0.0, 0.0, 0.0};
    for (int it = 0; it < 200; ++it) {
        for (int t = 0; t < 3; ++t) xm[t] = 0.5 * (xa[t] + xb[t]);
        const double dd[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
        if (norm2(dd) < 1.0e-10) break;
        const bool la = in_body(xa, ib, g), lm = in_body(xm, ib, g);
        double* dst = (lm == la) ? xa : xb;
        for (int t = 0; t < 3; ++t) dst[t] = xm[t];
    }
    for (int t = 0; t < 3; ++t) xb_io[t] = xm[t];
}

}  // namespace

extern "C" int mdx_set_ibm_coeff(const mdx_grid_t* g, const mdx_ibm_geom_t* ib, double* coeff, int dix, int diy, int diz) {
    if (!g || !ib || !coeff) return MDX_ERR_ARG;
    if (ib->geometry == 1 && !(ib->lambda != 0.0)) return MDX_ERR_ARG;
    const int ni = g->nx + 2, nj = g->ny + 2, nk = g->nz + 2;
    static const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    auto coord = [&](int ix, int iy, int iz, double* x) {   // ibm.f90:161-163
        x[0] = ((double)ix - (double)dix * 0.5 - 1.5) * g->dx;
        x[1] = ((double)iy - (double)diy * 0.5 - 1.5) * g->dy;
        x[2] = ((double)iz - (double)diz * 0.5 - 1.5) * g->dz;
    };
    for (int iz = 1; iz <= nk; ++iz)
        for (int iy = 1; iy <= nj; ++iy)
            for (int ix = 1; ix <= ni; ++ix) {
                double xa[3];
                coord(ix, iy, iz, xa);
                double c = 0.0;
                if (in_body(xa, ib, g)) {
                    c = 1.0e30;   // SOLID, ibm.f90:20
                } else {
                    for (int n = 0; n < 6; ++n) {
                        double xb[3];
                        coord(ix + nb[n][0], iy + nb[n][1], iz + nb[n][2], xb);
                        const double d0v[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
                        const double d0 = norm2(d0v);
                        if (in_body(xb, ib, g)) {
                            bisect(xa, xb, ib, g);
                            const double dv[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
                            const double d = norm2(dv);
                            c = c + ((d0 - d) / d) / (d0 * d0);
                        }
                    }
                }
                coeff[(size_t)(ix - 1) + (size_t)ni * ((size_t)(iy - 1) + (size_t)nj * (size_t)(iz - 1))] = c;
            }
    const size_t n = (size_t)ni * nj * nk;
    for (size_t t = 0; t < n; ++t) coeff[t] = coeff[t] / g->re;   // ibm.f90:186
    return MDX_OK;
}
