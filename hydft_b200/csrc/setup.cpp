// Host-side setup of a simulation: the reference's params_t (namelist input
// and derived defaults), units, structure source, free-energy term list,
// transport, stress closure, external potential and the grid band, turned
// into the constants and tables the device solver consumes.
//
//   params      src/core/params.f90:17-180
//   units       src/core/units.f90:41-70
//   species     src/model/species.f90:49-153
//   transport   src/transport/transport.f90:61-111, stanton_murillo.f90:63-154
//   stress      src/closure/stress.f90:37-57
//   grid/mask   src/core/grid.f90:34-113
//   vext        src/model/external_potential.f90:39-93
#include "setup.hpp"

#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "fermi_dirac.cuh"
#include "setup_gpu.hpp"

namespace hydft {

static const double PI = 3.14159265358979323846264338327950288;
static const double TWOPI = 2.0 * PI;
static const double SQRT2 = 1.41421356237309504880168872420969808;

static void cpy(char *dst, size_t n, const std::string &s)
{
    std::snprintf(dst, n, "%s", s.c_str());
}

static std::string lower(std::string s)
{
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

static std::string trim(const std::string &s)
{
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

void params_default(hydft_params *p)
{
    std::memset(p, 0, sizeof(*p));
    p->nx = 64; p->ny = 1; p->nz = 1;
    p->lx = 20.0; p->ly = 1.0; p->lz = 1.0;
    p->dealias = 1;
    cpy(p->kind, sizeof(p->kind), "ion");
    p->gamma = 2.0; p->kappa = 0.1; p->rs = 1.86; p->theta = -1.0; p->mass = 1.0;
    cpy(p->terms, sizeof(p->terms), "");
    p->tfk_gamma = 1.0 / 9.0;
    cpy(p->closure, sizeof(p->closure), "newtonian");
    cpy(p->transport, sizeof(p->transport), "constant");
    p->eta = 0.0; p->xi = 0.0; p->tau = 0.0;
    cpy(p->tau_model, sizeof(p->tau_model), "ichimaru");
    p->adiabatic_index = 5.0 / 3.0;
    cpy(p->structure, sizeof(p->structure), "hnc");
    cpy(p->structure_kind, sizeof(p->structure_kind), "s");
    p->hnc_nr = 8192; p->hnc_maxiter = 20000;
    p->hnc_rmax = 80.0; p->hnc_tol = 1.0e-9; p->hnc_mix = 0.2;
    p->dt = 0.0; p->cfl = 0.4; p->tend = 50.0;
    p->nsteps_max = 10000000; p->iout = 0; p->iprobe = 1; p->idiag = 10;
    cpy(p->ic, sizeof(p->ic), "mode");
    p->ic_amplitude = 1.0e-4;
    p->ic_mode[0] = 1; p->ic_mode[1] = 0; p->ic_mode[2] = 0;
    p->ic_width = 1.0;
    p->ic_seed = 1234;
    cpy(p->vext, sizeof(p->vext), "none");
    p->vext_amplitude = 0.0;
    p->vext_mode[0] = 1; p->vext_mode[1] = 0; p->vext_mode[2] = 0;
    p->vext_omega = 0.0; p->vext_width = 1.0; p->vext_ramp = 0.0;
    p->probe_mode[0] = 1; p->probe_mode[1] = 0; p->probe_mode[2] = 0;
    cpy(p->prefix, sizeof(p->prefix), "out");
    cpy(p->gpu_precision, sizeof(p->gpu_precision), "fp64");
}

// params.f90:161-172
void params_finalize(hydft_params *p)
{
    auto lw = [](char *s, size_t n) { std::string t = lower(trim(s)); cpy(s, n, t); };
    lw(p->kind, sizeof(p->kind));
    lw(p->terms, sizeof(p->terms));
    lw(p->closure, sizeof(p->closure));
    lw(p->transport, sizeof(p->transport));
    lw(p->tau_model, sizeof(p->tau_model));
    lw(p->structure, sizeof(p->structure));
    lw(p->structure_kind, sizeof(p->structure_kind));
    lw(p->ic, sizeof(p->ic));
    lw(p->vext, sizeof(p->vext));
    lw(p->gpu_precision, sizeof(p->gpu_precision));
    if (std::strlen(p->terms) == 0) {
        if (std::string(p->kind) == "electron") cpy(p->terms, sizeof(p->terms), "tf,gradient,hartree,ry");
        else cpy(p->terms, sizeof(p->terms), "ideal,hartree,ry");
    }
    if (std::string(p->kind) == "electron" && p->theta > 0.0)
        p->gamma = 2.0 * p->rs / (p->theta * std::pow(9.0 * PI / 4.0, 2.0 / 3.0));
    if (std::string(p->kind) == "electron") p->kappa = 0.0;
}

// ------------------------------------------------------------- namelists
// A Fortran namelist subset: &group key=value[, value...] ... /  with
// quoted strings, .true./.false./T/F logicals and ! comments.
namespace {

struct Tok {
    std::string key;
    std::vector<std::string> vals;
};

std::string strip_comments(const std::string &s)
{
    std::string out;
    char q = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        char c = s[i];
        if (q) {
            out += c;
            if (c == q) q = 0;
        } else if (c == '\'' || c == '"') {
            q = c;
            out += c;
        } else if (c == '!') {
            while (i < s.size() && s[i] != '\n') ++i;
            out += '\n';
        } else {
            out += c;
        }
    }
    return out;
}

// group name -> body text (between &name and the terminating / or &end)
bool find_group(const std::string &text, const std::string &name, std::string &body)
{
    const std::string lt = lower(text);
    size_t pos = 0;
    while ((pos = lt.find('&', pos)) != std::string::npos) {
        size_t e = pos + 1;
        while (e < lt.size() && (std::isalnum((unsigned char)lt[e]) || lt[e] == '_')) ++e;
        if (lt.substr(pos + 1, e - pos - 1) == name) {
            char q = 0;
            size_t i = e;
            for (; i < text.size(); ++i) {
                char c = text[i];
                if (q) { if (c == q) q = 0; continue; }
                if (c == '\'' || c == '"') { q = c; continue; }
                if (c == '/') break;
                if (c == '&' && lt.compare(i, 4, "&end") == 0) break;
            }
            body = text.substr(e, i - e);
            return true;
        }
        pos = e;
    }
    return false;
}

bool parse_body(const std::string &body, std::vector<Tok> &out, std::string &err)
{
    // split into tokens: key = v1, v2 ...
    std::vector<std::string> items;
    std::string cur;
    char q = 0;
    for (char c : body) {
        if (q) { cur += c; if (c == q) q = 0; continue; }
        if (c == '\'' || c == '"') { q = c; cur += c; continue; }
        if (c == ',' || std::isspace((unsigned char)c)) {
            if (!cur.empty()) { items.push_back(cur); cur.clear(); }
            continue;
        }
        if (c == '=') {
            if (!cur.empty()) { items.push_back(cur); cur.clear(); }
            items.push_back("=");
            continue;
        }
        cur += c;
    }
    if (!cur.empty()) items.push_back(cur);
    for (size_t i = 0; i < items.size(); ++i) {
        if (i + 1 < items.size() && items[i + 1] == "=") {
            Tok t;
            t.key = lower(items[i]);
            // array element syntax key(2)= is not supported
            i += 2;
            while (i < items.size() && !(i + 1 < items.size() && items[i + 1] == "=")) {
                t.vals.push_back(items[i]);
                ++i;
            }
            --i;
            out.push_back(t);
        } else if (items[i] != "=") {
            err = "namelist: cannot parse '" + items[i] + "'";
            return false;
        }
    }
    return true;
}

std::string unq(const std::string &v)
{
    if (v.size() >= 2 && (v[0] == '\'' || v[0] == '"') && v.back() == v[0]) return v.substr(1, v.size() - 2);
    return v;
}

bool to_d(const std::string &v, double &d)
{
    std::string s = lower(v);
    for (auto &c : s) if (c == 'd') c = 'e';
    char *e = nullptr;
    d = std::strtod(s.c_str(), &e);
    return e && *e == 0;
}

bool to_i(const std::string &v, int &i)
{
    char *e = nullptr;
    long l = std::strtol(v.c_str(), &e, 10);
    i = (int)l;
    return e && *e == 0;
}

bool to_b(const std::string &v, int &b)
{
    std::string s = lower(unq(v));
    if (s == ".true." || s == "t" || s == ".t." || s == "true") { b = 1; return true; }
    if (s == ".false." || s == "f" || s == ".f." || s == "false") { b = 0; return true; }
    return false;
}

}  // namespace

int params_read(const char *path, hydft_params *p, std::string &err)
{
    std::ifstream f(path);
    if (!f) { err = std::string("cannot open file ") + path; return HYDFT_ERR_IO; }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = strip_comments(ss.str());
    struct Spec { const char *group; const char *key; char type; void *ptr; size_t n; };
    std::vector<Spec> specs = {
        {"grid", "nx", 'i', &p->nx, 1}, {"grid", "ny", 'i', &p->ny, 1}, {"grid", "nz", 'i', &p->nz, 1},
        {"grid", "lx", 'd', &p->lx, 1}, {"grid", "ly", 'd', &p->ly, 1}, {"grid", "lz", 'd', &p->lz, 1},
        {"grid", "dealias", 'b', &p->dealias, 1},
        {"species", "kind", 's', p->kind, sizeof(p->kind)}, {"species", "gamma", 'd', &p->gamma, 1},
        {"species", "kappa", 'd', &p->kappa, 1}, {"species", "rs", 'd', &p->rs, 1},
        {"species", "theta", 'd', &p->theta, 1}, {"species", "mass", 'd', &p->mass, 1},
        {"species", "terms", 's', p->terms, sizeof(p->terms)}, {"species", "tfk_gamma", 'd', &p->tfk_gamma, 1},
        {"species", "closure", 's', p->closure, sizeof(p->closure)},
        {"species", "transport", 's', p->transport, sizeof(p->transport)},
        {"species", "eta", 'd', &p->eta, 1}, {"species", "xi", 'd', &p->xi, 1}, {"species", "tau", 'd', &p->tau, 1},
        {"species", "tau_model", 's', p->tau_model, sizeof(p->tau_model)},
        {"species", "adiabatic_index", 'd', &p->adiabatic_index, 1},
        {"species", "structure", 's', p->structure, sizeof(p->structure)},
        {"species", "structure_file", 's', p->structure_file, sizeof(p->structure_file)},
        {"species", "structure_kind", 's', p->structure_kind, sizeof(p->structure_kind)},
        {"hnc", "nr", 'i', &p->hnc_nr, 1}, {"hnc", "rmax", 'd', &p->hnc_rmax, 1}, {"hnc", "tol", 'd', &p->hnc_tol, 1},
        {"hnc", "mix", 'd', &p->hnc_mix, 1}, {"hnc", "maxiter", 'i', &p->hnc_maxiter, 1},
        {"time", "dt", 'd', &p->dt, 1}, {"time", "cfl", 'd', &p->cfl, 1}, {"time", "tend", 'd', &p->tend, 1},
        {"time", "nsteps_max", 'i', &p->nsteps_max, 1}, {"time", "iout", 'i', &p->iout, 1},
        {"time", "iprobe", 'i', &p->iprobe, 1}, {"time", "idiag", 'i', &p->idiag, 1},
        {"initial", "type", 's', p->ic, sizeof(p->ic)}, {"initial", "amplitude", 'd', &p->ic_amplitude, 1},
        {"initial", "mode", 'I', p->ic_mode, 3}, {"initial", "width", 'd', &p->ic_width, 1},
        {"initial", "seed", 'i', &p->ic_seed, 1},
        {"external", "type", 's', p->vext, sizeof(p->vext)},
        {"external", "amplitude", 'd', &p->vext_amplitude, 1}, {"external", "mode", 'I', p->vext_mode, 3},
        {"external", "omega", 'd', &p->vext_omega, 1}, {"external", "width", 'd', &p->vext_width, 1},
        {"external", "ramp", 'd', &p->vext_ramp, 1},
        {"probe", "mode", 'I', p->probe_mode, 3},
        {"output", "prefix", 's', p->prefix, sizeof(p->prefix)},
        {"gpu", "precision", 's', p->gpu_precision, sizeof(p->gpu_precision)},
    };
    const char *groups[] = {"grid", "species", "hnc", "time", "initial", "external", "probe", "linear", "output", "gpu"};
    for (const char *gname : groups) {
        std::string body;
        if (!find_group(text, gname, body)) continue;   // absent namelist keeps the defaults
        std::vector<Tok> toks;
        if (!parse_body(body, toks, err)) {
            err = std::string("error reading namelist &") + gname + " in " + path + ": " + err;
            return HYDFT_ERR_BAD_ARG;
        }
        for (const Tok &t : toks) {
            bool found = false, ok = true;
            for (const Spec &s : specs) {
                if (std::strcmp(s.group, gname) || t.key != s.key) continue;
                found = true;
                if (t.vals.empty()) { ok = false; break; }
                switch (s.type) {
                case 'i': ok = to_i(t.vals[0], *(int *)s.ptr); break;
                case 'd': ok = to_d(t.vals[0], *(double *)s.ptr); break;
                case 'b': ok = to_b(t.vals[0], *(int *)s.ptr); break;
                case 's': cpy((char *)s.ptr, s.n, unq(t.vals[0])); break;
                case 'I':
                    for (size_t i = 0; i < s.n && i < t.vals.size(); ++i) ok = ok && to_i(t.vals[i], ((int *)s.ptr)[i]);
                    break;
                }
                break;
            }
            if (!std::strcmp(gname, "linear")) { found = true; ok = true; }   // &linear is read but unused here
            if (!found || !ok) {
                err = std::string("error reading namelist &") + gname + " in " + path + ": item '" + t.key + "'";
                return HYDFT_ERR_BAD_ARG;
            }
        }
    }
    params_finalize(p);
    return 0;
}

// ------------------------------------------------------ transport fits
static double sm_knm(int idx, double g)
{
    static const double A[4][5] = {{1.4660, -1.7836, 1.4313, -0.55833, 0.061162},
                                   {0.52094, 0.25153, -1.1337, 1.2155, -0.43784},
                                   {0.30346, 0.23739, -0.62167, 0.56110, -0.18046},
                                   {0.85401, -0.22898, -0.60059, 0.80591, -0.30555}};
    static const double B[4][5] = {{0.081033, -0.091336, 0.051760, -0.50026, 0.17044},
                                   {0.20572, -0.16536, 0.061572, -0.12770, 0.066993},
                                   {0.68375, -0.38459, 0.10711, 0.10649, 0.028760},
                                   {0.43475, -0.21147, 0.11116, 0.19665, 0.15195}};
    static const int NI[4] = {1, 1, 1, 2}, MI[4] = {1, 2, 3, 2};
    const int i = idx - 1;
    double fact = 1.0;
    for (int q = 2; q <= MI[i] - 1; ++q) fact *= q;
    if (g < 1.0) {
        double s = 0.0;
        const double gg = std::max(g, DBL_MIN);
        for (int q = 4; q >= 0; --q) s = (s + A[i][q]) * gg;
        return -0.25 * NI[i] * fact * std::log(s);
    }
    const double lg = std::log(g);
    return (B[i][0] + B[i][1] * lg + B[i][2] * lg * lg) / (1.0 + B[i][3] * g + B[i][4] * g * g);
}

static const double SQRT3PI = 3.0699801238394655;

// ------------------------------------------------------------ model setup
static bool fft_plan(int n, FFTPlan &p)
{
    p.L = n;
    p.nrad = 0;
    int m = n;
    while (m % 8 == 0 && p.nrad < MAX_RAD) { p.rad[p.nrad++] = 8; m /= 8; }
    while (m % 4 == 0 && p.nrad < MAX_RAD) { p.rad[p.nrad++] = 4; m /= 4; }
    while (m % 2 == 0 && p.nrad < MAX_RAD) { p.rad[p.nrad++] = 2; m /= 2; }
    while (m % 3 == 0 && p.nrad < MAX_RAD) { p.rad[p.nrad++] = 3; m /= 3; }
    return m == 1 && n <= MAX_L;
}

// largest kept |m| along one axis, evaluating the mask condition as grid.f90 does
static int band_limit(int n, double L, int dealias)
{
    if (n == 1) return 0;
    if (!dealias) return n / 2 - 1;
    const double kc = TWOPI * (n / 2) / L * (2.0 / 3.0);
    int M = 0;
    for (int m = 0; m <= n / 2; ++m)
        if (std::fabs(TWOPI * m / L) < kc) M = m;
    return M;
}

double footprint_bytes(const hydft_params *pin)
{
    hydft_params p = *pin;
    params_finalize(&p);
    if (p.nx < 2 || p.ny < 1 || p.nz < 1) return -1.0;
    const double b = std::string(p.gpu_precision) == "fp32" ? 4.0 : 8.0, cb = 2.0 * b;
    const int Mx = band_limit(p.nx, p.lx, p.dealias), My = band_limit(p.ny, p.ly, p.dealias),
              Mz = band_limit(p.nz, p.lz, p.dealias);
    const double pkx = (double)((Mx + 1 + 3) / 4 * 4), nkyc = 2.0 * My + 1, nkzc = 2.0 * Mz + 1;
    const double csize = nkzc * nkyc * pkx, zsize = (double)p.nz * nkyc * pkx, ysize = (double)p.nz * p.ny * pkx;
    const double ncell = (double)p.nx * p.ny * p.nz;
    const int nm = p.nz > 1 ? 3 : (p.ny > 1 ? 2 : 1);
    const bool grad = std::string(p.terms).find("gradient") != std::string::npos;
    const bool evolve = std::string(p.closure) == "maxwell";
    const int ninA = 1 + nm + (grad ? nm + 1 : 0), noutA = nm + nm * (nm + 1) / 2 + 1;
    const int ninB = nm + (evolve ? 6 * nm : 0), noutB = nm + (evolve ? 6 : 0);
    const int nin = std::max({ninA, ninB, 10}), nout = std::max({noutA, noutB, 10});
    double bytes = cb * (68.0 * csize + nin * zsize + (p.ny > 1 ? nin * ysize : 0.0) + nout * ysize) +
                   b * (14.0 * ncell + csize) + 8.0 * ncell;   // + the FP64 staging field
    const std::string terms = p.terms;
    if (terms.find("hartree") != std::string::npos) bytes += b * csize;   // v(k) for the energy
    if (terms.find("ry") != std::string::npos) bytes += b * csize;        // c_cor(k) for the energy
    if (std::string(p.vext) == "gaussian") bytes += b * 4.0 * ncell + cb * csize;
    if (std::string(p.kind) == "electron") bytes += 8.0 * 6 * 6601;
    bytes += 96.0 * 1024;   // twiddles, control block, reduction partials
    return bytes;
}

int build_setup(const hydft_params *pin, const hydft_structure *st_in, int device, ModelHost &mh, std::string &err)
{
    hydft_params p = *pin;
    params_finalize(&p);
    mh.p = p;
    const std::string kind = p.kind;
    if (kind != "ion" && kind != "electron") { err = "unknown species kind: " + kind; return HYDFT_ERR_BAD_ARG; }
    // grid.f90:45-48
    if (p.nx < 2) { err = "grid: nx must be >= 2"; return HYDFT_ERR_BAD_ARG; }
    if (p.nx % 2) { err = "grid: nx must be even"; return HYDFT_ERR_BAD_ARG; }
    if (p.ny > 1 && p.ny % 2) { err = "grid: ny must be even (or 1)"; return HYDFT_ERR_BAD_ARG; }
    if (p.nz > 1 && p.nz % 2) { err = "grid: nz must be even (or 1)"; return HYDFT_ERR_BAD_ARG; }
    if (p.ny < 1 || p.nz < 1) { err = "grid: ny and nz must be >= 1"; return HYDFT_ERR_BAD_ARG; }
    const std::string prec = p.gpu_precision;
    if (prec != "fp64" && prec != "fp32") { err = "gpu precision must be fp64 or fp32"; return HYDFT_ERR_BAD_ARG; }
    mh.precision = prec == "fp32" ? 32 : 64;

    SolverSetup &S = mh.S;
    Grid &g = S.g;
    std::memset(&g, 0, sizeof(g));
    g.nx = p.nx; g.ny = p.ny; g.nz = p.nz;
    g.ndim = p.nz > 1 ? 3 : (p.ny > 1 ? 2 : 1);
    if (!fft_plan(p.nx, g.px) || !fft_plan(p.ny, g.py) || !fft_plan(p.nz, g.pz)) {
        err = "grid sizes must be 2^a 3^b and at most 512 on the GPU path";
        return HYDFT_ERR_UNSUPPORTED;
    }
    g.Mx = band_limit(p.nx, p.lx, p.dealias);
    g.My = band_limit(p.ny, p.ly, p.dealias);
    g.Mz = band_limit(p.nz, p.lz, p.dealias);
    g.nkxc = g.Mx + 1;
    g.nkyc = 2 * g.My + 1;
    g.nkzc = 2 * g.Mz + 1;
    g.pkx = (g.nkxc + 3) / 4 * 4;
    g.kx0 = TWOPI / p.lx;
    g.ky0 = p.ny > 1 ? TWOPI / p.ly : 0.0;
    g.kz0 = p.nz > 1 ? TWOPI / p.lz : 0.0;
    g.dx = p.lx / p.nx; g.dy = p.ly / p.ny; g.dz = p.lz / p.nz;
    S.nm = g.ndim;
    double volume = p.lx;
    if (p.ny > 1) volume *= p.ly;
    if (p.nz > 1) volume *= p.lz;
    S.volume = volume;
    // kmax_dealiased (grid.f90:109): largest |k| in the band
    {
        double km = 0.0;
        for (int a = 0; a <= g.Mx; ++a)
            for (int b = -g.My; b <= g.My; ++b)
                for (int c = -g.Mz; c <= g.Mz; ++c) {
                    const double kx = TWOPI * a / p.lx, ky = p.ny > 1 ? TWOPI * b / p.ly : 0.0,
                                 kz = p.nz > 1 ? TWOPI * c / p.lz : 0.0;
                    km = std::max(km, std::sqrt(kx * kx + ky * ky + kz * kz));
                }
        mh.kmax_dealiased = km;
    }

    // units.f90:41-70
    const bool quantum = kind == "electron";
    mh.quantum = quantum;
    mh.n0 = 3.0 / (4.0 * PI);
    mh.e2 = 1.0 / 3.0;
    mh.gamma = p.gamma;
    mh.kappa = quantum ? 0.0 : p.kappa;
    mh.mass = p.mass;
    mh.beta = 3.0 * p.gamma;
    const double kT = 1.0 / mh.beta;
    if (quantum || std::string(p.terms).find("tf") != std::string::npos ||
        std::string(p.terms).find("gradient") != std::string::npos) {
        if (int rc = gpu_fd_table(device, mh.fdtab, err)) return rc;
    }
    if (quantum) {
        mh.hbar = 1.0 / std::sqrt(3.0 * p.rs);
        mh.cn = SQRT2 / (PI * PI * std::pow(mh.hbar, 3) * std::pow(mh.beta, 1.5)) * std::pow(mh.mass, 1.5);
        bool ok = true;
        mh.alpha0 = fd::alpha_from_ip12(mh.fdtab.data(), mh.n0 / mh.cn, &ok);
        const double tf = mh.hbar * mh.hbar * std::pow(3.0 * PI * PI * mh.n0, 2.0 / 3.0) / (2.0 * mh.mass);
        mh.theta = kT / tf;
        mh.lambda_qsp = 2.0 * std::sqrt(PI * p.gamma / p.rs);
        mh.lambda_tf = 1.0 / std::sqrt(4.0 * PI * mh.e2 * mh.beta * mh.cn * 0.5 * fd::im12(mh.fdtab.data(), mh.alpha0));
    } else {
        mh.hbar = 0.0;
        mh.theta = DBL_MAX;
        mh.lambda_tf = 1.0 / std::sqrt(3.0 * p.gamma);
    }

    // term list (species.f90:104-151)
    std::vector<std::string> terms;
    {
        std::string t = p.terms, item;
        std::stringstream ts(t);
        while (std::getline(ts, item, ',')) {
            item = trim(item);
            if (!item.empty()) terms.push_back(item);
        }
    }
    bool has_hartree = false, has_ry = false;
    for (auto &t : terms) {
        if (t == "hartree") has_hartree = true;
        if (t == "ry") has_ry = true;
        if (t != "ideal" && t != "tf" && t != "gradient" && t != "hartree" && t != "ry") {
            err = "unknown free-energy term: " + t;
            return HYDFT_ERR_UNSUPPORTED;
        }
        if ((t == "tf" || t == "gradient") && !quantum) { err = t + " term needs kind = electron"; return HYDFT_ERR_BAD_ARG; }
    }
    mh.terms = terms;

    // structure (species.f90:80-101)
    const bool maxwell = std::string(p.closure) == "maxwell";
    if (!maxwell && std::string(p.closure) != "newtonian") {
        err = std::string("unknown stress closure: ") + p.closure;
        return HYDFT_ERR_UNSUPPORTED;
    }
    const bool need_deriv = maxwell && std::string(p.tau_model) == "ichimaru";
    const std::string ssrc = p.structure;
    mh.has_st = false;
    if (st_in && st_in->n > 0) {
        mh.st_k.assign(st_in->k, st_in->k + st_in->n);
        mh.st_c.assign(st_in->c, st_in->c + st_in->n);
        mh.u_ex = st_in->u_ex;
        mh.du_dgamma = st_in->du_dgamma;
        mh.has_energy = st_in->has_energy != 0;
        mh.has_st = true;
    } else if (ssrc == "hnc") {
        if (has_ry || need_deriv) {
            Potential pot;
            if (quantum) { pot.kind = 2; pot.gamma = mh.gamma; pot.kappa = 0.0; pot.lambda = mh.lambda_qsp; }
            else { pot.kind = 0; pot.gamma = mh.gamma; pot.kappa = mh.kappa; pot.lambda = 1.0; }
            HncOut res;
            if (int rc = gpu_hnc_solve(device, pot, mh.n0, p.hnc_nr, p.hnc_rmax, p.hnc_tol, p.hnc_mix,
                                       p.hnc_maxiter, res, err)) return rc;
            if (!res.converged) { err = "structure: HNC did not converge"; return HYDFT_ERR_HNC; }
            mh.st_k = res.k;
            mh.st_c = res.ck;
            mh.u_ex = res.u_ex;
            mh.has_energy = true;
            mh.has_st = true;
            mh.hnc_niter = res.niter;
            if (need_deriv) {
                const double g0 = pot.gamma, dg = 0.02 * g0;
                HncOut rp1, rm1;
                pot.gamma = g0 + dg;
                if (int rc = gpu_hnc_solve(device, pot, mh.n0, p.hnc_nr, p.hnc_rmax, p.hnc_tol, p.hnc_mix,
                                           p.hnc_maxiter, rp1, err)) return rc;
                pot.gamma = g0 - dg;
                if (int rc = gpu_hnc_solve(device, pot, mh.n0, p.hnc_nr, p.hnc_rmax, p.hnc_tol, p.hnc_mix,
                                           p.hnc_maxiter, rm1, err)) return rc;
                if (!(rp1.converged && rm1.converged)) {
                    err = "structure: HNC derivative runs did not converge";
                    return HYDFT_ERR_HNC;
                }
                mh.du_dgamma = (rp1.u_ex - rm1.u_ex) / (2.0 * dg);
            }
        }
    } else if (ssrc == "file") {
        // structure_source.f90:87-138
        std::ifstream f(p.structure_file);
        if (!f) { err = std::string("cannot open file ") + p.structure_file; return HYDFT_ERR_IO; }
        std::string line;
        std::vector<double> kk, vv;
        while (std::getline(f, line)) {
            line = trim(line);
            if (line.empty() || line[0] == '#') continue;
            std::stringstream ls(line);
            double a, b;
            if (ls >> a >> b) { kk.push_back(a); vv.push_back(b); }
        }
        if (kk.size() < 2) { err = std::string("structure file has fewer than two data rows: ") + p.structure_file; return HYDFT_ERR_BAD_ARG; }
        const char sk = (char)std::tolower((unsigned char)p.structure_kind[0]);
        mh.st_k = kk;
        mh.st_c.resize(kk.size());
        for (size_t i = 0; i < kk.size(); ++i) {
            if (sk == 's') mh.st_c[i] = (1.0 - 1.0 / vv[i]) / mh.n0;
            else if (sk == 'c') mh.st_c[i] = vv[i];
            else { err = "structure file kind must be s or c"; return HYDFT_ERR_BAD_ARG; }
        }
        for (size_t i = 1; i < kk.size(); ++i)
            if (kk[i] <= kk[i - 1]) { err = "structure file: k must be strictly increasing"; return HYDFT_ERR_BAD_ARG; }
        if (kk[0] <= 0.0) { err = "structure file: k must be positive"; return HYDFT_ERR_BAD_ARG; }
        mh.has_st = true;
        mh.has_energy = false;
    } else if (ssrc != "none") {
        err = "unknown structure source: " + ssrc;
        return HYDFT_ERR_UNSUPPORTED;
    }
    if (has_ry && !mh.has_st) { err = "ry term needs a structure source (hnc or file)"; return HYDFT_ERR_BAD_ARG; }
    mh.ry_subtract = has_hartree;

    // cg of the gradient term (species.f90:127)
    mh.cg = p.tfk_gamma * (3.0 * SQRT2 * PI * PI / 8.0) * std::pow(mh.hbar, 5) * std::pow(mh.beta, 1.5) /
            std::pow(mh.mass, 2.5);

    // transport.f90:61-111
    const std::string tr = p.transport;
    if (tr == "constant") {
        mh.eta = p.eta;
        mh.xi = p.xi;
    } else if (tr == "yukawa_fit") {
        const double geff = mh.gamma * (1.0 + mh.kappa + 0.5 * mh.kappa * mh.kappa) * std::exp(-mh.kappa);
        mh.eta = 0.482 / (geff * geff) + 0.629 / std::pow(geff, 0.878) + 1.88e-3 * geff;
        mh.xi = p.xi;
    } else if (tr == "stanton_murillo") {
        if (quantum) { err = "transport = stanton_murillo is the ion (Yukawa) fit; use electron_fit for electrons"; return HYDFT_ERR_BAD_ARG; }
        const double gg = mh.gamma * std::sqrt(mh.kappa * mh.kappa + 3.0 * mh.gamma / (1.0 + 3.0 * mh.gamma));
        mh.eta = 5.0 * SQRT3PI / (36.0 * std::pow(mh.gamma, 2.5) * sm_knm(4, gg));
        mh.xi = p.xi;
    } else if (tr == "electron_fit") {
        if (!quantum) { err = "transport = electron_fit needs kind = electron"; return HYDFT_ERR_BAD_ARG; }
        const double rs = p.rs;
        const double cv = 1.0 / std::sqrt(3.0 * rs) /
                          (60.0 * std::pow(rs, -1.5) + 80.0 / rs - 40.0 * std::pow(rs, -2.0 / 3.0) + 62.0 * std::pow(rs, -1.0 / 3.0));
        const double sm = 5.0 * SQRT3PI / (36.0 * std::pow(mh.gamma, 2.5) * sm_knm(4, mh.gamma / mh.lambda_tf));
        const double el = 4.0 / 3.0 * (cv + mh.theta * sm) / (1.0 + mh.theta);
        mh.eta = 0.75 * el;
        mh.xi = 0.0;
    } else {
        err = "unknown transport model: " + tr;
        return HYDFT_ERR_UNSUPPORTED;
    }
    mh.eta_l = 4.0 * mh.eta / 3.0 + mh.xi;
    mh.tau = 0.0;
    if (maxwell) {
        const std::string tm = p.tau_model;
        if (tm == "constant") {
            mh.tau = p.tau;
        } else if (tm == "ichimaru") {
            if (!mh.has_energy) { err = "tau_model = ichimaru needs the HNC structure source (for E_c)"; return HYDFT_ERR_BAD_ARG; }
            const double u = mh.u_ex, du = mh.du_dgamma;
            const double muc = u / 3.0 + mh.gamma * du / 9.0;
            const double em = 1.0 - p.adiabatic_index * muc + 4.0 * u / 15.0;
            if (em <= 0.0) { err = "ichimaru tau: 1 - gamma mu + 4u/15 <= 0; use tau_model = constant"; return HYDFT_ERR_BAD_ARG; }
            mh.tau = 3.0 * mh.gamma * mh.eta_l / em;
        } else {
            err = "unknown tau model: " + tm;
            return HYDFT_ERR_UNSUPPORTED;
        }
    }
    // stress.f90:37-57
    mh.evolve = maxwell && mh.tau > 0.0;
    mh.s_tau = maxwell ? mh.tau : 0.0;
    mh.s_eta = mh.eta * mh.n0;
    mh.s_xi = mh.xi * mh.n0;

    // solver constants
    S.beta = mh.beta;
    S.mass = mh.mass;
    S.n0 = mh.n0;
    S.nterms_local = 0;
    for (auto &t : terms) {
        if (t == "ideal") S.term_order[S.nterms_local++] = 1;
        else if (t == "tf") S.term_order[S.nterms_local++] = 2;
        else if (t == "gradient") S.term_order[S.nterms_local++] = 3;
    }
    S.cn = mh.cn;
    S.cg = mh.cg;
    S.alpha_ref = mh.alpha0;
    S.evolve = mh.evolve;
    S.newtonian = !mh.evolve;
    S.eta = mh.s_eta;
    S.xi = mh.s_xi;
    S.tau = mh.s_tau;
    if (!mh.fdtab.empty()) S.fdtab = mh.fdtab;

    // spectral mu kernels on the compact band: hartree v(k), RY -c_cor(k)/beta
    const size_t csize = (size_t)g.nkzc * g.nkyc * g.pkx;
    S.klin.assign(csize, 0.0);
    for (int kzc = 0; kzc < g.nkzc; ++kzc)
        for (int kyc = 0; kyc < g.nkyc; ++kyc)
            for (int kxc = 0; kxc < g.nkxc; ++kxc) {
                const int my = signed_idx(kyc, g.My), mz = signed_idx(kzc, g.Mz);
                const double kx = TWOPI * kxc / p.lx;
                const double ky = p.ny > 1 ? TWOPI * my / p.ly : 0.0;
                const double kz = p.nz > 1 ? TWOPI * mz / p.lz : 0.0;
                const double kabs = std::sqrt(kx * kx + ky * ky + kz * kz);
                double v = 0.0;
                for (auto &t : terms) {
                    if (t == "hartree") v += mh.hartree_kernel(kabs);
                    if (t == "ry") v += -mh.c_cor(kabs) / mh.beta;
                }
                S.klin[((size_t)kzc * g.nkyc + kyc) * g.pkx + kxc] = v;
            }

    // free-energy terms in input order and the hartree / RY kernels apart
    S.neterms = 0;
    for (auto &t : terms) {
        int id = 0;
        if (t == "ideal") id = 1;
        else if (t == "tf") id = 2;
        else if (t == "gradient") id = 3;
        else if (t == "hartree") id = 4;
        else if (t == "ry") id = 5;
        if (id && S.neterms < 8) S.eterm_order[S.neterms++] = id;
    }
    {
        bool hh = false, rr = false;
        for (auto &t : terms) {
            hh = hh || t == "hartree";
            rr = rr || t == "ry";
        }
        if (hh) S.kh.assign(csize, 0.0);
        if (rr) S.kr.assign(csize, 0.0);
        S.vk0 = hh ? mh.hartree_kernel(0.0) : 0.0;
        S.ck0 = rr ? mh.c_cor(0.0) : 0.0;
        if (hh || rr)
            for (int kzc = 0; kzc < g.nkzc; ++kzc)
                for (int kyc = 0; kyc < g.nkyc; ++kyc)
                    for (int kxc = 0; kxc < g.nkxc; ++kxc) {
                        const int my = signed_idx(kyc, g.My), mz = signed_idx(kzc, g.Mz);
                        const double kx = TWOPI * kxc / p.lx;
                        const double ky = p.ny > 1 ? TWOPI * my / p.ly : 0.0;
                        const double kz = p.nz > 1 ? TWOPI * mz / p.lz : 0.0;
                        const double kabs = std::sqrt(kx * kx + ky * ky + kz * kz);
                        const size_t q = ((size_t)kzc * g.nkyc + kyc) * g.pkx + kxc;
                        if (hh) S.kh[q] = mh.hartree_kernel(kabs);
                        if (rr) S.kr[q] = mh.c_cor(kabs);
                    }
    }

    // external potential (external_potential.f90:39-63)
    const std::string vx = p.vext;
    S.ext_active = 0;
    if (vx == "none") {
    } else if (vx == "mode" || vx == "driven" || vx == "gaussian") {
        S.ext_active = 1;
        S.ext_kind = vx == "mode" ? 1 : (vx == "driven" ? 2 : 3);
        S.ext_td = vx == "driven";
    } else {
        err = "unknown external potential: " + vx;
        return HYDFT_ERR_UNSUPPORTED;
    }
    if (S.ext_kind == 3) {
        // v = -A exp(-r^2 / (2 w^2)) about the box centre (external_potential.f90:81-91)
        const size_t nc = (size_t)p.nx * p.ny * p.nz;
        S.gauss_v.assign(nc, 0.0);
        const double w2 = p.vext_width * p.vext_width;
        for (int k = 0; k < p.nz; ++k)
            for (int j = 0; j < p.ny; ++j)
                for (int i = 0; i < p.nx; ++i) {
                    const double x = i * (p.lx / p.nx) - 0.5 * p.lx;
                    const double y = p.ny > 1 ? j * (p.ly / p.ny) - 0.5 * p.ly : 0.0;
                    const double z = p.nz > 1 ? k * (p.lz / p.nz) - 0.5 * p.lz : 0.0;
                    const double r2 = x * x + y * y + z * z;
                    S.gauss_v[i + (size_t)p.nx * (j + (size_t)p.ny * k)] = -p.vext_amplitude * std::exp(-0.5 * r2 / w2);
                }
    }
    S.ext_k[0] = TWOPI * p.vext_mode[0] / p.lx;
    S.ext_k[1] = p.ny > 1 ? TWOPI * p.vext_mode[1] / p.ly : 0.0;
    S.ext_k[2] = p.nz > 1 ? TWOPI * p.vext_mode[2] / p.lz : 0.0;
    S.ext_amp = p.vext_amplitude;
    S.ext_omega = p.vext_omega;
    S.ext_ramp = p.vext_ramp;
    mh.ext_omega = p.vext_omega;
    S.ex.resize(p.nx); S.ey.resize(p.ny); S.ez.resize(p.nz);
    for (int i = 0; i < p.nx; ++i) S.ex[i] = std::polar(1.0, S.ext_k[0] * (i * (p.lx / p.nx)));
    for (int j = 0; j < p.ny; ++j) S.ey[j] = std::polar(1.0, S.ext_k[1] * (j * (p.ly / p.ny)));
    for (int k = 0; k < p.nz; ++k) S.ez[k] = std::polar(1.0, S.ext_k[2] * (k * (p.lz / p.nz)));
    // compact index of the drive mode (for the mean of n F_ext)
    {
        int mx = p.vext_mode[0], my = p.ny > 1 ? p.vext_mode[1] : 0, mz = p.nz > 1 ? p.vext_mode[2] : 0;
        int conj = 0;
        if (mx < 0) { mx = -mx; my = -my; mz = -mz; conj = 1; }
        S.drive_conj = conj;
        S.drive_in_band = mx <= g.Mx && std::abs(my) <= g.My && std::abs(mz) <= g.Mz;
        if (S.drive_in_band) {
            const int kyc = my >= 0 ? my : my + g.nkyc, kzc = mz >= 0 ? mz : mz + g.nkzc;
            S.drive_idx = (int)(((size_t)kzc * g.nkyc + kyc) * g.pkx + mx);
        }
    }

    // compute_dt constants (model.f90:159-170): omega_max over the band
    {
        double wmax = 0.0;
        for (int kzc = 0; kzc < g.nkzc; ++kzc)
            for (int kyc = 0; kyc < g.nkyc; ++kyc)
                for (int kxc = 0; kxc < g.nkxc; ++kxc) {
                    const int my = signed_idx(kyc, g.My), mz = signed_idx(kzc, g.Mz);
                    const double kx = TWOPI * kxc / p.lx;
                    const double ky = p.ny > 1 ? TWOPI * my / p.ly : 0.0;
                    const double kz = p.nz > 1 ? TWOPI * mz / p.lz : 0.0;
                    const double k = std::sqrt(kx * kx + ky * ky + kz * kz);
                    if (k == 0.0) continue;
                    double c2 = mh.n0 * mh.kernel(k) / mh.mass;
                    if (mh.evolve) c2 += mh.eta_l / (mh.mass * mh.s_tau);
                    wmax = std::max(wmax, std::sqrt(k * k * std::max(c2, 0.0)));
                }
        mh.wmax = wmax;
        mh.numax = mh.evolve ? 0.0 : mh.eta_l / mh.mass * mh.kmax_dealiased * mh.kmax_dealiased;
        mh.dxmin = g.dx;
        if (p.ny > 1) mh.dxmin = std::min(mh.dxmin, g.dy);
        if (p.nz > 1) mh.dxmin = std::min(mh.dxmin, g.dz);
    }
    return 0;
}

// fe_hartree.f90:56-64
double ModelHost::hartree_kernel(double k) const
{
    if (k * k + kappa * kappa > 0.0) return 4.0 * PI * e2 / (k * k + kappa * kappa);
    return 0.0;
}

// utils.f90:30-55, structure_source.f90:37-41
double ModelHost::c_of_k(double k) const
{
    const int n = (int)st_k.size();
    const double xq = std::min(k, st_k[n - 1]);
    if (n == 1) return st_c[0];
    int lo;
    if (xq <= st_k[0]) lo = 0;
    else if (xq >= st_k[n - 1]) lo = n - 2;
    else {
        lo = (int)(std::upper_bound(st_k.begin(), st_k.end(), xq) - st_k.begin()) - 1;
        lo = std::min(std::max(lo, 0), n - 2);
    }
    const double w = (xq - st_k[lo]) / (st_k[lo + 1] - st_k[lo]);
    return (1.0 - w) * st_c[lo] + w * st_c[lo + 1];
}

// fe_correlation_ry.f90:39-49
double ModelHost::c_cor(double k) const
{
    const double k1 = std::max(k, st_k[0]);
    double c = c_of_k(k1);
    if (ry_subtract) c += beta * 4.0 * PI * e2 / (k1 * k1 + kappa * kappa);
    return c;
}

// functional.f90:72-80 with the terms' kernels
double ModelHost::kernel(double k) const
{
    double kk = 0.0;
    for (auto &t : terms) {
        if (t == "ideal") kk += 1.0 / (beta * n0);
        else if (t == "tf") kk += 2.0 / (beta * cn * fd::im12(fdtab.data(), alpha0));
        else if (t == "gradient") kk += 2.0 * cg * fd::xi(fdtab.data(), alpha0) * k * k;
        else if (t == "hartree") kk += hartree_kernel(k);
        else if (t == "ry") kk += -c_cor(k) / beta;
    }
    return kk;
}

}  // namespace hydft
