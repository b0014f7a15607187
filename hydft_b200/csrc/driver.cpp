// The reference's run loop and field files, over the GPU model.
//
// hydft_gpu_run follows hydft_run (src/hydft.f90:30-60): dt from compute_dt
// every 20 steps, the last step shortened to end at tend, probes every
// iprobe steps, budgets every idiag steps, fields every iout steps, into
// <prefix>_probe.dat, <prefix>_diag.dat and <prefix>_fld_NNNNNN.bin in the
// reference's formats (diagnostics.f90:32-77, io.f90:19-35).  The steps
// between two host events (a dt update, a budget line, a field file, the
// last step before tend) run back to back as graph replays; the probes of
// those steps are recorded on the device and written at the next event, so
// the loop does not wait for the device every step.
//
// hydft_gpu_write_fields / hydft_gpu_read_fields write and read the .bin
// field files (read: resume from one, with the step number taken from the
// file name).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydft_gpu.h"
#include "handle.hpp"

using namespace hydft;

namespace {

int fail(hydft_gpu *h, int rc, const std::string &msg)
{
    h->err = msg;
    return rc;
}

// Fortran ESw.dEe edit descriptor (w = 18, d = 9, e = 3): one leading
// digit, d decimals, an exponent of e digits, right-justified in w
std::string es(double v, int w = 18, int d = 9, int e = 3)
{
    char buf[64];
    if (!std::isfinite(v)) {
        std::snprintf(buf, sizeof buf, "%*s", w, std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
        return buf;
    }
    char m[48];
    std::snprintf(m, sizeof m, "%.*E", d, v);   // d.dddE+xx
    std::string s(m);
    const size_t p = s.find('E');
    std::string mant = s.substr(0, p);
    int ex = std::atoi(s.c_str() + p + 1);
    char tail[16];
    std::snprintf(tail, sizeof tail, "E%c%0*d", ex < 0 ? '-' : '+', e, std::abs(ex));
    std::snprintf(buf, sizeof buf, "%*s", w, (mant + tail).c_str());
    return buf;
}

struct Files {
    FILE *diag = nullptr, *probe = nullptr;
    ~Files()
    {
        if (diag) std::fclose(diag);
        if (probe) std::fclose(probe);
    }
};

// diag_write: step t dt mass mom(3) E_kin F E_tot n_min n_max
int write_diag(hydft_gpu *h, FILE *f)
{
    double t, dt, mass, mom[3], ekin, fe, nmin, nmax;
    int64_t step;
    h->s->get_time(&t, &dt, &step);
    int rc = hydft_gpu_budgets(h, &mass, mom, &ekin, &fe, &nmin, &nmax);
    if (rc) return rc;
    std::fprintf(f, "%9lld%s%s%s%s%s%s%s%s%s%s%s\n", (long long)step, es(t).c_str(), es(dt).c_str(),
                 es(mass).c_str(), es(mom[0]).c_str(), es(mom[1]).c_str(), es(mom[2]).c_str(), es(ekin).c_str(),
                 es(fe).c_str(), es(ekin + fe).c_str(), es(nmin).c_str(), es(nmax).c_str());
    return HYDFT_OK;
}

// diag_probe: t Re(a) Im(a) |a| Re(b) Im(b), a = n_k / n0, b = mom_x,k
void write_probe(FILE *f, double t, double nr, double ni, double mr, double mi, double n0)
{
    const double ar = nr / n0, ai = ni / n0;
    std::fprintf(f, "%s%s%s%s%s%s\n", es(t).c_str(), es(ar).c_str(), es(ai).c_str(), es(std::hypot(ar, ai)).c_str(),
                 es(mr).c_str(), es(mi).c_str());
}

}  // namespace

extern "C" {

int hydft_gpu_write_fields(hydft_gpu *h, const char *prefix)
{
    if (!h || !prefix) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    const hydft_params &p = h->mh.p;
    const size_t nc = (size_t)p.nx * p.ny * p.nz;
    const bool evolve = h->s->setup().evolve != 0;
    std::vector<double> n(nc), mom(3 * nc), pi(evolve ? 6 * nc : 0);
    int rc = hydft_gpu_get_state(h, n.data(), mom.data(), evolve ? pi.data() : nullptr);
    if (rc) return rc;
    double t, dt;
    int64_t step;
    h->s->get_time(&t, &dt, &step);
    char name[600];
    std::snprintf(name, sizeof name, "%s_fld_%06lld.bin", prefix, (long long)step);
    FILE *f = std::fopen(name, "wb");
    if (!f) return fail(h, HYDFT_ERR_IO, std::string("cannot write ") + name);
    const int32_t hdr[5] = {p.nx, p.ny, p.nz, h->mh.S.g.ndim, evolve ? 6 : 0};
    const double hd[4] = {t, p.lx, p.ly, p.lz};
    bool ok = std::fwrite(hdr, sizeof(int32_t), 5, f) == 5 && std::fwrite(hd, sizeof(double), 4, f) == 4 &&
              std::fwrite(n.data(), sizeof(double), nc, f) == nc &&
              std::fwrite(mom.data(), sizeof(double), 3 * nc, f) == 3 * nc;
    if (ok && evolve) ok = std::fwrite(pi.data(), sizeof(double), 6 * nc, f) == 6 * nc;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(h, HYDFT_ERR_IO, std::string("cannot write ") + name);
    return HYDFT_OK;
}

int hydft_gpu_read_fields(hydft_gpu *h, const char *path)
{
    if (!h || !path) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    const hydft_params &p = h->mh.p;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(h, HYDFT_ERR_IO, std::string("cannot open ") + path);
    int32_t hdr[5];
    double hd[4];
    if (std::fread(hdr, sizeof(int32_t), 5, f) != 5 || std::fread(hd, sizeof(double), 4, f) != 4) {
        std::fclose(f);
        return fail(h, HYDFT_ERR_IO, std::string("truncated field file ") + path);
    }
    if (hdr[0] != p.nx || hdr[1] != p.ny || hdr[2] != p.nz || hdr[3] != h->mh.S.g.ndim) {
        std::fclose(f);
        return fail(h, HYDFT_ERR_BAD_ARG, std::string("field file grid does not match the model: ") + path);
    }
    if (hdr[4] != 0 && hdr[4] != 6) {
        std::fclose(f);
        return fail(h, HYDFT_ERR_BAD_ARG, std::string("field file has an unknown Pi component count: ") + path);
    }
    const size_t nc = (size_t)p.nx * p.ny * p.nz;
    std::vector<double> n(nc), mom(3 * nc), pi(6 * nc, 0.0);
    bool ok = std::fread(n.data(), sizeof(double), nc, f) == nc && std::fread(mom.data(), sizeof(double), 3 * nc, f) == 3 * nc;
    if (ok && hdr[4] == 6) ok = std::fread(pi.data(), sizeof(double), 6 * nc, f) == 6 * nc;
    std::fclose(f);
    if (!ok) return fail(h, HYDFT_ERR_IO, std::string("truncated field file ") + path);
    const bool evolve = h->s->setup().evolve != 0;
    int rc = hydft_gpu_set_state(h, n.data(), mom.data(), evolve ? pi.data() : nullptr);
    if (rc) return rc;
    double t, dt;
    int64_t step;
    h->s->get_time(&t, &dt, &step);
    h->s->set_time(hd[0], dt);
    // <prefix>_fld_NNNNNN.bin: the step number of the file
    std::string s(path);
    const size_t k = s.rfind("_fld_");
    long long fstep = 0;
    if (k != std::string::npos && std::sscanf(s.c_str() + k + 5, "%lld", &fstep) == 1) h->s->set_step(fstep);
    return HYDFT_OK;
}

int hydft_gpu_run(hydft_gpu *h)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    const hydft_params &p = h->mh.p;
    const std::string prefix = p.prefix;
    Files fl;
    fl.diag = std::fopen((prefix + "_diag.dat").c_str(), "w");
    fl.probe = std::fopen((prefix + "_probe.dat").c_str(), "w");
    if (!fl.diag || !fl.probe) return fail(h, HYDFT_ERR_IO, "cannot open the output files of prefix " + prefix);
    std::fprintf(fl.diag, "# step   t   dt   mass   momx   momy   momz   E_kin   F   E_tot   n_min   n_max\n");
    std::fprintf(fl.probe, "# probe mode%4d%4d%4d:   t   Re(dn_k/n0)   Im(dn_k/n0)   |dn_k/n0|   Re(mom_k)   Im(mom_k)\n",
                 p.probe_mode[0], p.probe_mode[1], p.probe_mode[2]);
    const double n0 = h->mh.n0;
    int rc = h->s->probe_setup(p.probe_mode[0], p.probe_mode[1], p.probe_mode[2]);
    if (rc) return fail(h, rc, h->s->err);
    auto probe_now = [&]() -> int {
        double t, dt, nr, ni, mr, mi;
        int64_t step;
        h->s->get_time(&t, &dt, &step);
        int r = hydft_gpu_mode(h, 0, p.probe_mode[0], p.probe_mode[1], p.probe_mode[2], &nr, &ni);
        if (!r) r = hydft_gpu_mode(h, 1, p.probe_mode[0], p.probe_mode[1], p.probe_mode[2], &mr, &mi);
        if (!r) write_probe(fl.probe, t, nr, ni, mr, mi, n0);
        return r;
    };
    auto flush_probes = [&]() -> int {
        std::vector<double> rec;
        int r = h->s->read_probes(rec);
        if (r) return fail(h, r, h->s->err);
        for (size_t i = 0; i + 4 < rec.size(); i += 5) write_probe(fl.probe, rec[i], rec[i + 1], rec[i + 2], rec[i + 3], rec[i + 4], n0);
        return HYDFT_OK;
    };
    double dt = 0.0;
    if ((rc = hydft_gpu_compute_dt(h, &dt))) return rc;
    if ((rc = write_diag(h, fl.diag))) return rc;
    if ((rc = probe_now())) return rc;
    if (p.iout > 0 && (rc = hydft_gpu_write_fields(h, prefix.c_str()))) return rc;
    double t;
    int64_t step;
    h->s->get_time(&t, &dt, &step);
    const int iprobe = std::max(1, p.iprobe), idiag = std::max(1, p.idiag);
    int irecompute = 0;
    while (t < p.tend && step < p.nsteps_max) {
        if (irecompute == 0) {
            if ((rc = hydft_gpu_compute_dt(h, &dt))) return rc;
        }
        // the steps up to the next host event run back to back: the next dt
        // update, budget line, field file, the end, or a shortened last step
        int k = 0;
        double tk = t;
        for (;;) {
            if (tk + dt > p.tend) {
                if (k == 0) {   // this step ends exactly at tend
                    dt = p.tend - tk;
                    h->s->set_time(tk, dt);
                    k = 1;
                }
                break;
            }
            tk = tk + dt;
            ++k;
            const int64_t sk = step + k;
            const int irec = (irecompute + k) % 20;
            if (irec == 0 || sk % idiag == 0 || (p.iout > 0 && sk % p.iout == 0) || !(tk < p.tend) ||
                sk >= p.nsteps_max || k >= h->s->probe_capacity())
                break;
        }
        if ((rc = h->s->launch_steps_probed(k, iprobe))) return fail(h, rc, h->s->err);
        if ((rc = h->s->poll_status())) return fail(h, rc, h->s->err);
        irecompute = (irecompute + k) % 20;
        h->s->get_time(&t, &dt, &step);
        if ((rc = flush_probes())) return rc;
        if (step % idiag == 0 && (rc = write_diag(h, fl.diag))) return rc;
        if (p.iout > 0 && step % p.iout == 0 && (rc = hydft_gpu_write_fields(h, prefix.c_str()))) return rc;
    }
    if (step % idiag != 0 && (rc = write_diag(h, fl.diag))) return rc;
    return HYDFT_OK;
}

}  // extern "C"
