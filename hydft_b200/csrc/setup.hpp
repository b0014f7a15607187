// Host-side model setup (units, structure, terms, transport, stress, grid).
#pragma once

#include <string>
#include <vector>

#include "../../include/hydft_gpu.h"
#include "solver.hpp"

namespace hydft {

// The setup-time state of model_t that stays on the host: scalars of
// units_t, transport_t and stress_t, the structure table and the term list.
struct ModelHost {
    hydft_params p;
    int precision = 64;
    bool quantum = false;
    double n0 = 0, e2 = 0, gamma = 0, kappa = 0, mass = 1, beta = 3;
    double hbar = 0, theta = 0, alpha0 = 0, cn = 0, lambda_qsp = 0, lambda_tf = 0, cg = 0;
    std::vector<std::string> terms;
    bool has_st = false, has_energy = false, ry_subtract = false;
    std::vector<double> st_k, st_c;
    double u_ex = 0, du_dgamma = 0;
    int hnc_niter = 0;
    double eta = 0, xi = 0, eta_l = 0, tau = 0;
    bool evolve = false;
    double s_tau = 0, s_eta = 0, s_xi = 0;
    double ext_omega = 0;
    double kmax_dealiased = 0, wmax = 0, numax = 0, dxmin = 1;
    std::vector<double> fdtab;
    SolverSetup S;

    double hartree_kernel(double k) const;
    double c_of_k(double k) const;
    double c_cor(double k) const;
    double kernel(double k) const;
};

void params_default(hydft_params *p);
void params_finalize(hydft_params *p);
int params_read(const char *path, hydft_params *p, std::string &err);
int build_setup(const hydft_params *p, const hydft_structure *st, int device, ModelHost &mh, std::string &err);
// device bytes a model of these parameters allocates (the solver's buffers,
// assuming Pi evolves whenever the closure is Maxwell); -1 if invalid
double footprint_bytes(const hydft_params *p);

}  // namespace hydft
