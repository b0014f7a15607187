// FP64 setup kernels on the GPU: Fermi-Dirac table and inverse, OZ-HNC.
#pragma once

#include <string>
#include <vector>

namespace hydft {

// pair potential (pair_potential.f90): kind 0 yukawa, 1 coulomb, 2 hansen-mcdonald
struct Potential {
    int kind = 0;
    double gamma = 1.0, kappa = 0.0, ksplit = 1.0, lambda = 1.0;
    int pauli = 1;
};

struct HncOut {
    int nr = 0;
    std::vector<double> r, k, g, ck, sk;
    double u_ex = 0.0;
    bool converged = false;
    int niter = 0;
    double residual = 0.0;
};

void gauss_legendre(int n, double *x, double *w);
int gpu_fd_table(int device, std::vector<double> &out, std::string &err);
int gpu_fd_alpha(int device, const std::vector<double> &tab, const double *y, double *alpha, int n,
                 std::string &err);
int gpu_fourier_bessel(int device, const double *fin, double *fout, int n, double rmax, int direction,
                       std::string &err);
int gpu_hnc_solve(int device, const Potential &pot, double n0, int nr, double rmax, double tol, double mix,
                  int maxiter, HncOut &res, std::string &err);

}  // namespace hydft
