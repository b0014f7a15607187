// Solver instantiation in FP64.
#define HYDFT_REAL double
#define HYDFT_MAKE_FN make_solver_f64
#include "solver_impl.cuh"
