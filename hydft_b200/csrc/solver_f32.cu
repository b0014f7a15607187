// Solver instantiation in FP32.
#define HYDFT_REAL float
#define HYDFT_MAKE_FN make_solver_f32
#include "solver_impl.cuh"
