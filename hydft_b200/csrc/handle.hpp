// The simulation handle behind the C ABI (hydft_gpu in include/hydft_gpu.h),
// shared by the single-model entry points and the ensemble.
#pragma once

#include <string>

#include "setup.hpp"
#include "solver.hpp"

struct hydft_gpu {
    hydft::ModelHost mh;
    hydft::SolverBase *s = nullptr;
    int device = 0;
    bool owned_by_batch = false;   // members of an ensemble are destroyed with it
    std::string err;
};

namespace hydft {
// message of a failed handle-less call, returned by hydft_gpu_create_error()
void set_thread_error(const std::string &msg);
}  // namespace hydft
