// Precision dispatch of the device solver.
#include "solver.hpp"

namespace hydft {

SolverBase *make_solver_f32(const SolverSetup &s, int device, std::string &err);
SolverBase *make_solver_f64(const SolverSetup &s, int device, std::string &err);

SolverBase *make_solver(const SolverSetup &s, int precision, int device, std::string &err)
{
    return precision == 32 ? make_solver_f32(s, device, err) : make_solver_f64(s, device, err);
}

}  // namespace hydft
