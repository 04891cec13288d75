// Solver instantiations: float, neumann boundary.
#include "sh_inst.cuh"
namespace shb {
SolverBase* make_solver_f32_neumann(int n) { return make_solver<float, true>(n); }
}  // namespace shb
