// Solver instantiations: float, neumann boundary.
#include "sh_inst.cuh"
namespace shb {
SolverBase* make_solver_f32_neumann(int n, int variant) { return make_solver<float, true>(n, variant); }
}  // namespace shb
