// Solver instantiations: double, neumann boundary.
#include "sh_inst.cuh"
namespace shb {
SolverBase* make_solver_f64_neumann(int n, int variant) { return make_solver<double, true>(n, variant); }
}  // namespace shb
