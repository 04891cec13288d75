// Solver instantiations: double, periodic boundary.
#include "sh_inst.cuh"
namespace shb {
SolverBase* make_solver_f64_periodic(int n) { return make_solver<double, false>(n); }
}  // namespace shb
