// Solver instantiations: double, periodic boundary.
#include "sh_inst.cuh"
namespace shb {
SolverBase* make_solver_f64_periodic(int n, int variant) { return make_solver<double, false>(n, variant); }
}  // namespace shb
