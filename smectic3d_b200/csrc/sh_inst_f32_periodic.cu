// Solver instantiations: float, periodic boundary.
#include "sh_inst.cuh"
namespace shb {
SolverBase* make_solver_f32_periodic(int n, int variant) { return make_solver<float, false>(n, variant); }
}  // namespace shb
