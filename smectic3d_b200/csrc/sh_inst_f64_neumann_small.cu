// Solver instantiations: double, neumann boundary, N = 16, 32, 64.
#include "sh_inst.cuh"
SHB_INST_UNIT(f64, neumann, double, true, 16)
SHB_INST_UNIT(f64, neumann, double, true, 32)
SHB_INST_UNIT(f64, neumann, double, true, 64)
