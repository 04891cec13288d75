// Solver instantiations: double, neumann boundary, N = 128.
#include "sh_inst.cuh"
SHB_INST_UNIT(f64, neumann, double, true, 128)
