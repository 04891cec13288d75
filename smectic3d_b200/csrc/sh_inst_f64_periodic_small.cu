// Solver instantiations: double, periodic boundary, N = 16, 32, 64.
#include "sh_inst.cuh"
SHB_INST_UNIT(f64, periodic, double, false, 16)
SHB_INST_UNIT(f64, periodic, double, false, 32)
SHB_INST_UNIT(f64, periodic, double, false, 64)
