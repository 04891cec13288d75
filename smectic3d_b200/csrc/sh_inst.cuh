// Instantiation of the solver for every supported grid size.  Included by one
// translation unit per (precision, boundary) so that they compile in parallel.
#pragma once
#include "sh_solver.cuh"

namespace shb {

// Default cluster size CL of the plane pass (NC = N / (2 CL) column lines per
// CTA); ``variant`` selects another built CL for the same N (0 = default).
template <int N> constexpr int cluster_for() {
  return N <= 64 ? 1 : (N == 128 ? 2 : (N == 256 ? 4 : 16));
}

template <typename T, bool DCT>
SolverBase* make_solver(int n, int variant) {
  const int cl = variant ? variant : 0;
  switch (n) {
    case 16: return cl == 0 || cl == 1 ? new Solver<T, 16, 1, DCT>() : nullptr;
    case 32: return cl == 0 || cl == 1 ? new Solver<T, 32, 1, DCT>() : nullptr;
    case 64:
      if (cl == 0 || cl == 1) return new Solver<T, 64, 1, DCT>();
      if (cl == 2) return new Solver<T, 64, 2, DCT>();
      return nullptr;
    case 128:
      if (cl == 0 || cl == 2) return new Solver<T, 128, 2, DCT>();
      if (cl == 1) return new Solver<T, 128, 1, DCT>();
      if (cl == 4) return new Solver<T, 128, 4, DCT>();
      return nullptr;
    case 256:
      if (cl == 0 || cl == 4) return new Solver<T, 256, 4, DCT>();
      if (cl == 8) return new Solver<T, 256, 8, DCT>();
      if (cl == 16) return new Solver<T, 256, 16, DCT>();
      return nullptr;
#ifdef SHB_WITH_512
    case 512:
      if (cl == 0 || cl == 16) return new Solver<T, 512, 16, DCT>();
      if constexpr (sizeof(T) == 4) {
        if (cl == 8) return new Solver<T, 512, 8, DCT>();
      }
      return nullptr;
#endif
    default: return nullptr;
  }
}

}  // namespace shb
