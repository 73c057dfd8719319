// Multi-tissue CSD's solver through the ICLS drop-in: the caller builds the
// forward matrix C and the constraint matrix A (as MSMT_CSD::Shared::init
// does, msmt_csd.h:90-204), then solves every voxel of a volume at once.
//   g++ -std=c++17 -O2 -I include -I mrtrix3_b200/csrc -I /usr/local/cuda/include \
//       mrtrix3_b200/csrc/examples/icls_example.cpp -L mrtrix3_b200 -lcsd_b200 \
//       -L /usr/local/cuda/lib64 -lcudart -Wl,-rpath,$PWD/mrtrix3_b200 -o icls_example
#include <cstdio>
#include <vector>

#include "icls.hpp"

int main() {
  using namespace MR::Math::ICLS;
  // a 2-parameter non-negative least-squares problem, as a small stand-in
  const std::vector<double> H = {1.0, 0.0, 0.0, 1.0, 1.0, 1.0};  // [3][2]
  const std::vector<double> A = {1.0, 0.0, 0.0, 1.0};            // x >= 0
  Problem<double> problem(H, 3, 2, A, 2, {}, 0, 1e-10, 1e-10);
  Solver<double> solve(problem);
  std::vector<double> x;
  const size_t niter = solve(x, {1.0, -2.0, 0.5});
  std::printf("x = [%g %g] after %zu rounds\n", x[0], x[1], niter);
  // many voxels at once on host buffers
  const std::vector<float> b = {1.0f, -2.0f, 0.5f, 2.0f, 1.0f, 3.0f};
  std::vector<float> xs(4);
  std::vector<int32_t> it(2);
  solve.solve_batch(b.data(), 2, xs.data(), it.data());
  std::printf("voxel 1: [%g %g]\n", xs[2], xs[3]);
  return 0;
}
