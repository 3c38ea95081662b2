// C++ twin of DerivativeTests.ElastostaticResidual3D / InternalElasticEnergy3D
// (unit_tests/DerivativeTests.cpp:273-700) through include/pa_b200.hpp.
// Reads the mesh (C, N, cells, coords) from the file given as argv[1], sets
// u_i = 1e-4 (i+1), z = 1, E = 1e6, nu = 0.3, SIMP p = 1, min 0, and prints
// the residual, the compliance and its control gradient, one number per line.
#include <cstdio>
#include <fstream>
#include <vector>

#include "pa_b200.hpp"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::ifstream in(argv[1]);
  int64_t C = 0, N = 0;
  in >> C >> N;
  std::vector<int32_t> cells(4 * C);
  std::vector<double> coords(3 * N);
  for (auto& c : cells) in >> c;
  for (auto& x : coords) in >> x;
  try {
    pa_b200::Mesh mesh(cells.data(), C, coords.data(), N);
    pa_elastic_params prm{1.0e6, 0.3, 1.0, 0.0, PA_CONTROL_NODAL};
    pa_b200::Problem problem(mesh, prm);
    std::vector<double> u(3 * N), z(N, 1.0), r(3 * N), gz(N);
    for (int64_t i = 0; i < 3 * N; ++i) u[i] = 1e-4 * double(i + 1);
    problem.vectorFunction().value(u.data(), z.data(), r.data());
    const double f = problem.criterionValue(z.data(), u.data());
    problem.criterion().gradient_z(u.data(), z.data(), gz.data());
    for (double v : r) std::printf("%.17g\n", v);
    std::printf("%.17g\n", f);
    for (double v : gz) std::printf("%.17g\n", v);
  } catch (const pa_b200::Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
