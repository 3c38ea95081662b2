// Drives include/pa_b200_app.hpp (the MPMD_App-shaped application) the way a
// Plato Engine stage sequence would: import "Topology", run named operations,
// export named values and fields.  Box nx x ny x nz of unit hexes (nodal
// controls read from argv[1], one per node), x = 0 clamped, unit total
// traction -z on x = nx.  Prints, one block per line group:
//   value of "Objective Value", then "Objective Gradient" (N), then
//   "Objective GradientX" (3N), "Shifted Value", "Solution Z" (N), and the
//   messages of two requests that must fail.
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "pa_b200_app.hpp"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const int nx = 6, ny = 3, nz = 3;
  const int64_t N = int64_t(nx + 1) * (ny + 1) * (nz + 1);
  std::vector<double> topo(N);
  std::ifstream in(argv[1]);
  for (auto& v : topo) in >> v;
  try {
    pa_b200::Mesh mesh = pa_b200::Mesh::box(nx, ny, nz, nx, ny, nz);
    pa_elastic_params prm{1.0, 0.3, 3.0, 1e-9, PA_CONTROL_NODAL};
    pa_b200::Problem problem(mesh, prm);
    int64_t nf = 0;
    pa_b200::check(pa_mesh_boundary_faces(mesh.handle(), 0, double(nx), nullptr, &nf), "faces");
    std::vector<int32_t> faces(3 * nf);
    pa_b200::check(pa_mesh_boundary_faces(mesh.handle(), 0, double(nx), faces.data(), &nf), "faces");
    const double flux[3] = {0.0, 0.0, -1.0 / (ny * nz)};
    problem.addTraction(faces, flux);
    std::vector<int32_t> dofs;
    std::vector<double> vals;
    for (int k = 0; k <= nz; ++k)
      for (int j = 0; j <= ny; ++j) {
        const int32_t v = int32_t((nx + 1) * (j + (ny + 1) * k));  // x-fastest numbering, i = 0
        for (int d = 0; d < 3; ++d) {
          dofs.push_back(3 * v + d);
          vals.push_back(0.0);
        }
      }
    problem.setEssentialBoundaryConditions(dofs, vals);

    pa_solve_options so{};
    pa_b200::check(pa_solve_options_default(&so), "options");
    so.method = PA_SOLVER_PCG_FP64;
    so.rel_tol = 1e-12;
    pa_b200::MpmdApp app(problem, N, N, /*self_adjoint=*/true, &so);
    using L = pa_b200::MpmdApp::Layout;
    app.defineComputeSolution("Compute Displacement Solution");
    app.defineComputeCriterion("Compute Objective", "Internal Elastic Energy", "Objective Value", "Objective Gradient");
    app.defineComputeCriterionGradientX("Compute Objective GradientX", "Internal Elastic Energy", "Objective GradientX");
    app.defineComputeCriterionValue("Compute Shifted Value", "Internal Elastic Energy", "Shifted Value", 0.25);

    app.importData("Topology", L::ScalarField, topo.data(), topo.size());
    app.compute("Compute Displacement Solution");
    app.compute("Compute Objective");
    app.compute("Compute Objective GradientX");
    double f = 0.0;
    app.exportData("Objective Value", L::Scalar, &f, 1);
    std::vector<double> gz(N), gx(3 * N), sz(N);
    app.exportData("Objective Gradient", L::ScalarField, gz.data(), gz.size());
    app.exportData("Objective GradientX", L::ScalarField, gx.data(), gx.size());
    std::printf("%.17g\n", f);
    for (double v : gz) std::printf("%.17g\n", v);
    for (double v : gx) std::printf("%.17g\n", v);
    app.compute("Compute Shifted Value");
    double fs = 0.0;
    app.exportData("Shifted Value", L::Scalar, &fs, 1);
    std::printf("%.17g\n", fs);
    app.exportData("Solution Z", L::ScalarField, sz.data(), sz.size());
    for (double v : sz) std::printf("%.17g\n", v);
    // requests the reference rejects
    try {
      app.exportData("No Such Value", L::Scalar, &f, 1);
      std::printf("no error\n");
    } catch (const pa_b200::Error& e) {
      std::printf("ERR %s\n", e.what());
    }
    try {
      app.defineComputeCriterion("Bad", "Maximize Stiffness", "v", "g");
      std::printf("no error\n");
    } catch (const pa_b200::Error& e) {
      std::printf("ERR %s\n", e.what());
    }
  } catch (const pa_b200::Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
