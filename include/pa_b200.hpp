// pa_b200.hpp -- header-only C++ view of the C ABI in pa_b200.h, shaped like
// the reference's classes so that a Kokkos-free C++ caller can swap it in:
//
//   Plato::Elliptic::VectorFunction<Mechanics<3>>   -> pa_b200::VectorFunction
//     value / gradient_u / gradient_z               (src/elliptic/VectorFunction.hpp:231,505,598)
//   Plato::Elliptic::PhysicsScalarFunction          -> pa_b200::PhysicsScalarFunction
//     value / gradient_u / gradient_z               (src/elliptic/PhysicsScalarFunction.hpp:225,365,432)
//   Plato::Elliptic::Problem                        -> pa_b200::Problem
//     solution / criterionValue / criterionGradient (src/elliptic/Problem.hpp:259,320,413)
//
// Errors become pa_b200::Error exceptions, as the reference reports errors with
// THROWERR (src/AnalyzeMacros.hpp).  Arrays are raw pointers (device or host)
// sized by the mesh; ownership stays with the caller.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pa_b200.h"

namespace pa_b200 {

struct Error : public std::runtime_error {
  pa_status status;
  Error(pa_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(pa_status s, const char* what) {
  if (s != PA_OK) throw Error(s, std::string(what) + ": " + pa_last_error());
}

class Mesh {
 public:
  Mesh(const int32_t* cells2nodes, int64_t num_cells, const double* coords, int64_t num_nodes) {
    check(pa_mesh_create(cells2nodes, num_cells, coords, num_nodes, &h_), "pa_mesh_create");
  }
  static Mesh box(int nx, int ny, int nz, double lx, double ly, double lz) {
    Mesh m;
    check(pa_mesh_create_box(nx, ny, nz, lx, ly, lz, &m.h_), "pa_mesh_create_box");
    return m;
  }
  Mesh(Mesh&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
  Mesh(const Mesh&) = delete;
  ~Mesh() { if (h_) pa_mesh_destroy(h_); }
  int64_t numCells() const { int64_t c; check(pa_mesh_sizes(h_, &c, nullptr, nullptr, nullptr), "sizes"); return c; }
  int64_t numNodes() const { int64_t n; check(pa_mesh_sizes(h_, nullptr, &n, nullptr, nullptr), "sizes"); return n; }
  int64_t numBlocks() const { int64_t b; check(pa_mesh_sizes(h_, nullptr, nullptr, &b, nullptr), "sizes"); return b; }
  pa_mesh* handle() const { return h_; }

 private:
  Mesh() = default;
  pa_mesh* h_ = nullptr;
};

class VectorFunction {
 public:
  explicit VectorFunction(pa_problem* p) : p_(p) {}
  void value(const double* u, const double* z, double* r) const { check(pa_vf_value(p_, u, z, r), "value"); }
  void gradient_u(const double* u, const double* z, double* entries) const {
    check(pa_vf_gradient_u(p_, u, z, entries), "gradient_u");
  }
  void gradient_z(const double* u, const double* z, double* entries) const {
    check(pa_vf_gradient_z(p_, u, z, entries), "gradient_z");
  }

 private:
  pa_problem* p_;
};

class PhysicsScalarFunction {
 public:
  explicit PhysicsScalarFunction(pa_problem* p) : p_(p) {}
  double value(const double* u, const double* z) const {
    double v = 0.0;
    check(pa_sf_value(p_, u, z, &v), "value");
    return v;
  }
  void gradient_u(const double* u, const double* z, double* g) const { check(pa_sf_gradient_u(p_, u, z, g), "gradient_u"); }
  void gradient_z(const double* u, const double* z, double* g) const { check(pa_sf_gradient_z(p_, u, z, g), "gradient_z"); }

 private:
  pa_problem* p_;
};

class Problem {
 public:
  Problem(const Mesh& mesh, const pa_elastic_params& params, void* stream = nullptr) {
    check(pa_problem_create(mesh.handle(), &params, stream, &h_), "pa_problem_create");
  }
  Problem(const Problem&) = delete;
  ~Problem() { if (h_) pa_problem_destroy(h_); }
  void addTraction(const std::vector<int32_t>& faces, const double flux[3]) {
    check(pa_problem_add_traction(h_, faces.data(), int64_t(faces.size() / 3), flux), "add_traction");
  }
  void setEssentialBoundaryConditions(const std::vector<int32_t>& dofs, const std::vector<double>& values) {
    check(pa_problem_set_dirichlet(h_, dofs.data(), values.data(), int64_t(dofs.size())), "set_dirichlet");
  }
  VectorFunction vectorFunction() const { return VectorFunction(h_); }
  PhysicsScalarFunction criterion() const { return PhysicsScalarFunction(h_); }
  pa_solve_stats solution(const double* z, double* u, const pa_solve_options* opts = nullptr) {
    pa_solve_stats st{};
    check(pa_problem_solution(h_, z, u, opts, &st), "solution");
    return st;
  }
  double criterionValue(const double* z, const double* u) const { return criterion().value(u, z); }
  void criterionGradient(const double* z, const double* u, double* g, bool selfAdjoint = true,
                         const pa_solve_options* opts = nullptr) {
    check(pa_problem_criterion_gradient(h_, z, u, g, selfAdjoint ? 1 : 0, opts), "criterion_gradient");
  }
  pa_problem* handle() const { return h_; }

 private:
  pa_problem* h_ = nullptr;
};

}  // namespace pa_b200
