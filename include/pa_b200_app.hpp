// pa_b200_app.hpp -- header-only plugin-facing application over the C ABI,
// shaped like the reference's MPMD_App (src/Analyze_App.hpp:68-740,
// src/Analyze_App.cpp:660-1110): the object an optimizer drives through named
// operations and named shared data.
//
//   MPMD_App::ComputeSolution             -> compute() of a ComputeSolution operation
//   MPMD_App::ComputeCriterion            -> ComputeCriterion          (value - target and gradient_z)
//   MPMD_App::ComputeCriterionValue       -> ComputeCriterionValue     (solves first: the energy is not linear)
//   MPMD_App::ComputeCriterionGradient    -> ComputeCriterionGradient  (at the current state)
//   MPMD_App::ComputeCriterionX           -> ComputeCriterionX         (value - target and gradient_x)
//   MPMD_App::ComputeCriterionGradientX   -> ComputeCriterionGradientX
//   MPMD_App::importData / exportData     -> importData / exportData   ("Topology", "Solution", value and
//                                            gradient names mapped to their criterion, as the reference's
//                                            mValueNameToCriterionName / mGradientZNameToCriterionName)
//
// The reference parses its operations from the Plato Engine's XML; here they
// are defined by calls.  Criteria: "Internal Elastic Energy" (the compliance
// of the hot path).  Shared data lives in host memory (the reference copies
// Plato Engine's shared fields into device views, copyFieldIntoAnalyze); the
// library accepts host arrays.  Errors are pa_b200::Error exceptions, as the
// reference throws Plato::ParsingException / THROWERR.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "pa_b200.hpp"

namespace pa_b200 {

class MpmdApp {
 public:
  // Plato::data::layout_t values the operations use
  enum class Layout { ScalarField, ElementField, Scalar };
  enum class OpKind { ComputeSolution, ComputeCriterion, ComputeCriterionValue, ComputeCriterionGradient,
                      ComputeCriterionX, ComputeCriterionGradientX };

  // problem: set up with its loads and boundary conditions; num_controls is
  // the control length (nodes for the reference's nodal layout, cells for
  // per-cell controls).  self_adjoint: the reference's "Self-Adjoint" problem
  // parameter (criterion gradients are then -df/dz and -df/dx).
  MpmdApp(Problem& problem, int64_t num_nodes, int64_t num_controls, bool self_adjoint = true,
          const pa_solve_options* solver = nullptr)
      : problem_(problem), num_nodes_(num_nodes), self_adjoint_(self_adjoint),
        control_(size_t(num_controls), 1.0), state_(size_t(3 * num_nodes), 0.0) {
    // the reference initialises the control to 1 (src/Analyze_App.cpp:330-331)
    if (solver) {
      solver_ = *solver;
    } else {
      check(pa_solve_options_default(&solver_), "pa_solve_options_default");
    }
  }

  // ------------------------------------------------------- operations ---
  void defineComputeSolution(const std::string& op) { add(op, Op{OpKind::ComputeSolution}); }
  void defineComputeCriterion(const std::string& op, const std::string& criterion, const std::string& value_name,
                              const std::string& gradient_name, double target = 0.0) {
    Op o{OpKind::ComputeCriterion, criterion, target};
    mapValue(value_name, criterion);
    mapGradientZ(gradient_name, criterion);
    add(op, o);
  }
  void defineComputeCriterionValue(const std::string& op, const std::string& criterion, const std::string& value_name,
                                   double target = 0.0) {
    mapValue(value_name, criterion);
    add(op, Op{OpKind::ComputeCriterionValue, criterion, target});
  }
  void defineComputeCriterionGradient(const std::string& op, const std::string& criterion,
                                      const std::string& gradient_name) {
    mapGradientZ(gradient_name, criterion);
    add(op, Op{OpKind::ComputeCriterionGradient, criterion});
  }
  void defineComputeCriterionX(const std::string& op, const std::string& criterion, const std::string& value_name,
                               const std::string& gradient_name, double target = 0.0) {
    mapValue(value_name, criterion);
    mapGradientX(gradient_name, criterion);
    add(op, Op{OpKind::ComputeCriterionX, criterion, target});
  }
  void defineComputeCriterionGradientX(const std::string& op, const std::string& criterion,
                                       const std::string& gradient_name) {
    mapGradientX(gradient_name, criterion);
    add(op, Op{OpKind::ComputeCriterionGradientX, criterion});
  }

  // Plato::Application::compute(operationName)
  void compute(const std::string& op_name) {
    auto it = ops_.find(op_name);
    if (it == ops_.end()) throw Error(PA_ERR_INVALID_ARG, "no operation named '" + op_name + "'");
    const Op& op = it->second;
    switch (op.kind) {
      case OpKind::ComputeSolution:
        solve();
        break;
      case OpKind::ComputeCriterion:
        solve();
        values_[op.criterion] = value(op.criterion) - op.target;
        gradientZ(op.criterion);
        break;
      case OpKind::ComputeCriterionValue:
        solve();  // criterionIsLinear() is false for the energy
        values_[op.criterion] = value(op.criterion) - op.target;
        break;
      case OpKind::ComputeCriterionGradient:
        gradientZ(op.criterion);
        break;
      case OpKind::ComputeCriterionX:
        solve();
        values_[op.criterion] = value(op.criterion) - op.target;
        gradientX(op.criterion);
        break;
      case OpKind::ComputeCriterionGradientX:
        gradientX(op.criterion);
        break;
    }
  }

  // ------------------------------------------------------ shared data ---
  // importData: "Topology" (the control field) or "Solution" (the state).
  void importData(const std::string& name, Layout layout, const double* data, size_t n) {
    if (layout != Layout::ScalarField) return;  // parameters and values are not read by these operations
    if (name == "Topology") {
      copyIn(control_, data, n, name);
    } else if (name == "Solution") {
      copyIn(state_, data, n, name);
    }
  }

  // exportData: a criterion value by its value name (Scalar), a gradient by
  // its gradient name, "Topology", "Solution" (the x displacement,
  // component 0, as the reference exports a scalar field of the state) or
  // "Solution X|Y|Z" (ScalarField).
  void exportData(const std::string& name, Layout layout, double* data, size_t n) const {
    if (layout == Layout::Scalar) {
      auto v = value_names_.find(name);
      if (v == value_names_.end())
        throw Error(PA_ERR_INVALID_ARG, "Attempted to export SharedValue ('" + name + "') that doesn't exist.");
      auto c = values_.find(v->second);
      if (c == values_.end() || n < 1) throw Error(PA_ERR_INVALID_ARG, "criterion '" + v->second + "' not computed");
      data[0] = c->second;
      return;
    }
    if (name == "Topology") return copyOut(control_, data, n, name);
    auto gz = gradz_names_.find(name);
    if (gz != gradz_names_.end()) return copyOut(at(grad_z_, gz->second), data, n, name);
    auto gx = gradx_names_.find(name);
    if (gx != gradx_names_.end()) return copyOut(at(grad_x_, gx->second), data, n, name);
    int comp = -1;
    if (name == "Solution" || name == "Solution X") comp = 0;
    if (name == "Solution Y") comp = 1;
    if (name == "Solution Z") comp = 2;
    if (comp >= 0) {
      if (n != size_t(num_nodes_)) throw Error(PA_ERR_INVALID_ARG, "'" + name + "': size mismatch");
      for (int64_t v = 0; v < num_nodes_; ++v) data[v] = state_[size_t(3 * v + comp)];
      return;
    }
    throw Error(PA_ERR_INVALID_ARG, "Attempted to export field ('" + name + "') that doesn't exist.");
  }

  const std::vector<double>& control() const { return control_; }
  const std::vector<double>& state() const { return state_; }
  const pa_solve_stats& lastSolve() const { return last_; }

 private:
  struct Op {
    OpKind kind;
    std::string criterion;
    double target = 0.0;
  };

  static void checkCriterion(const std::string& c) {
    if (c != "Internal Elastic Energy") throw Error(PA_ERR_INVALID_ARG, "REQUESTED CRITERION NOT DEFINED: " + c);
  }
  void add(const std::string& name, const Op& op) {
    if (op.kind != OpKind::ComputeSolution) checkCriterion(op.criterion);
    if (ops_.count(name)) throw Error(PA_ERR_INVALID_ARG, "operation '" + name + "' defined twice");
    ops_[name] = op;
  }
  // addUnique: one value / gradient name per criterion (src/Analyze_App.cpp:657-665)
  static void addUnique(std::map<std::string, std::string>& m, const std::string& key, const std::string& c) {
    auto it = m.find(key);
    if (it != m.end() && it->second != c)
      throw Error(PA_ERR_INVALID_ARG, "shared data name '" + key + "' already maps to criterion '" + it->second + "'");
    m[key] = c;
  }
  void mapValue(const std::string& n, const std::string& c) { addUnique(value_names_, n, c); }
  void mapGradientZ(const std::string& n, const std::string& c) { addUnique(gradz_names_, n, c); }
  void mapGradientX(const std::string& n, const std::string& c) { addUnique(gradx_names_, n, c); }

  void solve() { last_ = problem_.solution(control_.data(), state_.data(), &solver_); }
  double value(const std::string&) const { return problem_.criterionValue(control_.data(), state_.data()); }
  void gradientZ(const std::string& c) {
    std::vector<double>& g = grad_z_[c];
    g.assign(control_.size(), 0.0);
    problem_.criterionGradient(control_.data(), state_.data(), g.data(), self_adjoint_, &solver_);
  }
  void gradientX(const std::string& c) {
    // Problem::criterionGradientX (src/elliptic/Problem.hpp:510-531): the
    // self-adjoint energy's total derivative is -df/dx
    if (!self_adjoint_) throw Error(PA_ERR_INVALID_ARG, "gradient_x is built for the self-adjoint criterion only");
    std::vector<double>& g = grad_x_[c];
    g.assign(size_t(3 * num_nodes_), 0.0);
    check(pa_sf_gradient_x(problem_.handle(), state_.data(), control_.data(), g.data()), "gradient_x");
    for (double& v : g) v = -v;
  }
  static const std::vector<double>& at(const std::map<std::string, std::vector<double>>& m, const std::string& c) {
    auto it = m.find(c);
    if (it == m.end()) throw Error(PA_ERR_INVALID_ARG, "gradient of '" + c + "' not computed");
    return it->second;
  }
  static void copyIn(std::vector<double>& dst, const double* src, size_t n, const std::string& name) {
    if (n != dst.size()) throw Error(PA_ERR_INVALID_ARG, "'" + name + "': size mismatch");
    dst.assign(src, src + n);
  }
  static void copyOut(const std::vector<double>& src, double* dst, size_t n, const std::string& name) {
    if (n != src.size()) throw Error(PA_ERR_INVALID_ARG, "'" + name + "': size mismatch");
    for (size_t i = 0; i < n; ++i) dst[i] = src[i];
  }

  Problem& problem_;
  int64_t num_nodes_;
  bool self_adjoint_;
  pa_solve_options solver_{};
  pa_solve_stats last_{};
  std::vector<double> control_, state_;
  std::map<std::string, Op> ops_;
  std::map<std::string, std::string> value_names_, gradz_names_, gradx_names_;
  std::map<std::string, double> values_;
  std::map<std::string, std::vector<double>> grad_z_, grad_x_;
};

}  // namespace pa_b200
