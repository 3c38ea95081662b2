// pa_problem.cuh -- the problem handle behind pa_problem* (not part of the ABI).
#pragma once
#include <memory>

#include "pa_internal.cuh"

namespace pa {

// Device workspace of the PCG solvers; sized on first use, reused across solves.
struct SolverWorkspace {
  int64_t ndof = 0;
  // FP64 vectors
  DevBuf<double> x, b, r, p0, p1, ap, dinv, t, w64, diag;
  // FP32 vectors (mixed precision)
  DevBuf<float> r32, p32a, p32b, ap32, dinv32, dx32, w32;
  DevBuf<float> coords32;
  DevBuf<float> ones32, z32;   // flexible CG: all-ones "diagonal", preconditioned residual
  DevBuf<float4> dinv4, ones4; // D^-1 (and the all-ones diagonal) as N x (x, y, z, 0) for the FP32 tile kernel
  DevBuf<double> fcg_state;    // flexible CG scalars
  DevBuf<double> partials;
  DevBuf<unsigned int> counters;
  DevBuf<PcgScalars> sc;
  DevBuf<double> rr_hist;
  void ensure(int64_t ndof_, int64_t C, int grid, bool mixed);
};

// The operator a solve uses: SIMP weights per cell (tile order), optional J2
// tangent records (8 per cell, tile order) and the interleaved Jacobi diagonal.
struct SolveOperator {
  const double* w64 = nullptr;
  const float* w32 = nullptr;
  const double* plas64 = nullptr;
  const float* plas32 = nullptr;
  const double* diag_aos = nullptr;
  bool homogeneous_bc = false;  // impose zero (not the problem's) Dirichlet values
  double bc_scale = 1.0;        // otherwise impose bc_scale times the problem's values
};

struct LearnedPC;
struct MgHierarchy;
struct BoxHierarchy;

struct Problem {
  Mesh* mesh = nullptr;
  LearnedPC* pc = nullptr;  // network of PA_SOLVER_FCG_LEARNED (not owned)
  LearnedPC* coarse_pc = nullptr;  // learned level-1 weight correction of the box multigrid (not owned)
  MgHierarchy* mg = nullptr;  // coarse levels of PA_SOLVER_PCG_MG (owned; mg_release)
  BoxHierarchy* boxmg = nullptr;  // the same on box kernels (owned; boxmg_release)
  ElasticParams ep{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // natural BCs
  std::vector<int32_t> faces;     // 3 per face
  std::vector<double> face_flux;  // 3 per face
  DevBuf<int32_t> d_faces;
  DevBuf<double> d_face_flux;
  // essential BCs
  std::vector<int32_t> bc_dofs;
  std::vector<double> bc_vals;
  DevBuf<int32_t> d_bc_dofs;
  DevBuf<double> d_bc_vals;
  DevBuf<uint8_t> d_node_mask;  // N, bit d = dof d constrained
  DevBuf<uint32_t> d_tile_nodes_bc;  // the mesh's flagged tile node ids with the mask bits of these BCs
  // scratch for reductions / staging
  DevBuf<double> d_partials;
  DevBuf<double> d_scalar;
  DevBuf<unsigned int> d_counter;
  DevBuf<double> d_rhs;
  std::vector<std::unique_ptr<DevBuf<char>>> staging;  // host-array staging, reused across calls
  SolverWorkspace ws;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // per-part results of the last batched solve (parted meshes)
  std::vector<int32_t> part_iterations;
  std::vector<double> part_rel_residual;

  int64_t N() const { return mesh->N; }
  int64_t C() const { return mesh->C; }
  int64_t ndof() const { return 3 * mesh->N; }
  int64_t nz() const { return ep.layout == PA_CONTROL_CELL ? mesh->C : mesh->N; }
};

pa_status solve_batched(Problem& P, const SolveOperator& op, const double* b, double* x_out,
                        const pa_solve_options& o, pa_solve_stats* st);
// multigrid-preconditioned CG on box meshes (pa_mg.cu)
pa_status solve_mg(Problem& P, const SolveOperator& op, const double* b, double* x_out, const pa_solve_options& o,
                   pa_solve_stats* st);
void mg_release(Problem& P);

// Structured boxes (pa_boxmg.cu): the box kernel of pa_box.cuh applies the
// operator; multigrid CG with every level on it.
// Per-cell entry points on a box mesh in its own numbering with per-cell
// controls: y = K(z) u (interleaved), the internal energy (value, one
// device double; may be null) with dF/dz per cell (may be null), and dR/dz
// per cell (12 values in each cell's vertex order).
bool box_entry_eligible(const Problem& P);
// The assembled K(z) (block CRS entries) on a box mesh in its own numbering
// with sorted columns; false (nothing launched) on any other mesh.
bool box_gradient_u(Problem& P, const double* z, double* entries);
// dR/dx (the volume term) likewise; the caller adds the surface loads
bool box_gradient_x(Problem& P, const double* u, const double* z, double* entries);
void box_entry_apply(Problem& P, const double* z, const double* u, double* y);
void box_entry_energy(Problem& P, const double* z, const double* u, double* value, double* grad_z);
void box_entry_gradient_z(Problem& P, const double* z, const double* u, double* vals);
// Learned level-1 weights of the box multigrid (pa_boxmg.cu): the level-1 hex
// grid (false: no box multigrid), the network's input features for control z
// (5 per level-1 hex, device), and the loss and dL/ddelta of the V-cycle on
// residual/error pairs for an explicit correction delta (device arrays;
// energies and loss on the host).
bool boxmg_coarse_grid(const Problem& P, int dims[3]);
void boxmg_coarse_features(Problem& P, const double* z, float* feat);
void boxmg_coarse_sensitivity(Problem& P, const double* z, const float* delta, int nres, const double* res,
                              const double* energies, double* loss, float* grad);
bool box_apply_eligible(const Problem& P);
bool boxmg_eligible(const Problem& P);
// false (nothing written) when the coarsest operator is singular.  jacobi:
// the same FP64 outer CG on the box kernel preconditioned by the fine level's
// inverse diagonal instead of the V-cycle (PA_SOLVER_PCG_FP64 on box meshes:
// deterministic, no atomics)
bool solve_boxmg(Problem& P, const double* z, const double* b, double* x_out, const pa_solve_options& o,
                 pa_solve_stats* st, pa_status* status, bool jacobi = false);
// interleaved x, y in the caller's order; xs, ys: 3N scratch
template <typename T>
void box_apply(Problem& P, const double* z, const T* x, T* y, bool constrained, T* xs, T* ys);
double time_box_apply(Problem& P, const double* z, bool fp32, int reps, int64_t* bytes);
void boxmg_release(Problem& P);

}  // namespace pa
