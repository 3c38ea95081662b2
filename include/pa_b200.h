/*
 * pa_b200.h -- C ABI of libpa_b200.so, a B200 (sm_100a) implementation of
 * Plato Analyze's per-cell linear-tetrahedron hot path: SIMP elastostatics
 * (residual, state/control Jacobians), the "Internal Elastic Energy"
 * (compliance) criterion, a matrix-free Jacobi-PCG solve of the constrained
 * system, and the J2 radial return.
 *
 * Conventions
 *  - Every entry point returns pa_status (0 = success).  No C++ exception
 *    crosses this boundary; pa_last_error() returns the calling thread's
 *    last message.
 *  - Array arguments may be device pointers or host pointers (pageable or
 *    pinned).  Host arrays are staged through library-owned device buffers;
 *    an entry point that was given a host output returns after the result
 *    is on the host.  Device-only calls are asynchronous on the problem's
 *    stream, except those that return a host scalar.
 *  - Sizes are implied by the mesh: N nodes, C cells, 3N state dofs, B CRS
 *    blocks (pa_mesh_sizes).  Nodal vectors are interleaved (x,y,z) per
 *    node, as the reference's ScalarVector of a 3-dof-per-node physics.
 *  - Handles are not reentrant: one host thread drives one pa_problem at a
 *    time.  Several problems may share a mesh.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the platoanalyze source tree).
 */
#ifndef PA_B200_H
#define PA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  PA_OK = 0,
  PA_ERR_INVALID_ARG = 1,  /* bad pointer, size or parameter */
  PA_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  PA_ERR_NOT_CONVERGED = 3,/* iteration cap reached before the tolerance */
  PA_ERR_BREAKDOWN = 4,    /* Krylov breakdown (p.Ap <= 0 or non-finite) */
  PA_ERR_NONFINITE = 5,    /* NaN/Inf in an input or a reduction */
  PA_ERR_NO_DEVICE = 6,    /* no CUDA device visible */
  PA_ERR_UNSUPPORTED = 7   /* valid request this build does not serve */
} pa_status;

typedef struct pa_mesh pa_mesh;
typedef struct pa_problem pa_problem;
typedef struct pa_pc pa_pc;

/* Library version string and the calling thread's last error message. */
const char* pa_version(void);
const char* pa_last_error(void);

/* ---------------------------------------------------------------- mesh --- */

/* Linear-tet mesh from connectivity (C x 4, int32) and coordinates (N x 3).
 * Replaces the Omega_h::Mesh the reference's SpatialModel wraps
 * (src/SpatialModel.hpp:15-149) and the node-star CRS graph of
 * CreateBlockMatrix (src/ImplicitFunctors.hpp:735-808).  Builds the
 * block-CRS graph (columns sorted ascending, diagonal included) and the
 * shared-memory cell tiles the kernels use. */
pa_status pa_mesh_create(const int32_t* cells2nodes, int64_t num_cells, const double* coords,
                         int64_t num_nodes, pa_mesh** out);

/* Exodus II mesh input, the mesh and node sets the reference reads with
 * Omega_h::exodus::read (src/PlatoDriver.hpp:76).  Host-only: a netCDF
 * classic file (CDF-1, CDF-2 or CDF-5; netCDF-4/HDF5 files are refused with
 * PA_ERR_INVALID_ARG) with num_dim 3, coordinates coordx/coordy/coordz (or
 * coord), element blocks connect1..B of 4-node tetrahedra (elem_type TETRA,
 * TETRA4, TET4 or TET; any other type is refused) concatenated in block
 * order, and node sets node_ns1..S named by ns_names (else "ns_<id>" from
 * ns_prop1).  Indices are 0-based on output.  Typical use: open, sizes, mesh
 * into caller arrays, pa_mesh_create, node sets for the Dirichlet dofs,
 * close. */
typedef struct pa_exodus pa_exodus;
pa_status pa_exodus_open(const char* path, pa_exodus** out);
pa_status pa_exodus_sizes(const pa_exodus* exodus, int64_t* num_nodes, int64_t* num_cells, int32_t* num_node_sets);
/* coords: 3 x num_nodes (x, y, z per node); cells2nodes: 4 x num_cells */
pa_status pa_exodus_mesh(const pa_exodus* exodus, double* coords, int32_t* cells2nodes);
/* Node set `index` (0 .. num_node_sets - 1): its name (truncated to
 * name_capacity - 1 characters, NUL-terminated; may be NULL), its size and,
 * when nodes is not NULL, its node ids. */
pa_status pa_exodus_node_set(const pa_exodus* exodus, int32_t index, char* name, int32_t name_capacity,
                             int64_t* count, int32_t* nodes);
void pa_exodus_close(pa_exodus* exodus);

/* Structured box [0,lx]x[0,ly]x[0,lz] with nx*ny*nz hexes, each split into
 * six tets around its (0,0,0)-(1,1,1) diagonal in the order of the
 * reference's single-hex box (unit_tests/OmegaHUtilitiesTests.cpp:258-287).
 * Nodes are numbered x fastest.  Stands in for Omega_h::build_box
 * (unit_tests/PlatoTestHelpers.hpp:240-249) with this build's own numbering. */
pa_status pa_mesh_create_box(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                             pa_mesh** out);

/* Handles may be destroyed in any order: a mesh (or a network, pa_pc_destroy)
 * still used by problems is released when the last of them is destroyed. */
pa_status pa_mesh_destroy(pa_mesh* mesh);

/* Sizes: cells C, nodes N, CRS blocks B, cell tiles T. Any output may be NULL. */
pa_status pa_mesh_sizes(const pa_mesh* mesh, int64_t* num_cells, int64_t* num_nodes,
                        int64_t* num_blocks, int64_t* num_tiles);

/* Host copies of the connectivity (C x 4) and coordinates (N x 3). */
pa_status pa_mesh_get(const pa_mesh* mesh, int32_t* cells2nodes, double* coords);

/* Host copy of the block-CRS graph: rowmap (N+1), cols (B). */
pa_status pa_mesh_graph(const pa_mesh* mesh, int32_t* rowmap, int32_t* cols);

/* Replace the CRS graph by a caller's graph with the same nonzero pattern but
 * any in-row column order, e.g. the Omega_h star order the reference's
 * CrsMatrix carries (src/alg/CrsMatrix.hpp:28-30).  gradient_u and
 * gradient_z then fill entries in that order. */
pa_status pa_mesh_set_graph(pa_mesh* mesh, const int32_t* rowmap, const int32_t* cols, int64_t num_blocks);

/* Uniform hex geometry.  When every cell belongs to a six-tet hex and all
 * hexes are translates of one another (a structured voxel grid, any hex
 * shape; edge vectors equal to 1e-9 of the hex size), the FP32 matrix-free
 * kernels take each template tet's shape gradients and volume from a per-mesh
 * table computed once in FP64 instead of recomputing them per tet from
 * gathered coordinates; the FP64 kernels do so when the hexes agree to
 * rounding level (1e-12 of the hex size).  No reference counterpart: the
 * reference recomputes them per cell (src/ImplicitFunctors.hpp:165-217).  enable = 1 (the default) uses the table
 * when the mesh qualifies, 0 forces the per-tet geometry, -1 only queries;
 * *active (may be NULL) receives 1 when the table is in use.  Changing it is
 * allowed only before problems are created on the mesh. */
pa_status pa_mesh_uniform_geometry(pa_mesh* mesh, int32_t enable, int32_t* active);

/* Box kernels.  On a box lattice (made by pa_mesh_create_box, or given to
 * pa_mesh_create as arrays that form such a box -- equal axis-aligned hexes
 * split into the same six tets along one cube diagonal, as Omega_h build_box
 * does -- under any node, cell and vertex order) the matrix-free operator
 * (pa_apply) and every level of the multigrid solve (PA_SOLVER_PCG_MG) run on
 * a kernel that derives node ids from the lattice and works on the tets as
 * edge differences of their hex (no connectivity, coordinates or geometry
 * arithmetic), with the vector updates fused into it.  No reference
 * counterpart (the reference gathers through cells2nodes,
 * src/ImplicitFunctors.hpp:15-58).  enable = 1 (the default) uses them when
 * the mesh qualifies, 0 keeps the tile kernels, -1 only queries; *active (may
 * be NULL) receives 1 when they are in use.  Takes effect on the next call. */
pa_status pa_mesh_box_kernels(pa_mesh* mesh, int32_t enable, int32_t* active);

/* Visualisation output: the mesh, the displacement u (3N, interleaved; may be
 * NULL) and the control (N nodal or C per-cell values by control_layout; may
 * be NULL) as a VTK XML unstructured grid (.vtu, base64 binary arrays,
 * tetrahedra) with the reference's field names "Displacements" and "Control"
 * -- Plato::write / Plato::output through Omega_h's VTK writer
 * (src/AnalyzeOutput.hpp:469-482).  u and control may be host or device
 * arrays. */
pa_status pa_write_vtu(const pa_mesh* mesh, const char* path, const double* u, const double* control,
                       int32_t control_layout);

/* Boundary faces (triangles, 3 node ids each) lying on the plane
 * coord[axis] == value.  Call with faces == NULL to get the count. */
pa_status pa_mesh_boundary_faces(const pa_mesh* mesh, int32_t axis, double value, int32_t* faces,
                                 int64_t* num_faces);

/* ------------------------------------------------------------- problem --- */

#define PA_CONTROL_NODAL 0 /* reference layout: N nodal controls, cell density = mean of 4 */
#define PA_CONTROL_CELL 1  /* one density per cell; gradient_z is per cell */

/* Material and penalty, the "Isotropic Linear Elastic" material
 * (src/IsotropicLinearElasticMaterial.cpp:86-108) and the SIMP "Penalty
 * Function" keys Exponent / Minimum Value (src/Simp.hpp:41-50). */
typedef struct {
  double youngs_modulus;
  double poissons_ratio;
  double simp_exponent;
  double simp_min;
  int32_t control_layout;
} pa_elastic_params;

/* Elliptic mechanics problem on `mesh` (src/elliptic/Problem.hpp:93-114).
 * `stream` is a cudaStream_t.  NULL: the library creates its own blocking
 * stream, which the legacy default stream orders against in both directions
 * (device arrays written there before a call are read after them; results
 * are visible there after the call).  With any other stream the caller
 * orders its own work against it. */
pa_status pa_problem_create(pa_mesh* mesh, const pa_elastic_params* params, void* stream, pa_problem** out);
pa_status pa_problem_destroy(pa_problem* problem);

/* Uniform traction `flux` on boundary triangles: NaturalBC "Uniform" with
 * SurfaceLoadIntegral (src/NaturalBC.hpp:41-110, src/SurfaceLoadIntegral.hpp:96-160).
 * Adds to the problem's load set. */
pa_status pa_problem_add_traction(pa_problem* problem, const int32_t* faces, int64_t num_faces,
                                  const double flux[3]);
pa_status pa_problem_clear_tractions(pa_problem* problem);

/* Essential BCs: dof ids (3*node + component) and values
 * (Elliptic::Problem::setEssentialBoundaryConditions, src/elliptic/Problem.hpp:636-650). */
pa_status pa_problem_set_dirichlet(pa_problem* problem, const int32_t* dofs, const double* values, int64_t n);

/* --------------------------------------- Elliptic::VectorFunction --------- */

/* r = K(z) u - F_traction: VectorFunction::value (src/elliptic/VectorFunction.hpp:231-310). */
pa_status pa_vf_value(pa_problem* problem, const double* u, const double* z, double* r);

/* dR/du into 9*B block-CRS entries [block][i][j] on the mesh graph:
 * VectorFunction::gradient_u (src/elliptic/VectorFunction.hpp:505-594). */
pa_status pa_vf_gradient_u(pa_problem* problem, const double* u, const double* z, double* entries);

/* dR/dz, transposed: nodal layout -> 3*B entries of 1x3 blocks (row =
 * control node, col = state node) on the mesh graph; cell layout -> 12*C
 * entries (row = cell, its 4 nodes x 3 dofs in local order).
 * VectorFunction::gradient_z (src/elliptic/VectorFunction.hpp:598-689). */
pa_status pa_vf_gradient_z(pa_problem* problem, const double* u, const double* z, double* entries);

/* dR/dx (shape sensitivity), transposed into 9*B block-CRS entries on the mesh
 * graph: block (row = node of the coordinate, col = node of the residual dof),
 * entry [coordinate component][residual component]; includes the surface
 * load's dependence on the face areas.  VectorFunction::gradient_x
 * (src/elliptic/VectorFunction.hpp:317-408). */
pa_status pa_vf_gradient_x(pa_problem* problem, const double* u, const double* z, double* entries);

/* --------------------- PhysicsScalarFunction "Internal Elastic Energy" ---- */

/* f = sum_c 1/2 vol p(rho) eps:C:eps  (src/elliptic/PhysicsScalarFunction.hpp:225,
 * src/elliptic/InternalElasticEnergy.hpp:100-158).  `value` is a host pointer. */
pa_status pa_sf_value(pa_problem* problem, const double* u, const double* z, double* value);
/* df/du, 3N (src/elliptic/PhysicsScalarFunction.hpp:365). */
pa_status pa_sf_gradient_u(pa_problem* problem, const double* u, const double* z, double* grad);
/* df/dz, N (nodal) or C (cell) (src/elliptic/PhysicsScalarFunction.hpp:432). */
pa_status pa_sf_gradient_z(pa_problem* problem, const double* u, const double* z, double* grad);
/* df/dx, 3N (PhysicsScalarFunction::gradient_x, src/elliptic/PhysicsScalarFunction.hpp:293-360). */
pa_status pa_sf_gradient_x(pa_problem* problem, const double* u, const double* z, double* grad);

/* Allocation-free compliance value.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory while they run (a host
 * framework that owns all device memory through its own pool, a timed loop
 * where cudaMalloc's implicit device synchronisation is not acceptable, code
 * that cannot create library handles).  Same value as pa_sf_value, from raw
 * DEVICE arrays (cells2nodes 16-byte aligned, int32 C x 4; coords N x 3; u 3N;
 * z N or C per params->control_layout) into the DEVICE scalar `value`, on
 * `stream` (a cudaStream_t, NULL = default stream), asynchronously.  The
 * library allocates nothing: block partial sums live in a fixed 256 KB
 * __device__ array, which limits a call to 8,388,608 cells (larger meshes are
 * rejected with PA_ERR_INVALID_ARG).  The first call on a device looks up that
 * array's address (do it before any stream capture); calls whose kernels
 * overlap on the GPU race on the shared array, so serialise them on one stream.
 * All arrays must belong to the current device.  A node id outside
 * [0, num_nodes) makes *value NaN (the kernel skips that cell's reads); the
 * lengths of coords, u and z cannot be checked from the host, and arrays
 * shorter than stated are undefined behaviour. */
pa_status pa_sf_value_noalloc(const int32_t* cells2nodes, int64_t num_cells, const double* coords,
                              int64_t num_nodes, const double* u, const double* z,
                              const pa_elastic_params* params, double* value, void* stream);

/* ----------------------------------------------------- matrix-free ------- */

#define PA_FP64 0
#define PA_FP32 1

/* y = K(z) x without assembling K.  precision PA_FP64 (x, y double) or
 * PA_FP32 (x, y float).  constrained != 0 applies the symmetric Dirichlet
 * elimination of applyBlockConstraints (src/ApplyConstraints.hpp:11-79):
 * constrained rows and columns removed, identity on the diagonal.  No
 * reference counterpart (the reference always assembles). */
pa_status pa_apply(pa_problem* problem, const double* z, const void* x, void* y, int32_t precision,
                   int32_t constrained);

/* Symmetric Dirichlet elimination on an assembled block CRS + rhs with the
 * problem's BCs times `scale`: applyBlockConstraints<3> (src/ApplyConstraints.hpp:11-79). */
pa_status pa_apply_block_constraints(pa_problem* problem, double* entries, double* rhs, double scale);

/* ----------------------------------------------------------- solver ------ */

#define PA_SOLVER_PCG_FP64 0  /* matrix-free Jacobi-PCG, FP64 throughout */
#define PA_SOLVER_PCG_MIXED 1 /* FP32 apply/vectors, FP64 dots, FP64 true-residual updates */
#define PA_SOLVER_PCG_MG 3    /* FP64 CG preconditioned by a geometric multigrid V-cycle (FP32 Chebyshev
                                 smoothing); meshes that are a structured box under some node, cell and
                                 vertex numbering (pa_mesh_create_box or arrays), any hex counts */
#define PA_SOLVER_FCG_LEARNED 2 /* flexible CG preconditioned by the problem's learned network
                                   (pa_problem_set_preconditioner), precision as PA_SOLVER_PCG_MIXED;
                                   continues as PA_SOLVER_PCG_MIXED when the residual stalls or the
                                   network's direction is not a descent direction */

typedef struct {
  int32_t method;        /* PA_SOLVER_* */
  double rel_tol;        /* ||b - K x|| / ||b|| target */
  int32_t max_iters;     /* <= 0: 20 * sqrt(ndof) + 1000 */
  int32_t check_every;   /* iterations between convergence checks / residual replacement */
  int32_t use_initial_guess; /* 0: start from x = 0 (as Problem::solution does) */
  int32_t mg_coarse_solver;  /* PA_SOLVER_PCG_MG: PA_MG_COARSE_* (0, the default, is AUTO) */
} pa_solve_options;

/* Coarsest multigrid level: AUTO solves it with a dense FP64 inverse (built by
 * Gauss-Jordan elimination for each solve's weights) when the operator is
 * elastic and the level has at most 2048 dofs and is nonsingular, else (J2
 * tangent solves included) by Chebyshev iteration; CHEBYSHEV always iterates
 * (degree 40 on [lmax/1000, 1.1 lmax] of D^-1 K). */
#define PA_MG_COARSE_AUTO 0
#define PA_MG_COARSE_CHEBYSHEV 1

typedef struct {
  int32_t iterations;     /* CG iterations */
  int32_t replacements;   /* FP64 true-residual replacements (mixed) */
  double rel_residual;    /* final FP64 ||b - K x|| / ||b|| of the constrained system */
  double seconds;         /* device time of the solve */
  int32_t converged;
  int64_t kernel_launches; /* kernels this library launched for the solve */
  int32_t fallback_iterations; /* PA_SOLVER_FCG_LEARNED: iterations run by the Jacobi fallback */
} pa_solve_stats;

pa_status pa_solve_options_default(pa_solve_options* options);

/* Solve the Dirichlet-constrained system K(z) x = b (b unconstrained; the
 * problem's BC values are imposed as applyBlockConstraints does) -- the
 * AbstractSolver::solve boundary (src/alg/PlatoAbstractSolver.hpp:19-27). */
pa_status pa_solve(pa_problem* problem, const double* z, const double* b, double* x,
                   const pa_solve_options* options, pa_solve_stats* stats);

/* Elliptic::Problem::solution (src/elliptic/Problem.hpp:259-311): u = 0,
 * R = value(u, z), solve K du = -R with BCs, u += du. */
pa_status pa_problem_solution(pa_problem* problem, const double* z, double* u,
                              const pa_solve_options* options, pa_solve_stats* stats);

/* Elliptic::Problem::criterionGradient for the energy criterion
 * (src/elliptic/Problem.hpp:413-468).  self_adjoint != 0: -df/dz.  Otherwise
 * the adjoint route: K lambda = -df/du with zero BCs, g = df/dz + (dR/dz)^T lambda. */
pa_status pa_problem_criterion_gradient(pa_problem* problem, const double* z, const double* u, double* grad,
                                        int32_t self_adjoint, const pa_solve_options* options);

/* Diagnostic, no reference counterpart: average device time (ms) of one
 * fused CG kernel launch (p update + matrix-free K p + p.Kp, the solver's
 * hot kernel) over `reps` back-to-back launches on the problem's stream,
 * and its algorithmic bytes per launch:
 * C*(16 + s) + N*6*3*s, s = 4 (PA_FP32) or 8 (PA_FP64). */
pa_status pa_time_cg_apply(pa_problem* problem, const double* z, int32_t precision, int32_t reps,
                           double* ms_per_launch, int64_t* algorithmic_bytes);

/* Diagnostic, no reference counterpart: the same for the plain constrained
 * apply y = K x (the multigrid smoother's kernel, VectorFunction::value's
 * stiffness part), algorithmic bytes C*(16 + s) + N*3*3*s. */
pa_status pa_time_apply(pa_problem* problem, const double* z, int32_t precision, int32_t reps,
                        double* ms_per_launch, int64_t* algorithmic_bytes);

/* ---------------------------------------------------------- J2 return ---- */

/* J2 parameters: "Isotropic Linear Elastic" + "J2 Plasticity" keys of
 * J2PlasticityLocalResidual::initialize (src/J2PlasticityLocalResidual.hpp:130-200). */
typedef struct {
  double youngs_modulus;
  double poissons_ratio;
  double initial_yield_stress;
  double hardening_modulus_isotropic;
  double hardening_modulus_kinematic;
  double elastic_penalty_exponent;   /* reference default 1.0 */
  double elastic_min_ersatz;         /* reference default 1e-9 */
  double plastic_penalty_exponent;   /* reference default 0.5 */
  double plastic_min_ersatz;         /* reference default 1e-4 */
} pa_j2_params;

/* Radial return of every cell: J2PlasticityLocalResidual::updateLocalState
 * (src/J2PlasticityLocalResidual.hpp:421-523).  u: 3N displacements;
 * z: N nodal densities; prev_local / local: C x 14 local states
 * [acc. plastic strain, dgamma, plastic strain (6), backstress (6)]. */
pa_status pa_j2_radial_return(pa_problem* problem, const pa_j2_params* params, const double* u, const double* z,
                              const double* prev_local, double* local);

/* J2 local residual: J2PlasticityLocalResidual::evaluate
 * (src/J2PlasticityLocalResidual.hpp:291-409), 14 equations per cell at local
 * states `local` (current) and `prev_local`; u: 3N, z: N nodal; residual: C x 14. */
pa_status pa_j2_local_residual(pa_problem* problem, const pa_j2_params* params, const double* u, const double* z,
                               const double* local, const double* prev_local, double* residual);

typedef struct {
  int32_t steps;       /* pseudo-time load steps; Dirichlet values ramp as (k+1)/steps */
  int32_t max_newton;  /* Newton iterations per step */
  double newton_tol;   /* ||R_free|| <= newton_tol * (||R_free|| at the step's first iteration) */
  int32_t adaptive_forcing; /* 0: every tangent solve to linear->rel_tol; 1: inexact Newton, tolerance
                               eta_k = 0.9 (||R_k|| / ||R_k-1||)^2 (Eisenstat-Walker choice 2,
                               safeguarded, at most 0.1, at least linear->rel_tol and half the
                               remaining Newton reduction).  The Newton stopping test is unchanged. */
} pa_j2_solve_options;

typedef struct {
  int32_t steps;
  int32_t newton_iterations;  /* tangent solves over all steps */
  int64_t cg_iterations;      /* PCG iterations over all tangent solves */
  double seconds;             /* device time */
  double final_rel_residual;  /* largest over the steps of the relative Newton residual at the step's end */
  int32_t converged;
  int32_t linear_unconverged; /* tangent solves that stopped at their iteration cap */
  int32_t line_search_halvings; /* step halvings of the Newton line search */
} pa_j2_stats;

/* Elasto-plastic solve, displacement-form small-strain J2 with linear
 * isotropic/kinematic hardening: load steps over the problem's Dirichlet
 * values (the final values), Newton with per-cell radial return (FP64) and the
 * consistent tangent applied matrix-free inside the problem's PCG
 * (`linear`: FP64 or mixed).  Replaces PlasticityProblem::solution's forward
 * solve (src/PlasticityProblem.hpp:352, :791-846) with
 * NewtonRaphsonSolver::solve (src/NewtonRaphsonSolver.hpp:570-640); the
 * reference's global residual is the stabilized u-p form, this one the
 * displacement form.  Each step starts as the reference's does
 * (src/NewtonRaphsonSolver.hpp:127-131): tangent at the converged state with
 * the Dirichlet increment imposed in the solve; the Newton iterations that
 * follow use a backtracking line search on the residual norm.  A step ends
 * when ||R_free|| <= newton_tol x ||R_free|| of the new boundary values on the
 * previous field.  Outputs u (3N) and the final local states (C x 14). */
pa_status pa_j2_solve(pa_problem* problem, const pa_j2_params* params, const double* z,
                      const pa_j2_solve_options* options, const pa_solve_options* linear, double* u, double* local,
                      pa_j2_stats* stats);

/* Stabilized u-p plasticity residual, InfinitesimalStrainPlasticityResidual::
 * evaluate (src/InfinitesimalStrainPlasticityResidual.hpp:398-516): state is
 * 4 dofs per node (u_x, u_y, u_z, p; 4N), local the C x 14 local states, z the
 * N nodal controls, ppg the projected pressure gradient, per node (3N,
 * ppg_per_cell = 0) or per cell node (C x 12, ppg_per_cell = 1, the
 * reference's workset).  residual: per cell (C x 16, node-major, assembled =
 * 0, the reference's result workset) or assembled (4N, assembled = 1). */
typedef struct {
  double youngs_modulus;
  double poissons_ratio;
  double penalty_exponent;  /* SIMP on the elastic moduli */
  double penalty_min;
  double pressure_scaling;  /* "Pressure Scaling", default 1 */
} pa_up_params;

pa_status pa_up_residual(pa_problem* problem, const pa_up_params* params, const double* state, const double* local,
                         const double* ppg, int32_t ppg_per_cell, const double* z, double* residual,
                         int32_t assembled);

/* Stabilized u-p J2 plasticity solve, PlasticityProblem::solution's forward
 * problem (src/PlasticityProblem.hpp:791-846) with NewtonRaphsonSolver::solve
 * (src/NewtonRaphsonSolver.hpp:570-640): load steps over the problem's
 * Dirichlet values (displacement dofs 3 v + i, the final values; the
 * pressures are free), each Newton iterate returning the local states from
 * the previous step's (the J2 return mapping of `params`) and solving with the
 * condensed tangent dR/du - dR/dc (dH/dc)^-1 dH/du; the projected pressure
 * gradient of step k+1 is the lumped projection of step k's pressure
 * (PlasticityProblem::updateProjectedPressureGradient, :877-897), zero in the
 * first step.  The tangent is symmetric indefinite: MINRES with the inverse
 * absolute diagonal, to linear->rel_tol (default 1e-12) within
 * linear->max_iters (0: 100000); linear->method is ignored.  A step ends when
 * ||R_free|| <= newton_tol x ||R_free|| of the new boundary values on the
 * previous field (backtracking line search as pa_j2_solve).  Outputs the
 * state (u_x, u_y, u_z, p per node; 4N), the local states (C x 14) and, when
 * ppg is not NULL, the projected pressure gradient of the last step (3N).
 * stats->cg_iterations counts MINRES iterations. */
pa_status pa_up_solve(pa_problem* problem, const pa_up_params* up, const pa_j2_params* params, const double* z,
                      const pa_j2_solve_options* options, const pa_solve_options* linear, double* state,
                      double* local, double* ppg, pa_j2_stats* stats);

/* The "Elastic Work" criterion of the u-p plasticity problem and its
 * gradient with respect to the nodal controls (PlasticityProblem::
 * criterionValue / criterionGradient, src/PlasticityProblem.hpp:411-560, with
 * ElasticWorkCriterion, src/ElasticWorkCriterion.hpp, and the path-dependent
 * adjoint, src/PathDependentAdjointSolver.hpp:154-940).  Runs pa_up_solve
 * (same arguments and outputs), then *value = sum over the steps of each
 * step's elastic work V (sigma_n + sigma_{n-1}) . (e_n - e_{n-1}) / 2, with
 * e = eps(u) - eps_p and sigma the isotropic stress of up's moduli penalized
 * by the criterion's own SIMP (penalty_exponent, penalty_min), and gradient
 * (N) = d value / d z through every step (local states, pressures and the
 * lagged projection included).  The adjoint solves use MINRES like the
 * forward ones; stats->cg_iterations counts both. */
pa_status pa_up_elastic_work(pa_problem* problem, const pa_up_params* up, const pa_j2_params* params,
                             double penalty_exponent, double penalty_min, const double* z,
                             const pa_j2_solve_options* options, const pa_solve_options* linear, double* value,
                             double* gradient, double* state, double* local, pa_j2_stats* stats);

/* ------------------------------------------------------ batched solves --- */
/* No counterpart in the reference (one Problem solves one mesh).  A parted
 * mesh is the disjoint union of independent sub-meshes: part p owns the nodes
 * [node_offsets[p], node_offsets[p+1]) and every cell whose nodes lie there
 * (a cell spanning two parts is rejected).  On a parted mesh,
 * PA_SOLVER_PCG_MIXED runs one independent Jacobi-PCG per part (its own
 * alpha, beta, stopping test and iteration count) with all parts advanced by
 * the same kernels, so each part's result is that of solving it alone.
 * Call pa_mesh_set_parts before creating problems on the mesh; at most 4096
 * parts. */
pa_status pa_mesh_set_parts(pa_mesh* mesh, int32_t num_parts, const int64_t* node_offsets);
/* Per-part iteration counts and final relative residuals of the last batched
 * solve (num_parts entries each; either output may be NULL). */
pa_status pa_problem_part_stats(pa_problem* problem, int32_t* iterations, double* rel_residuals);
/* Tile-size autotuner: times the fused FP32 CG kernel at density z for tiles
 * of 64, 128 and 256 clusters, keeps the fastest (rebuilding the mesh's tiles)
 * and returns it; ms_per_apply (3 entries, may be NULL) gets the timings.  The
 * problem must be the only one on its mesh. */
pa_status pa_problem_autotune_tiles(pa_problem* problem, const double* z, int32_t* tile_clusters,
                                    double* ms_per_apply);

/* ------------------------------------------------ learned preconditioner --- */
/* No counterpart in the reference (its solvers are AmgX / AztecOO / Belos).
 * A small convolutional network on the nodal grid of a structured box mesh
 * (pa_mesh_create_box numbering: node i + gx (j + gy k)) maps the residual of
 * the constrained system to a correction:
 *   M r = D^-1 r + s D^-1/2 f(D^-1/2 r / s, stiffness, Dirichlet),  s = RMS(D^-1/2 r),
 * with D the Jacobi diagonal and f four 3x3x3 convolutions (5 -> 32 -> 32 ->
 * 32 -> 3 channels, ReLU between them), BF16 weights and activations, FP32
 * accumulation on the tensor cores.  Input features per node: the three
 * scaled residual components, 1 + log10(mean diagonal / max diagonal) / 9
 * clipped to [0, 1], and the constrained fraction of the node's dofs.  A new
 * network has zero weights in its last layer, so M starts as Jacobi. */

typedef struct {
  int32_t steps;        /* optimizer steps (Adam) */
  int32_t batch;        /* samples per step */
  double learning_rate; /* Adam step size; cosine-decayed to 5% over the steps */
  uint64_t seed;        /* sample order */
} pa_pc_train_options;

typedef struct {
  double initial_loss;  /* mean loss of the first step */
  double final_loss;    /* mean loss of the last min(10, steps) steps */
  double seconds;       /* device time of the training */
  int32_t steps;
  int64_t kernel_launches;
} pa_pc_train_stats;

/* Network for a grid of gx x gy x gz nodes; hidden-layer weights He-normal
 * from `seed`, last layer zero. */
pa_status pa_pc_create(int32_t gx, int32_t gy, int32_t gz, uint64_t seed, pa_pc** pc);
pa_status pa_pc_destroy(pa_pc* pc);
/* Parameters as one FP32 vector: per layer the weights [out][in][kz][ky][kx]
 * then the biases [out]. */
pa_status pa_pc_num_params(const pa_pc* pc, int64_t* count);
pa_status pa_pc_get_params(pa_pc* pc, float* params);
pa_status pa_pc_set_params(pa_pc* pc, const float* params);
/* The network alone on given input features (G x 5 FP32 per node; G = gx gy gz),
 * output G x 3 FP32 (the correction f before scaling). */
pa_status pa_pc_forward(pa_pc* pc, const float* features, float* out);
/* Gradient of sum(grad_out . f(features)) with respect to the parameters. */
pa_status pa_pc_backward(pa_pc* pc, const float* features, const float* grad_out, float* grad_params);
/* Diagnostics: average device time of the network's four convolutions over
 * `reps` back-to-back launches on the last input, and their algorithmic FLOPs
 * (2 x 27 x in x out per node and layer, real channel counts). */
pa_status pa_pc_time_forward(pa_pc* pc, int32_t reps, double* ms_per_forward, int64_t* flops);
/* out = M r for the problem at density z (interleaved 3N vectors). */
pa_status pa_pc_apply(pa_problem* problem, pa_pc* pc, const double* z, const double* r, double* out);
/* Train on residual/error pairs: sample s has residual r_s (3N, interleaved,
 * zero on constrained dofs) of the problem at density densities[sample_density[s]]
 * (each num_densities x nz), and e_s . r_s = energies[s] where K e_s = r_s.
 * Loss per sample: ||e_s - M r_s||_K^2 / ||e_s||_K^2, evaluated with the
 * matrix-free operator; gradients by the library's own backward kernels. */
pa_status pa_pc_train(pa_problem* problem, pa_pc* pc, int32_t num_densities, const double* densities,
                      int32_t num_samples, const int32_t* sample_density, const double* residuals,
                      const double* energies, const pa_pc_train_options* options, pa_pc_train_stats* stats);
/* Attach (or detach with NULL) the network PA_SOLVER_FCG_LEARNED uses; the
 * mesh must be the network's grid.  The problem does not own the network. */
pa_status pa_problem_set_preconditioner(pa_problem* problem, pa_pc* pc);

/* ------------------------------------ learned coarse-level multigrid weights --
 * No counterpart in the reference (it solves with AmgX / Belos).  The box
 * multigrid of PA_SOLVER_PCG_MG gives each level-1 hex the mean weight of its
 * children; a network (pa_pc on the level-1 hex grid: gx, gy, gz = its hex
 * counts) may multiply it by exp(0.5 tanh(delta)), delta its first output channel, fed
 * with 5 features per level-1 hex (logarithms of the mean, geometric mean,
 * minimum and maximum child weight, and the fraction of children inside the
 * box).  A network whose last layer is zero (a new one) leaves the method
 * unchanged.  Arrays may be device or host pointers. */
/* Level-1 hex counts of the problem's box multigrid; PA_ERR_INVALID_ARG when
 * the mesh has none. */
pa_status pa_boxmg_coarse_grid(pa_problem* problem, int32_t dims[3]);
/* The network's input features for control z: 5 per level-1 hex, channel-last. */
pa_status pa_boxmg_coarse_features(pa_problem* problem, const double* z, float* features);
/* Training loss and gradient for an explicit correction delta (one per
 * level-1 hex): the mean over the residual/error pairs (residuals: num x 3N,
 * interleaved, K e_s = r_s at control z, energies[s] = e_s . r_s) of
 * ||e_s - V r_s||_K^2 / ||e_s||_K^2, V the V-cycle, and its gradient in delta
 * (exact for a two-level hierarchy; deeper levels and level 1's smoother are
 * held fixed otherwise).  The fine smoother's spectral estimate is made from
 * its cold start in every call, so equal inputs give equal results. */
pa_status pa_boxmg_coarse_sensitivity(pa_problem* problem, const double* z, const float* delta,
                                      int32_t num_residuals, const double* residuals, const double* energies,
                                      double* loss, float* grad_delta);
/* Attach (or detach with NULL) the network that corrects the level-1 weights
 * of every later PA_SOLVER_PCG_MG solve; the problem does not own it. */
pa_status pa_problem_set_coarse_network(pa_problem* problem, pa_pc* pc);

#ifdef __cplusplus
}
#endif
#endif /* PA_B200_H */
