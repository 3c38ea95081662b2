// pa_abi.cu -- the extern "C" entry points of libpa_b200.so.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>

#include "pa_problem.cuh"
#include "pa_cell.cuh"
#include "pa_learned.cuh"

namespace pa {

pa_status solve_device(Problem& P, const double* z, const double* b, double* x_out, const pa_solve_options& o,
                       pa_solve_stats* st);
void launch_dRdz_transpose_times(const Problem& P, const double* u, const double* z, const double* lambda,
                                 double* g, cudaStream_t s);
void launch_block_constraints(const Problem& P, double* entries, double* rhs, double scale, cudaStream_t s);
void launch_scale(double* v, int64_t n, double a, cudaStream_t s);
void launch_gradient_x(Problem& P, const double* u, const double* z, double* entries, cudaStream_t s);
void launch_energy_grad_x(const Problem& P, const double* u, const double* z, double* gx, cudaStream_t s);
double time_cg_apply(Problem& P, const double* z, bool fp32, int reps);
double time_apply(Problem& P, const double* z, bool fp32, int reps);
void launch_j2_local_residual(const Problem& P, const pa_j2_params& jp, const double* u, const double* z,
                              const double* loc, const double* prev, double* H, cudaStream_t s);
pa_status j2_solve(Problem& P, const pa_j2_params& jp, const double* z, const pa_j2_solve_options& jo,
                   const pa_solve_options& lo, double* u, double* local, pa_j2_stats* js);
pa_status up_solve(Problem& P, const pa_up_params& up, const pa_j2_params& jp, const double* z,
                   const pa_j2_solve_options& jo, const pa_solve_options& lo, double* state, double* local,
                   double* ppg, pa_j2_stats* js);
pa_status up_elastic_work(Problem& P, const pa_up_params& up, const pa_j2_params& jp, double fpe, double fpmin,
                          const double* z, const pa_j2_solve_options& jo, const pa_solve_options& lo, double* value,
                          double* grad, double* state, double* local, pa_j2_stats* js);

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  PA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) dev = 0;
  if (!cached[dev]) PA_CUDA(cudaDeviceGetAttribute(&cached[dev], cudaDevAttrMultiProcessorCount, dev));
  return cached[dev];
}

namespace {

template <typename F>
pa_status guard(F&& f) {
  try {
    f();
    return PA_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return PA_ERR_CUDA;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return PA_ERR_INVALID_ARG;
  }
}

template <typename F>
pa_status guard_status(F&& f) {
  try {
    const pa_status st = f();
    if (st == PA_ERR_NOT_CONVERGED) set_last_error("the iteration cap was reached before the tolerance");
    else if (st == PA_ERR_BREAKDOWN) set_last_error("Krylov breakdown (p.Kp <= 0 or non-finite)");
    else if (st == PA_ERR_NONFINITE) set_last_error("non-finite value in a reduction");
    return st;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return PA_ERR_INVALID_ARG;
  }
}

void require_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw Error(PA_ERR_NO_DEVICE, "no CUDA device is visible to libpa_b200");
  }
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Maps caller arrays to device arrays for one call: device pointers pass
// through; host arrays are copied into staging buffers (in) and back (out).
class Stage {
 public:
  explicit Stage(Problem& P) : P_(P) {}
  template <typename T>
  const T* in(const T* p, int64_t count, const char* name) {
    PA_CHECK(p != nullptr, std::string("null pointer: ") + name);
    if (is_device_pointer(p)) return p;
    T* d = reinterpret_cast<T*>(buffer(count * sizeof(T)));
    PA_CUDA(cudaMemcpyAsync(d, p, count * sizeof(T), cudaMemcpyHostToDevice, P_.stream));
    return d;
  }
  template <typename T>
  T* out(T* p, int64_t count, const char* name, bool copy_in = false) {
    PA_CHECK(p != nullptr, std::string("null pointer: ") + name);
    if (is_device_pointer(p)) return p;
    T* d = reinterpret_cast<T*>(buffer(count * sizeof(T)));
    if (copy_in) PA_CUDA(cudaMemcpyAsync(d, p, count * sizeof(T), cudaMemcpyHostToDevice, P_.stream));
    outs_.push_back({p, d, size_t(count * sizeof(T))});
    return d;
  }
  void finish() {
    for (auto& o : outs_) PA_CUDA(cudaMemcpyAsync(o.host, o.dev, o.bytes, cudaMemcpyDeviceToHost, P_.stream));
    if (!outs_.empty()) PA_CUDA(cudaStreamSynchronize(P_.stream));
    PA_CUDA(cudaGetLastError());
  }

 private:
  struct Out {
    void* host;
    void* dev;
    size_t bytes;
  };
  void* buffer(size_t bytes) {
    auto& pool = P_.staging;
    if (slot_ >= pool.size()) pool.emplace_back(new DevBuf<char>());
    DevBuf<char>& b = *pool[slot_++];
    if (b.n < bytes) b.resize(bytes);
    return b.get();
  }
  Problem& P_;
  size_t slot_ = 0;
  std::vector<Out> outs_;
};

}  // namespace

}  // namespace pa

struct pa_mesh {
  pa::Mesh m;
  bool destroy_requested = false;  // pa_mesh_destroy while problems still use the mesh
};
struct pa_pc;
struct pa_problem {
  pa::Problem P;
  pa_mesh* mesh = nullptr;  // the problem keeps its mesh alive until it is destroyed
  pa_pc* pc = nullptr;      // and its attached network
  pa_pc* cpc = nullptr;     // and its coarse-weight network
};
struct pa_pc {
  pa::LearnedPC* pc = nullptr;
  int32_t attached = 0;            // problems using this network
  bool destroy_requested = false;  // released by the last of them
  ~pa_pc() { pa::pc_delete(pc); }
};

using pa::Error;
using pa::guard;
using pa::Problem;

namespace {

Problem& prob(pa_problem* h) {
  if (!h) throw Error(PA_ERR_INVALID_ARG, "null pa_problem");
  PA_CUDA(cudaSetDevice(h->P.mesh->device));
  return h->P;
}

void upload_bcs(Problem& P) {
  const int64_t N = P.N();
  std::vector<uint8_t> mask(N, 0);
  for (int32_t d : P.bc_dofs) mask[d / 3] |= uint8_t(1u << (d % 3));
  P.d_node_mask.upload(mask.data(), mask.size(), P.stream);
  std::vector<uint32_t> tn = P.mesh->h_tile_nodes;
  for (uint32_t& f : tn) f |= uint32_t(mask[f & pa::kNodeIdMask]) << pa::kMaskShift;
  P.d_tile_nodes_bc.upload(tn.data(), tn.size(), P.stream);
  if (!P.bc_dofs.empty()) {
    P.d_bc_dofs.upload(P.bc_dofs.data(), P.bc_dofs.size(), P.stream);
    P.d_bc_vals.upload(P.bc_vals.data(), P.bc_vals.size(), P.stream);
  }
  PA_CUDA(cudaStreamSynchronize(P.stream));
}

}  // namespace

extern "C" {

const char* pa_version(void) { return "pa_b200 0.1 (sm_100a)"; }
const char* pa_last_error(void) { return pa::g_last_error.c_str(); }

pa_status pa_mesh_create(const int32_t* cells2nodes, int64_t num_cells, const double* coords, int64_t num_nodes,
                         pa_mesh** out) {
  return guard([&] {
    PA_CHECK(out && cells2nodes && coords, "null argument");
    PA_CHECK(num_cells > 0 && num_nodes > 0, "empty mesh");
    pa::require_device();
    std::unique_ptr<pa_mesh> h(new pa_mesh());
    h->m.C = num_cells;
    h->m.N = num_nodes;
    h->m.cells.assign(cells2nodes, cells2nodes + 4 * num_cells);
    h->m.coords.assign(coords, coords + 3 * num_nodes);
    pa::mesh_build(h->m);
    *out = h.release();
  });
}

pa_status pa_mesh_create_box(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz, pa_mesh** out) {
  return guard([&] {
    PA_CHECK(out, "null argument");
    PA_CHECK(nx > 0 && ny > 0 && nz > 0, "box needs positive hex counts");
    PA_CHECK(lx > 0 && ly > 0 && lz > 0, "box needs positive lengths");
    pa::require_device();
    std::unique_ptr<pa_mesh> h(new pa_mesh());
    pa::mesh_make_box(h->m, nx, ny, nz, lx, ly, lz);
    *out = h.release();
  });
}

// A mesh destroyed while problems still use it is released by the last of
// them (handles may be destroyed in any order).
pa_status pa_mesh_destroy(pa_mesh* mesh) {
  return guard([&] {
    if (!mesh) return;
    if (mesh->m.live_problems > 0) {
      mesh->destroy_requested = true;
      return;
    }
    delete mesh;
  });
}

pa_status pa_mesh_sizes(const pa_mesh* mesh, int64_t* num_cells, int64_t* num_nodes, int64_t* num_blocks,
                        int64_t* num_tiles) {
  return guard([&] {
    PA_CHECK(mesh, "null pa_mesh");
    if (num_cells) *num_cells = mesh->m.C;
    if (num_nodes) *num_nodes = mesh->m.N;
    if (num_blocks) *num_blocks = mesh->m.B;
    if (num_tiles) *num_tiles = mesh->m.T;
  });
}

pa_status pa_mesh_get(const pa_mesh* mesh, int32_t* cells2nodes, double* coords) {
  return guard([&] {
    PA_CHECK(mesh, "null pa_mesh");
    if (cells2nodes) std::memcpy(cells2nodes, mesh->m.cells.data(), sizeof(int32_t) * mesh->m.cells.size());
    if (coords) std::memcpy(coords, mesh->m.coords.data(), sizeof(double) * mesh->m.coords.size());
  });
}

pa_status pa_mesh_graph(const pa_mesh* mesh, int32_t* rowmap, int32_t* cols) {
  return guard([&] {
    PA_CHECK(mesh, "null pa_mesh");
    if (rowmap) std::memcpy(rowmap, mesh->m.rowmap.data(), sizeof(int32_t) * mesh->m.rowmap.size());
    if (cols) std::memcpy(cols, mesh->m.cols.data(), sizeof(int32_t) * mesh->m.cols.size());
  });
}

pa_status pa_mesh_set_graph(pa_mesh* mesh, const int32_t* rowmap, const int32_t* cols, int64_t num_blocks) {
  return guard([&] {
    PA_CHECK(mesh && rowmap && cols, "null argument");
    pa::Mesh& m = mesh->m;
    PA_CHECK(num_blocks == m.B, "graph has a different number of blocks than the mesh's node-star pattern");
    PA_CHECK(rowmap[0] == 0 && rowmap[m.N] == num_blocks, "rowmap does not span the blocks");
    std::vector<int32_t> a, b;
    for (int64_t v = 0; v < m.N; ++v) {
      PA_CHECK(rowmap[v + 1] - rowmap[v] == m.rowmap[v + 1] - m.rowmap[v], "row lengths differ from the mesh pattern");
      a.assign(cols + rowmap[v], cols + rowmap[v + 1]);
      b.assign(m.cols.begin() + m.rowmap[v], m.cols.begin() + m.rowmap[v + 1]);
      std::sort(a.begin(), a.end());
      std::sort(b.begin(), b.end());
      PA_CHECK(a == b, "row columns differ from the mesh pattern");
    }
    m.cols.assign(cols, cols + num_blocks);
    m.cols_sorted = true;
    for (int64_t v = 0; v < m.N && m.cols_sorted; ++v)
      m.cols_sorted = std::is_sorted(m.cols.begin() + m.rowmap[v], m.cols.begin() + m.rowmap[v + 1]);
    if (m.d_cell_entry.n) m.build_graph_entries();
  });
}

pa_status pa_write_vtu(const pa_mesh* mesh, const char* path, const double* u, const double* control,
                       int32_t control_layout) {
  return guard([&] {
    PA_CHECK(mesh && path, "null argument");
    PA_CHECK(control_layout == PA_CONTROL_NODAL || control_layout == PA_CONTROL_CELL, "unknown control layout");
    pa::write_vtu(mesh->m, path, u, control, control_layout);
  });
}

pa_status pa_mesh_boundary_faces(const pa_mesh* mesh, int32_t axis, double value, int32_t* faces,
                                 int64_t* num_faces) {
  return guard([&] {
    PA_CHECK(mesh && num_faces, "null argument");
    PA_CHECK(axis >= 0 && axis < 3, "axis must be 0, 1 or 2");
    const pa::Mesh& m = mesh->m;
    const double tol = 1e-12 * (1.0 + std::fabs(value));
    int64_t nf = 0;
    for (int64_t c = 0; c < m.C; ++c)
      for (int drop = 0; drop < 4; ++drop) {
        int32_t f[3];
        int k = 0;
        bool on = true;
        for (int n = 0; n < 4; ++n) {
          if (n == drop) continue;
          f[k++] = m.cells[4 * c + n];
          on = on && std::fabs(m.coords[3 * int64_t(m.cells[4 * c + n]) + axis] - value) <= tol;
        }
        if (!on) continue;
        if (faces) std::memcpy(faces + 3 * nf, f, sizeof(f));
        ++nf;
      }
    *num_faces = nf;
  });
}

pa_status pa_problem_create(pa_mesh* mesh, const pa_elastic_params* params, void* stream, pa_problem** out) {
  return guard([&] {
    PA_CHECK(mesh && params && out, "null argument");
    PA_CHECK(params->youngs_modulus > 0, "Youngs Modulus must be positive");
    PA_CHECK(params->poissons_ratio > -1.0 && params->poissons_ratio < 0.5, "Poissons Ratio must lie in (-1, 0.5)");
    PA_CHECK(params->control_layout == PA_CONTROL_NODAL || params->control_layout == PA_CONTROL_CELL,
             "unknown control layout");
    PA_CUDA(cudaSetDevice(mesh->m.device));
    std::unique_ptr<pa_problem> h(new pa_problem());
    Problem& P = h->P;
    PA_CHECK(!mesh->destroy_requested, "mesh already destroyed");
    P.mesh = &mesh->m;
    h->mesh = mesh;
    P.ep = pa::ElasticParams{params->youngs_modulus, params->poissons_ratio, params->simp_exponent, params->simp_min,
                             params->control_layout};
    if (stream) {
      P.stream = reinterpret_cast<cudaStream_t>(stream);
    } else {
      // a blocking stream: ordered against the legacy default stream, so that
      // a caller working there (e.g. torch's default stream) sees the
      // library's results, and the library sees the caller's inputs
      PA_CUDA(cudaStreamCreateWithFlags(&P.stream, cudaStreamDefault));
      P.own_stream = true;
    }
    upload_bcs(P);
    mesh->m.live_problems += 1;
    *out = h.release();
  });
}

pa_status pa_problem_destroy(pa_problem* problem) {
  return guard([&] {
    if (!problem) return;
    Problem& P = problem->P;
    pa_mesh* mh = problem->mesh;
    PA_CUDA(cudaSetDevice(P.mesh->device));
    cudaStreamSynchronize(P.stream);
    if (P.ev0) cudaEventDestroy(P.ev0);
    if (P.ev1) cudaEventDestroy(P.ev1);
    cudaStream_t s = P.own_stream ? P.stream : nullptr;
    pa_pc* pc = problem->pc;
    pa_pc* cpc = problem->cpc;
    pa::mg_release(P);
    pa::boxmg_release(P);
    delete problem;
    if (s) cudaStreamDestroy(s);
    mh->m.live_problems -= 1;
    if (mh->m.live_problems == 0 && mh->destroy_requested) delete mh;
    if (pc && --pc->attached == 0 && pc->destroy_requested) delete pc;
    if (cpc && --cpc->attached == 0 && cpc->destroy_requested) delete cpc;
  });
}

pa_status pa_problem_add_traction(pa_problem* problem, const int32_t* faces, int64_t num_faces, const double flux[3]) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(flux && (faces || num_faces == 0) && num_faces >= 0, "null argument");
    for (int64_t i = 0; i < 3 * num_faces; ++i)
      PA_CHECK(faces[i] >= 0 && faces[i] < P.N(), "face node id out of range");
    P.faces.insert(P.faces.end(), faces, faces + 3 * num_faces);
    for (int64_t f = 0; f < num_faces; ++f) P.face_flux.insert(P.face_flux.end(), flux, flux + 3);
    P.d_faces.upload(P.faces.data(), P.faces.size(), P.stream);
    P.d_face_flux.upload(P.face_flux.data(), P.face_flux.size(), P.stream);
    PA_CUDA(cudaStreamSynchronize(P.stream));
  });
}

pa_status pa_problem_clear_tractions(pa_problem* problem) {
  return guard([&] {
    Problem& P = prob(problem);
    P.faces.clear();
    P.face_flux.clear();
  });
}

pa_status pa_problem_set_dirichlet(pa_problem* problem, const int32_t* dofs, const double* values, int64_t n) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(n >= 0 && (n == 0 || (dofs && values)), "null argument");
    for (int64_t i = 0; i < n; ++i) {
      PA_CHECK(dofs[i] >= 0 && dofs[i] < P.ndof(), "Dirichlet dof out of range");
      PA_CHECK(std::isfinite(values[i]), "non-finite Dirichlet value");
    }
    P.bc_dofs.assign(dofs, dofs + n);
    P.bc_vals.assign(values, values + n);
    upload_bcs(P);
  });
}

// y = K(z) u (interleaved, unconstrained) through the FP64 tile kernel: the
// tets of a tile sum into shared memory and only nodes shared with other
// tiles are added globally, instead of 12 global atomics per tet.
static void apply_k64(Problem& P, const double* du, const double* dz, double* dy) {
  if (pa::box_entry_eligible(P)) {  // the box kernel, penalty and interleaving fused
    pa::box_entry_apply(P, dz, du, dy);
    return;
  }
  const int64_t n = P.ndof();
  P.ws.w64.resize(P.C());
  pa::launch_cell_weights(P, dz, P.ws.w64.get(), nullptr, P.stream);
  pa::DevBuf<double>& xs = P.ws.x;
  pa::DevBuf<double>& ys = P.ws.t;
  if (xs.n < size_t(n)) xs.resize(n);
  if (ys.n < size_t(n)) ys.resize(n);
  pa::launch_aos_to_soa<double, double>(du, xs.get(), P.N(), P.stream);
  pa::launch_apply_tiled<double>(P, P.ws.w64.get(), xs.get(), ys.get(), false, P.stream);
  pa::launch_soa_to_aos<double, double>(ys.get(), dy, P.N(), P.stream);
}

pa_status pa_vf_value(pa_problem* problem, const double* u, const double* z, double* r) {
  return guard([&] {
    Problem& P = prob(problem);
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.nz(), "z");
    double* dr = st.out(r, P.ndof(), "r");
    apply_k64(P, du, dz, dr);  // linear elasticity: the volume term is K(z) u
    pa::launch_traction(P, dr, -1.0, P.stream);
    st.finish();
  });
}

pa_status pa_vf_gradient_u(pa_problem* problem, const double* u, const double* z, double* entries) {
  return guard([&] {
    Problem& P = prob(problem);
    (void)u;  // K does not depend on u for linear elasticity; kept for the reference's signature
    if (!P.mesh->d_cell_entry.n) P.mesh->build_graph_entries();
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    double* de = st.out(entries, 9 * P.mesh->B, "entries");
    if (!pa::box_gradient_u(P, dz, de)) pa::launch_gradient_u(P, dz, de, P.stream);
    st.finish();
  });
}

pa_status pa_vf_gradient_z(pa_problem* problem, const double* u, const double* z, double* entries) {
  return guard([&] {
    Problem& P = prob(problem);
    if (!P.mesh->d_cell_entry.n) P.mesh->build_graph_entries();
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.nz(), "z");
    const int64_t n = P.ep.layout == PA_CONTROL_CELL ? 12 * P.C() : 3 * P.mesh->B;
    double* de = st.out(entries, n, "entries");
    if (pa::box_entry_eligible(P))
      pa::box_entry_gradient_z(P, dz, du, de);
    else
      pa::launch_gradient_z(P, du, dz, de, P.stream);
    st.finish();
  });
}

pa_status pa_vf_gradient_x(pa_problem* problem, const double* u, const double* z, double* entries) {
  return guard([&] {
    Problem& P = prob(problem);
    if (!P.mesh->d_cell_entry.n) P.mesh->build_graph_entries();
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.nz(), "z");
    double* de = st.out(entries, 9 * P.mesh->B, "entries");
    pa::launch_gradient_x(P, du, dz, de, P.stream);
    st.finish();
  });
}

pa_status pa_sf_gradient_x(pa_problem* problem, const double* u, const double* z, double* grad) {
  return guard([&] {
    Problem& P = prob(problem);
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.nz(), "z");
    double* dg = st.out(grad, P.ndof(), "grad");
    pa::launch_energy_grad_x(P, du, dz, dg, P.stream);
    st.finish();
  });
}

static void energy_call(pa_problem* problem, const double* u, const double* z, double* value, double* gu, double* gz) {
  Problem& P = prob(problem);
  pa::Stage st(P);
  const double* du = st.in(u, P.ndof(), "u");
  const double* dz = st.in(z, P.nz(), "z");
  double* dgu = gu ? st.out(gu, P.ndof(), "grad") : nullptr;
  double* dgz = gz ? st.out(gz, P.nz(), "grad") : nullptr;
  const int64_t grid = (P.C() + 255) / 256;
  if (value) {
    if (P.d_partials.n < size_t(grid)) P.d_partials.resize(grid);
    if (P.d_scalar.n < 2) P.d_scalar.resize(2);
  }
  if (!dgu && pa::box_entry_eligible(P))
    pa::box_entry_energy(P, dz, du, value ? P.d_scalar.get() : nullptr, dgz);
  else
    pa::launch_energy(P, du, dz, P.d_partials.get(), value ? P.d_scalar.get() : nullptr, dgu, dgz, P.stream);
  if (value) {
    PA_CUDA(cudaMemcpyAsync(value, P.d_scalar.get(), sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    PA_CUDA(cudaStreamSynchronize(P.stream));
  }
  st.finish();
}

pa_status pa_sf_value(pa_problem* problem, const double* u, const double* z, double* value) {
  return guard([&] {
    PA_CHECK(value, "null value pointer");
    energy_call(problem, u, z, value, nullptr, nullptr);
  });
}

pa_status pa_sf_gradient_u(pa_problem* problem, const double* u, const double* z, double* grad) {
  return guard([&] {
    PA_CHECK(grad, "null grad pointer");
    // f = 1/2 u^T K(z) u, so df/du = K(z) u
    Problem& P = prob(problem);
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.nz(), "z");
    double* dg = st.out(grad, P.ndof(), "grad");
    apply_k64(P, du, dz, dg);
    st.finish();
  });
}

pa_status pa_sf_gradient_z(pa_problem* problem, const double* u, const double* z, double* grad) {
  return guard([&] {
    PA_CHECK(grad, "null grad pointer");
    energy_call(problem, u, z, nullptr, nullptr, grad);
  });
}

pa_status pa_apply(pa_problem* problem, const double* z, const void* x, void* y, int32_t precision,
                   int32_t constrained) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(precision == PA_FP64 || precision == PA_FP32, "precision must be PA_FP64 or PA_FP32");
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    const int64_t n = P.ndof();
    P.ws.w64.resize(P.C());
    if (precision == PA_FP32) P.ws.w32.resize(P.C());
    pa::launch_cell_weights(P, dz, P.ws.w64.get(), precision == PA_FP32 ? P.ws.w32.get() : nullptr, P.stream);
    const int64_t nbc = constrained ? int64_t(P.bc_dofs.size()) : 0;
    const bool box = pa::box_apply_eligible(P);
    if (precision == PA_FP64) {
      const double* dx = st.in(static_cast<const double*>(x), n, "x");
      double* dy = st.out(static_cast<double*>(y), n, "y");
      pa::DevBuf<double>& xs = P.ws.x;
      pa::DevBuf<double>& ys = P.ws.t;
      if (xs.n < size_t(n)) xs.resize(n);
      if (ys.n < size_t(n)) ys.resize(n);
      if (box) {
        pa::box_apply<double>(P, dz, dx, dy, constrained != 0, xs.get(), ys.get());
      } else {
        pa::launch_aos_to_soa<double, double>(dx, xs.get(), P.N(), P.stream);
        pa::launch_apply_tiled<double>(P, P.ws.w64.get(), xs.get(), ys.get(), constrained != 0, P.stream);
        pa::launch_soa_to_aos<double, double>(ys.get(), dy, P.N(), P.stream);
      }
      pa::launch_copy_dofs<double>(P.d_bc_dofs.get(), nbc, dx, dy, P.stream);  // identity rows
    } else {
      const float* dx = st.in(static_cast<const float*>(x), n, "x");
      float* dy = st.out(static_cast<float*>(y), n, "y");
      pa::DevBuf<float>& xs = P.ws.r32;
      pa::DevBuf<float>& ys = P.ws.ap32;
      if (xs.n < size_t(n)) xs.resize(n);
      if (ys.n < size_t(n)) ys.resize(n);
      if (box) {
        pa::box_apply<float>(P, dz, dx, dy, constrained != 0, xs.get(), ys.get());
      } else {
        pa::launch_aos_to_soa<float, float>(dx, xs.get(), P.N(), P.stream);
        pa::launch_apply_tiled<float>(P, P.ws.w32.get(), xs.get(), ys.get(), constrained != 0, P.stream);
        pa::launch_soa_to_aos<float, float>(ys.get(), dy, P.N(), P.stream);
      }
      pa::launch_copy_dofs<float>(P.d_bc_dofs.get(), nbc, dx, dy, P.stream);
    }
    st.finish();
  });
}

pa_status pa_apply_block_constraints(pa_problem* problem, double* entries, double* rhs, double scale) {
  return guard([&] {
    Problem& P = prob(problem);
    if (!P.mesh->d_cell_entry.n) P.mesh->build_graph_entries();
    pa::Stage st(P);
    double* de = st.out(entries, 9 * P.mesh->B, "entries", true);
    double* dr = st.out(rhs, P.ndof(), "rhs", true);
    pa::launch_block_constraints(P, de, dr, scale, P.stream);
    st.finish();
  });
}

pa_status pa_solve_options_default(pa_solve_options* o) {
  return guard([&] {
    PA_CHECK(o, "null options");
    o->method = PA_SOLVER_PCG_FP64;
    o->rel_tol = 1e-10;
    o->max_iters = 0;
    o->check_every = 64;
    o->use_initial_guess = 0;
    o->mg_coarse_solver = PA_MG_COARSE_AUTO;
  });
}

pa_status pa_solve(pa_problem* problem, const double* z, const double* b, double* x, const pa_solve_options* options,
                   pa_solve_stats* stats) {
  return pa::guard_status([&] {
    Problem& P = prob(problem);
    pa_solve_options o;
    pa_solve_options_default(&o);
    if (options) o = *options;
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    const double* db = st.in(b, P.ndof(), "b");
    double* dx = st.out(x, P.ndof(), "x", o.use_initial_guess != 0);
    pa_status s = pa::solve_device(P, dz, db, dx, o, stats);
    st.finish();
    return s;
  });
}

pa_status pa_problem_solution(pa_problem* problem, const double* z, double* u, const pa_solve_options* options,
                              pa_solve_stats* stats) {
  return pa::guard_status([&] {
    Problem& P = prob(problem);
    pa_solve_options o;
    pa_solve_options_default(&o);
    if (options) o = *options;
    o.use_initial_guess = 0;
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    double* du = st.out(u, P.ndof(), "u");
    // R = value(0, z) = -F; solve K du = -R; u = du
    P.d_rhs.resize(P.ndof());
    double* rhs = P.d_rhs.get();
    PA_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * P.ndof(), P.stream));
    pa::launch_traction(P, rhs, 1.0, P.stream);  // -R(u=0) = F
    pa_status s = pa::solve_device(P, dz, rhs, du, o, stats);
    st.finish();
    return s;
  });
}

pa_status pa_problem_criterion_gradient(pa_problem* problem, const double* z, const double* u, double* grad,
                                        int32_t self_adjoint, const pa_solve_options* options) {
  return pa::guard_status([&] {
    Problem& P = prob(problem);
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.nz(), "z");
    double* dg = st.out(grad, P.nz(), "grad");
    pa::launch_energy(P, du, dz, nullptr, nullptr, nullptr, dg, P.stream);  // df/dz
    pa_status s = PA_OK;
    if (self_adjoint) {
      // -df/dz (src/elliptic/Problem.hpp:438-441)
      pa::launch_scale(dg, P.nz(), -1.0, P.stream);
    } else {
      // lambda: K lambda = -df/du with homogeneous BCs; g += (dR/dz)^T lambda
      pa_solve_options o;
      pa_solve_options_default(&o);
      if (options) o = *options;
      o.use_initial_guess = 0;
      pa::DevBuf<double> dfdu(P.ndof()), lam(P.ndof());
      pa::launch_energy(P, du, dz, nullptr, nullptr, dfdu.get(), nullptr, P.stream);
      pa::launch_scale(dfdu.get(), P.ndof(), -1.0, P.stream);
      std::vector<double> saved = P.bc_vals;
      std::fill(P.bc_vals.begin(), P.bc_vals.end(), 0.0);
      upload_bcs(P);
      s = pa::solve_device(P, dz, dfdu.get(), lam.get(), o, nullptr);
      P.bc_vals = saved;
      upload_bcs(P);
      pa::launch_dRdz_transpose_times(P, du, dz, lam.get(), dg, P.stream);
    }
    st.finish();
    return s;
  });
}

pa_status pa_j2_radial_return(pa_problem* problem, const pa_j2_params* params, const double* u, const double* z,
                              const double* prev_local, double* local) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(params, "null J2 parameters");
    PA_CHECK(params->youngs_modulus > 0 && params->initial_yield_stress > 0, "J2 moduli must be positive");
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.N(), "z");
    const double* dp = st.in(prev_local, 14 * P.C(), "prev_local");
    double* dl = st.out(local, 14 * P.C(), "local");
    pa::launch_j2(P, *params, du, dz, dp, dl, P.stream);
    st.finish();
  });
}

pa_status pa_time_apply(pa_problem* problem, const double* z, int32_t precision, int32_t reps,
                        double* ms_per_launch, int64_t* algorithmic_bytes) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(precision == PA_FP64 || precision == PA_FP32, "precision must be PA_FP64 or PA_FP32");
    PA_CHECK(reps > 0 && ms_per_launch, "need reps > 0 and an output");
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    if (pa::box_apply_eligible(P)) {
      // the box kernel: weights (one per hex when the six tets share it), x in,
      // y out and the node's Dirichlet mask; no connectivity, no coordinates
      int64_t nb = 0;
      *ms_per_launch = pa::time_box_apply(P, dz, precision == PA_FP32, reps, &nb);
      if (algorithmic_bytes) *algorithmic_bytes = nb;
    } else {
      *ms_per_launch = pa::time_apply(P, dz, precision == PA_FP32, reps);
      if (algorithmic_bytes) {
        const int64_t sv = precision == PA_FP32 ? 4 : 8;
        // cells: 4 int32 node ids + penalty weight; nodes: coords, x in, y out
        *algorithmic_bytes = P.C() * (16 + sv) + P.N() * (3 * sv) * 3;
      }
    }
    st.finish();
  });
}

pa_status pa_time_cg_apply(pa_problem* problem, const double* z, int32_t precision, int32_t reps,
                           double* ms_per_launch, int64_t* algorithmic_bytes) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(precision == PA_FP64 || precision == PA_FP32, "precision must be PA_FP64 or PA_FP32");
    PA_CHECK(reps > 0 && ms_per_launch, "need reps > 0 and an output");
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    *ms_per_launch = pa::time_cg_apply(P, dz, precision == PA_FP32, reps);
    if (algorithmic_bytes) {
      const int64_t sv = precision == PA_FP32 ? 4 : 8;
      // cells: 4 int32 node ids + penalty weight; nodes: coords, p_old, r, D^-1 in, p_new, K p out
      *algorithmic_bytes = P.C() * (16 + sv) + P.N() * (3 * sv) * 6;
    }
    st.finish();
  });
}

pa_status pa_j2_local_residual(pa_problem* problem, const pa_j2_params* params, const double* u, const double* z,
                               const double* local, const double* prev_local, double* residual) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(params, "null J2 parameters");
    pa::Stage st(P);
    const double* du = st.in(u, P.ndof(), "u");
    const double* dz = st.in(z, P.N(), "z");
    const double* dl = st.in(local, 14 * P.C(), "local");
    const double* dp = st.in(prev_local, 14 * P.C(), "prev_local");
    double* dh = st.out(residual, 14 * P.C(), "residual");
    pa::launch_j2_local_residual(P, *params, du, dz, dl, dp, dh, P.stream);
    st.finish();
  });
}

pa_status pa_up_residual(pa_problem* problem, const pa_up_params* params, const double* state, const double* local,
                         const double* ppg, int32_t ppg_per_cell, const double* z, double* residual,
                         int32_t assembled) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(params, "null u-p parameters");
    PA_CHECK(params->youngs_modulus > 0 && params->poissons_ratio > -1.0 && params->poissons_ratio < 0.5,
             "u-p moduli out of range");
    pa::Stage st(P);
    const double* ds = st.in(state, 4 * P.N(), "state");
    const double* dl = st.in(local, 14 * P.C(), "local");
    const double* dp = st.in(ppg, ppg_per_cell ? 12 * P.C() : 3 * P.N(), "projected pressure gradient");
    const double* dz = st.in(z, P.N(), "z");
    double* dr = st.out(residual, assembled ? 4 * P.N() : 16 * P.C(), "residual");
    pa::launch_up_residual(P, *params, ds, dl, dp, ppg_per_cell ? 1 : 0, dz, dr, assembled ? 1 : 0, P.stream);
    st.finish();
  });
}

pa_status pa_j2_solve(pa_problem* problem, const pa_j2_params* params, const double* z,
                      const pa_j2_solve_options* options, const pa_solve_options* linear, double* u, double* local,
                      pa_j2_stats* stats) {
  return pa::guard_status([&] {
    Problem& P = prob(problem);
    PA_CHECK(params && options, "null J2 parameters or options");
    PA_CHECK(params->youngs_modulus > 0 && params->initial_yield_stress > 0, "J2 moduli must be positive");
    pa_solve_options lo;
    pa_solve_options_default(&lo);
    if (linear) lo = *linear;
    lo.use_initial_guess = 0;
    pa::Stage st(P);
    const double* dz = st.in(z, P.N(), "z");
    double* du = st.out(u, P.ndof(), "u");
    double* dl = st.out(local, 14 * P.C(), "local");
    pa_status s = pa::j2_solve(P, *params, dz, *options, lo, du, dl, stats);
    st.finish();
    return s;
  });
}

pa_status pa_up_solve(pa_problem* problem, const pa_up_params* up, const pa_j2_params* params, const double* z,
                      const pa_j2_solve_options* options, const pa_solve_options* linear, double* state,
                      double* local, double* ppg, pa_j2_stats* stats) {
  return pa::guard_status([&] {
    Problem& P = prob(problem);
    PA_CHECK(up && params && options, "null u-p parameters or options");
    PA_CHECK(up->youngs_modulus > 0 && up->poissons_ratio > -1.0 && up->poissons_ratio < 0.5,
             "u-p moduli out of range");
    PA_CHECK(params->youngs_modulus > 0 && params->initial_yield_stress > 0, "J2 moduli must be positive");
    pa_solve_options lo;
    pa_solve_options_default(&lo);
    lo.rel_tol = 1e-12;
    lo.max_iters = 0;
    if (linear) lo = *linear;
    pa::Stage st(P);
    const double* dz = st.in(z, P.N(), "z");
    double* ds = st.out(state, 4 * P.N(), "state");
    double* dl = st.out(local, 14 * P.C(), "local");
    double* dp = ppg ? st.out(ppg, 3 * P.N(), "projected pressure gradient") : nullptr;
    pa_status s = pa::up_solve(P, *up, *params, dz, *options, lo, ds, dl, dp, stats);
    st.finish();
    return s;
  });
}

pa_status pa_up_elastic_work(pa_problem* problem, const pa_up_params* up, const pa_j2_params* params,
                             double penalty_exponent, double penalty_min, const double* z,
                             const pa_j2_solve_options* options, const pa_solve_options* linear, double* value,
                             double* gradient, double* state, double* local, pa_j2_stats* stats) {
  return pa::guard_status([&] {
    Problem& P = prob(problem);
    PA_CHECK(up && params && options && value, "null u-p parameters, options or value");
    PA_CHECK(up->youngs_modulus > 0 && up->poissons_ratio > -1.0 && up->poissons_ratio < 0.5,
             "u-p moduli out of range");
    PA_CHECK(params->youngs_modulus > 0 && params->initial_yield_stress > 0, "J2 moduli must be positive");
    pa_solve_options lo;
    pa_solve_options_default(&lo);
    lo.rel_tol = 1e-12;
    lo.max_iters = 0;
    if (linear) lo = *linear;
    pa::Stage st(P);
    const double* dz = st.in(z, P.N(), "z");
    double* dg = st.out(gradient, P.N(), "gradient");
    double* ds = st.out(state, 4 * P.N(), "state");
    double* dl = st.out(local, 14 * P.C(), "local");
    pa_status s = pa::up_elastic_work(P, *up, *params, penalty_exponent, penalty_min, dz, *options, lo, value, dg, ds,
                                      dl, stats);
    st.finish();
    return s;
  });
}

}  // extern "C"

/* ------------------------------------------------ learned preconditioner --- */

namespace {

pa::LearnedPC& pcref(pa_pc* h) {
  if (!h || !h->pc) throw Error(PA_ERR_INVALID_ARG, "null pa_pc");
  PA_CUDA(cudaSetDevice(pa::pc_device(*h->pc)));
  return *h->pc;
}

// Device view of a caller array for a network-only call (host arrays copied in).
template <typename T>
const T* pc_in(const T* p, int64_t count, pa::DevBuf<char>& tmp, cudaStream_t s, const char* name) {
  PA_CHECK(p != nullptr, std::string("null pointer: ") + name);
  if (pa::is_device_pointer(p)) return p;
  tmp.resize(size_t(count) * sizeof(T));
  PA_CUDA(cudaMemcpyAsync(tmp.get(), p, size_t(count) * sizeof(T), cudaMemcpyHostToDevice, s));
  return reinterpret_cast<const T*>(tmp.get());
}

// Device output for a network-only call; copied back to a host array by pc_out_finish.
template <typename T>
T* pc_out(T* p, int64_t count, pa::DevBuf<char>& tmp, const char* name) {
  PA_CHECK(p != nullptr, std::string("null pointer: ") + name);
  if (pa::is_device_pointer(p)) return p;
  tmp.resize(size_t(count) * sizeof(T));
  return reinterpret_cast<T*>(tmp.get());
}
template <typename T>
void pc_out_finish(T* p, const T* d, int64_t count, cudaStream_t s) {
  if (static_cast<const void*>(p) != static_cast<const void*>(d))
    PA_CUDA(cudaMemcpyAsync(p, d, size_t(count) * sizeof(T), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" {

pa_status pa_pc_create(int32_t gx, int32_t gy, int32_t gz, uint64_t seed, pa_pc** out) {
  return guard([&] {
    PA_CHECK(out, "null argument");
    pa::require_device();
    std::unique_ptr<pa_pc> h(new pa_pc());
    h->pc = pa::pc_new(gx, gy, gz, seed);
    *out = h.release();
  });
}

pa_status pa_pc_destroy(pa_pc* pc) {
  return guard([&] {
    if (!pc) return;
    if (pc->attached > 0) {
      pc->destroy_requested = true;  // released when the last problem using it detaches
      return;
    }
    if (pc->pc) PA_CUDA(cudaSetDevice(pa::pc_device(*pc->pc)));
    delete pc;
  });
}

pa_status pa_pc_num_params(const pa_pc* pc, int64_t* count) {
  return guard([&] {
    PA_CHECK(pc && count, "null argument");
    *count = pa::pc_num_params();
  });
}

pa_status pa_pc_get_params(pa_pc* pc, float* params) {
  return guard([&] {
    pa::LearnedPC& L = pcref(pc);
    cudaStream_t s = pa::pc_stream(L);
    pa::DevBuf<char> t;
    const int64_t n = pa::pc_num_params();
    float* d = pc_out(params, n, t, "params");
    pa::pc_get_params(L, d, s);
    pc_out_finish(params, d, n, s);
  });
}

pa_status pa_pc_set_params(pa_pc* pc, const float* params) {
  return guard([&] {
    pa::LearnedPC& L = pcref(pc);
    cudaStream_t s = pa::pc_stream(L);
    pa::DevBuf<char> t;
    pa::pc_set_params(L, pc_in(params, pa::pc_num_params(), t, s, "params"), s);
    PA_CUDA(cudaStreamSynchronize(s));
  });
}

pa_status pa_pc_forward(pa_pc* pc, const float* features, float* out) {
  return guard([&] {
    pa::LearnedPC& L = pcref(pc);
    cudaStream_t s = pa::pc_stream(L);
    const int64_t G = pa::pc_grid_points(L);
    pa::DevBuf<char> ti, to;
    const float* df = pc_in(features, 5 * G, ti, s, "features");
    float* dout = pc_out(out, 3 * G, to, "out");
    pa::pc_forward_features(L, df, dout, s);
    pc_out_finish(out, dout, 3 * G, s);
  });
}

pa_status pa_pc_backward(pa_pc* pc, const float* features, const float* grad_out, float* grad_params) {
  return guard([&] {
    pa::LearnedPC& L = pcref(pc);
    cudaStream_t s = pa::pc_stream(L);
    const int64_t G = pa::pc_grid_points(L), np = pa::pc_num_params();
    pa::DevBuf<char> tf, tg, to;
    const float* df = pc_in(features, 5 * G, tf, s, "features");
    const float* dg = pc_in(grad_out, 3 * G, tg, s, "grad_out");
    float* dp = pc_out(grad_params, np, to, "grad_params");
    pa::pc_backward_features(L, df, dg, dp, s);
    pc_out_finish(grad_params, dp, np, s);
  });
}

pa_status pa_pc_time_forward(pa_pc* pc, int32_t reps, double* ms_per_forward, int64_t* flops) {
  return guard([&] {
    pa::LearnedPC& L = pcref(pc);
    PA_CHECK(reps > 0 && ms_per_forward, "bad arguments");
    *ms_per_forward = pa::pc_time_forward(L, reps);
    if (flops) *flops = pa::pc_forward_flops(L);
  });
}

pa_status pa_pc_apply(pa_problem* problem, pa_pc* pc, const double* z, const double* r, double* out) {
  return guard([&] {
    Problem& P = prob(problem);
    pa::LearnedPC& L = pcref(pc);
    pa::pc_check_grid(L, *P.mesh);
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    const double* dr = st.in(r, P.ndof(), "r");
    double* dout = st.out(out, P.ndof(), "out");
    pa::pc_apply(L, P, dz, dr, dout);
    st.finish();
  });
}

pa_status pa_pc_train(pa_problem* problem, pa_pc* pc, int32_t num_densities, const double* densities,
                      int32_t num_samples, const int32_t* sample_density, const double* residuals,
                      const double* energies, const pa_pc_train_options* options, pa_pc_train_stats* stats) {
  return guard([&] {
    Problem& P = prob(problem);
    pa::LearnedPC& L = pcref(pc);
    PA_CHECK(options != nullptr, "null options");
    PA_CHECK(num_densities > 0 && num_samples > 0, "empty training set");
    PA_CHECK(sample_density && energies, "null argument");
    pa::pc_check_grid(L, *P.mesh);
    pa::Stage st(P);
    pa::PcTrainSet set;
    set.num_densities = num_densities;
    set.num_samples = num_samples;
    set.densities = st.in(densities, int64_t(num_densities) * P.nz(), "densities");
    set.residuals = st.in(residuals, int64_t(num_samples) * P.ndof(), "residuals");
    set.sample_density.resize(num_samples);
    set.sample_energy.resize(num_samples);
    if (pa::is_device_pointer(sample_density))
      PA_CUDA(cudaMemcpy(set.sample_density.data(), sample_density, sizeof(int32_t) * num_samples,
                         cudaMemcpyDeviceToHost));
    else
      std::copy(sample_density, sample_density + num_samples, set.sample_density.begin());
    if (pa::is_device_pointer(energies))
      PA_CUDA(cudaMemcpy(set.sample_energy.data(), energies, sizeof(double) * num_samples, cudaMemcpyDeviceToHost));
    else
      std::copy(energies, energies + num_samples, set.sample_energy.begin());
    pa::pc_train(L, P, set, *options, stats);
    st.finish();
  });
}

pa_status pa_problem_set_preconditioner(pa_problem* problem, pa_pc* pc) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(P.ep.layout == PA_CONTROL_CELL || P.ep.layout == PA_CONTROL_NODAL, "bad problem");
    auto detach = [&]() {
      pa_pc* old = problem->pc;
      problem->pc = nullptr;
      P.pc = nullptr;
      if (old && --old->attached == 0 && old->destroy_requested) delete old;
    };
    if (!pc) {
      detach();
      return;
    }
    PA_CHECK(!pc->destroy_requested, "network already destroyed");
    pa::LearnedPC& L = pcref(pc);
    PA_CHECK(pa::pc_device(L) == P.mesh->device, "network and problem live on different devices");
    pa::pc_check_grid(L, *P.mesh);
    if (problem->pc == pc) return;
    detach();
    problem->pc = pc;
    pc->attached += 1;
    P.pc = &L;
  });
}

pa_status pa_problem_set_coarse_network(pa_problem* problem, pa_pc* pc) {
  return guard([&] {
    Problem& P = prob(problem);
    auto detach = [&]() {
      pa_pc* old = problem->cpc;
      problem->cpc = nullptr;
      P.coarse_pc = nullptr;
      if (old && --old->attached == 0 && old->destroy_requested) delete old;
    };
    if (!pc) {
      detach();
      return;
    }
    PA_CHECK(!pc->destroy_requested, "network already destroyed");
    pa::LearnedPC& L = pcref(pc);
    PA_CHECK(pa::pc_device(L) == P.mesh->device, "network and problem live on different devices");
    int dims[3];
    PA_CHECK(pa::boxmg_coarse_grid(P, dims), "the problem's mesh has no box multigrid");
    PA_CHECK(pa::pc_grid_points(L) == int64_t(dims[0]) * dims[1] * dims[2],
             "the network's grid is not the level-1 hex grid (pa_boxmg_coarse_grid)");
    if (problem->cpc == pc) return;
    detach();
    problem->cpc = pc;
    pc->attached += 1;
    P.coarse_pc = &L;
  });
}

pa_status pa_boxmg_coarse_grid(pa_problem* problem, int32_t dims[3]) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(dims, "null argument");
    int d[3];
    PA_CHECK(pa::boxmg_coarse_grid(P, d), "the problem's mesh has no box multigrid");
    for (int a = 0; a < 3; ++a) dims[a] = d[a];
  });
}

pa_status pa_boxmg_coarse_features(pa_problem* problem, const double* z, float* features) {
  return guard([&] {
    Problem& P = prob(problem);
    int d[3];
    PA_CHECK(pa::boxmg_coarse_grid(P, d), "the problem's mesh has no box multigrid");
    const int64_t H1 = int64_t(d[0]) * d[1] * d[2];
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    float* df = st.out(features, 5 * H1, "features");
    pa::boxmg_coarse_features(P, dz, df);
    st.finish();
  });
}

pa_status pa_boxmg_coarse_sensitivity(pa_problem* problem, const double* z, const float* delta,
                                      int32_t num_residuals, const double* residuals, const double* energies,
                                      double* loss, float* grad_delta) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(loss && energies && num_residuals > 0, "null argument or no residuals");
    int d[3];
    PA_CHECK(pa::boxmg_coarse_grid(P, d), "the problem's mesh has no box multigrid");
    const int64_t H1 = int64_t(d[0]) * d[1] * d[2];
    std::vector<double> en(static_cast<size_t>(num_residuals));
    if (pa::is_device_pointer(energies))
      PA_CUDA(cudaMemcpy(en.data(), energies, sizeof(double) * en.size(), cudaMemcpyDeviceToHost));
    else
      std::copy(energies, energies + num_residuals, en.begin());
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    const float* dd = st.in(delta, H1, "delta");
    const double* dr = st.in(residuals, int64_t(num_residuals) * P.ndof(), "residuals");
    float* dg = st.out(grad_delta, H1, "grad_delta");
    pa::boxmg_coarse_sensitivity(P, dz, dd, num_residuals, dr, en.data(), loss, dg);
    st.finish();
  });
}

/* ------------------------------------------------------ batched solves --- */

pa_status pa_mesh_set_parts(pa_mesh* mesh, int32_t num_parts, const int64_t* node_offsets) {
  return guard([&] {
    PA_CHECK(mesh && node_offsets, "null argument");
    pa::Mesh& m = mesh->m;
    PA_CHECK(m.live_problems == 0, "set the parts before creating problems on the mesh");
    PA_CHECK(num_parts >= 1 && num_parts <= pa::kMaxParts, "num_parts out of range");
    PA_CHECK(node_offsets[0] == 0 && node_offsets[num_parts] == m.N, "part node offsets must run from 0 to N");
    for (int32_t p = 0; p < num_parts; ++p) PA_CHECK(node_offsets[p + 1] > node_offsets[p], "empty or unsorted part");
    PA_CUDA(cudaSetDevice(m.device));
    std::vector<int64_t> saved = m.part_node_offsets;
    const int32_t saved_n = m.num_parts;
    m.num_parts = num_parts;
    m.part_node_offsets.assign(node_offsets, node_offsets + num_parts + 1);
    try {
      pa::mesh_rebuild_tiles(m);
    } catch (...) {
      m.num_parts = saved_n;
      m.part_node_offsets = saved;
      pa::mesh_rebuild_tiles(m);
      throw;
    }
  });
}

pa_status pa_mesh_uniform_geometry(pa_mesh* mesh, int32_t enable, int32_t* active) {
  return guard([&] {
    PA_CHECK(mesh, "null pa_mesh");
    pa::Mesh& m = mesh->m;
    if (enable >= 0 && bool(enable) != m.allow_uniform_geometry) {
      PA_CHECK(m.live_problems == 0, "change the geometry mode before creating problems on the mesh");
      PA_CUDA(cudaSetDevice(m.device));
      m.allow_uniform_geometry = enable != 0;
      pa::mesh_rebuild_tiles(m);
    }
    if (active) *active = m.uniform_hex ? 1 : 0;
  });
}

pa_status pa_mesh_box_kernels(pa_mesh* mesh, int32_t enable, int32_t* active) {
  return guard([&] {
    PA_CHECK(mesh, "null pa_mesh");
    pa::Mesh& m = mesh->m;
    if (enable >= 0) m.box_kernels = enable != 0;
    if (active) *active = (m.box_kernels && m.lat_n[0] > 0) ? 1 : 0;
  });
}

pa_status pa_problem_part_stats(pa_problem* problem, int32_t* iterations, double* rel_residuals) {
  return guard([&] {
    Problem& P = prob(problem);
    PA_CHECK(!P.part_iterations.empty(), "no batched solve has run on this problem");
    if (iterations) std::copy(P.part_iterations.begin(), P.part_iterations.end(), iterations);
    if (rel_residuals) std::copy(P.part_rel_residual.begin(), P.part_rel_residual.end(), rel_residuals);
  });
}

pa_status pa_problem_autotune_tiles(pa_problem* problem, const double* z, int32_t* tile_clusters,
                                    double* ms_per_apply) {
  return guard([&] {
    Problem& P = prob(problem);
    pa::Mesh& m = *P.mesh;
    PA_CHECK(m.live_problems == 1, "autotuning rebuilds the mesh's tiles: the problem must be its mesh's only one");
    pa::Stage st(P);
    const double* dz = st.in(z, P.nz(), "z");
    const int sizes[3] = {64, 128, 256};
    double best = 1e300;
    int best_k = m.tile_clusters;
    for (int i = 0; i < 3; ++i) {
      m.tile_clusters = sizes[i];
      pa::mesh_rebuild_tiles(m);
      upload_bcs(P);
      pa::time_cg_apply(P, dz, true, 3);  // warm
      const double ms = pa::time_cg_apply(P, dz, true, 10);
      if (ms_per_apply) ms_per_apply[i] = ms;
      if (ms < best) {
        best = ms;
        best_k = sizes[i];
      }
    }
    m.tile_clusters = best_k;
    pa::mesh_rebuild_tiles(m);
    upload_bcs(P);
    if (tile_clusters) *tile_clusters = best_k;
    st.finish();
  });
}

}  // extern "C"
