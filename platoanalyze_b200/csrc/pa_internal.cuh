// pa_internal.cuh -- shared declarations of libpa_b200 (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <stdexcept>

#include "pa_b200.h"  // include/ is on the compiler include path

namespace pa {

// ------------------------------------------------------------------ errors --
struct Error : public std::runtime_error {
  pa_status status;
  Error(pa_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);

#define PA_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      throw ::pa::Error(PA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + \
                                         __FILE__ + ":" + std::to_string(__LINE__));               \
  } while (0)

#define PA_CHECK(cond, msg)                                         \
  do {                                                              \
    if (!(cond)) throw ::pa::Error(PA_ERR_INVALID_ARG, (msg));      \
  } while (0)

// Launch-error check after a kernel launch.
#define PA_LAUNCHED() PA_CUDA(cudaGetLastError())

// ----------------------------------------------------------- device buffer --
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { resize(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void resize(size_t count) {
    if (count == n && p) return;
    release();
    if (count) PA_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void upload(const T* h, size_t count, cudaStream_t s = 0) {
    resize(count);
    if (count) PA_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  T* get() const { return p; }
};

// ------------------------------------------------------------- tile layout --
// Cells are grouped into clusters (six tets of one hex, or a single tet) and
// clusters into tiles of at most tile_clusters clusters (64, 128 or 256)
// touching at most 2 * tile_clusters distinct nodes.  A tile's nodes are staged in shared memory;
// each cluster stores up to 8 tile-local node ids as uint16.  tile_nodes
// entries are a 27-bit node id plus flags: kShared (the node also belongs to
// another tile, so its sum is added atomically), kOwner (this tile writes
// per-node outputs of the node; exactly one tile per node) and three
// Dirichlet-mask bits (bit d: dof d constrained; set in a problem's copy).
constexpr int kMaxTileClusters = 256;  // tile sizes: 64, 128 or 256 clusters (= threads per CTA)
constexpr uint32_t kShared = 0x80000000u;
constexpr uint32_t kOwner = 0x40000000u;
constexpr int kMaskShift = 27;
constexpr uint32_t kNodeIdMask = (1u << kMaskShift) - 1u;

struct TileView {
  const int32_t* tile_cluster_start;  // T+1
  const int32_t* tile_cell_start;     // T+1, internal cell index
  const int32_t* tile_hex_count;      // T: the first tile_hex_count clusters of a tile are hexes
  const int32_t* tile_node_start;     // T+1
  const uint32_t* tile_nodes;         // flagged global node ids
  const uint4* cluster_nodes;         // 8 x uint16 tile-local node ids (hex slot order / cell order)
  const int32_t* cell_perm;           // C, internal -> user cell id
  int32_t num_tiles;
};

// Geometry shared by every hex cluster of a mesh whose hexes are translates
// of one another (a structured voxel grid): per template tet k the rows of
// det * J^-1 (h[k][0..2] for the tet's vertices 0, a, b in the tile kernel's
// relative form) and s[k] = 1 / (6 |det|).  The tile kernel reads it from its
// parameter block instead of recomputing the geometry per tet.
template <typename T>
struct HexGeo {
  T h[6][9];
  T s[6];
};

struct Mesh {
  int device = 0;
  int64_t C = 0, N = 0, B = 0, T = 0;
  std::vector<int32_t> cells;    // C*4 user order
  std::vector<double> coords;    // N*3
  std::vector<int32_t> rowmap;   // N+1
  std::vector<int32_t> cols;     // B
  DevBuf<int32_t> d_cells;
  DevBuf<double> d_coords;           // N*3 interleaved (cell kernels)
  DevBuf<double> d_coords_soa;       // 3N component-major (tile kernel, FP64)
  DevBuf<float> d_coords32_soa;      // 3N component-major (tile kernel, FP32)
  DevBuf<float4> d_coords32_aos4;    // N x (x, y, z, 0): one 16-byte gather per node (FP32 PCG modes)
  DevBuf<int32_t> d_rowmap, d_cols;
  DevBuf<int32_t> d_cell_entry;  // C*16 CRS block index of (a,b) pairs
  bool cols_sorted = true;       // every row's columns in increasing node order
  int64_t num_clusters = 0, num_hex = 0;
  // every cluster a hex and every hex a translate of the first (edge vectors
  // equal to 1e-9 of the hex size): the FP32 tile kernel then takes the
  // geometry from geo32 and gathers no coordinates; the FP64 kernel does the
  // same from geo64 when the largest deviation (hex_geo_dev, relative to the
  // hex size) is at rounding level, <= 1e-12
  bool uniform_hex = false;
  double hex_geo_dev = 0.0;
  bool allow_uniform_geometry = true;  // false: always the per-tet geometry
  HexGeo<double> geo64{};
  HexGeo<float> geo32{};
  int tile_clusters = 128;  // clusters per tile (threads per CTA); a tile touches <= 2x as many nodes
  // structured box (mesh_make_box): hex counts and lengths; 0 for other meshes
  int box_n[3] = {0, 0, 0};
  double box_l[3] = {0.0, 0.0, 0.0};
  bool box_kernels = true;  // structured boxes: apply and multigrid on the box kernel (pa_box.cuh)
  // Lattice of the box kernels: set for mesh_make_box boxes (identity
  // numbering) and for meshes given as arrays that are such a box under some
  // numbering (detect_lattice, pa_lattice.cu); lat_n[0] == 0 otherwise.
  int lat_n[3] = {0, 0, 0};
  double lat_l[3] = {0.0, 0.0, 0.0};
  bool lat_permuted = false;           // the caller's numbering differs from the lattice order
  int lat_flip = 0;                    // bit a: lattice axis a runs against the caller's axis a
                                       // (vector components along it change sign)
  DevBuf<int32_t> d_lat_node;          // lattice node -> caller's node (permuted only)
  DevBuf<int32_t> d_lat_of_node;       // caller's node -> lattice node (permuted only)
  DevBuf<int32_t> d_lat_cell;          // 6 h + t (hex h, box template tet t) -> caller's cell (permuted only)
  std::vector<int32_t> h_lat_of_node;  // caller's node -> lattice node (permuted only)
  DevBuf<int32_t> d_tile_cluster_start, d_tile_cell_start, d_tile_hex_count, d_tile_node_start, d_cell_perm;
  DevBuf<int32_t> d_cell_iperm;  // user -> internal cell id
  DevBuf<uint32_t> d_tile_nodes;
  DevBuf<uint4> d_cluster_nodes;
  std::vector<int32_t> h_cell_perm;  // internal -> user
  std::vector<uint32_t> h_tile_nodes; // flagged ids without mask bits
  // Parts: independent sub-meshes solved side by side (batched solves).  Part
  // p owns nodes [part_node_offsets[p], part_node_offsets[p+1]); no cell spans
  // two parts and no tile holds cells of two parts.
  int32_t num_parts = 1;
  int32_t live_problems = 0;               // problems created on this mesh and not destroyed
  std::vector<int64_t> part_node_offsets;  // P+1 (empty: one part)
  std::vector<int32_t> h_tile_part;        // T
  DevBuf<uint16_t> d_node_part;            // N (parts > 1)
  DevBuf<int32_t> d_tile_part;             // T (parts > 1)
  TileView tiles() const {
    return TileView{d_tile_cluster_start.get(), d_tile_cell_start.get(), d_tile_hex_count.get(),
                    d_tile_node_start.get(), d_tile_nodes.get(), d_cluster_nodes.get(), d_cell_perm.get(), int32_t(T)};
  }
  void build_graph_entries();
};

void mesh_build(Mesh& m);  // tiles + graph + device upload
// Recognise a mesh given as arrays as a box of equal axis-aligned hexes, each
// split into the six tets of mesh_make_box (up to a reflection of the axes),
// under any node, cell and vertex numbering; sets lat_* (pa_lattice.cu).
void detect_lattice(Mesh& m);
// Structured box [0,lx]x[0,ly]x[0,lz] of nx*ny*nz hexes x 6 tets (nodes and
// hexes numbered x fastest), then mesh_build.
void mesh_make_box(Mesh& m, int nx, int ny, int nz, double lx, double ly, double lz);
// .vtu output of the mesh, u (3N or null) and the control (N or C values, or null)
void write_vtu(const Mesh& m, const std::string& path, const double* u, const double* control, int control_layout);
void mesh_rebuild_tiles(Mesh& m);  // tiles only (after a change of parts or tile size)

// ----------------------------------------------------------------- material --
template <typename T>
struct Iso {
  T lam, mu;  // Lame parameters; C = lam I(x)I + 2 mu on normal, mu on engineering shear
};

struct ElasticParams {
  double E, nu, p, pmin;
  int layout;
  Iso<double> iso() const {
    double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    return Iso<double>{c * nu, 0.5 * c * (1.0 - 2.0 * nu)};
  }
};

// Per-iteration scalars of the PCG kernels, resident in device memory.
struct PcgScalars {
  double rz;       // r . z of the current residual
  double rz_prev;  // previous r . z
  double pap;      // p . K p
  double alpha, beta;
  double rr;       // ||r||^2 (recursive residual)
  double bb;       // ||b||^2
  double stop2;    // stop when rr <= stop2
  int32_t done;    // 1 once converged (kernels become no-ops)
  int32_t breakdown;
  int32_t iters;   // iterations completed
  int32_t pad;
};

// Per-part scalars of the batched PCG (one independent CG per part).
struct PartScalars {
  double rz, pap, alpha, beta, rr, stop2;
  int32_t done, breakdown, iters, pad;
};
constexpr int kMaxParts = 4096;

struct Problem;

// ------------------------------------------------------------ kernel APIs --
// (implemented in pa_elastic.cu)
void launch_traction(const Problem& P, double* r, double scale, cudaStream_t s);
void launch_gradient_u(const Problem& P, const double* z, double* entries, cudaStream_t s);
void launch_gradient_z(const Problem& P, const double* u, const double* z, double* entries, cudaStream_t s);
void launch_energy(const Problem& P, const double* u, const double* z, double* cell_partials /*>=grid*/,
                   double* value_out /*device scalar or null*/, double* grad_u, double* grad_z, cudaStream_t s);
void launch_cell_weights(const Problem& P, const double* z, double* w64, float* w32, cudaStream_t s);
// y = K x with the tile kernel on component-major (SoA) vectors;
// constrained = mask the problem's Dirichlet dofs.
template <typename T>
void launch_apply_tiled(const Problem& P, const T* w, const T* x, T* y, bool constrained, cudaStream_t s,
                        const T* plas = nullptr);
// interleaved (AoS, the ABI's layout) <-> component-major (SoA) copies
template <typename S, typename T>
void launch_aos_to_soa(const S* aos, T* soa, int64_t N, cudaStream_t s);
template <typename T, typename S>
void launch_soa_to_aos(const T* soa, S* aos, int64_t N, cudaStream_t s);
template <typename T>
void launch_copy_dofs(const int32_t* dofs, int64_t n, const T* src, T* dst, cudaStream_t s);
void launch_diag(const Problem& P, const double* w, double* diag, cudaStream_t s);
void launch_j2(const Problem& P, const pa_j2_params& jp, const double* u, const double* z, const double* prev,
               double* cur, cudaStream_t s);
void launch_up_residual(const Problem& P, const pa_up_params& up, const double* state, const double* local,
                        const double* ppg, int ppg_per_cell, const double* z, double* out, int assemble,
                        cudaStream_t s);

// out[v] = (soa[v], soa[N + v], soa[2N + v], 0)
void launch_pack4(int64_t N, const float* soa, float4* out, cudaStream_t s);

int num_sms();

}  // namespace pa
