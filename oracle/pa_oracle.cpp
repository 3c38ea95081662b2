// pa_oracle.cpp -- FP64 CPU restatement of Plato Analyze's linear-tet
// elastostatics / compliance / J2 radial-return hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
// platoanalyze_b200/: only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it.  Nothing in the shipped library links it.
//
// Structure deliberately mirrors the reference (gather -> per-cell functors ->
// atomic scatter-add), with derivatives produced by a forward-mode dual number
// of our own (the role Sacado SFad plays in the reference), so that the CUDA
// product's hand-derived gradients are checked against an independent
// differentiation route.  Each function names the reference lines it restates
// (paths relative to the platoanalyze source tree).
//
// Build: oracle/build.py  ->  oracle/_build/libpa_oracle.so  (g++ -O3 -fopenmp)

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

// ---------------------------------------------------------------------------
// Forward-mode dual number (value + N partials).  Plays the role of
// Sacado::Fad::SFad<double,N> (src/SimplexFadTypes.hpp:13-15).
// ---------------------------------------------------------------------------
template <int N>
struct Dual {
  double v;
  double d[N];
  Dual() : v(0) { for (int i = 0; i < N; ++i) d[i] = 0; }
  Dual(double x) : v(x) { for (int i = 0; i < N; ++i) d[i] = 0; }
};
template <int N> inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v + b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
template <int N> inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v - b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
template <int N> inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v * b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <int N> inline Dual<N> operator*(double s, const Dual<N>& a) { Dual<N> r; r.v = s * a.v; for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i]; return r; }
template <int N> inline Dual<N> operator*(const Dual<N>& a, double s) { return s * a; }
template <int N> inline Dual<N> operator/(const Dual<N>& a, double s) { return (1.0 / s) * a; }
template <int N> inline Dual<N> operator+(double s, const Dual<N>& a) { Dual<N> r = a; r.v += s; return r; }
template <int N> inline Dual<N> operator+(const Dual<N>& a, double s) { return s + a; }
template <int N> inline Dual<N> operator-(const Dual<N>& a, double s) { Dual<N> r = a; r.v -= s; return r; }
template <int N> inline Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { a = a + b; return a; }
template <int N> inline Dual<N> dpow(const Dual<N>& a, double p) {
  Dual<N> r; r.v = std::pow(a.v, p);
  double dp = (a.v == 0.0) ? (p == 1.0 ? 1.0 : 0.0) : p * std::pow(a.v, p - 1.0);
  for (int i = 0; i < N; ++i) r.d[i] = dp * a.d[i];
  return r;
}
inline double dpow(double a, double p) { return std::pow(a, p); }
template <int N> inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r; r.v = a.v / b.v;
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v);
  return r;
}
template <int N> inline Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }
template <int N> inline Dual<N> operator-(const Dual<N>& a) { Dual<N> r; r.v = -a.v; for (int i = 0; i < N; ++i) r.d[i] = -a.d[i]; return r; }
template <int N> inline Dual<N> dabs(const Dual<N>& a) { return a.v < 0 ? -a : a; }
inline double dabs(double a) { return std::fabs(a); }
template <int N> inline Dual<N> dsqrt(const Dual<N>& a) {
  Dual<N> r; r.v = std::sqrt(a.v);
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / (2.0 * r.v);
  return r;
}
inline double dsqrt(double a) { return std::sqrt(a); }
inline double val(double x) { return x; }
template <int N> inline double val(const Dual<N>& x) { return x.v; }

struct Elastic {
  double C[6][6];
  double simp_p, simp_min;
};

// Isotropic stiffness, IsotropicLinearElasticMaterial<3> ctor
// (src/IsotropicLinearElasticMaterial.cpp:86-108): lambda+2mu diagonal,
// lambda off-diagonal, mu on the (engineering) shear terms.
Elastic make_elastic(double E, double nu, double p, double pmin) {
  Elastic m;
  std::memset(m.C, 0, sizeof(m.C));
  double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m.C[i][j] = c * nu;
  for (int i = 0; i < 3; ++i) { m.C[i][i] = c * (1.0 - nu); m.C[i + 3][i + 3] = 0.5 * c * (1.0 - 2.0 * nu); }
  m.simp_p = p;
  m.simp_min = pmin;
  return m;
}

// ComputeGradientWorkset<3> (src/ImplicitFunctors.hpp:165-217): J columns are
// x_n - x_3, gradients are the rows of J^-1, node 3 closes the partition of
// unity, volume = |det J|; the caller multiplies by the 1-point weight 1/6
// (src/elliptic/ElastostaticResidual.hpp:181-182).
void cell_gradients(const double X[4][3], double g[4][3], double& vol) {
  double j11 = X[0][0] - X[3][0], j12 = X[1][0] - X[3][0], j13 = X[2][0] - X[3][0];
  double j21 = X[0][1] - X[3][1], j22 = X[1][1] - X[3][1], j23 = X[2][1] - X[3][1];
  double j31 = X[0][2] - X[3][2], j32 = X[1][2] - X[3][2], j33 = X[2][2] - X[3][2];
  double det = j11 * j22 * j33 + j12 * j23 * j31 + j13 * j21 * j32 - j11 * j23 * j32 - j12 * j21 * j33 - j13 * j22 * j31;
  g[0][0] = (j22 * j33 - j23 * j32) / det; g[0][1] = (j13 * j32 - j12 * j33) / det; g[0][2] = (j12 * j23 - j13 * j22) / det;
  g[1][0] = (j23 * j31 - j21 * j33) / det; g[1][1] = (j11 * j33 - j13 * j31) / det; g[1][2] = (j13 * j21 - j11 * j23) / det;
  g[2][0] = (j21 * j32 - j22 * j31) / det; g[2][1] = (j12 * j31 - j11 * j32) / det; g[2][2] = (j11 * j22 - j12 * j21) / det;
  for (int d = 0; d < 3; ++d) g[3][d] = -(g[0][d] + g[1][d] + g[2][d]);
  vol = std::fabs(det) / 6.0;
}

// Same as cell_gradients for a differentiable configuration type (gradient_x).
template <typename T>
void cell_gradients_t(const T X[4][3], T g[4][3], T& vol) {
  T j11 = X[0][0] - X[3][0], j12 = X[1][0] - X[3][0], j13 = X[2][0] - X[3][0];
  T j21 = X[0][1] - X[3][1], j22 = X[1][1] - X[3][1], j23 = X[2][1] - X[3][1];
  T j31 = X[0][2] - X[3][2], j32 = X[1][2] - X[3][2], j33 = X[2][2] - X[3][2];
  T det = j11 * j22 * j33 + j12 * j23 * j31 + j13 * j21 * j32 - j11 * j23 * j32 - j12 * j21 * j33 - j13 * j22 * j31;
  g[0][0] = (j22 * j33 - j23 * j32) / det; g[0][1] = (j13 * j32 - j12 * j33) / det; g[0][2] = (j12 * j23 - j13 * j22) / det;
  g[1][0] = (j23 * j31 - j21 * j33) / det; g[1][1] = (j11 * j33 - j13 * j31) / det; g[1][2] = (j13 * j21 - j11 * j23) / det;
  g[2][0] = (j21 * j32 - j22 * j31) / det; g[2][1] = (j12 * j31 - j11 * j32) / det; g[2][2] = (j11 * j22 - j12 * j21) / det;
  for (int d = 0; d < 3; ++d) g[3][d] = -(g[0][d] + g[1][d] + g[2][d]);
  vol = dabs(det) / 6.0;
}

// Strain<3> (src/Strain.hpp:56-94): Voigt {xx,yy,zz,yz,xz,xy}, engineering shears.
template <typename T, typename G>
void strain(const G g[4][3], const T u[12], T e[6]) {
  for (int i = 0; i < 6; ++i) e[i] = T(0.0);
  for (int n = 0; n < 4; ++n) {
    e[0] += u[3 * n + 0] * g[n][0];
    e[1] += u[3 * n + 1] * g[n][1];
    e[2] += u[3 * n + 2] * g[n][2];
    e[3] += u[3 * n + 2] * g[n][1] + u[3 * n + 1] * g[n][2];
    e[4] += u[3 * n + 2] * g[n][0] + u[3 * n + 0] * g[n][2];
    e[5] += u[3 * n + 1] * g[n][0] + u[3 * n + 0] * g[n][1];
  }
}

// LinearStress<3> (src/LinearStress.hpp:61-77) with zero reference strain.
template <typename T>
void stress(const Elastic& m, const T e[6], T s[6]) {
  for (int i = 0; i < 6; ++i) {
    s[i] = T(0.0);
    for (int j = 0; j < 6; ++j) s[i] += e[j] * m.C[i][j];
  }
}

// MSIMP (src/Simp.hpp:130-134).
template <typename T>
T simp(const Elastic& m, const T& rho) {
  return m.simp_min + (1.0 - m.simp_min) * dpow(rho, m.simp_p);
}

// StressDivergence<3> (src/StressDivergence.hpp:70-90).
template <typename T, typename G, typename V>
void divergence(const G g[4][3], V vol, const T s[6], T r[12]) {
  static const int voigt[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
  for (int i = 0; i < 3; ++i)
    for (int n = 0; n < 4; ++n)
      for (int j = 0; j < 3; ++j) r[3 * n + i] += vol * s[voigt[i][j]] * g[n][j];
}

void gather_X(const int32_t* cells, const double* coords, int64_t c, double X[4][3]) {
  for (int n = 0; n < 4; ++n) {
    int64_t v = cells[4 * c + n];
    for (int d = 0; d < 3; ++d) X[n][d] = coords[3 * v + d];
  }
}

// Cell density: mean of the 4 nodal controls (src/ApplyWeighting.hpp:56-60)
// for the nodal layout; the per-cell layout reads one value per cell.
template <typename T>
T cell_rho(const T zc[4], int layout) {
  if (layout == 1) return zc[0];
  return (zc[0] + zc[1] + zc[2] + zc[3]) / 4.0;
}

// Residual of one cell: ElastostaticResidual::evaluate
// (src/elliptic/ElastostaticResidual.hpp:147-214).
template <typename TU, typename TZ, typename TR>
void cell_residual(const Elastic& m, const double g[4][3], double vol, const TU u[12], const TZ zc[4], int layout, TR r[12]) {
  TU e[6], s[6];
  strain(g, u, e);
  stress(m, e, s);
  TZ w = simp(m, cell_rho(zc, layout));
  TR sw[6];
  for (int i = 0; i < 6; ++i) sw[i] = s[i] * w;
  for (int i = 0; i < 12; ++i) r[i] = TR(0.0);
  divergence(g, vol, sw, r);
}

// Internal elastic energy of one cell: InternalElasticEnergy::evaluate
// (src/elliptic/InternalElasticEnergy.hpp:100-158), ScalarProduct scale 0.5
// (src/ScalarProduct.hpp:28-42).
template <typename TU, typename TZ, typename TR>
TR cell_energy(const Elastic& m, const double g[4][3], double vol, const TU u[12], const TZ zc[4], int layout) {
  TU e[6], s[6];
  strain(g, u, e);
  stress(m, e, s);
  TZ w = simp(m, cell_rho(zc, layout));
  TR acc = TR(0.0);
  for (int i = 0; i < 6; ++i) acc += (s[i] * w) * e[i];
  return 0.5 * acc * vol;
}

inline void atomic_add(double* p, double v) {
#pragma omp atomic
  *p += v;
}

void load_zc(const double* z, const int32_t* cells, int64_t c, int layout, double zc[4]) {
  if (layout == 1) { zc[0] = zc[1] = zc[2] = zc[3] = z[c]; return; }
  for (int n = 0; n < 4; ++n) zc[n] = z[cells[4 * c + n]];
}

int64_t find_entry(const int32_t* rowmap, const int32_t* cols, int32_t row, int32_t col) {
  // BlockMatrixEntryOrdinal (src/ImplicitFunctors.hpp:662-680): linear search.
  for (int32_t k = rowmap[row]; k < rowmap[row + 1]; ++k)
    if (cols[k] == col) return k;
  return -1;
}

}  // namespace

extern "C" {

int pao_num_threads(void) { return omp_get_max_threads(); }
void pao_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// Structured box -> 6 linear tets per hex.  Nodes are numbered x fastest:
// id = i + (nx+1)*(j + (ny+1)*k).  Hexes are visited x fastest; each hex is
// split into the six tets of the reference's single-hex box
// (unit_tests/OmegaHUtilitiesTests.cpp:258-287), in that order and with that
// local vertex order, all sharing the hex diagonal (0,0,0)-(1,1,1).
void pao_box_mesh(int nx, int ny, int nz, double lx, double ly, double lz, int32_t* cells, double* coords) {
  static const int tet[6][4][3] = {
      {{0, 0, 0}, {1, 1, 0}, {0, 1, 0}, {1, 1, 1}}, {{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}},
      {{0, 0, 0}, {0, 1, 1}, {0, 0, 1}, {1, 1, 1}}, {{0, 0, 0}, {1, 0, 1}, {1, 1, 1}, {0, 0, 1}},
      {{1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {0, 0, 0}}, {{1, 0, 0}, {1, 1, 1}, {1, 1, 0}, {0, 0, 0}}};
  int64_t px = nx + 1, py = ny + 1;
  for (int64_t k = 0; k <= nz; ++k)
    for (int64_t j = 0; j <= ny; ++j)
      for (int64_t i = 0; i <= nx; ++i) {
        int64_t v = i + px * (j + py * k);
        coords[3 * v + 0] = lx * double(i) / nx;
        coords[3 * v + 1] = ly * double(j) / ny;
        coords[3 * v + 2] = lz * double(k) / nz;
      }
  int64_t c = 0;
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i)
        for (int t = 0; t < 6; ++t, ++c)
          for (int n = 0; n < 4; ++n) {
            const int* o = tet[t][n];
            cells[4 * c + n] = int32_t((i + o[0]) + px * ((j + o[1]) + py * (k + o[2])));
          }
}

// VectorFunction::value (src/elliptic/VectorFunction.hpp:231-310): gather,
// per-cell residual, atomic scatter (src/Assembly.hpp:1189-1209), then the
// uniform surface load with scale -1 (src/SurfaceLoadIntegral.hpp:96-160:
// weight = scale * (1/6) * |(x0-x2) x (x1-x2)| per face node).
void pao_residual(int64_t C, int64_t N, const int32_t* cells, const double* coords, const double* u,
                  const double* z, int layout, double E, double nu, double p, double pmin,
                  int64_t nfaces, const int32_t* faces, const double* flux, double* r) {
  Elastic m = make_elastic(E, nu, p, pmin);
  std::memset(r, 0, sizeof(double) * 3 * N);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < C; ++c) {
    double X[4][3], g[4][3], vol, ue[12], zc[4], re[12];
    gather_X(cells, coords, c, X);
    cell_gradients(X, g, vol);
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) ue[3 * n + d] = u[3 * cells[4 * c + n] + d];
    load_zc(z, cells, c, layout, zc);
    cell_residual(m, g, vol, ue, zc, layout, re);
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) atomic_add(&r[3 * cells[4 * c + n] + d], re[3 * n + d]);
  }
  for (int64_t f = 0; f < nfaces; ++f) {
    const int32_t* v = faces + 3 * f;
    double a[3], b[3], cr[3];
    for (int d = 0; d < 3; ++d) { a[d] = coords[3 * v[0] + d] - coords[3 * v[2] + d]; b[d] = coords[3 * v[1] + d] - coords[3 * v[2] + d]; }
    cr[0] = a[1] * b[2] - a[2] * b[1]; cr[1] = a[2] * b[0] - a[0] * b[2]; cr[2] = a[0] * b[1] - a[1] * b[0];
    double w = -1.0 * (1.0 / 6.0) * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int n = 0; n < 3; ++n)
      for (int d = 0; d < 3; ++d) r[3 * v[n] + d] += w * flux[d];
  }
}

// Nodal-graph CRS (block rows = nodes, columns sorted ascending, diagonal
// included); the same node-star graph CreateBlockMatrix builds
// (src/ImplicitFunctors.hpp:735-808).  Returns nnz blocks; call with
// cols == nullptr to size.
int64_t pao_crs_graph(int64_t C, int64_t N, const int32_t* cells, int32_t* rowmap, int32_t* cols) {
  std::vector<std::vector<int32_t>> adj(N);
  for (int64_t c = 0; c < C; ++c)
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) adj[cells[4 * c + a]].push_back(cells[4 * c + b]);
  int64_t nnz = 0;
  for (int64_t i = 0; i < N; ++i) {
    auto& v = adj[i];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    if (rowmap) rowmap[i] = int32_t(nnz);
    if (cols) std::copy(v.begin(), v.end(), cols + nnz);
    nnz += int64_t(v.size());
  }
  if (rowmap) rowmap[N] = int32_t(nnz);
  return nnz;
}

// VectorFunction::gradient_u (src/elliptic/VectorFunction.hpp:505-594) with
// the Jacobian evaluation type (12 state partials per cell) and
// assemble_jacobian_fad (src/Assembly.hpp:1341-1363): entry
// block*9 + i*3 + j for row dof i of node a, column dof j of node b.
void pao_jacobian(int64_t C, int64_t N, const int32_t* cells, const double* coords, const double* u,
                  const double* z, int layout, double E, double nu, double p, double pmin,
                  const int32_t* rowmap, const int32_t* cols, double* vals) {
  Elastic m = make_elastic(E, nu, p, pmin);
  std::memset(vals, 0, sizeof(double) * 9 * rowmap[N]);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < C; ++c) {
    double X[4][3], g[4][3], vol, zc[4];
    gather_X(cells, coords, c, X);
    cell_gradients(X, g, vol);
    Dual<12> ue[12], re[12];
    for (int i = 0; i < 12; ++i) { ue[i] = Dual<12>(u[3 * cells[4 * c + i / 3] + i % 3]); ue[i].d[i] = 1.0; }
    load_zc(z, cells, c, layout, zc);
    cell_residual(m, g, vol, ue, zc, layout, re);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        int64_t k = find_entry(rowmap, cols, cells[4 * c + a], cells[4 * c + b]);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) atomic_add(&vals[9 * k + 3 * i + j], re[3 * a + i].d[3 * b + j]);
      }
  }
}

// VectorFunction::gradient_z (src/elliptic/VectorFunction.hpp:598-689),
// control partials (4 per cell) and assemble_transpose_jacobian
// (src/Assembly.hpp:1422-1445): rows = control nodes, 1x3 blocks over state
// nodes, entry block*3 + dof.  Per-cell layout: row c has the 12 partials of
// cell c in local (node, dof) order.
void pao_gradient_z(int64_t C, int64_t N, const int32_t* cells, const double* coords, const double* u,
                    const double* z, int layout, double E, double nu, double p, double pmin,
                    const int32_t* rowmap, const int32_t* cols, double* vals) {
  Elastic m = make_elastic(E, nu, p, pmin);
  if (layout == 0) std::memset(vals, 0, sizeof(double) * 3 * rowmap[N]);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < C; ++c) {
    double X[4][3], g[4][3], vol, ue[12], zv[4];
    gather_X(cells, coords, c, X);
    cell_gradients(X, g, vol);
    for (int i = 0; i < 12; ++i) ue[i] = u[3 * cells[4 * c + i / 3] + i % 3];
    load_zc(z, cells, c, layout, zv);
    Dual<4> zc[4], re[12];
    for (int k = 0; k < 4; ++k) { zc[k] = Dual<4>(zv[k]); zc[k].d[k] = 1.0; }
    cell_residual(m, g, vol, ue, zc, layout, re);
    if (layout == 1) {
      for (int i = 0; i < 12; ++i) vals[12 * c + i] = re[i].d[0];
      continue;
    }
    for (int k = 0; k < 4; ++k)
      for (int b = 0; b < 4; ++b) {
        int64_t e = find_entry(rowmap, cols, cells[4 * c + k], cells[4 * c + b]);
        for (int d = 0; d < 3; ++d) atomic_add(&vals[3 * e + d], re[3 * b + d].d[k]);
      }
  }
}

// PhysicsScalarFunction value / gradient_u / gradient_z for "Internal Elastic
// Energy" (src/elliptic/PhysicsScalarFunction.hpp:225,365,432), local sums
// via local_result_sum (src/Assembly.hpp:21-30) and
// assemble_vector_gradient_fad / assemble_scalar_gradient_fad
// (src/Assembly.hpp:417-490, :526-590).  grad_u/grad_z may be null.
double pao_energy(int64_t C, int64_t N, const int32_t* cells, const double* coords, const double* u,
                  const double* z, int layout, double E, double nu, double p, double pmin,
                  double* grad_u, double* grad_z) {
  Elastic m = make_elastic(E, nu, p, pmin);
  if (grad_u) std::memset(grad_u, 0, sizeof(double) * 3 * N);
  if (grad_z) std::memset(grad_z, 0, sizeof(double) * (layout == 1 ? C : N));
  double total = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : total)
  for (int64_t c = 0; c < C; ++c) {
    double X[4][3], g[4][3], vol, ue[12], zv[4];
    gather_X(cells, coords, c, X);
    cell_gradients(X, g, vol);
    for (int i = 0; i < 12; ++i) ue[i] = u[3 * cells[4 * c + i / 3] + i % 3];
    load_zc(z, cells, c, layout, zv);
    total += cell_energy<double, double, double>(m, g, vol, ue, zv, layout);
    if (grad_u) {
      Dual<12> ud[12];
      for (int i = 0; i < 12; ++i) { ud[i] = Dual<12>(ue[i]); ud[i].d[i] = 1.0; }
      Dual<12> f = cell_energy<Dual<12>, double, Dual<12>>(m, g, vol, ud, zv, layout);
      for (int i = 0; i < 12; ++i) atomic_add(&grad_u[3 * cells[4 * c + i / 3] + i % 3], f.d[i]);
    }
    if (grad_z) {
      Dual<4> zd[4];
      for (int k = 0; k < 4; ++k) { zd[k] = Dual<4>(zv[k]); zd[k].d[k] = 1.0; }
      Dual<4> f = cell_energy<double, Dual<4>, Dual<4>>(m, g, vol, ue, zd, layout);
      if (layout == 1) grad_z[c] = f.d[0];
      else
        for (int k = 0; k < 4; ++k) atomic_add(&grad_z[cells[4 * c + k]], f.d[k]);
    }
  }
  return total;
}

// Symmetric Dirichlet elimination on a block CRS: applyBlockConstraints<3>
// (src/ApplyConstraints.hpp:11-79).
void pao_apply_block_constraints(int64_t N, const int32_t* rowmap, const int32_t* cols, double* vals, double* rhs,
                                 int64_t nbc, const int32_t* bc_dofs, const double* bc_values, double scale) {
  for (int64_t b = 0; b < nbc; ++b) {
    int32_t rdof = bc_dofs[b];
    double value = scale * bc_values[b];
    int32_t rnode = rdof / 3, rl = rdof % 3;
    for (int32_t k = rowmap[rnode]; k < rowmap[rnode + 1]; ++k)
      for (int cl = 0; cl < 3; ++cl) {
        int32_t cnode = cols[k];
        int64_t e = 9LL * k + 3 * rl + cl;
        int32_t cdof = 3 * cnode + cl;
        if (cdof == rdof) { vals[e] = 1.0; continue; }
        rhs[cdof] -= vals[e] * value;
        vals[e] = 0.0;
        for (int32_t kk = rowmap[cnode]; kk < rowmap[cnode + 1]; ++kk)
          if (3 * cols[kk] + rl == rdof) vals[9LL * kk + 3 * cl + rl] = 0.0;
      }
  }
  for (int64_t b = 0; b < nbc; ++b) rhs[bc_dofs[b]] = scale * bc_values[b];
}

// Block-CRS SpMV y = A x  (the product MatrixTimesVectorPlusVector builds on,
// src/PlatoMathHelpers.hpp:89-115).
void pao_block_spmv(int64_t N, const int32_t* rowmap, const int32_t* cols, const double* vals, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    double a0 = 0, a1 = 0, a2 = 0;
    for (int32_t k = rowmap[i]; k < rowmap[i + 1]; ++k) {
      const double* v = vals + 9LL * k;
      const double* xv = x + 3LL * cols[k];
      a0 += v[0] * xv[0] + v[1] * xv[1] + v[2] * xv[2];
      a1 += v[3] * xv[0] + v[4] * xv[1] + v[5] * xv[2];
      a2 += v[6] * xv[0] + v[7] * xv[1] + v[8] * xv[2];
    }
    y[3 * i + 0] = a0; y[3 * i + 1] = a1; y[3 * i + 2] = a2;
  }
}

static double dot(int64_t n, const double* a, const double* b) {
  double s = 0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

// Jacobi-preconditioned CG on the assembled, constrained block CRS (FP64).
// The reference hands this system to AmgX / AztecOO (src/alg/*LinearSolver.cpp);
// the oracle solves the same linear system.  max_iters <= 0 means 10*ndof.
// Returns the iteration count; *relres_out = ||b - A x|| / ||b||.
int pao_pcg(int64_t N, const int32_t* rowmap, const int32_t* cols, const double* vals, const double* b, double* x,
            double rel_tol, int max_iters, double* relres_out) {
  int64_t n = 3 * N;
  std::vector<double> diag(n), r(n), zz(n), pp(n), ap(n);
  for (int64_t i = 0; i < N; ++i)
    for (int32_t k = rowmap[i]; k < rowmap[i + 1]; ++k)
      if (cols[k] == i)
        for (int d = 0; d < 3; ++d) diag[3 * i + d] = vals[9LL * k + 4 * d];
  pao_block_spmv(N, rowmap, cols, vals, x, ap.data());
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ap[i];
  double bn = std::sqrt(dot(n, b, b));
  if (bn == 0) bn = 1;
  for (int64_t i = 0; i < n; ++i) { zz[i] = r[i] / diag[i]; pp[i] = zz[i]; }
  double rz = dot(n, r.data(), zz.data());
  if (max_iters <= 0) max_iters = int(10 * n);
  int it = 0;
  double rr = std::sqrt(dot(n, r.data(), r.data()));
  while (it < max_iters && rr / bn > rel_tol) {
    pao_block_spmv(N, rowmap, cols, vals, pp.data(), ap.data());
    double alpha = rz / dot(n, pp.data(), ap.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) { x[i] += alpha * pp[i]; r[i] -= alpha * ap[i]; zz[i] = r[i] / diag[i]; }
    double rz1 = dot(n, r.data(), zz.data());
    double beta = rz1 / rz;
    rz = rz1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) pp[i] = zz[i] + beta * pp[i];
    rr = std::sqrt(dot(n, r.data(), r.data()));
    ++it;
  }
  pao_block_spmv(N, rowmap, cols, vals, x, ap.data());
  double tr = 0;
  for (int64_t i = 0; i < n; ++i) tr += (b[i] - ap[i]) * (b[i] - ap[i]);
  if (relres_out) *relres_out = std::sqrt(tr) / bn;
  return it;
}

// The same Jacobi-PCG as pao_pcg, started from x, with a checkpoint: when the
// relative recursive residual first reaches report_tol, the iteration count
// and the wall time since entry are stored (info[0], info[1]); the loop goes
// on to rel_tol (info[2] = iterations, info[3] = total seconds, info[4] =
// true relative residual ||b - A x|| / ||b||).  max_iters <= 0 means 10*ndof;
// max_iters caps a bounded run (a timing sample of a longer solve).
void pao_pcg_run(int64_t N, const int32_t* rowmap, const int32_t* cols, const double* vals, const double* b,
                 double* x, double report_tol, double rel_tol, int max_iters, double* info) {
  const double t0 = omp_get_wtime();
  int64_t n = 3 * N;
  std::vector<double> dinv(n), r(n), zz(n), pp(n), ap(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i)
    for (int32_t k = rowmap[i]; k < rowmap[i + 1]; ++k)
      if (cols[k] == i)
        for (int d = 0; d < 3; ++d) dinv[3 * i + d] = 1.0 / vals[9LL * k + 4 * d];
  pao_block_spmv(N, rowmap, cols, vals, x, ap.data());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    r[i] = b[i] - ap[i];
    zz[i] = r[i] * dinv[i];
    pp[i] = zz[i];
  }
  double bn = std::sqrt(dot(n, b, b));
  if (bn == 0) bn = 1;
  double rz = dot(n, r.data(), zz.data());
  if (max_iters <= 0) max_iters = int(10 * n);
  int it = 0;
  double rr = std::sqrt(dot(n, r.data(), r.data()));
  info[0] = -1.0;
  info[1] = 0.0;
  if (rr / bn <= report_tol) { info[0] = 0.0; info[1] = omp_get_wtime() - t0; }
  while (it < max_iters && rr / bn > rel_tol) {
    pao_block_spmv(N, rowmap, cols, vals, pp.data(), ap.data());
    const double alpha = rz / dot(n, pp.data(), ap.data());
    double rz1 = 0.0, rr2 = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz1, rr2)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * pp[i];
      r[i] -= alpha * ap[i];
      zz[i] = r[i] * dinv[i];
      rz1 += r[i] * zz[i];
      rr2 += r[i] * r[i];
    }
    const double beta = rz1 / rz;
    rz = rz1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) pp[i] = zz[i] + beta * pp[i];
    rr = std::sqrt(rr2);
    ++it;
    if (info[0] < 0.0 && rr / bn <= report_tol) { info[0] = it; info[1] = omp_get_wtime() - t0; }
  }
  pao_block_spmv(N, rowmap, cols, vals, x, ap.data());
  double tr = 0;
#pragma omp parallel for schedule(static) reduction(+ : tr)
  for (int64_t i = 0; i < n; ++i) tr += (b[i] - ap[i]) * (b[i] - ap[i]);
  info[2] = it;
  info[3] = omp_get_wtime() - t0;
  info[4] = std::sqrt(tr) / bn;
}

// Matrix-free K u (no constraints) with hand-derived cell operator; used to
// cross-check the dual-number Jacobian and as a CPU timing of one apply.
void pao_apply(int64_t C, int64_t N, const int32_t* cells, const double* coords, const double* u,
               const double* z, int layout, double E, double nu, double p, double pmin, double* y) {
  pao_residual(C, N, cells, coords, u, z, layout, E, nu, p, pmin, 0, nullptr, nullptr, y);
}

// ---------------------------------------------------------------------------
// J2 radial return: J2PlasticityLocalResidual::updateLocalState
// (src/J2PlasticityLocalResidual.hpp:421-523) for the displacement-only
// small-strain form.  Local state per cell (14): [0] accumulated plastic
// strain, [1] plastic multiplier increment, [2..7] plastic strain (Voigt,
// engineering shears), [8..13] backstress.
//   elastic strain  = total - plastic     (src/ThermoPlasticityUtilities.hpp:101-121)
//   deviatoric s    = 2 mu dev(eps_e), shear mu*gamma (src/ComputeDeviatoricStress.hpp:110-130)
//   n = (s - a)/||s - a|| with shear terms doubled in the norm
//                                          (src/J2PlasticityUtilities.hpp:378-407)
//   plastic step updates                   (src/J2PlasticityUtilities.hpp:250-273)
// `u` holds 3 dofs per node.  Parameters: shear modulus mu, yield stress,
// isotropic/kinematic hardening, SIMP (exponent, minimum) for the elastic and
// plastic properties, nodal density z (mean of 4 nodes).
void pao_j2_update(int64_t C, const int32_t* cells, const double* coords, const double* u, const double* z,
                   double mu, double sigma_y0, double h_iso, double h_kin, double pe, double pe_min,
                   double pp_, double pp_min, const double* prev, double* cur) {
  const double s32 = std::sqrt(1.5), s23 = std::sqrt(2.0 / 3.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < C; ++c) {
    double X[4][3], g[4][3], vol, ue[12], e[6];
    gather_X(cells, coords, c, X);
    cell_gradients(X, g, vol);
    for (int i = 0; i < 12; ++i) ue[i] = u[3 * cells[4 * c + i / 3] + i % 3];
    strain(g, ue, e);
    const double* pv = prev + 14 * c;
    double* cv = cur + 14 * c;
    cv[0] = pv[0];
    cv[1] = 0.0;
    for (int i = 2; i < 14; ++i) cv[i] = pv[i];
    double ee[6];
    for (int i = 0; i < 6; ++i) ee[i] = e[i] - cv[2 + i];
    double rho = 0.25 * (z[cells[4 * c]] + z[cells[4 * c + 1]] + z[cells[4 * c + 2]] + z[cells[4 * c + 3]]);
    double mu_p = (pe_min + (1.0 - pe_min) * std::pow(rho, pe)) * mu;
    double tr3 = (ee[0] + ee[1] + ee[2]) / 3.0;
    double s[6] = {2 * mu_p * (ee[0] - tr3), 2 * mu_p * (ee[1] - tr3), 2 * mu_p * (ee[2] - tr3),
                   mu_p * ee[3], mu_p * ee[4], mu_p * ee[5]};
    double nrm[6];
    for (int i = 0; i < 6; ++i) nrm[i] = s[i] - cv[8 + i];
    double norm = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2] +
                            2 * (nrm[3] * nrm[3] + nrm[4] * nrm[4] + nrm[5] * nrm[5]));
    for (int i = 0; i < 6; ++i) nrm[i] /= norm;
    double ppen = pp_min + (1.0 - pp_min) * std::pow(rho, pp_);
    double hi = ppen * h_iso, hk = ppen * h_kin, sy0 = ppen * sigma_y0;
    double sy = sy0 + hi * cv[0];
    double ftr = s32 * norm - sy;
    if (ftr > 1.0e-10) {
      cv[1] = ftr / (3.0 * mu_p + hi + hk);
      cv[0] = pv[0] + cv[1];
      double m1 = cv[1] * s32;
      for (int i = 0; i < 3; ++i) cv[2 + i] = pv[2 + i] + m1 * nrm[i];
      for (int i = 3; i < 6; ++i) cv[2 + i] = pv[2 + i] + 2.0 * m1 * nrm[i];
      double m2 = cv[1] * s23 * hk;
      for (int i = 0; i < 6; ++i) cv[8 + i] = pv[8 + i] + m2 * nrm[i];
    }
  }
}

// updatePlasticStrainAndBackstressPlasticStep<3> alone
// (src/J2PlasticityUtilities.hpp:250-273), for the reference's known-answer
// unit test of that utility.
void pao_j2_plastic_step(int64_t C, const double* prev, const double* normal, double h_kin, double* cur) {
  const double s32 = std::sqrt(1.5), s23 = std::sqrt(2.0 / 3.0);
  for (int64_t c = 0; c < C; ++c) {
    const double* pv = prev + 14 * c;
    const double* n = normal + 6 * c;
    double* cv = cur + 14 * c;
    double m1 = cv[1] * s32;
    for (int i = 0; i < 3; ++i) cv[2 + i] = pv[2 + i] + m1 * n[i];
    for (int i = 3; i < 6; ++i) cv[2 + i] = pv[2 + i] + 2.0 * m1 * n[i];
    double m2 = cv[1] * s23 * h_kin;
    for (int i = 0; i < 6; ++i) cv[8 + i] = pv[8 + i] + m2 * n[i];
  }
}

// VectorFunction::gradient_x (src/elliptic/VectorFunction.hpp:317-408): the
// configuration evaluation type (12 coordinate partials per cell) and the
// transposed block assembly -- block (row = node of coordinate dof k,
// col = node of residual dof i), entry [k % 3][i % 3] -- plus the uniform
// surface load's dependence on the face area (scale -1).
void pao_gradient_x(int64_t C, int64_t N, const int32_t* cells, const double* coords, const double* u,
                    const double* z, int layout, double E, double nu, double p, double pmin,
                    int64_t nfaces, const int32_t* faces, const double* flux,
                    const int32_t* rowmap, const int32_t* cols, double* vals) {
  Elastic m = make_elastic(E, nu, p, pmin);
  std::memset(vals, 0, sizeof(double) * 9 * rowmap[N]);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < C; ++c) {
    Dual<12> X[4][3], g[4][3], vol, ue[12], re[12];
    double zc[4];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) {
        X[n][d] = Dual<12>(coords[3 * int64_t(cells[4 * c + n]) + d]);
        X[n][d].d[3 * n + d] = 1.0;
      }
    cell_gradients_t(X, g, vol);
    for (int i = 0; i < 12; ++i) ue[i] = Dual<12>(u[3 * cells[4 * c + i / 3] + i % 3]);
    load_zc(z, cells, c, layout, zc);
    Dual<12> e[6], s[6], sw[6];
    strain(g, ue, e);
    stress(m, e, s);
    double w = simp(m, cell_rho(zc, layout));
    for (int i = 0; i < 6; ++i) sw[i] = s[i] * w;
    for (int i = 0; i < 12; ++i) re[i] = Dual<12>(0.0);
    divergence(g, vol, sw, re);
    for (int a = 0; a < 4; ++a)       // config node (row)
      for (int b = 0; b < 4; ++b) {   // state node (column)
        int64_t k = find_entry(rowmap, cols, cells[4 * c + a], cells[4 * c + b]);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) atomic_add(&vals[9 * k + 3 * i + j], re[3 * b + j].d[3 * a + i]);
      }
  }
  for (int64_t f = 0; f < nfaces; ++f) {
    const int32_t* v = faces + 3 * f;
    Dual<9> a[3], b[3], cr[3], xs[3][3];
    for (int n = 0; n < 3; ++n)
      for (int d = 0; d < 3; ++d) { xs[n][d] = Dual<9>(coords[3 * v[n] + d]); xs[n][d].d[3 * n + d] = 1.0; }
    for (int d = 0; d < 3; ++d) { a[d] = xs[0][d] - xs[2][d]; b[d] = xs[1][d] - xs[2][d]; }
    cr[0] = a[1] * b[2] - a[2] * b[1]; cr[1] = a[2] * b[0] - a[0] * b[2]; cr[2] = a[0] * b[1] - a[1] * b[0];
    Dual<9> w = (-1.0 / 6.0) * dsqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int an = 0; an < 3; ++an)
      for (int bn = 0; bn < 3; ++bn) {
        int64_t k = find_entry(rowmap, cols, v[an], v[bn]);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) vals[9 * k + 3 * i + j] += w.d[3 * an + i] * flux[j];
      }
  }
}

// PhysicsScalarFunction::gradient_x for the internal energy: df/dx (3N).
void pao_energy_grad_x(int64_t C, int64_t N, const int32_t* cells, const double* coords, const double* u,
                       const double* z, int layout, double E, double nu, double p, double pmin, double* gx) {
  Elastic m = make_elastic(E, nu, p, pmin);
  std::memset(gx, 0, sizeof(double) * 3 * N);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < C; ++c) {
    Dual<12> X[4][3], g[4][3], vol, ue[12];
    double zc[4];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) {
        X[n][d] = Dual<12>(coords[3 * int64_t(cells[4 * c + n]) + d]);
        X[n][d].d[3 * n + d] = 1.0;
      }
    cell_gradients_t(X, g, vol);
    for (int i = 0; i < 12; ++i) ue[i] = Dual<12>(u[3 * cells[4 * c + i / 3] + i % 3]);
    load_zc(z, cells, c, layout, zc);
    Dual<12> e[6], s[6], acc(0.0);
    strain(g, ue, e);
    stress(m, e, s);
    double w = simp(m, cell_rho(zc, layout));
    for (int i = 0; i < 6; ++i) acc += (s[i] * w) * e[i];
    Dual<12> f = 0.5 * acc * vol;
    for (int k = 0; k < 12; ++k) atomic_add(&gx[3 * int64_t(cells[4 * c + k / 3]) + k % 3], f.d[k]);
  }
}

}  // extern "C"
