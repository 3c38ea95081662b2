// pa_elastic.cu -- per-cell kernels of the elastostatics VectorFunction and
// the Internal Elastic Energy ScalarFunction (value and hand-derived
// gradients), Jacobi diagonal and SIMP cell weights.
//
// These entry points are called once per design iteration (not inside the
// Krylov loop), so they use one thread per cell in the caller's cell order
// with global atomics for the scatter; the Krylov hot loop uses the
// tile-staged kernel of pa_tiled.cuh, and so do the residual and dF/du entry
// points (K(z) u, pa_abi.cu), which would otherwise add 12 atomics per tet.
#include <algorithm>

#include "pa_problem.cuh"
#include "pa_tiled.cuh"

namespace pa {

namespace {

constexpr int kThreads = 256;

inline int grid_for(int64_t n, int threads = kThreads) {
  int64_t g = (n + threads - 1) / threads;
  return int(g < 1 ? 1 : g);
}

struct CellIn {
  const int32_t* cells;
  const double* coords;
  int64_t C;
};

__device__ __forceinline__ void load_cell(const CellIn& m, int64_t c, int v[4], double x[4][3]) {
  const int4 q = reinterpret_cast<const int4*>(m.cells)[c];
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int d = 0; d < 3; ++d) x[n][d] = __ldg(&m.coords[3 * int64_t(v[n]) + d]);
}

__device__ __forceinline__ void load_u(const double* u, const int v[4], double ue[12]) {
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int d = 0; d < 3; ++d) ue[3 * n + d] = __ldg(&u[3 * int64_t(v[n]) + d]);
}

// Cell density: mean of the 4 nodal controls (src/ApplyWeighting.hpp:56-60)
// or the cell's own value in the per-cell layout.
__device__ __forceinline__ double cell_density(const double* z, int layout, int64_t c, const int v[4]) {
  if (layout == PA_CONTROL_CELL) return __ldg(&z[c]);
  return (__ldg(&z[v[0]]) + __ldg(&z[v[1]]) + __ldg(&z[v[2]]) + __ldg(&z[v[3]])) / 4.0;
}

struct Mat64 {
  Iso<double> iso;
  double p, pmin;
  int layout;
};

// SurfaceLoadIntegral (src/SurfaceLoadIntegral.hpp:96-160): per face node
// weight = scale * (1/6) |(x0 - x2) x (x1 - x2)|, times the face's flux.
__global__ void k_traction(const int32_t* __restrict__ faces, const double* __restrict__ flux, int64_t nf,
                           const double* __restrict__ coords, double scale, double* __restrict__ r) {
  const int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (f >= nf) return;
  const int64_t v0 = faces[3 * f], v1 = faces[3 * f + 1], v2 = faces[3 * f + 2];
  double a[3], b[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    a[d] = coords[3 * v0 + d] - coords[3 * v2 + d];
    b[d] = coords[3 * v1 + d] - coords[3 * v2 + d];
  }
  const double cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2], cz = a[0] * b[1] - a[1] * b[0];
  const double w = scale * (1.0 / 6.0) * sqrt(cx * cx + cy * cy + cz * cz);
  const int64_t vs[3] = {v0, v1, v2};
#pragma unroll
  for (int n = 0; n < 3; ++n)
#pragma unroll
    for (int d = 0; d < 3; ++d) atomicAdd(&r[3 * vs[n] + d], w * flux[3 * f + d]);
}

// gradient_u: closed-form K_e blocks scattered into the block CRS through the
// precomputed cell -> block map (replaces the per-entry linear column search
// of BlockMatrixEntryOrdinal, src/ImplicitFunctors.hpp:662-680).
__global__ void k_gradient_u(CellIn m, Mat64 mat, const double* __restrict__ z, const int32_t* __restrict__ cell_entry,
                             double* __restrict__ vals) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= m.C) return;
  int v[4];
  double x[4][3], g[4][3], vol;
  load_cell(m, c, v, x);
  tet_geometry(x, g, vol);
  const double s = vol * simp(cell_density(z, mat.layout, c, v), mat.p, mat.pmin);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      double k[9];
      tet_kblock(mat.iso, s, g[a], g[b], k);
      double* dst = vals + 9 * int64_t(cell_entry[16 * c + 4 * a + b]);
#pragma unroll
      for (int q = 0; q < 9; ++q) atomicAdd(&dst[q], k[q]);
    }
}

// gradient_z: dR_e/dz_k = dp/drho * drho/dz_k * vol B^T C B u_e.
__global__ void k_gradient_z(CellIn m, Mat64 mat, const double* __restrict__ u, const double* __restrict__ z,
                             const int32_t* __restrict__ cell_entry, double* __restrict__ vals) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= m.C) return;
  int v[4];
  double x[4][3], g[4][3], vol, ue[12], e[6], sig[6], re[12];
  load_cell(m, c, v, x);
  load_u(u, v, ue);
  tet_geometry(x, g, vol);
  tet_strain(g, ue, e);
  const double rho = cell_density(z, mat.layout, c, v);
  if (mat.layout == PA_CONTROL_CELL) {
    tet_stress(mat.iso, vol * simp_deriv(rho, mat.p, mat.pmin), e, sig);
    tet_divergence(g, sig, re);
#pragma unroll
    for (int i = 0; i < 12; ++i) vals[12 * c + i] = re[i];
    return;
  }
  tet_stress(mat.iso, vol * 0.25 * simp_deriv(rho, mat.p, mat.pmin), e, sig);
  tet_divergence(g, sig, re);
  for (int k = 0; k < 4; ++k)
    for (int b = 0; b < 4; ++b) {
      double* dst = vals + 3 * int64_t(cell_entry[16 * c + 4 * k + b]);
#pragma unroll
      for (int d = 0; d < 3; ++d) atomicAdd(&dst[d], re[3 * b + d]);
    }
}

// Internal Elastic Energy: value (block partials), gradient_u, gradient_z.
__global__ void k_energy(CellIn m, Mat64 mat, const double* __restrict__ u, const double* __restrict__ z,
                         double* __restrict__ partials, double* __restrict__ grad_u, double* __restrict__ grad_z) {
  __shared__ double s_red[32];
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double f = 0.0;
  if (c < m.C) {
    int v[4];
    double x[4][3], g[4][3], vol, ue[12], e[6], sig[6];
    load_cell(m, c, v, x);
    load_u(u, v, ue);
    tet_geometry(x, g, vol);
    tet_strain(g, ue, e);
    const double rho = cell_density(z, mat.layout, c, v);
    tet_stress(mat.iso, vol, e, sig);  // unpenalized, volume-weighted
    const double e0 = 0.5 * voigt_dot(sig, e);
    const double w = simp(rho, mat.p, mat.pmin);
    f = w * e0;
    if (grad_u) {
      double re[12];
#pragma unroll
      for (int i = 0; i < 6; ++i) sig[i] *= w;
      tet_divergence(g, sig, re);
#pragma unroll
      for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int d = 0; d < 3; ++d) atomicAdd(&grad_u[3 * int64_t(v[n]) + d], re[3 * n + d]);
    }
    if (grad_z) {
      const double dw = simp_deriv(rho, mat.p, mat.pmin);
      if (mat.layout == PA_CONTROL_CELL) {
        grad_z[c] = dw * e0;
      } else {
#pragma unroll
        for (int n = 0; n < 4; ++n) atomicAdd(&grad_z[v[n]], 0.25 * dw * e0);
      }
    }
  }
  const double b = block_sum(f, s_red);
  if (partials && threadIdx.x == 0) partials[blockIdx.x] = b;
}

__global__ void k_sum_partials(const double* __restrict__ partials, int n, double* __restrict__ out) {
  __shared__ double s_red[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
  v = block_sum(v, s_red);
  if (threadIdx.x == 0) *out = v;
}

// SIMP weight per cell in tile (internal) order, FP64 and FP32.
__global__ void k_cell_weights(CellIn m, Mat64 mat, const int32_t* __restrict__ perm, const double* __restrict__ z,
                               double* __restrict__ w64, float* __restrict__ w32) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= m.C) return;
  const int64_t c = perm[i];
  const int4 q = reinterpret_cast<const int4*>(m.cells)[c];
  const int v[4] = {q.x, q.y, q.z, q.w};
  const double w = simp(cell_density(z, mat.layout, c, v), mat.p, mat.pmin);
  if (w64) w64[i] = w;
  if (w32) w32[i] = float(w);
}

// Jacobi diagonal: K_aa,ii = s [(lam + mu) g_ai^2 + mu |g_a|^2].
__global__ void k_diag(CellIn m, Mat64 mat, const int32_t* __restrict__ perm, const double* __restrict__ w,
                       double* __restrict__ diag) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= m.C) return;
  const int64_t c = perm[i];
  int v[4];
  double x[4][3], g[4][3], vol;
  load_cell(m, c, v, x);
  tet_geometry(x, g, vol);
  const double s = vol * w[i];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const double gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      atomicAdd(&diag[3 * int64_t(v[n]) + d], s * ((mat.iso.lam + mat.iso.mu) * g[n][d] * g[n][d] + mat.iso.mu * gg));
  }
}


// (dR/dz)^T lambda added into g: per cell dp/drho * lambda_e . (vol B^T C B u_e),
// spread to the 4 nodal controls (1/4 each) or the cell's own control; the
// matrix-free form of MatrixTimesVectorPlusVector(dgdz, lambda, dfdz)
// (src/PlatoMathHelpers.hpp:58-137).
__global__ void k_dRdz_T(CellIn m, Mat64 mat, const double* __restrict__ u, const double* __restrict__ z,
                         const double* __restrict__ lam, double* __restrict__ g) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= m.C) return;
  int v[4];
  double x[4][3], gr[4][3], vol, ue[12], le[12], e[6], el[6], sig[6];
  load_cell(m, c, v, x);
  load_u(u, v, ue);
  load_u(lam, v, le);
  tet_geometry(x, gr, vol);
  tet_strain(gr, ue, e);
  tet_strain(gr, le, el);
  tet_stress(mat.iso, vol, e, sig);
  const double dw = simp_deriv(cell_density(z, mat.layout, c, v), mat.p, mat.pmin);
  const double val = dw * voigt_dot(sig, el);
  if (mat.layout == PA_CONTROL_CELL) {
    g[c] += val;
  } else {
#pragma unroll
    for (int n = 0; n < 4; ++n) atomicAdd(&g[v[n]], 0.25 * val);
  }
}

// applyBlockConstraints<3> (src/ApplyConstraints.hpp:11-79), first loop: one
// thread per constrained dof zeroes its row and column (diagonal 1) and lifts
// the rhs.
__global__ void k_bc_first(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals, double scale,
                           const int32_t* __restrict__ rowmap, const int32_t* __restrict__ cols,
                           double* __restrict__ entries, double* __restrict__ rhs) {
  const int64_t b = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (b >= nbc) return;
  const int32_t rdof = dofs[b];
  const double value = scale * vals[b];
  const int32_t rnode = rdof / 3, rl = rdof % 3;
  for (int32_t k = rowmap[rnode]; k < rowmap[rnode + 1]; ++k) {
    const int32_t cnode = cols[k];
    for (int cl = 0; cl < 3; ++cl) {
      const int64_t e = 9LL * k + 3 * rl + cl;
      const int32_t cdof = 3 * cnode + cl;
      if (cdof == rdof) {
        entries[e] = 1.0;
        continue;
      }
      atomicAdd(&rhs[cdof], -entries[e] * value);
      entries[e] = 0.0;
      for (int32_t kk = rowmap[cnode]; kk < rowmap[cnode + 1]; ++kk)
        if (3 * cols[kk] + rl == rdof) entries[9LL * kk + 3 * cl + rl] = 0.0;
    }
  }
}

// second loop: rhs at constrained dofs = scaled value.
__global__ void k_bc_second(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                            double scale, double* __restrict__ rhs) {
  const int64_t b = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (b < nbc) rhs[dofs[b]] = scale * vals[b];
}

__global__ void k_scale(double* __restrict__ v, int64_t n, double a) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    v[i] *= a;
}

// ------------------------------------------------------------ gradient_x --
// Configuration derivatives by forward-mode directional differentiation: each
// of the 12 coordinate dofs of a cell is seeded in turn on a one-partial dual
// number D1, so the per-cell chain of pa_cell.cuh is reused unchanged.
struct D1 {
  double v, d;
  __device__ D1() : v(0.0), d(0.0) {}
  __device__ D1(double x) : v(x), d(0.0) {}
  __device__ D1(double x, double dx) : v(x), d(dx) {}
};
__device__ __forceinline__ D1 operator+(D1 a, D1 b) { return D1(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ D1 operator-(D1 a, D1 b) { return D1(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ D1 operator-(D1 a) { return D1(-a.v, -a.d); }
__device__ __forceinline__ D1 operator*(D1 a, D1 b) { return D1(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ D1 operator/(D1 a, D1 b) { return D1(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
__device__ __forceinline__ D1& operator+=(D1& a, D1 b) { a = a + b; return a; }
__device__ __forceinline__ D1 fabs(D1 a) { return a.v < 0.0 ? -a : a; }
__device__ __forceinline__ D1 sqrt(D1 a) {
  const double r = ::sqrt(a.v);
  return D1(r, a.d / (2.0 * r));
}

// dR/dx transposed into the block CRS: block (row = node of coordinate dof k,
// col = node of residual dof i), entry [k % 3][i % 3]
// (VectorFunction::gradient_x, src/elliptic/VectorFunction.hpp:317-408).
__global__ void k_gradient_x(CellIn m, Mat64 mat, const double* __restrict__ u, const double* __restrict__ z,
                             const int32_t* __restrict__ cell_entry, double* __restrict__ vals) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= m.C) return;
  int v[4];
  double x0[4][3], ue0[12];
  load_cell(m, c, v, x0);
  load_u(u, v, ue0);
  const double w = simp(cell_density(z, mat.layout, c, v), mat.p, mat.pmin);
  const Iso<D1> iso{D1(mat.iso.lam), D1(mat.iso.mu)};
  for (int k = 0; k < 12; ++k) {
    D1 x[4][3], g[4][3], vol, ue[12], e[6], sig[6], re[12];
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int d = 0; d < 3; ++d) x[n][d] = D1(x0[n][d], (3 * n + d == k) ? 1.0 : 0.0);
#pragma unroll
    for (int i = 0; i < 12; ++i) ue[i] = D1(ue0[i]);
    tet_geometry(x, g, vol);
    tet_strain(g, ue, e);
    tet_stress(iso, vol * D1(w), e, sig);
    tet_divergence(g, sig, re);
    const int a = k / 3, ka = k % 3;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      double* dst = vals + 9 * int64_t(cell_entry[16 * c + 4 * a + b]) + 3 * ka;
#pragma unroll
      for (int j = 0; j < 3; ++j) atomicAdd(&dst[j], re[3 * b + j].d);
    }
  }
}

__device__ __forceinline__ int64_t find_block(const int32_t* __restrict__ rowmap, const int32_t* __restrict__ cols,
                                              int32_t row, int32_t col) {
  for (int32_t k = rowmap[row]; k < rowmap[row + 1]; ++k)
    if (cols[k] == col) return k;
  return -1;
}

// Surface load's dependence on the face area, scale -1 (SurfaceLoadIntegral,
// src/SurfaceLoadIntegral.hpp:96-160): weight = -(1/6)|(x0-x2) x (x1-x2)|.
__global__ void k_traction_x(const int32_t* __restrict__ faces, const double* __restrict__ flux, int64_t nf,
                             const double* __restrict__ coords, const int32_t* __restrict__ rowmap,
                             const int32_t* __restrict__ cols, double* __restrict__ vals) {
  const int64_t f = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (f >= nf) return;
  const int32_t vs[3] = {faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]};
  for (int k = 0; k < 9; ++k) {
    D1 xs[3][3];
    for (int n = 0; n < 3; ++n)
      for (int d = 0; d < 3; ++d) xs[n][d] = D1(coords[3 * int64_t(vs[n]) + d], (3 * n + d == k) ? 1.0 : 0.0);
    D1 a[3], b[3];
    for (int d = 0; d < 3; ++d) {
      a[d] = xs[0][d] - xs[2][d];
      b[d] = xs[1][d] - xs[2][d];
    }
    const D1 cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2], cz = a[0] * b[1] - a[1] * b[0];
    const D1 wgt = D1(-1.0 / 6.0) * sqrt(cx * cx + cy * cy + cz * cz);
    const int an = k / 3, ka = k % 3;
    for (int bn = 0; bn < 3; ++bn) {
      const int64_t e = find_block(rowmap, cols, vs[an], vs[bn]);
      if (e < 0) continue;
      for (int j = 0; j < 3; ++j) atomicAdd(&vals[9 * e + 3 * ka + j], wgt.d * flux[3 * f + j]);
    }
  }
}

// df/dx of the internal energy (PhysicsScalarFunction::gradient_x).
__global__ void k_energy_grad_x(CellIn m, Mat64 mat, const double* __restrict__ u, const double* __restrict__ z,
                                double* __restrict__ gx) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= m.C) return;
  int v[4];
  double x0[4][3], ue0[12];
  load_cell(m, c, v, x0);
  load_u(u, v, ue0);
  const double w = simp(cell_density(z, mat.layout, c, v), mat.p, mat.pmin);
  const Iso<D1> iso{D1(mat.iso.lam), D1(mat.iso.mu)};
  for (int k = 0; k < 12; ++k) {
    D1 x[4][3], g[4][3], vol, ue[12], e[6], sig[6];
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int d = 0; d < 3; ++d) x[n][d] = D1(x0[n][d], (3 * n + d == k) ? 1.0 : 0.0);
#pragma unroll
    for (int i = 0; i < 12; ++i) ue[i] = D1(ue0[i]);
    tet_geometry(x, g, vol);
    tet_strain(g, ue, e);
    tet_stress(iso, vol * D1(w), e, sig);
    const D1 f = D1(0.5) * voigt_dot(sig, e);
    atomicAdd(&gx[3 * int64_t(v[k / 3]) + k % 3], f.d);
  }
}

CellIn cell_in(const Problem& P) { return CellIn{P.mesh->d_cells.get(), P.mesh->d_coords.get(), P.mesh->C}; }
Mat64 mat64(const Problem& P) { return Mat64{P.ep.iso(), P.ep.p, P.ep.pmin, P.ep.layout}; }

}  // namespace

void launch_traction(const Problem& P, double* r, double scale, cudaStream_t s) {
  const int64_t nf = int64_t(P.faces.size() / 3);
  if (!nf) return;
  k_traction<<<grid_for(nf), kThreads, 0, s>>>(P.d_faces.get(), P.d_face_flux.get(), nf, P.mesh->d_coords.get(),
                                               scale, r);
  PA_LAUNCHED();
}

void launch_gradient_u(const Problem& P, const double* z, double* entries, cudaStream_t s) {
  PA_CUDA(cudaMemsetAsync(entries, 0, sizeof(double) * 9 * P.mesh->B, s));
  k_gradient_u<<<grid_for(P.C()), kThreads, 0, s>>>(cell_in(P), mat64(P), z, P.mesh->d_cell_entry.get(), entries);
  PA_LAUNCHED();
}

void launch_gradient_z(const Problem& P, const double* u, const double* z, double* entries, cudaStream_t s) {
  if (P.ep.layout != PA_CONTROL_CELL) PA_CUDA(cudaMemsetAsync(entries, 0, sizeof(double) * 3 * P.mesh->B, s));
  k_gradient_z<<<grid_for(P.C()), kThreads, 0, s>>>(cell_in(P), mat64(P), u, z, P.mesh->d_cell_entry.get(), entries);
  PA_LAUNCHED();
}

void launch_energy(const Problem& P, const double* u, const double* z, double* partials, double* value_out,
                   double* grad_u, double* grad_z, cudaStream_t s) {
  if (grad_u) PA_CUDA(cudaMemsetAsync(grad_u, 0, sizeof(double) * P.ndof(), s));
  if (grad_z && P.ep.layout != PA_CONTROL_CELL) PA_CUDA(cudaMemsetAsync(grad_z, 0, sizeof(double) * P.N(), s));
  const int grid = grid_for(P.C());
  k_energy<<<grid, kThreads, 0, s>>>(cell_in(P), mat64(P), u, z, value_out ? partials : nullptr, grad_u, grad_z);
  PA_LAUNCHED();
  if (value_out) {
    k_sum_partials<<<1, 1024, 0, s>>>(partials, grid, value_out);
    PA_LAUNCHED();
  }
}

void launch_cell_weights(const Problem& P, const double* z, double* w64, float* w32, cudaStream_t s) {
  k_cell_weights<<<grid_for(P.C()), kThreads, 0, s>>>(cell_in(P), mat64(P), P.mesh->d_cell_perm.get(), z, w64, w32);
  PA_LAUNCHED();
}

void launch_diag(const Problem& P, const double* w, double* diag, cudaStream_t s) {
  PA_CUDA(cudaMemsetAsync(diag, 0, sizeof(double) * P.ndof(), s));
  k_diag<<<grid_for(P.C()), kThreads, 0, s>>>(cell_in(P), mat64(P), P.mesh->d_cell_perm.get(), w, diag);
  PA_LAUNCHED();
}

void launch_dRdz_transpose_times(const Problem& P, const double* u, const double* z, const double* lambda, double* g,
                                 cudaStream_t s) {
  k_dRdz_T<<<grid_for(P.C()), kThreads, 0, s>>>(cell_in(P), mat64(P), u, z, lambda, g);
  PA_LAUNCHED();
}

void launch_block_constraints(const Problem& P, double* entries, double* rhs, double scale, cudaStream_t s) {
  const int64_t nbc = int64_t(P.bc_dofs.size());
  if (!nbc) return;
  k_bc_first<<<grid_for(nbc), kThreads, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), scale,
                                                P.mesh->d_rowmap.get(), P.mesh->d_cols.get(), entries, rhs);
  PA_LAUNCHED();
  k_bc_second<<<grid_for(nbc), kThreads, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), scale, rhs);
  PA_LAUNCHED();
}

void launch_gradient_x(Problem& P, const double* u, const double* z, double* entries, cudaStream_t s) {
  if (!box_gradient_x(P, u, z, entries)) {  // box meshes: every block written once, no atomics
    PA_CUDA(cudaMemsetAsync(entries, 0, sizeof(double) * 9 * P.mesh->B, s));
    k_gradient_x<<<grid_for(P.C(), 128), 128, 0, s>>>(cell_in(P), mat64(P), u, z, P.mesh->d_cell_entry.get(), entries);
    PA_LAUNCHED();
  }
  const int64_t nf = int64_t(P.faces.size() / 3);
  if (nf) {
    k_traction_x<<<grid_for(nf), kThreads, 0, s>>>(P.d_faces.get(), P.d_face_flux.get(), nf, P.mesh->d_coords.get(),
                                                   P.mesh->d_rowmap.get(), P.mesh->d_cols.get(), entries);
    PA_LAUNCHED();
  }
}

void launch_energy_grad_x(const Problem& P, const double* u, const double* z, double* gx, cudaStream_t s) {
  PA_CUDA(cudaMemsetAsync(gx, 0, sizeof(double) * P.ndof(), s));
  k_energy_grad_x<<<grid_for(P.C(), 128), 128, 0, s>>>(cell_in(P), mat64(P), u, z, gx);
  PA_LAUNCHED();
}

void launch_scale(double* v, int64_t n, double a, cudaStream_t s) {
  k_scale<<<grid_for(std::min<int64_t>(n, 148LL * 8 * kThreads)), kThreads, 0, s>>>(v, n, a);
  PA_LAUNCHED();
}

template <typename T>
void launch_apply_tiled(const Problem& P, const T* w, const T* x, T* y, bool constrained, cudaStream_t s,
                        const T* plas) {
  ApplyArgs<T> a{};
  a.plas = plas;
  a.tv = P.mesh->tiles();
  a.tile_nodes = constrained ? P.d_tile_nodes_bc.get() : P.mesh->d_tile_nodes.get();
  a.N = P.N();
  a.coords = std::is_same<T, double>::value ? reinterpret_cast<const T*>(P.mesh->d_coords_soa.get())
                                            : reinterpret_cast<const T*>(P.mesh->d_coords32_soa.get());
  a.w = w;
  Iso<double> i64 = P.ep.iso();
  a.iso = Iso<T>{T(i64.lam), T(i64.mu)};
  a.x = x;
  a.y = y;
  PA_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * P.ndof(), s));
  const int grid = apply_kernel_setup<T, 0>(*P.mesh);
  launch_apply_kernel<T, 0>(*P.mesh, grid, s, a);
  PA_LAUNCHED();
}

template <typename S, typename T>
__global__ void k_aos_to_soa(const S* __restrict__ aos, T* __restrict__ soa, int64_t N) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t v = i / 3, d = i - 3 * v;
    soa[d * N + v] = T(aos[i]);
  }
}
template <typename T, typename S>
__global__ void k_soa_to_aos(const T* __restrict__ soa, S* __restrict__ aos, int64_t N) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t v = i / 3, d = i - 3 * v;
    aos[i] = S(soa[d * N + v]);
  }
}
template <typename T>
__global__ void k_copy_dofs(const int32_t* __restrict__ dofs, int64_t n, const T* __restrict__ src, T* __restrict__ dst) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) dst[dofs[i]] = src[dofs[i]];
}

template <typename S, typename T>
void launch_aos_to_soa(const S* aos, T* soa, int64_t N, cudaStream_t s) {
  k_aos_to_soa<S, T><<<grid_for(std::min<int64_t>(3 * N, 148LL * 8 * kThreads)), kThreads, 0, s>>>(aos, soa, N);
  PA_LAUNCHED();
}
template <typename T, typename S>
void launch_soa_to_aos(const T* soa, S* aos, int64_t N, cudaStream_t s) {
  k_soa_to_aos<T, S><<<grid_for(std::min<int64_t>(3 * N, 148LL * 8 * kThreads)), kThreads, 0, s>>>(soa, aos, N);
  PA_LAUNCHED();
}
template <typename T>
void launch_copy_dofs(const int32_t* dofs, int64_t n, const T* src, T* dst, cudaStream_t s) {
  if (!n) return;
  k_copy_dofs<T><<<grid_for(n), kThreads, 0, s>>>(dofs, n, src, dst);
  PA_LAUNCHED();
}
template void launch_aos_to_soa<double, double>(const double*, double*, int64_t, cudaStream_t);
template void launch_aos_to_soa<float, float>(const float*, float*, int64_t, cudaStream_t);
template void launch_soa_to_aos<double, double>(const double*, double*, int64_t, cudaStream_t);
template void launch_soa_to_aos<float, float>(const float*, float*, int64_t, cudaStream_t);
template void launch_aos_to_soa<double, float>(const double*, float*, int64_t, cudaStream_t);
template void launch_soa_to_aos<float, double>(const float*, double*, int64_t, cudaStream_t);
template void launch_copy_dofs<double>(const int32_t*, int64_t, const double*, double*, cudaStream_t);
template void launch_copy_dofs<float>(const int32_t*, int64_t, const float*, float*, cudaStream_t);

template void launch_apply_tiled<double>(const Problem&, const double*, const double*, double*, bool, cudaStream_t,
                                         const double*);
template void launch_apply_tiled<float>(const Problem&, const float*, const float*, float*, bool, cudaStream_t,
                                        const float*);

}  // namespace pa
