// pa_mg.cu -- CG preconditioned by a geometric multigrid V-cycle on
// structured box meshes (mesh_make_box): PA_SOLVER_PCG_MG.
//
// The reference solves the constrained system with AmgX's aggregation AMG
// preconditioning a Krylov method (src/alg/AmgXConfigs.cpp,
// src/alg/AmgXLinearSolver.cpp:34-73) or with AztecOO's ILU domain
// decomposition.  On a box mesh the hierarchy is geometric instead:
//  * level l+1 is the box with half the hexes per axis (same lengths), its
//    tets weighted by the mean SIMP weight of the 48 child tets; the
//    Dirichlet dofs of node (I,J,K) are those of fine node (2I,2J,2K);
//  * prolongation P: trilinear interpolation on the node lattice;
//    restriction R = P^T;
//  * smoothing: Chebyshev polynomial of degree 2 in D^-1 K on
//    [lmax/10, 1.15 lmax], lmax from 20 power iterations (FP32, matrix-free
//    tile kernel, zero-mean start); the same polynomial before and after the coarse correction, so
//    the V-cycle is a symmetric positive definite operator;
//  * coarsest level (10x5x5 hexes for a 160x80x80 box): solved exactly with
//    a dense FP64 inverse built per solve by blocked Gauss-Jordan elimination
//    (one matrix-vector product per V-cycle) when it has at most 2048 dofs
//    and the operator is elastic; otherwise (J2 tangents), or on request,
//    Chebyshev of degree 40 on [lmax/1000, 1.1 lmax].
// The outer CG runs in FP64 with the FP64 apply; it stops on the recursive
// residual and confirms on the true residual b' - K x.  For a J2 tangent
// solve the fine level (smoothing and outer CG) applies the consistent
// tangent and the coarse levels the elastic operator of the averaged weights
// (still a symmetric positive definite V-cycle).
#include <cmath>
#include <memory>
#include <vector>

#include "pa_cell.cuh"
#include "pa_dense.cuh"
#include "pa_problem.cuh"
#include "pa_tiled.cuh"

namespace pa {

namespace {

constexpr int kT = 256;
// grid-stride kernels
int grid_of(int64_t n) { return int(std::min<int64_t>((n + kT - 1) / kT, 148 * 16)); }
// one thread per item (no stride loop): every item needs its thread
int grid_all(int64_t n) { return int((n + kT - 1) / kT); }

// kernels of this library launched by the current multigrid solve (one
// host thread drives a problem at a time)
thread_local int64_t g_launches = 0;

// ------------------------------------------------------------- kernels --
// Mean SIMP weight of the 8 child hexes (48 tets) of each coarse hex.
__global__ void k_mg_coarse_weights(int64_t Cc, const int32_t* __restrict__ cperm, int cnx, int cny,
                                    const int32_t* __restrict__ fiperm, int fnx, int fny,
                                    const double* __restrict__ wf, double* __restrict__ w64, float* __restrict__ w32) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= Cc) return;
  const int64_t hex = cperm[i] / 6;
  const int64_t I = hex % cnx, J = (hex / cnx) % cny, K = hex / (int64_t(cnx) * cny);
  double s = 0.0;
  for (int c = 0; c < 2; ++c)
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        const int64_t fh = (2 * I + a) + fnx * ((2 * J + b) + int64_t(fny) * (2 * K + c));
        for (int t = 0; t < 6; ++t) s += wf[fiperm[6 * fh + t]];
      }
  const double w = s / 48.0;
  w64[i] = w;
  w32[i] = float(w);
}

// dinv = masked 1 / diag (diag interleaved FP64, dinv component-major FP32)
__global__ void k_mg_inv_diag(int64_t N, const double* __restrict__ diag, const uint8_t* __restrict__ mask,
                              float* __restrict__ dinv) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t v = i / 3, d = i - 3 * v;
    const double g = diag[i];
    dinv[d * N + v] = ((mask[v] >> d) & 1) || !(g > 0.0) ? 0.0f : float(1.0 / g);
  }
}

// Restriction (R = P^T of trilinear interpolation), coarse masked dofs zero.
__global__ void k_mg_restrict(int cnx, int cny, int cnz, const float* __restrict__ f, int64_t Nf,
                              const uint8_t* __restrict__ cmask, float* __restrict__ c, int64_t Nc) {
  const int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (v >= Nc) return;
  const int cpx = cnx + 1, cpy = cny + 1;
  const int I = int(v % cpx), J = int((v / cpx) % cpy), K = int(v / (int64_t(cpx) * cpy));
  const int fpx = 2 * cnx + 1, fpy = 2 * cny + 1, fpz = 2 * cnz + 1;
  float s[3] = {0.f, 0.f, 0.f};
  for (int dc = -1; dc <= 1; ++dc) {
    const int k = 2 * K + dc;
    if (k < 0 || k >= fpz) continue;
    const float wc = dc ? 0.5f : 1.0f;
    for (int db = -1; db <= 1; ++db) {
      const int j = 2 * J + db;
      if (j < 0 || j >= fpy) continue;
      const float wb = wc * (db ? 0.5f : 1.0f);
      for (int da = -1; da <= 1; ++da) {
        const int i = 2 * I + da;
        if (i < 0 || i >= fpx) continue;
        const float w = wb * (da ? 0.5f : 1.0f);
        const int64_t fv = i + int64_t(fpx) * (j + int64_t(fpy) * k);
#pragma unroll
        for (int d = 0; d < 3; ++d) s[d] += w * f[d * Nf + fv];
      }
    }
  }
  const uint8_t mk = cmask[v];
#pragma unroll
  for (int d = 0; d < 3; ++d) c[d * Nc + v] = ((mk >> d) & 1) ? 0.f : s[d];
}

// x_fine += P e (trilinear), fine masked dofs untouched.
__global__ void k_mg_prolong_add(int cnx, int cny, const float* __restrict__ e, int64_t Nc,
                                 const uint8_t* __restrict__ fmask, float* __restrict__ x, int64_t Nf) {
  const int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (v >= Nf) return;
  const int fpx = 2 * cnx + 1, fpy = 2 * cny + 1;
  const int i = int(v % fpx), j = int((v / fpx) % fpy), k = int(v / (int64_t(fpx) * fpy));
  const int cpx = cnx + 1, cpy = cny + 1;
  int ia[2], ja[2], ka[2];
  float wi[2], wj[2], wk[2];
  int ni, nj, nk;
  auto axis = [](int q, int (&idx)[2], float (&w)[2], int& n) {
    if (q % 2 == 0) {
      idx[0] = q / 2; w[0] = 1.f; n = 1;
    } else {
      idx[0] = q / 2; idx[1] = q / 2 + 1; w[0] = w[1] = 0.5f; n = 2;
    }
  };
  axis(i, ia, wi, ni);
  axis(j, ja, wj, nj);
  axis(k, ka, wk, nk);
  float s[3] = {0.f, 0.f, 0.f};
  for (int c = 0; c < nk; ++c)
    for (int b = 0; b < nj; ++b)
      for (int a = 0; a < ni; ++a) {
        const float w = wi[a] * wj[b] * wk[c];
        const int64_t cv = ia[a] + int64_t(cpx) * (ja[b] + int64_t(cpy) * ka[c]);
#pragma unroll
        for (int d = 0; d < 3; ++d) s[d] += w * e[d * Nc + cv];
      }
  const uint8_t mk = fmask[v];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (!((mk >> d) & 1)) x[d * Nf + v] += s[d];
}

// Chebyshev start: r = dinv (b - Ax) (Ax may be null: x = 0), d = r / theta
__global__ void k_cheb_start(int64_t n, const float* __restrict__ b, const float* __restrict__ ax,
                             const float* __restrict__ dinv, float inv_theta, float* __restrict__ r,
                             float* __restrict__ d) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float ri = dinv[i] * (ax ? b[i] - ax[i] : b[i]);
    r[i] = ri;
    d[i] = ri * inv_theta;
  }
}

// Chebyshev step: x += d; r -= dinv A d; d = c1 d + c2 r
__global__ void k_cheb_step(int64_t n, float* __restrict__ x, float* __restrict__ r, float* __restrict__ d,
                            const float* __restrict__ ad, const float* __restrict__ dinv, float c1, float c2) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float di = d[i];
    x[i] += di;
    const float ri = r[i] - dinv[i] * ad[i];
    r[i] = ri;
    d[i] = c1 * di + c2 * ri;
  }
}

__global__ void k_mg_add(int64_t n, float* __restrict__ x, const float* __restrict__ d) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] += d[i];
}

// out = a - b
__global__ void k_mg_sub(int64_t n, const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = a[i] - b[i];
}

// y = dinv * x (power iteration), plus ||y||^2 into acc
__global__ void k_mg_scale_norm(int64_t n, const float* __restrict__ x, const float* __restrict__ dinv,
                                float* __restrict__ y, double* __restrict__ acc);
__global__ void k_mg_norm2(int64_t n, const float* __restrict__ x, double* __restrict__ acc);


// x *= 1 / sqrt(*norm2) (a zero or non-finite norm leaves x unchanged)
__global__ void k_mg_scale_dev(int64_t n, float* __restrict__ x, const double* __restrict__ norm2) {
  const double q = *norm2;
  if (!(q > 0.0) || !isfinite(q)) return;
  const float sc = float(1.0 / sqrt(q));
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] *= sc;
}


// deterministic zero-mean start vector in [-1, 1], masked
__global__ void k_mg_seed(int64_t N, const uint8_t* __restrict__ mask, float* __restrict__ x) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t v = i % N, d = i / N;
    uint32_t h = uint32_t(i) * 2654435761u + 0x9e3779b9u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    x[i] = ((mask[v] >> d) & 1) ? 0.f : float(int(h % 2001u) - 1000) * 1e-3f;
  }
}

__global__ void k_mg_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    b[i] = float(a[i]);
}
__global__ void k_mg_to_f64(int64_t n, const float* __restrict__ a, double* __restrict__ b) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    b[i] = double(a[i]);
}

// FP64 outer-CG helpers.  Sums: warp shuffles, then one atomic per block.
__device__ __forceinline__ void block_add(double s, double* acc) {
  __shared__ double w[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? w[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(acc, s);
  }
}

__global__ void k_mg_dot(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                         double* __restrict__ acc) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += a[i] * b[i];
  block_add(s, acc);
}
// y = dinv * x (power iteration), plus ||y||^2 into acc
__global__ void k_mg_scale_norm(int64_t n, const float* __restrict__ x, const float* __restrict__ dinv,
                                float* __restrict__ y, double* __restrict__ acc) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float v = dinv[i] * x[i];
    y[i] = v;
    s += double(v) * v;
  }
  block_add(s, acc);
}

__global__ void k_mg_norm2(int64_t n, const float* __restrict__ x, double* __restrict__ acc) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += double(x[i]) * x[i];
  block_add(s, acc);
}

// sc = {rz, pq, rr, rz_new, alpha, beta, breakdown}
__global__ void k_mg_alpha(double* sc) {
  const double pq = sc[1];
  if (!(pq > 0.0) || !isfinite(pq)) {
    sc[4] = 0.0;
    sc[6] = 1.0;
  } else {
    sc[4] = sc[0] / pq;
  }
}
__global__ void k_mg_beta(double* sc) {
  sc[5] = sc[3] / sc[0];
  sc[0] = sc[3];
}
// x += alpha p; r -= alpha q (alpha on the device)
__global__ void k_mg_xr_dev(int64_t n, const double* __restrict__ sc, const double* __restrict__ p,
                            const double* __restrict__ q, double* __restrict__ x, double* __restrict__ r) {
  const double a = sc[4];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += a * p[i];
    r[i] -= a * q[i];
  }
}
// p = z + beta p (beta on the device)
__global__ void k_mg_p_dev(int64_t n, const double* __restrict__ sc, const double* __restrict__ z,
                           double* __restrict__ p) {
  const double beta = sc[5];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

// out = mask ? 0 : a - b   (SoA; b may be null)
__global__ void k_mg_res64(int64_t N, const double* __restrict__ a, const double* __restrict__ b,
                           const uint8_t* __restrict__ mask, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t v = i % N, d = i / N;
    out[i] = ((mask[v] >> d) & 1) ? 0.0 : a[i] - (b ? b[i] : 0.0);
  }
}
// x_soa[d N + v] = scale * value for each Dirichlet dof (dof = 3 v + d)
__global__ void k_mg_scatter_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                                double scale, int64_t N, double* __restrict__ x) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nbc) return;
  const int32_t dof = dofs[i];
  x[(dof % 3) * N + dof / 3] = scale * vals[i];
}
__global__ void k_mg_set_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                            double scale, double* __restrict__ x_aos) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nbc) return;
  x_aos[dofs[i]] = scale * vals[i];
}

// ---- coarsest level: dense inverse ---------------------------------------
// The coarsest box (10x5x5 hexes for 160x80x80, 1188 dofs) is solved exactly:
// its masked elastic operator is assembled as a dense FP64 matrix (component-
// major dofs d*N + v, padded to nd, a multiple of kGJ), Dirichlet and padding
// dofs carry identity rows/columns (the restricted right-hand side is zero
// there), and the matrix is inverted in place by blocked Gauss-Jordan
// elimination without pivoting (symmetric positive definite).  A V-cycle
// then costs one matrix-vector product at the bottom.
constexpr int64_t kDirectMaxDofs = 2048;

// one thread per tet: A[row, col] += the masked 12x12 stiffness
__global__ void k_mg_dense_assemble(int64_t C, const int32_t* __restrict__ perm, const int32_t* __restrict__ cells,
                                    const double* __restrict__ coords, const double* __restrict__ w,
                                    const uint8_t* __restrict__ mask, Iso<double> iso, int64_t N, int64_t nd,
                                    double* __restrict__ A) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= C) return;
  const int64_t u = perm[i];
  int64_t v[4];
  double x[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cells[4 * u + k];
#pragma unroll
    for (int d = 0; d < 3; ++d) x[k][d] = coords[3 * v[k] + d];
  }
  double g[4][3], vol;
  tet_geometry(x, g, vol);
  const double s = vol * w[i];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      double k9[9];
      tet_kblock(iso, s, g[a], g[b], k9);
      for (int di = 0; di < 3; ++di) {
        if ((mask[v[a]] >> di) & 1) continue;
        for (int dj = 0; dj < 3; ++dj) {
          if ((mask[v[b]] >> dj) & 1) continue;
          atomicAdd(&A[(di * N + v[a]) * nd + dj * N + v[b]], k9[3 * di + dj]);
        }
      }
    }
}

// identity on Dirichlet and padding dofs; diag0 = the diagonal before elimination
__global__ void k_mg_dense_ident(int64_t N, int64_t nd, const uint8_t* __restrict__ mask, double* __restrict__ A,
                                 double* __restrict__ diag0) {
  const int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (r >= nd) return;
  const bool fixed = r >= 3 * N || ((mask[r % N] >> (r / N)) & 1);
  if (fixed) A[r * nd + r] = 1.0;
  diag0[r] = A[r * nd + r];
}

}  // namespace

// ------------------------------------------------------------ hierarchy --
struct MgLevel {
  int n[3] = {0, 0, 0};
  int64_t N = 0, C = 0;
  Problem* P = nullptr;                // level 0: the caller's problem
  std::unique_ptr<Mesh> own_mesh;      // levels >= 1
  std::unique_ptr<Problem> own_prob;
  DevBuf<double> w64, diag;
  DevBuf<float> w32, dinv, x, b, r, d, ad;
  const float* plas = nullptr;  // level 0 of a J2 tangent solve: the FP32 tangent records
  float lmax = 0.f;
  DevBuf<float> ev;  // the power iteration's last vector: the next elastic solve starts from it
  bool ev_valid = false;  // ev (and lmax) come from an elastic operator
  // coarsest level, direct solve: the dense inverse (nd x nd) and its scratch
  int64_t nd = 0;
  DevBuf<double> dense, gj_c, gj_p, diag0, gj_flag;
  DevBuf<unsigned> gj_sync;
};

struct MgHierarchy {
  std::vector<std::unique_ptr<MgLevel>> L;
  int fine_n[3] = {0, 0, 0};
  double fine_l[3] = {0, 0, 0};
  bool coarse_direct = false;  // this solve's coarsest level uses the dense inverse
};

void mg_release(Problem& P) {
  delete P.mg;
  P.mg = nullptr;
}

namespace {

double host_dot(cudaStream_t s, DevBuf<double>& acc, int64_t n, const double* a, const double* b) {
  g_launches += 1;
  PA_CUDA(cudaMemsetAsync(acc.get(), 0, sizeof(double), s));
  k_mg_dot<<<grid_of(n), kT, 0, s>>>(n, a, b, acc.get());
  PA_LAUNCHED();
  double h = 0.0;
  PA_CUDA(cudaMemcpyAsync(&h, acc.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  return h;
}

// Dense inverse of the coarsest level's operator for this solve's weights;
// false when elimination met a non-positive pivot (a singular operator, e.g.
// no Dirichlet dofs), in which case the level keeps the Chebyshev solve.
bool coarse_factor(MgLevel& L, cudaStream_t s) {
  const int64_t n3 = 3 * L.N, nd = (n3 + kGJ - 1) / kGJ * kGJ;
  if (L.nd != nd) {
    L.dense.resize(nd * nd);
    L.gj_c.resize(nd * kGJ);
    L.gj_p.resize(2 * kGJ * kGJ);
    L.gj_sync.resize(1);
    L.diag0.resize(nd);
    L.gj_flag.resize(1);
    L.nd = nd;
  }
  const Mesh& m = *L.P->mesh;
  PA_CUDA(cudaMemsetAsync(L.dense.get(), 0, sizeof(double) * nd * nd, s));
  PA_CUDA(cudaMemsetAsync(L.gj_flag.get(), 0, sizeof(double), s));
  k_mg_dense_assemble<<<grid_all(L.C), kT, 0, s>>>(L.C, m.d_cell_perm.get(), m.d_cells.get(), m.d_coords.get(),
                                                   L.w64.get(), L.P->d_node_mask.get(), L.P->ep.iso(), L.N, nd,
                                                   L.dense.get());
  k_mg_dense_ident<<<grid_all(nd), kT, 0, s>>>(L.N, nd, L.P->d_node_mask.get(), L.dense.get(), L.diag0.get());
  PA_LAUNCHED();
  gj_invert(s, nd, L.dense.get(), L.diag0.get(), L.gj_c.get(), L.gj_p.get(), L.gj_sync.get(), L.gj_flag.get());
  g_launches += 3;
  double flag = 0.0;
  PA_CUDA(cudaMemcpyAsync(&flag, L.gj_flag.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  if (flag >= 2.0) throw Error(PA_ERR_CUDA, "coarsest factorization: a grid barrier timed out");
  return flag == 0.0;
}

// Dirichlet masks of a coarse level by injection from the fine level's node mask.
void coarse_bcs(const MgLevel& f, MgLevel& c, const std::vector<uint8_t>& fmask, std::vector<uint8_t>& cmask) {
  const int64_t fpx = f.n[0] + 1, fpy = f.n[1] + 1;
  const int64_t cpx = c.n[0] + 1, cpy = c.n[1] + 1, cpz = c.n[2] + 1;
  cmask.assign(size_t(c.N), 0);
  Problem& P = *c.P;
  P.bc_dofs.clear();
  P.bc_vals.clear();
  for (int64_t K = 0; K < cpz; ++K)
    for (int64_t J = 0; J < cpy; ++J)
      for (int64_t I = 0; I < cpx; ++I) {
        const int64_t cv = I + cpx * (J + cpy * K);
        const uint8_t m = fmask[size_t(2 * I + fpx * (2 * J + fpy * 2 * K))];
        cmask[size_t(cv)] = m;
        for (int d = 0; d < 3; ++d)
          if ((m >> d) & 1) {
            P.bc_dofs.push_back(int32_t(3 * cv + d));
            P.bc_vals.push_back(0.0);
          }
      }
  P.d_node_mask.upload(cmask.data(), cmask.size(), P.stream);
  std::vector<uint32_t> tn = P.mesh->h_tile_nodes;
  for (uint32_t& t : tn) t |= uint32_t(cmask[t & kNodeIdMask]) << kMaskShift;
  P.d_tile_nodes_bc.upload(tn.data(), tn.size(), P.stream);
  if (!P.bc_dofs.empty()) {
    P.d_bc_dofs.upload(P.bc_dofs.data(), P.bc_dofs.size(), P.stream);
    P.d_bc_vals.upload(P.bc_vals.data(), P.bc_vals.size(), P.stream);
  }
}

// Build (first use) or refresh the hierarchy for the problem's box mesh,
// weights w64 / w32 (tile order) and Dirichlet set.
void mg_setup(Problem& P, const double* w64, const float* w32, const double* diag_aos, const float* plas32,
              bool coarse_direct) {
  const Mesh& m = *P.mesh;
  PA_CHECK(m.box_n[0] > 0, "PA_SOLVER_PCG_MG needs a structured box mesh (pa_mesh_create_box)");
  PA_CHECK(m.box_n[0] % 2 == 0 && m.box_n[1] % 2 == 0 && m.box_n[2] % 2 == 0,
           "PA_SOLVER_PCG_MG needs even hex counts on every axis");
  cudaStream_t s = P.stream;
  bool rebuild = P.mg == nullptr;
  if (!rebuild)
    for (int a = 0; a < 3; ++a)
      rebuild = rebuild || P.mg->fine_n[a] != m.box_n[a] || P.mg->fine_l[a] != m.box_l[a];
  if (rebuild) {
    mg_release(P);
    std::unique_ptr<MgHierarchy> H(new MgHierarchy());
    for (int a = 0; a < 3; ++a) {
      H->fine_n[a] = m.box_n[a];
      H->fine_l[a] = m.box_l[a];
    }
    int n[3] = {m.box_n[0], m.box_n[1], m.box_n[2]};
    for (int l = 0;; ++l) {
      std::unique_ptr<MgLevel> L(new MgLevel());
      for (int a = 0; a < 3; ++a) L->n[a] = n[a];
      if (l == 0) {
        L->P = &P;
      } else {
        L->own_mesh.reset(new Mesh());
        L->own_mesh->tile_clusters = m.tile_clusters;
        mesh_make_box(*L->own_mesh, n[0], n[1], n[2], m.box_l[0], m.box_l[1], m.box_l[2]);
        L->own_prob.reset(new Problem());
        L->own_prob->mesh = L->own_mesh.get();
        L->own_prob->ep = P.ep;
        L->own_prob->stream = s;
        L->P = L->own_prob.get();
        L->w64.resize(L->own_mesh->C);
        L->w32.resize(L->own_mesh->C);
        L->diag.resize(3 * L->own_mesh->N);
      }
      L->N = L->P->N();
      L->C = L->P->C();
      const int64_t n3 = 3 * L->N;
      L->dinv.resize(n3);
      L->x.resize(n3);
      L->b.resize(n3);
      L->r.resize(n3);
      L->d.resize(n3);
      L->ad.resize(n3);
      H->L.push_back(std::move(L));
      // coarsen while every axis stays even and the box keeps >= 2 hexes per axis
      if (n[0] % 2 || n[1] % 2 || n[2] % 2 || std::min(std::min(n[0], n[1]), n[2]) < 4) break;
      for (int a = 0; a < 3; ++a) n[a] /= 2;
    }
    PA_CHECK(H->L.size() >= 2, "PA_SOLVER_PCG_MG needs at least one coarse level");
    P.mg = H.release();
  }
  MgHierarchy& H = *P.mg;
  H.L[0]->plas = plas32;  // the coarse levels carry the elastic operator
  // of the fine problem's current material (a J2 solve sets its own E, nu)
  for (size_t l = 1; l < H.L.size(); ++l) H.L[l]->own_prob->ep = P.ep;
  // Dirichlet sets by injection
  std::vector<uint8_t> fmask(size_t(P.N()), 0);
  for (int32_t dof : P.bc_dofs) fmask[size_t(dof / 3)] |= uint8_t(1u << (dof % 3));
  for (size_t l = 1; l < H.L.size(); ++l) {
    std::vector<uint8_t> cmask;
    coarse_bcs(*H.L[l - 1], *H.L[l], fmask, cmask);
    fmask.swap(cmask);
  }
  // weights, inverse diagonals
  for (size_t l = 0; l < H.L.size(); ++l) {
    MgLevel& L = *H.L[l];
    const double* ldiag = diag_aos;
    if (l > 0) {
      MgLevel& F = *H.L[l - 1];
      k_mg_coarse_weights<<<grid_all(L.C), kT, 0, s>>>(L.C, L.P->mesh->d_cell_perm.get(), L.n[0], L.n[1],
                                                      F.P->mesh->d_cell_iperm.get(), F.n[0], F.n[1],
                                                      l == 1 ? w64 : F.w64.get(), L.w64.get(), L.w32.get());
      PA_LAUNCHED();
      launch_diag(*L.P, L.w64.get(), L.diag.get(), s);
      ldiag = L.diag.get();
      g_launches += 2;
    }
    k_mg_inv_diag<<<grid_of(3 * L.N), kT, 0, s>>>(L.N, ldiag, L.P->d_node_mask.get(), L.dinv.get());
    PA_LAUNCHED();
    g_launches += 1;
  }
  MgLevel& Lc = *H.L.back();
  H.coarse_direct = coarse_direct && 3 * Lc.N <= kDirectMaxDofs && coarse_factor(Lc, s);
  // lmax of D^-1 K per level: power iteration, all on the device (each
  // step's squared norm lands in norms[level][step]; the scaling kernel reads
  // it there), one host read for every level at the end.  An elastic solve
  // after an elastic solve on the same hierarchy (new SIMP weights) starts
  // from the previous vector, takes 5 steps and keeps at least 0.95 of the
  // previous estimate; every other solve starts from a seed and takes 20 (a
  // J2 tangent changes too much between Newton iterations for a warm start:
  // measured, the 80x40x40 bar then stopped converging).
  constexpr int kPower = 20, kPowerWarm = 5;
  const size_t NL = H.L.size();
  const size_t NP = H.coarse_direct ? NL - 1 : NL;  // levels that smooth (need lmax)
  DevBuf<double> norms(NL * (kPower + 1));
  PA_CUDA(cudaMemsetAsync(norms.get(), 0, sizeof(double) * NL * (kPower + 1), s));
  for (size_t l = 0; l < NP; ++l) {
    MgLevel& L = *H.L[l];
    const float* lw32 = l == 0 ? w32 : L.w32.get();
    const int64_t n3 = 3 * L.N;
    double* nl = norms.get() + l * (kPower + 1);
    if (L.ev.n != size_t(n3)) {
      L.ev.resize(n3);
      L.ev_valid = false;
    }
    const bool warm = L.ev_valid && plas32 == nullptr;
    if (warm)
      PA_CUDA(cudaMemcpyAsync(L.x.get(), L.ev.get(), sizeof(float) * n3, cudaMemcpyDeviceToDevice, s));
    else
      k_mg_seed<<<grid_of(n3), kT, 0, s>>>(L.N, L.P->d_node_mask.get(), L.x.get());
    k_mg_norm2<<<grid_of(n3), kT, 0, s>>>(n3, L.x.get(), nl);
    k_mg_scale_dev<<<grid_of(n3), kT, 0, s>>>(n3, L.x.get(), nl);  // unit start vector
    PA_LAUNCHED();
    g_launches += 3;
    const int steps = warm ? kPowerWarm : kPower;
    for (int it = 1; it <= steps; ++it) {
      launch_apply_tiled<float>(*L.P, lw32, L.x.get(), L.ad.get(), true, s, L.plas);
      k_mg_scale_norm<<<grid_of(n3), kT, 0, s>>>(n3, L.ad.get(), L.dinv.get(), L.x.get(), nl + it);
      k_mg_scale_dev<<<grid_of(n3), kT, 0, s>>>(n3, L.x.get(), nl + it);
      PA_LAUNCHED();
      g_launches += 3;
    }
    PA_CUDA(cudaMemcpyAsync(L.ev.get(), L.x.get(), sizeof(float) * n3, cudaMemcpyDeviceToDevice, s));
  }
  std::vector<double> h(NL * (kPower + 1));
  PA_CUDA(cudaMemcpyAsync(h.data(), norms.get(), sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  for (size_t l = 0; l < NP; ++l) {
    PA_CHECK(h[l * (kPower + 1)] > 0.0, "multigrid level without free dofs");
    double lam = 0.0;  // ||D^-1 K x|| with ||x|| = 1 approaches lmax from below
    for (int it = 1; it <= kPower; ++it) {
      const double v = h[l * (kPower + 1) + it];
      if (std::isfinite(v)) lam = std::max(lam, std::sqrt(v));
    }
    PA_CHECK(lam > 0.0, "multigrid: no spectral estimate (zero operator?)");
    MgLevel& L = *H.L[l];
    if (L.ev_valid && plas32 == nullptr) lam = std::max(lam, 0.95 * double(L.lmax));
    L.lmax = float(lam);
    L.ev_valid = plas32 == nullptr;
  }
}

struct Cheb {
  float inv_theta;
  std::vector<float> c1, c2;  // per step k >= 1
};

Cheb cheb_coeffs(float lmin, float lmax, int deg) {
  Cheb c;
  const double theta = 0.5 * (double(lmax) + lmin), delta = 0.5 * (double(lmax) - lmin), sigma = theta / delta;
  c.inv_theta = float(1.0 / theta);
  double rho = 1.0 / sigma;
  for (int k = 1; k < deg; ++k) {
    const double rn = 1.0 / (2.0 * sigma - rho);
    c.c1.push_back(float(rn * rho));
    c.c2.push_back(float(2.0 * rn / delta));
    rho = rn;
  }
  return c;
}

// x <- Chebyshev iteration on D^-1 K x = D^-1 b (x == 0 on entry if zero_x)
void cheb(MgLevel& L, const float* w32, const float* b, float* x, bool zero_x, const Cheb& c, int deg,
          cudaStream_t s) {
  const int64_t n3 = 3 * L.N;
  if (zero_x) {
    PA_CUDA(cudaMemsetAsync(x, 0, sizeof(float) * n3, s));
    k_cheb_start<<<grid_of(n3), kT, 0, s>>>(n3, b, nullptr, L.dinv.get(), c.inv_theta, L.r.get(), L.d.get());
  } else {
    launch_apply_tiled<float>(*L.P, w32, x, L.ad.get(), true, s, L.plas);
    k_cheb_start<<<grid_of(n3), kT, 0, s>>>(n3, b, L.ad.get(), L.dinv.get(), c.inv_theta, L.r.get(), L.d.get());
  }
  PA_LAUNCHED();
  g_launches += zero_x ? 1 : 2;
  for (int k = 1; k < deg; ++k) {
    g_launches += 2;
    launch_apply_tiled<float>(*L.P, w32, L.d.get(), L.ad.get(), true, s, L.plas);
    k_cheb_step<<<grid_of(n3), kT, 0, s>>>(n3, x, L.r.get(), L.d.get(), L.ad.get(), L.dinv.get(), c.c1[k - 1],
                                           c.c2[k - 1]);
    PA_LAUNCHED();
  }
  k_mg_add<<<grid_of(n3), kT, 0, s>>>(n3, x, L.d.get());
  PA_LAUNCHED();
  g_launches += 1;
}

constexpr int kSmoothDeg = 2, kCoarseDeg = 40;

// x_l = V(b_l): both in the level's buffers
void vcycle(MgHierarchy& H, size_t l, const float* w32_fine, cudaStream_t s) {
  MgLevel& L = *H.L[l];
  const float* w32 = l == 0 ? w32_fine : L.w32.get();
  if (l + 1 == H.L.size()) {
    if (H.coarse_direct) {
      const int64_t n3 = 3 * L.N;
      k_mg_dense_solve<<<grid_all(32 * n3), kT, 0, s>>>(n3, L.nd, L.dense.get(), L.b.get(), L.x.get());
      PA_LAUNCHED();
      g_launches += 1;
      return;
    }
    const Cheb c = cheb_coeffs(L.lmax * 1.1f / 1000.f, L.lmax * 1.1f, kCoarseDeg);
    cheb(L, w32, L.b.get(), L.x.get(), true, c, kCoarseDeg, s);
    return;
  }
  const Cheb c = cheb_coeffs(L.lmax * 1.15f / 10.f, L.lmax * 1.15f, kSmoothDeg);
  cheb(L, w32, L.b.get(), L.x.get(), true, c, kSmoothDeg, s);
  // residual -> coarse right-hand side
  const int64_t n3 = 3 * L.N;
  launch_apply_tiled<float>(*L.P, w32, L.x.get(), L.ad.get(), true, s, L.plas);
  k_mg_sub<<<grid_of(n3), kT, 0, s>>>(n3, L.b.get(), L.ad.get(), L.r.get());
  PA_LAUNCHED();
  MgLevel& Cl = *H.L[l + 1];
  k_mg_restrict<<<grid_all(Cl.N), kT, 0, s>>>(Cl.n[0], Cl.n[1], Cl.n[2], L.r.get(), L.N, Cl.P->d_node_mask.get(),
                                            Cl.b.get(), Cl.N);
  PA_LAUNCHED();
  g_launches += 3;
  vcycle(H, l + 1, w32_fine, s);
  g_launches += 1;
  k_mg_prolong_add<<<grid_all(L.N), kT, 0, s>>>(Cl.n[0], Cl.n[1], Cl.x.get(), Cl.N, L.P->d_node_mask.get(), L.x.get(),
                                              L.N);
  PA_LAUNCHED();
  cheb(L, w32, L.b.get(), L.x.get(), false, c, kSmoothDeg, s);
}

}  // namespace

// Solve K x = b (interleaved b, x_out) for the operator's weights with
// multigrid-preconditioned CG; options as pa_solve (rel_tol, max_iters).
pa_status solve_mg(Problem& P, const SolveOperator& op, const double* b, double* x_out, const pa_solve_options& o,
                   pa_solve_stats* st) {
  cudaStream_t s = P.stream;
  PA_CHECK(o.rel_tol > 0.0, "rel_tol must be positive");
  PA_CHECK(op.w32 != nullptr, "multigrid needs the FP32 weights");
  PA_CHECK((op.plas64 == nullptr) == (op.plas32 == nullptr), "J2 tangent records in both precisions");
  const int64_t N = P.N(), n = P.ndof();
  SolverWorkspace& ws = P.ws;
  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  g_launches = 0;
  P.ws.ensure(n, P.C(), 1, true);
  PA_CHECK(o.mg_coarse_solver == PA_MG_COARSE_AUTO || o.mg_coarse_solver == PA_MG_COARSE_CHEBYSHEV,
           "mg_coarse_solver must be PA_MG_COARSE_AUTO or PA_MG_COARSE_CHEBYSHEV");
  // AUTO: the dense coarse inverse for elastic operators.  A J2 tangent
  // solve keeps the Chebyshev coarse solve: its coarse levels carry the
  // elastic operator, only a model of the plastic tangent, and with
  // Eisenstat-Walker tolerances the exact coarse solve left one load step of
  // the 80x40x40 bar unconverged (measured; with tight tolerances both
  // coarse solves give the same Newton iterations).
  mg_setup(P, op.w64, op.w32, op.diag_aos, op.plas32,
           o.mg_coarse_solver == PA_MG_COARSE_AUTO && op.plas32 == nullptr);
  MgHierarchy& H = *P.mg;
  MgLevel& F = *H.L[0];
  const uint8_t* mask = P.d_node_mask.get();
  const int vg = grid_of(n);
  DevBuf<double> acc(1);
  // b' = mask(b - K x_D); vectors component-major
  double* bp = ws.b.get();
  double* x = ws.x.get();
  double* r = ws.r.get();
  double* z = ws.p0.get();
  double* p = ws.p1.get();
  double* q = ws.ap.get();
  double* t = ws.t.get();
  const int64_t nbc = op.homogeneous_bc ? 0 : int64_t(P.bc_dofs.size());
  launch_aos_to_soa<double, double>(b, t, N, s);
  if (nbc) {
    PA_CUDA(cudaMemsetAsync(z, 0, sizeof(double) * n, s));
    k_mg_scatter_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), op.bc_scale, N,
                                                           z);
    PA_LAUNCHED();
    launch_apply_tiled<double>(P, op.w64, z, q, false, s, op.plas64);
    k_mg_res64<<<vg, kT, 0, s>>>(N, t, q, mask, bp);
  } else {
    k_mg_res64<<<vg, kT, 0, s>>>(N, t, nullptr, mask, bp);
  }
  PA_LAUNCHED();
  double bb = host_dot(s, acc, n, bp, bp);
  if (!(bb > 0.0)) bb = 1.0;
  const double tol2 = o.rel_tol * o.rel_tol * bb;
  const int max_iters = o.max_iters > 0 ? o.max_iters : 1000;
  PA_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
  PA_CUDA(cudaMemcpyAsync(r, bp, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  // z = V(r): conversion, V-cycle, conversion, captured once per solve as a
  // CUDA graph (hundreds of small launches on the coarse levels) and replayed
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  struct GraphGuard {
    cudaGraph_t& g;
    cudaGraphExec_t& e;
    ~GraphGuard() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
    }
  } guard_graph{graph, gexec};
  const int64_t launches_before = g_launches;
  PA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  k_mg_to_f32<<<vg, kT, 0, s>>>(n, r, F.b.get());
  vcycle(H, 0, op.w32, s);
  k_mg_to_f64<<<vg, kT, 0, s>>>(n, F.x.get(), z);
  g_launches += 2;
  {
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) throw Error(PA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
  }
  PA_CUDA(cudaGraphInstantiate(&gexec, graph, 0));
  const int64_t per_precondition = g_launches - launches_before;
  g_launches = launches_before;
  auto precondition = [&]() {
    PA_CUDA(cudaGraphLaunch(gexec, s));
    g_launches += per_precondition;
  };
  // Outer CG with its scalars on the device: sc = {rz, pq, rr, rz_new, alpha,
  // beta, breakdown}; alpha and beta come from one-thread kernels, and the
  // host reads (rr, breakdown) once per iteration for the stopping test.
  DevBuf<double> scal(8);
  double* dsc = scal.get();
  auto dot_into = [&](const double* a, const double* b2, int slot) {
    PA_CUDA(cudaMemsetAsync(dsc + slot, 0, sizeof(double), s));
    k_mg_dot<<<vg, kT, 0, s>>>(n, a, b2, dsc + slot);
    PA_LAUNCHED();
    g_launches += 1;
  };
  auto read_rr = [&](double& rr, bool& bd) {
    double h[2];
    PA_CUDA(cudaMemcpyAsync(h, dsc + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaMemcpyAsync(h + 1, dsc + 6, sizeof(double), cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    rr = h[0];
    bd = h[1] != 0.0;
  };
  int iters = 0, restarts = 0;
  double rr_true = bb;
  bool converged = false, breakdown = false;
  while (!converged && iters < max_iters && !breakdown) {
    PA_CUDA(cudaMemsetAsync(dsc + 6, 0, sizeof(double), s));
    precondition();
    PA_CUDA(cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    dot_into(r, z, 0);  // rz
    dot_into(r, r, 2);  // rr
    double rr = 0.0;
    bool bd = false;
    read_rr(rr, bd);
    while (rr > tol2 && iters < max_iters) {
      launch_apply_tiled<double>(P, op.w64, p, q, true, s, op.plas64);
      dot_into(p, q, 1);  // pq
      k_mg_alpha<<<1, 1, 0, s>>>(dsc);
      k_mg_xr_dev<<<vg, kT, 0, s>>>(n, dsc, p, q, x, r);
      PA_LAUNCHED();
      g_launches += 3;
      ++iters;
      dot_into(r, r, 2);  // rr
      read_rr(rr, bd);
      if (bd) { breakdown = true; break; }
      if (rr <= tol2) break;
      precondition();
      dot_into(r, z, 3);  // rz_new
      k_mg_beta<<<1, 1, 0, s>>>(dsc);
      k_mg_p_dev<<<vg, kT, 0, s>>>(n, dsc, z, p);
      PA_LAUNCHED();
      g_launches += 2;
    }
    // confirm on the true residual r = b' - K x
    launch_apply_tiled<double>(P, op.w64, x, q, true, s, op.plas64);
    k_mg_res64<<<vg, kT, 0, s>>>(N, bp, q, mask, r);
    PA_LAUNCHED();
    g_launches += 2;
    rr_true = host_dot(s, acc, n, r, r);
    converged = rr_true <= tol2;
    if (!converged) ++restarts;
  }
  // x_out = x + x_D (interleaved)
  launch_soa_to_aos<double, double>(x, x_out, N, s);
  if (nbc) {
    k_mg_set_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), op.bc_scale, x_out);
    PA_LAUNCHED();
  }
  PA_CUDA(cudaEventRecord(P.ev1, s));
  PA_CUDA(cudaEventSynchronize(P.ev1));
  const double relres = std::sqrt(rr_true / bb);
  if (st) {
    st->iterations = iters;
    st->replacements = restarts;
    st->rel_residual = relres;
    st->converged = converged ? 1 : 0;
    st->kernel_launches = g_launches + 6;  // + the right-hand side and output conversions
    st->fallback_iterations = 0;
  }
  if (breakdown) return PA_ERR_BREAKDOWN;
  if (!std::isfinite(relres)) return PA_ERR_NONFINITE;
  return converged ? PA_OK : PA_ERR_NOT_CONVERGED;
}

}  // namespace pa
