// pa_solver.cu -- matrix-free Jacobi-preconditioned CG on the
// Dirichlet-constrained stiffness system, FP64 or mixed precision.
//
// The reference hands the assembled, symmetrically constrained block CRS to
// AmgX or AztecOO (AbstractSolver::solve, src/alg/PlatoAbstractSolver.hpp:19-27;
// constraints by applyBlockConstraints, src/ApplyConstraints.hpp:11-79).  This
// solver solves the same linear system without assembling it:
//   K_ff x_f = b_f - K_fc x_D,   x_c = x_D,
// i.e. the constrained rows/columns are masked in the matrix-free apply.
//
// One CG iteration is two kernels:
//   K1 (pa_tiled.cuh, mode 1): p = D^-1 r + beta p_old (formed while staging),
//      Ap = K p, and p.Ap from per-cell energies; its last CTA sets alpha.
//   K2 (k_cg_update): x += alpha p, r -= alpha Ap, Ap = 0, r.z and r.r; its
//      last CTA sets beta and the convergence flag.
// All scalars stay on the device; chunks of iterations are captured once in a
// CUDA graph and replayed; the host reads the scalars once per chunk.
//
// Mixed precision: K1/K2 run on FP32 vectors and the FP32 operator (dots
// accumulated in FP64); x is kept in FP64 and the FP32 update dx is folded in
// once per chunk, where the FP64 true residual b - K x is recomputed with the
// FP64 operator and replaces the recursive FP32 residual (reliable updates),
// and convergence is decided on that FP64 residual.
#include <cmath>
#include <cstddef>
#include <algorithm>

#include "pa_learned.cuh"
#include "pa_problem.cuh"
#include "pa_tiled.cuh"

namespace pa {

namespace {

constexpr int kVecThreads = 256;

int vec_grid(int64_t n) {
  const int64_t want = (n + kVecThreads - 1) / kVecThreads;
  const int64_t cap = int64_t(num_sms()) * 8;
  return int(std::max<int64_t>(1, std::min(want, cap)));
}

__device__ __forceinline__ void block_sum2(double& a, double& b, double* smem /*64*/) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) { smem[warp] = a; smem[32 + warp] = b; }
  __syncthreads();
  a = b = 0.0;
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    a = lane < nw ? smem[lane] : 0.0;
    b = lane < nw ? smem[32 + lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
  }
}

// 16-byte vector of T (float4 / double2) for the streaming kernels.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
};

template <typename T>
__device__ __forceinline__ void cg_update_one(T& x, T& r, T p, T& ap, T dinv, T a, double& rz, double& rr) {
  x += a * p;
  const T ri = r - a * ap;
  r = ri;
  ap = T(0);
  rz += double(ri) * double(dinv * ri);
  rr += double(ri) * double(ri);
}

// CG update (K2): x += alpha p, r -= alpha Ap, Ap = 0, r.z and r.r; the last
// CTA sets beta, the iteration count and the convergence flag.  All vectors
// are T (the iterate is an FP32 correction in mixed precision) and 16-byte
// aligned; the body streams them as 16-byte vectors.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_cg_update(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                                           const T* __restrict__ p, T* __restrict__ ap,
                                                           const T* __restrict__ dinv, PcgScalars* __restrict__ sc,
                                                           double* __restrict__ partials, unsigned int* counter,
                                                           double* __restrict__ rr_hist) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  __shared__ double s_red[64];
  if (sc->done) return;
  const T a = T(sc->alpha);
  double rz = 0.0, rr = 0.0;
  const int64_t nv = n / W;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += stride) {
    V xv = reinterpret_cast<V*>(x)[i], rv = reinterpret_cast<V*>(r)[i], av = reinterpret_cast<V*>(ap)[i];
    const V pv = reinterpret_cast<const V*>(p)[i], dv = reinterpret_cast<const V*>(dinv)[i];
    T* xs = reinterpret_cast<T*>(&xv);
    T* rs = reinterpret_cast<T*>(&rv);
    T* as = reinterpret_cast<T*>(&av);
    const T* ps = reinterpret_cast<const T*>(&pv);
    const T* ds = reinterpret_cast<const T*>(&dv);
#pragma unroll
    for (int k = 0; k < W; ++k) cg_update_one(xs[k], rs[k], ps[k], as[k], ds[k], a, rz, rr);
    reinterpret_cast<V*>(x)[i] = xv;
    reinterpret_cast<V*>(r)[i] = rv;
    reinterpret_cast<V*>(ap)[i] = av;
  }
  for (int64_t i = nv * W + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += stride)
    cg_update_one(x[i], r[i], p[i], ap[i], dinv[i], a, rz, rr);
  block_sum2(rz, rr, s_red);
  if (threadIdx.x == 0) { partials[2 * blockIdx.x] = rz; partials[2 * blockIdx.x + 1] = rr; }
  if (last_block_arrive(counter)) {
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
      t0 += __ldcg(&partials[2 * i]);
      t1 += __ldcg(&partials[2 * i + 1]);
    }
    block_sum2(t0, t1, s_red);
    if (threadIdx.x == 0) {
      sc->beta = t0 / sc->rz;
      sc->rz_prev = sc->rz;
      sc->rz = t0;
      sc->rr = t1;
      const int it = sc->iters + 1;
      sc->iters = it;
      if (rr_hist) rr_hist[it] = t1;
      if (!isfinite(t0) || !isfinite(t1)) { sc->breakdown = 1; sc->done = 1; }
      if (t1 <= sc->stop2) sc->done = 1;
      *counter = 0u;
    }
  }
}

// r.z, r.r of a fresh residual (z = D^-1 r); resets beta, sets stop2 = tol2 * bb.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_cg_init(int64_t n, const T* __restrict__ r, const T* __restrict__ dinv,
                                                         PcgScalars* __restrict__ sc, double* __restrict__ partials,
                                                         unsigned int* counter, double tol2, int reset) {
  __shared__ double s_red[64];
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double ri = double(r[i]);
    rz += ri * double(dinv[i] * r[i]);
    rr += ri * ri;
  }
  block_sum2(rz, rr, s_red);
  if (threadIdx.x == 0) { partials[2 * blockIdx.x] = rz; partials[2 * blockIdx.x + 1] = rr; }
  if (last_block_arrive(counter)) {
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
      t0 += __ldcg(&partials[2 * i]);
      t1 += __ldcg(&partials[2 * i + 1]);
    }
    block_sum2(t0, t1, s_red);
    if (threadIdx.x == 0) {
      sc->rz = t0;
      sc->rr = t1;
      if (reset) {
        sc->beta = 0.0;
        sc->bb = t1;
        sc->iters = 0;
        sc->breakdown = 0;
        sc->stop2 = tol2 * t1;
      }
      sc->done = (t1 <= sc->stop2) ? 1 : 0;
      *counter = 0u;
    }
  }
}

// Vectors inside the solver are component-major (SoA, v[d * N + node]); the
// ABI's vectors are interleaved (AoS, v[3 * node + d]).  mask[node] bit d
// marks a constrained dof.

// out_soa = mask ? 0 : a_aos - t_soa   (t may be null)
__global__ void k_aos_minus_soa(int64_t N, const double* __restrict__ a, const double* __restrict__ t,
                                const uint8_t* __restrict__ mask, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    const bool c = mask && ((mask[v] >> d) & 1);
    out[i] = c ? 0.0 : a[3 * v + d] - (t ? t[i] : 0.0);
  }
}

// out = mask ? 0 : a - b   (all SoA)
__global__ void k_sub_masked(int64_t N, const double* __restrict__ a, const double* __restrict__ b,
                             const uint8_t* __restrict__ mask, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    const bool c = mask && ((mask[v] >> d) & 1);
    out[i] = c ? 0.0 : a[i] - b[i];
  }
}

// D^-1 (SoA) from the interleaved diagonal; constrained and zero entries -> 0.
template <typename T>
__global__ void k_inv_diag(int64_t N, const double* __restrict__ diag_aos, const uint8_t* __restrict__ mask,
                           T* __restrict__ dinv) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    const bool c = mask && ((mask[v] >> d) & 1);
    const double g = diag_aos[3 * v + d];
    dinv[i] = (c || g == 0.0) ? T(0) : T(1.0 / g);
  }
}

__global__ void k_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(a[i]);
}

// x += dx; dx = 0
__global__ void k_fold(int64_t n, double* __restrict__ x, float* __restrict__ dx) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += double(dx[i]);
    dx[i] = 0.0f;
  }
}

// Dirichlet lift vector (SoA): xd[d * N + node] = scale * value for each BC dof.
__global__ void k_scatter_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                             double scale, int64_t N, double* __restrict__ xd) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < nbc) xd[(dofs[i] % 3) * N + dofs[i] / 3] = scale * vals[i];
}

// x[dof] = scale * value (final solution on constrained dofs).
__global__ void k_set_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals, double scale,
                         double* __restrict__ x) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < nbc) x[dofs[i]] = scale * vals[i];
}

__global__ void k_dot2(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
  __shared__ double s_red[64];
  double s = 0.0, t = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    s += a[i] * a[i];
    t += b[i] * b[i];
  }
  block_sum2(s, t, s_red);
  if (threadIdx.x == 0) { atomicAdd(&out[0], s); atomicAdd(&out[1], t); }
}

// ---------------------------------------------------------- flexible CG --
// Flexible CG (one-term truncation) with the learned preconditioner M:
//   z = M r,  beta = -(z . q_old) / (p_old . q_old),  p = z + beta p_old,
//   q = K p,  alpha = (z . r) / (p . q),  x += alpha p,  r -= alpha q.
// p, q and p.q come from the fused apply kernel in its PCG mode, given z in
// place of r and an all-ones vector in place of D^-1.
struct FcgState {
  double rdr;      // r . D^-1 r of the current residual (the network's input scale)
  double pq_prev;  // p . K p of the previous direction
  int32_t first;   // 1: the next direction is z itself
  int32_t pad;
  double gamma;    // weight of the network's correction in z
};

// Weight of the network's correction c = s D^-1/2 f: z = D^-1 r + gamma c with
// gamma = 1, reduced to 0.5 (r.D^-1 r) / (-c.r) when c.r < -0.5 r.D^-1 r, so
// that z.r >= 0.5 r.D^-1 r > 0 (z is always a descent direction).
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_fcg_gamma(int64_t N, const T* __restrict__ r,
                                                           const float* __restrict__ dsq,
                                                           const float* __restrict__ out, FcgState* __restrict__ fs,
                                                           double inv_nfree, PcgScalars* __restrict__ sc,
                                                           double* __restrict__ partials, unsigned int* counter) {
  __shared__ double s_red[64];
  if (sc->done) return;
  const double s2 = fs->rdr * inv_nfree;
  const double sig = s2 > 0.0 ? sqrt(s2) : 0.0;
  double cr = 0.0, unused = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    cr += double(dsq[i]) * double(out[4 * v + d]) * double(r[i]);
  }
  block_sum2(cr, unused, s_red);
  if (threadIdx.x == 0) partials[2 * blockIdx.x] = cr;
  if (last_block_arrive(counter)) {
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) t0 += __ldcg(&partials[2 * i]);
    block_sum2(t0, t1, s_red);
    if (threadIdx.x == 0) {
      const double c = sig * t0, a = fs->rdr;
      fs->gamma = (c < -0.5 * a) ? -0.5 * a / c : 1.0;
      *counter = 0u;
    }
  }
}

// z = D^-1 r + gamma s D^-1/2 f; z.q_old, z.r and p_old.r; q = 0 for the next
// apply.  Last CTA: beta = -z.q_old / p_old.q_old (flexible CG) and rz =
// p.r = z.r + beta p_old.r, the numerator of the exact line search
// alpha = p.r / p.Kp that the fused apply forms.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_fcg_z(int64_t N, const T* __restrict__ r, const T* __restrict__ dinv,
                                                       const float* __restrict__ dsq, const float* __restrict__ out,
                                                       const T* __restrict__ p_old, T* __restrict__ q,
                                                       T* __restrict__ z, FcgState* __restrict__ fs, double inv_nfree,
                                                       PcgScalars* __restrict__ sc, double* __restrict__ partials,
                                                       unsigned int* counter) {
  __shared__ double s_red[64];
  if (sc->done) return;
  const double s2 = fs->rdr * inv_nfree;
  const T sig = T((s2 > 0.0 ? sqrt(s2) : 0.0) * fs->gamma);
  double zq = 0.0, zr = 0.0, pr = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    const T ri = r[i];
    const T zi = dinv[i] * ri + sig * T(dsq[i]) * T(out[4 * v + d]);
    zq += double(zi) * double(q[i]);
    zr += double(zi) * double(ri);
    pr += double(p_old[i]) * double(ri);
    q[i] = T(0);
    z[i] = zi;
  }
  block_sum2(zq, zr, s_red);
  double unused = 0.0;
  block_sum2(pr, unused, s_red);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x] = zq;
    partials[3 * blockIdx.x + 1] = zr;
    partials[3 * blockIdx.x + 2] = pr;
  }
  if (last_block_arrive(counter)) {
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, u2 = 0.0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
      t0 += __ldcg(&partials[3 * i]);
      t1 += __ldcg(&partials[3 * i + 1]);
      t2 += __ldcg(&partials[3 * i + 2]);
    }
    block_sum2(t0, t1, s_red);
    block_sum2(t2, u2, s_red);
    if (threadIdx.x == 0) {
      const double beta = fs->first ? 0.0 : -t0 / fs->pq_prev;
      const double pr_new = t1 + beta * t2;
      if (!(t1 > 0.0) || !(pr_new > 0.0) || !isfinite(t0) || !isfinite(pr_new)) {
        sc->breakdown = 2;  // not a descent direction: the host falls back to Jacobi
        sc->done = 1;
      } else {
        sc->beta = beta;
        sc->rz = pr_new;
        fs->first = 0;
      }
      *counter = 0u;
    }
  }
}

template <typename T>
__device__ __forceinline__ void fcg_update_one(T& x, T& r, T p, T q, T dinv, T a, double& rdr, double& rr) {
  x += a * p;
  const T ri = r - a * q;
  r = ri;
  rdr += double(ri) * double(dinv * ri);
  rr += double(ri) * double(ri);
}

// x += alpha p, r -= alpha q (q kept for the next beta), r.D^-1 r and r.r; the
// last CTA keeps p.q, counts the iteration and sets the convergence flag.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_fcg_update(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                                            const T* __restrict__ p, const T* __restrict__ q,
                                                            const T* __restrict__ dinv, PcgScalars* __restrict__ sc,
                                                            FcgState* __restrict__ fs, double* __restrict__ partials,
                                                            unsigned int* counter) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  __shared__ double s_red[64];
  if (sc->done) return;
  const T a = T(sc->alpha);
  double rdr = 0.0, rr = 0.0;
  const int64_t nv = n / W;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += stride) {
    V xv = reinterpret_cast<V*>(x)[i], rv = reinterpret_cast<V*>(r)[i];
    const V pv = reinterpret_cast<const V*>(p)[i], qv = reinterpret_cast<const V*>(q)[i];
    const V dv = reinterpret_cast<const V*>(dinv)[i];
    T* xs = reinterpret_cast<T*>(&xv);
    T* rs = reinterpret_cast<T*>(&rv);
    const T* ps = reinterpret_cast<const T*>(&pv);
    const T* qs = reinterpret_cast<const T*>(&qv);
    const T* ds = reinterpret_cast<const T*>(&dv);
#pragma unroll
    for (int k = 0; k < W; ++k) fcg_update_one(xs[k], rs[k], ps[k], qs[k], ds[k], a, rdr, rr);
    reinterpret_cast<V*>(x)[i] = xv;
    reinterpret_cast<V*>(r)[i] = rv;
  }
  for (int64_t i = nv * W + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += stride)
    fcg_update_one(x[i], r[i], p[i], q[i], dinv[i], a, rdr, rr);
  block_sum2(rdr, rr, s_red);
  if (threadIdx.x == 0) { partials[2 * blockIdx.x] = rdr; partials[2 * blockIdx.x + 1] = rr; }
  if (last_block_arrive(counter)) {
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
      t0 += __ldcg(&partials[2 * i]);
      t1 += __ldcg(&partials[2 * i + 1]);
    }
    block_sum2(t0, t1, s_red);
    if (threadIdx.x == 0) {
      fs->rdr = t0;
      fs->pq_prev = sc->pap;
      sc->rr = t1;
      sc->iters = sc->iters + 1;
      if (!isfinite(t0) || !isfinite(t1)) { sc->breakdown = 1; sc->done = 1; }
      if (t1 <= sc->stop2) sc->done = 1;
      *counter = 0u;
    }
  }
}

// r.D^-1 r and r.r of a fresh residual; `reset` restarts the direction recurrence.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_fcg_init(int64_t n, const T* __restrict__ r, const T* __restrict__ dinv,
                                                          FcgState* __restrict__ fs, PcgScalars* __restrict__ sc,
                                                          double* __restrict__ partials, unsigned int* counter,
                                                          int reset) {
  __shared__ double s_red[64];
  double rdr = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double ri = double(r[i]);
    rdr += ri * double(dinv[i]) * ri;
    rr += ri * ri;
  }
  block_sum2(rdr, rr, s_red);
  if (threadIdx.x == 0) { partials[2 * blockIdx.x] = rdr; partials[2 * blockIdx.x + 1] = rr; }
  if (last_block_arrive(counter)) {
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
      t0 += __ldcg(&partials[2 * i]);
      t1 += __ldcg(&partials[2 * i + 1]);
    }
    block_sum2(t0, t1, s_red);
    if (threadIdx.x == 0) {
      fs->rdr = t0;
      if (reset) fs->first = 1;
      sc->rr = t1;
      sc->done = (t1 <= sc->stop2) ? 1 : 0;
      *counter = 0u;
    }
  }
}

__global__ void k_fill_f32(int64_t n, float v, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = v;
}

template <typename T>
int fused_apply_grid(const Mesh& m) {
  return apply_kernel_setup<T, 1>(m);
}

template <typename T>
ApplyArgs<T> fused_args(Problem& P, const T* coords, const T* w, const T* p_old, T* p_new, T* ap, const T* r,
                        const T* dinv, const T* plas = nullptr, const float4* dinv4 = nullptr) {
  SolverWorkspace& ws = P.ws;
  ApplyArgs<T> a{};
  a.tv = P.mesh->tiles();
  a.N = P.N();
  a.coords = coords;
  if constexpr (std::is_same<T, float>::value) a.coords4 = P.mesh->d_coords32_aos4.get();
  a.dinv4 = dinv4;
  a.w = w;
  a.plas = plas;
  a.tile_nodes = P.d_tile_nodes_bc.get();
  Iso<double> i64 = P.ep.iso();
  a.iso = Iso<T>{T(i64.lam), T(i64.mu)};
  a.x = p_old;
  a.y = ap;
  a.r = r;
  a.dinv = dinv;
  a.p_new = p_new;
  a.sc = ws.sc.get();
  a.partials = ws.partials.get();
  a.counter = ws.counters.get();
  return a;
}

}  // namespace

namespace {
__global__ void k_pack4(int64_t N, const float* __restrict__ soa, float4* __restrict__ out) {
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < N; v += int64_t(gridDim.x) * blockDim.x)
    out[v] = make_float4(soa[v], soa[N + v], soa[2 * N + v], 0.0f);
}
}  // namespace

void launch_pack4(int64_t N, const float* soa, float4* out, cudaStream_t s) {
  k_pack4<<<vec_grid(N), kVecThreads, 0, s>>>(N, soa, out);
  PA_LAUNCHED();
}

void SolverWorkspace::ensure(int64_t n, int64_t C, int grid, bool mixed) {
  if (ndof != n) {
    x.resize(n); b.resize(n); r.resize(n); p0.resize(n); p1.resize(n); ap.resize(n); dinv.resize(n); t.resize(n);
    diag.resize(n);
    w64.resize(C);
    ndof = n;
    r32.release(); p32a.release(); p32b.release(); ap32.release(); dinv32.release(); dx32.release(); w32.release();
  }
  if (mixed && r32.n != size_t(n)) {
    r32.resize(n); p32a.resize(n); p32b.resize(n); ap32.resize(n); dinv32.resize(n); dx32.resize(n); w32.resize(C);
    dinv4.resize(n / 3); ones4.resize(n / 3);
  }
  if (partials.n < size_t(3 * grid + 64)) partials.resize(3 * grid + 64);  // up to 3 per block
  if (counters.n < 4) {
    counters.resize(4);
    PA_CUDA(cudaMemset(counters.get(), 0, 4 * sizeof(unsigned int)));
  }
  if (sc.n < 1) sc.resize(1);
}

// A CUDA graph of `chunk` fused CG iterations (K1, K2 pairs), captured once
// per solve and replayed; p alternates between two buffers so that the
// staging pass of K1 never reads a p value another CTA already replaced.
template <typename T, typename X>
struct CgGraph {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  int chunk = 0;
  ~CgGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  void capture(Problem& P, const T* coords, const T* w, T* pa, T* pb, T* ap, T* r, const T* dinv, X* x, int chunk_,
               const T* plas = nullptr, const float4* dinv4 = nullptr) {
    cudaStream_t s = P.stream;
    SolverWorkspace& ws = P.ws;
    const int64_t n = P.ndof();
    const int vg = vec_grid(n);
    const int ag = fused_apply_grid<T>(*P.mesh);
    chunk = chunk_ + (chunk_ % 2);
    ApplyArgs<T> a_even = fused_args<T>(P, coords, w, pa, pb, ap, r, dinv, plas, dinv4);  // reads pa, writes pb
    ApplyArgs<T> a_odd = fused_args<T>(P, coords, w, pb, pa, ap, r, dinv, plas, dinv4);   // reads pb, writes pa
    PA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; ++k) {
      launch_apply_kernel<T, 1>(*P.mesh, ag, s, k % 2 == 0 ? a_even : a_odd);
      const T* pnew = (k % 2 == 0) ? pb : pa;
      k_cg_update<T><<<vg, kVecThreads, 0, s>>>(n, x, r, pnew, ap, dinv, ws.sc.get(), ws.partials.get(),
                                                   ws.counters.get() + 1, nullptr);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) throw Error(PA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    PA_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  }
  // One replay; returns the device scalars after it.
  PcgScalars run(Problem& P) {
    PcgScalars hs{};
    PA_CUDA(cudaGraphLaunch(exec, P.stream));
    PA_CUDA(cudaMemcpyAsync(&hs, P.ws.sc.get(), sizeof(PcgScalars), cudaMemcpyDeviceToHost, P.stream));
    PA_CUDA(cudaStreamSynchronize(P.stream));
    return hs;
  }
};

static double host_norm2(Problem& P, const double* v) {
  cudaStream_t s = P.stream;
  const int64_t n = P.ndof();
  if (P.d_scalar.n < 2) P.d_scalar.resize(2);
  PA_CUDA(cudaMemsetAsync(P.d_scalar.get(), 0, 2 * sizeof(double), s));
  k_dot2<<<vec_grid(n), kVecThreads, 0, s>>>(n, v, v, P.d_scalar.get());
  PA_LAUNCHED();
  double h[2];
  PA_CUDA(cudaMemcpyAsync(h, P.d_scalar.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  return h[0];
}

// (Re)start the recursive residual from r (FP64 or FP32 copy), keeping p and
// beta unless `reset`.  Writes the stop threshold (recursive hint) and clears
// the done flag.
template <typename T>
static PcgScalars restart_residual(Problem& P, const T* r, const T* dinv, bool reset, double stop2, double bb) {
  cudaStream_t s = P.stream;
  SolverWorkspace& ws = P.ws;
  const int64_t n = P.ndof();
  k_cg_init<T><<<vec_grid(n), kVecThreads, 0, s>>>(n, r, dinv, ws.sc.get(), ws.partials.get(), ws.counters.get(),
                                                   0.0, reset ? 1 : 0);
  PA_LAUNCHED();
  PcgScalars cur{};
  PA_CUDA(cudaMemcpyAsync(&cur, ws.sc.get(), sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  cur.stop2 = stop2;
  cur.bb = bb;
  cur.done = 0;
  if (reset) { cur.iters = 0; cur.beta = 0.0; cur.breakdown = 0; }
  PA_CUDA(cudaMemcpyAsync(ws.sc.get(), &cur, sizeof(PcgScalars), cudaMemcpyHostToDevice, s));
  return cur;
}

// Solve the constrained system K x = b for the given operator (weights,
// optional J2 tangent records, Jacobi diagonal); b and x_out are device
// pointers in the interleaved layout (3N).
pa_status solve_operator(Problem& P, const SolveOperator& op, const double* b, double* x_out,
                         const pa_solve_options& o, pa_solve_stats* st, bool record_start) {
  cudaStream_t s = P.stream;
  const int64_t n = P.ndof();
  const bool mixed = o.method == PA_SOLVER_PCG_MIXED;
  PA_CHECK(o.method == PA_SOLVER_PCG_FP64 || mixed, "unknown solver method");
  PA_CHECK(o.rel_tol > 0.0, "rel_tol must be positive");
  const int grid_need = std::max(std::max(fused_apply_grid<double>(*P.mesh), fused_apply_grid<float>(*P.mesh)),
                                vec_grid(n));
  P.ws.ensure(n, P.C(), grid_need, mixed);
  SolverWorkspace& ws = P.ws;
  const int max_iters = o.max_iters > 0 ? o.max_iters : int(20.0 * std::sqrt(double(n)) + 1000);
  const int chunk = o.check_every > 0 ? o.check_every : 64;
  const double tol2 = o.rel_tol * o.rel_tol;
  const int vg = vec_grid(n);
  const uint8_t* mask = P.d_node_mask.get();
  const int64_t nbc = op.homogeneous_bc ? 0 : int64_t(P.bc_dofs.size());
  int64_t launches = 0;  // kernels of this library launched by the solve (graph nodes included)

  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  if (record_start) PA_CUDA(cudaEventRecord(P.ev0, s));

  // masked inverse of the Jacobi diagonal
  const int64_t N = P.N();
  k_inv_diag<double><<<vg, kVecThreads, 0, s>>>(N, op.diag_aos, mask, ws.dinv.get());
  PA_LAUNCHED();
  launches += 1;
  if (mixed) {
    PA_CHECK(op.w32 != nullptr, "mixed precision needs FP32 weights");
    k_inv_diag<float><<<vg, kVecThreads, 0, s>>>(N, op.diag_aos, mask, ws.dinv32.get());
    PA_LAUNCHED();
    launch_pack4(N, ws.dinv32.get(), ws.dinv4.get(), s);
    launches += 2;
  }
  // b' = mask(b - K x_D), x_D = Dirichlet values (held in p0 for the moment).
  double* bprime = ws.b.get();
  if (nbc) {
    PA_CUDA(cudaMemsetAsync(ws.p0.get(), 0, sizeof(double) * n, s));
    k_scatter_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), op.bc_scale, N,
                                                        ws.p0.get());
    PA_LAUNCHED();
    launch_apply_tiled<double>(P, op.w64, ws.p0.get(), ws.t.get(), false, s, op.plas64);
    k_aos_minus_soa<<<vg, kVecThreads, 0, s>>>(N, b, ws.t.get(), mask, bprime);
    launches += 3;
  } else {
    k_aos_minus_soa<<<vg, kVecThreads, 0, s>>>(N, b, nullptr, nullptr, bprime);
    launches += 1;
  }
  PA_LAUNCHED();
  // initial free-dof iterate
  if (o.use_initial_guess) {
    k_aos_minus_soa<<<vg, kVecThreads, 0, s>>>(N, x_out, nullptr, mask, ws.x.get());
    launches += 1;
  } else {
    PA_CUDA(cudaMemsetAsync(ws.x.get(), 0, sizeof(double) * n, s));
  }
  PA_LAUNCHED();
  // FP64 true residual r = b' - K_masked x
  auto true_residual = [&]() {
    launch_apply_tiled<double>(P, op.w64, ws.x.get(), ws.t.get(), true, s, op.plas64);
    k_sub_masked<<<vg, kVecThreads, 0, s>>>(N, bprime, ws.t.get(), mask, ws.r.get());
    PA_LAUNCHED();
    launches += 3;
    return host_norm2(P, ws.r.get());
  };
  double bb = host_norm2(P, bprime);
  launches += 1;
  if (!(bb > 0.0)) bb = 1.0;
  double rr_true = true_residual();

  // Krylov vectors
  PA_CUDA(cudaMemsetAsync(ws.p0.get(), 0, sizeof(double) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.p1.get(), 0, sizeof(double) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.ap.get(), 0, sizeof(double) * n, s));
  if (mixed) {
    PA_CUDA(cudaMemsetAsync(ws.dx32.get(), 0, sizeof(float) * n, s));
    PA_CUDA(cudaMemsetAsync(ws.p32a.get(), 0, sizeof(float) * n, s));
    PA_CUDA(cudaMemsetAsync(ws.p32b.get(), 0, sizeof(float) * n, s));
    PA_CUDA(cudaMemsetAsync(ws.ap32.get(), 0, sizeof(float) * n, s));
  }
  CgGraph<double, double> g64;
  CgGraph<float, float> g32;
  if (mixed)
    g32.capture(P, P.mesh->d_coords32_soa.get(), op.w32, ws.p32a.get(), ws.p32b.get(), ws.ap32.get(), ws.r32.get(),
                ws.dinv32.get(), ws.dx32.get(), chunk, op.plas32, ws.dinv4.get());
  else
    g64.capture(P, P.mesh->d_coords_soa.get(), op.w64, ws.p0.get(), ws.p1.get(), ws.ap.get(), ws.r.get(),
                ws.dinv.get(), ws.x.get(), chunk, op.plas64);

  // Recursive-residual stop hint, confirmed on the FP64 true residual.
  const double hint = mixed ? 0.25 : 0.81;
  int replacements = 0, iters = 0;
  bool converged = rr_true <= tol2 * bb, breakdown = false, first = true;
  while (!converged) {
    PcgScalars hs{};
    if (mixed) {
      k_to_f32<<<vg, kVecThreads, 0, s>>>(n, ws.r.get(), ws.r32.get());
      PA_LAUNCHED();
      hs = restart_residual<float>(P, ws.r32.get(), ws.dinv32.get(), first, hint * tol2 * bb, bb);
      hs = g32.run(P);  // one chunk, then fold dx and replace the residual
      launches += 3 + 2LL * g32.chunk;
      // newest p in p32b after an odd number of iterations: keep p32a current
      if ((hs.iters - iters) % 2)
        PA_CUDA(cudaMemcpyAsync(ws.p32a.get(), ws.p32b.get(), sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
      k_fold<<<vg, kVecThreads, 0, s>>>(n, ws.x.get(), ws.dx32.get());
      PA_LAUNCHED();
    } else {
      hs = restart_residual<double>(P, ws.r.get(), ws.dinv.get(), first, hint * tol2 * bb, bb);
      const int start = hs.iters;
      launches += 1;
      do {
        hs = g64.run(P);
        launches += 2LL * g64.chunk;
      } while (!hs.done && hs.iters < max_iters);
      if ((hs.iters - start) % 2)
        PA_CUDA(cudaMemcpyAsync(ws.p0.get(), ws.p1.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    first = false;
    iters = hs.iters;
    rr_true = true_residual();
    ++replacements;
    converged = rr_true <= tol2 * bb;
    if (hs.breakdown) { breakdown = !converged; break; }
    if (iters >= max_iters) break;
  }
  const double relres = std::sqrt(rr_true / bb);

  // x_out = x_f + x_D (back to the interleaved layout); constrained dofs are 0 in x_f
  launch_soa_to_aos<double, double>(ws.x.get(), x_out, N, s);
  launches += 1;
  if (nbc) {
    k_set_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), op.bc_scale,
                                                    x_out);
    PA_LAUNCHED();
    launches += 1;
  }
  PA_CUDA(cudaEventRecord(P.ev1, s));
  PA_CUDA(cudaEventSynchronize(P.ev1));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, P.ev0, P.ev1));
  if (st) {
    st->iterations = iters;
    st->replacements = replacements;
    st->rel_residual = relres;
    st->seconds = ms * 1e-3;
    st->converged = converged ? 1 : 0;
    st->kernel_launches = launches;
    st->fallback_iterations = 0;
  }
  if (breakdown) return PA_ERR_BREAKDOWN;
  if (!std::isfinite(relres)) return PA_ERR_NONFINITE;
  return converged ? PA_OK : PA_ERR_NOT_CONVERGED;
}

// Flexible CG with the learned preconditioner, mixed precision as in
// solve_operator (FP32 vectors and apply, FP64 dots, FP64 x and true-residual
// replacement once per chunk).  One iteration = the network (pack + four
// convolutions), the correction weight, z/beta, the fused apply (p, K p, p.Kp,
// alpha), the update.
// The solve continues as mixed Jacobi-PCG from the current iterate when the
// network's direction is not a descent direction, the FP64 residual has not
// improved for 512 iterations, or half of the iteration budget is spent.
pa_status solve_fcg(Problem& P, const SolveOperator& op, LearnedPC& pc, const double* b, double* x_out,
                    const pa_solve_options& o, pa_solve_stats* st) {
  cudaStream_t s = P.stream;
  const int64_t n = P.ndof(), N = P.N();
  PA_CHECK(o.rel_tol > 0.0, "rel_tol must be positive");
  PA_CHECK(op.w32 != nullptr && op.plas32 == nullptr, "the learned preconditioner serves the elastic operator");
  const int grid_need = std::max(std::max(fused_apply_grid<double>(*P.mesh), fused_apply_grid<float>(*P.mesh)),
                                vec_grid(n));
  P.ws.ensure(n, P.C(), grid_need, true);
  SolverWorkspace& ws = P.ws;
  if (ws.ones32.n != size_t(n)) { ws.ones32.resize(n); ws.z32.resize(n); }
  static_assert(sizeof(FcgState) <= 8 * sizeof(double), "FcgState fits its buffer");
  if (ws.fcg_state.n < 8) ws.fcg_state.resize(8);
  FcgState* fs = reinterpret_cast<FcgState*>(ws.fcg_state.get());
  const int max_iters = o.max_iters > 0 ? o.max_iters : int(20.0 * std::sqrt(double(n)) + 1000);
  int chunk = o.check_every > 0 ? o.check_every : 64;
  chunk += chunk % 2;
  const double tol2 = o.rel_tol * o.rel_tol;
  const int vg = vec_grid(n);
  const uint8_t* mask = P.d_node_mask.get();
  const int64_t nbc = op.homogeneous_bc ? 0 : int64_t(P.bc_dofs.size());
  const double inv_nfree = 1.0 / double(free_dofs(P));
  int64_t launches = 0;

  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  cudaEvent_t t0;
  PA_CUDA(cudaEventCreate(&t0));
  PA_CUDA(cudaEventRecord(t0, s));

  // operator pieces: D^-1 (FP32, SoA), D^-1/2 and node features; ones for the fused apply
  pc_prepare_operator(pc, P, op.diag_aos, ws.dinv32.get(), s);
  k_fill_f32<<<vg, kVecThreads, 0, s>>>(n, 1.0f, ws.ones32.get());
  PA_LAUNCHED();
  launch_pack4(N, ws.ones32.get(), ws.ones4.get(), s);
  launches += 3;
  // b' = mask(b - K x_D)
  double* bprime = ws.b.get();
  if (nbc) {
    PA_CUDA(cudaMemsetAsync(ws.p0.get(), 0, sizeof(double) * n, s));
    k_scatter_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), op.bc_scale, N,
                                                        ws.p0.get());
    PA_LAUNCHED();
    launch_apply_tiled<double>(P, op.w64, ws.p0.get(), ws.t.get(), false, s);
    k_aos_minus_soa<<<vg, kVecThreads, 0, s>>>(N, b, ws.t.get(), mask, bprime);
    launches += 3;
  } else {
    k_aos_minus_soa<<<vg, kVecThreads, 0, s>>>(N, b, nullptr, nullptr, bprime);
    launches += 1;
  }
  PA_LAUNCHED();
  if (o.use_initial_guess) {
    k_aos_minus_soa<<<vg, kVecThreads, 0, s>>>(N, x_out, nullptr, mask, ws.x.get());
    launches += 1;
  } else {
    PA_CUDA(cudaMemsetAsync(ws.x.get(), 0, sizeof(double) * n, s));
  }
  PA_LAUNCHED();
  auto true_residual = [&]() {
    launch_apply_tiled<double>(P, op.w64, ws.x.get(), ws.t.get(), true, s);
    k_sub_masked<<<vg, kVecThreads, 0, s>>>(N, bprime, ws.t.get(), mask, ws.r.get());
    PA_LAUNCHED();
    launches += 3;
    return host_norm2(P, ws.r.get());
  };
  double bb = host_norm2(P, bprime);
  launches += 1;
  if (!(bb > 0.0)) bb = 1.0;
  double rr_true = true_residual();

  PA_CUDA(cudaMemsetAsync(ws.dx32.get(), 0, sizeof(float) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.p32a.get(), 0, sizeof(float) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.p32b.get(), 0, sizeof(float) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.ap32.get(), 0, sizeof(float) * n, s));

  // one chunk of iterations, captured once
  const int32_t* done = reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(ws.sc.get()) +
                                                         offsetof(PcgScalars, done));
  const int ag = fused_apply_grid<float>(*P.mesh);
  const float* coords32 = P.mesh->d_coords32_soa.get();
  ApplyArgs<float> a_even = fused_args<float>(P, coords32, op.w32, ws.p32a.get(), ws.p32b.get(), ws.ap32.get(),
                                              ws.z32.get(), ws.ones32.get(), nullptr, ws.ones4.get());
  ApplyArgs<float> a_odd = fused_args<float>(P, coords32, op.w32, ws.p32b.get(), ws.p32a.get(), ws.ap32.get(),
                                             ws.z32.get(), ws.ones32.get(), nullptr, ws.ones4.get());
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  PA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < chunk; ++k) {
    pc_launch_network<float>(pc, ws.r32.get(), &fs->rdr, inv_nfree, done, s);
    k_fcg_gamma<float><<<vg, kVecThreads, 0, s>>>(N, ws.r32.get(), pc_dsq(pc), pc_output(pc), fs, inv_nfree,
                                                  ws.sc.get(), ws.partials.get(), ws.counters.get() + 2);
    const float* pold = (k % 2 == 0) ? ws.p32a.get() : ws.p32b.get();
    k_fcg_z<float><<<vg, kVecThreads, 0, s>>>(N, ws.r32.get(), ws.dinv32.get(), pc_dsq(pc), pc_output(pc), pold,
                                              ws.ap32.get(), ws.z32.get(), fs, inv_nfree, ws.sc.get(),
                                              ws.partials.get(), ws.counters.get() + 2);
    launch_apply_kernel<float, 1>(*P.mesh, ag, s, k % 2 == 0 ? a_even : a_odd);
    const float* pnew = (k % 2 == 0) ? ws.p32b.get() : ws.p32a.get();
    k_fcg_update<float><<<vg, kVecThreads, 0, s>>>(n, ws.dx32.get(), ws.r32.get(), pnew, ws.ap32.get(),
                                                   ws.dinv32.get(), ws.sc.get(), fs, ws.partials.get(),
                                                   ws.counters.get() + 3);
  }
  {
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) throw Error(PA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
  }
  PA_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  struct GraphGuard {
    cudaGraph_t g;
    cudaGraphExec_t e;
    ~GraphGuard() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
    }
  } guard_graph{graph, exec};
  const int per_iter = kPcNetworkLaunches + 4;

  const double hint = 0.25;
  int replacements = 0, iters = 0;
  bool converged = rr_true <= tol2 * bb, fallback = false, first = true;
  std::vector<double> hist;
  while (!converged) {
    k_to_f32<<<vg, kVecThreads, 0, s>>>(n, ws.r.get(), ws.r32.get());
    PA_LAUNCHED();
    PcgScalars cur{};
    cur.stop2 = hint * tol2 * bb;
    cur.bb = bb;
    cur.iters = iters;
    PA_CUDA(cudaMemcpyAsync(ws.sc.get(), &cur, sizeof(cur), cudaMemcpyHostToDevice, s));
    k_fcg_init<float><<<vg, kVecThreads, 0, s>>>(n, ws.r32.get(), ws.dinv32.get(), fs, ws.sc.get(), ws.partials.get(),
                                                 ws.counters.get() + 2, first ? 1 : 0);
    PA_LAUNCHED();
    PA_CUDA(cudaGraphLaunch(exec, s));
    PcgScalars hs{};
    PA_CUDA(cudaMemcpyAsync(&hs, ws.sc.get(), sizeof(hs), cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    launches += 3 + int64_t(per_iter) * chunk;
    if ((hs.iters - iters) % 2)
      PA_CUDA(cudaMemcpyAsync(ws.p32a.get(), ws.p32b.get(), sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    k_fold<<<vg, kVecThreads, 0, s>>>(n, ws.x.get(), ws.dx32.get());
    PA_LAUNCHED();
    first = false;
    iters = hs.iters;
    rr_true = true_residual();
    ++replacements;
    converged = rr_true <= tol2 * bb;
    hist.push_back(rr_true);
    if (converged) break;
    if (iters >= max_iters / 2) {  // too slow: hand the rest of the solve to Jacobi-PCG
      fallback = true;
      break;
    }
    // stalled: no chunk of the last `window` (>= 512 iterations) improved on
    // the best residual before them (CG residuals are not monotone)
    bool stalled = false;
    const size_t window = size_t(std::max(4, (512 + chunk - 1) / chunk));
    if (hist.size() > window) {
      const double before = *std::min_element(hist.begin(), hist.end() - window);
      const double recent = *std::min_element(hist.end() - window, hist.end());
      stalled = !(recent < 0.99 * before);
    }
    if (hs.breakdown || stalled || !std::isfinite(rr_true)) {
      fallback = true;
      break;
    }
  }
  pc_check_error(pc, s);

  launch_soa_to_aos<double, double>(ws.x.get(), x_out, N, s);
  launches += 1;
  if (nbc) {
    k_set_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), op.bc_scale,
                                                    x_out);
    PA_LAUNCHED();
    launches += 1;
  }
  pa_status status = PA_OK;
  int fb_iters = 0;
  if (fallback) {
    pa_solve_options fo = o;
    fo.method = PA_SOLVER_PCG_MIXED;
    fo.use_initial_guess = 1;
    fo.max_iters = max_iters;  // the fallback is a solve of its own
    pa_solve_stats fst{};
    status = solve_operator(P, op, b, x_out, fo, &fst, false);
    fb_iters = fst.iterations;
    replacements += fst.replacements;
    launches += fst.kernel_launches;
    converged = fst.converged != 0;
    rr_true = fst.rel_residual * fst.rel_residual * bb;
  } else {
    const double relres = std::sqrt(rr_true / bb);
    status = converged ? PA_OK : (std::isfinite(relres) ? PA_ERR_NOT_CONVERGED : PA_ERR_NONFINITE);
  }
  PA_CUDA(cudaEventRecord(P.ev1, s));
  PA_CUDA(cudaEventSynchronize(P.ev1));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, t0, P.ev1));
  cudaEventDestroy(t0);
  if (st) {
    st->iterations = iters + fb_iters;
    st->fallback_iterations = fb_iters;
    st->replacements = replacements;
    st->rel_residual = std::sqrt(rr_true / bb);
    st->seconds = ms * 1e-3;
    st->converged = converged ? 1 : 0;
    st->kernel_launches = launches;
  }
  return status;
}

// Elastic solve for density z: SIMP weights and Jacobi diagonal from z, then
// solve_operator (or the flexible CG with the problem's learned network).
pa_status solve_device(Problem& P, const double* z, const double* b, double* x_out, const pa_solve_options& o,
                       pa_solve_stats* st) {
  if (o.method == PA_SOLVER_FCG_LEARNED) {
    PA_CHECK(P.pc != nullptr, "PA_SOLVER_FCG_LEARNED needs a network (pa_problem_set_preconditioner)");
    const int64_t n = P.ndof();
    const int grid_need = std::max(std::max(fused_apply_grid<double>(*P.mesh), fused_apply_grid<float>(*P.mesh)),
                                  vec_grid(n));
    P.ws.ensure(n, P.C(), grid_need, true);
    SolverWorkspace& ws = P.ws;
    if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
    cudaEvent_t t0;
    PA_CUDA(cudaEventCreate(&t0));
    PA_CUDA(cudaEventRecord(t0, P.stream));
    launch_cell_weights(P, z, ws.w64.get(), ws.w32.get(), P.stream);
    launch_diag(P, ws.w64.get(), ws.diag.get(), P.stream);
    SolveOperator op;
    op.w64 = ws.w64.get();
    op.w32 = ws.w32.get();
    op.diag_aos = ws.diag.get();
    pa_status status = solve_fcg(P, op, *P.pc, b, x_out, o, st);
    float ms = 0.f;
    PA_CUDA(cudaEventElapsedTime(&ms, t0, P.ev1));
    cudaEventDestroy(t0);
    if (st) {
      st->kernel_launches += 2;
      st->seconds = ms * 1e-3;  // weights and diagonal included
    }
    return status;
  }
  const bool mixed = o.method == PA_SOLVER_PCG_MIXED;
  const bool mg = o.method == PA_SOLVER_PCG_MG;
  const bool box_jacobi = o.method == PA_SOLVER_PCG_FP64 && !o.use_initial_guess && boxmg_eligible(P);
  const int64_t n = P.ndof();
  const int grid_need = std::max(std::max(fused_apply_grid<double>(*P.mesh), fused_apply_grid<float>(*P.mesh)),
                                vec_grid(n));
  P.ws.ensure(n, P.C(), grid_need, mixed || mg || box_jacobi);
  SolverWorkspace& ws = P.ws;
  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  if ((mg && o.mg_coarse_solver == PA_MG_COARSE_AUTO && boxmg_eligible(P)) || box_jacobi) {
    // structured box: every level (or, for FP64 Jacobi-PCG, the fine level) on
    // the box kernel, deterministic
    cudaEvent_t t0;
    PA_CUDA(cudaEventCreate(&t0));
    PA_CUDA(cudaEventRecord(t0, P.stream));
    pa_status status = PA_OK;
    const bool done = solve_boxmg(P, z, b, x_out, o, st, &status, box_jacobi);
    if (done) {
      float ms = 0.f;
      PA_CUDA(cudaEventElapsedTime(&ms, t0, P.ev1));
      cudaEventDestroy(t0);
      if (st) st->seconds = ms * 1e-3;  // weights, diagonals and the hierarchy's set-up included
      return status;
    }
    cudaEventDestroy(t0);  // singular coarsest operator: the tile-kernel hierarchy below
  }
  if (mg) {
    PA_CHECK(P.mesh->num_parts == 1, "PA_SOLVER_PCG_MG solves one box (not a parted mesh)");
    cudaEvent_t t0;
    PA_CUDA(cudaEventCreate(&t0));
    PA_CUDA(cudaEventRecord(t0, P.stream));
    launch_cell_weights(P, z, ws.w64.get(), ws.w32.get(), P.stream);
    launch_diag(P, ws.w64.get(), ws.diag.get(), P.stream);
    SolveOperator op;
    op.w64 = ws.w64.get();
    op.w32 = ws.w32.get();
    op.diag_aos = ws.diag.get();
    pa_status status = solve_mg(P, op, b, x_out, o, st);
    float ms = 0.f;
    PA_CUDA(cudaEventElapsedTime(&ms, t0, P.ev1));
    cudaEventDestroy(t0);
    if (st) {
      st->kernel_launches += 2;
      st->seconds = ms * 1e-3;  // weights, diagonal and the hierarchy's set-up included
    }
    return status;
  }
  if (mixed && P.mesh->num_parts > 1) {
    // parted mesh: one independent CG per part
    cudaEvent_t t0;
    PA_CUDA(cudaEventCreate(&t0));
    PA_CUDA(cudaEventRecord(t0, P.stream));
    launch_cell_weights(P, z, ws.w64.get(), ws.w32.get(), P.stream);
    launch_diag(P, ws.w64.get(), ws.diag.get(), P.stream);
    SolveOperator op;
    op.w64 = ws.w64.get();
    op.w32 = ws.w32.get();
    op.diag_aos = ws.diag.get();
    pa_status status = solve_batched(P, op, b, x_out, o, st);
    float ms = 0.f;
    PA_CUDA(cudaEventElapsedTime(&ms, t0, P.ev1));
    cudaEventDestroy(t0);
    if (st) {
      st->kernel_launches += 2;
      st->seconds = ms * 1e-3;
    }
    return status;
  }
  PA_CUDA(cudaEventRecord(P.ev0, P.stream));  // the solve time includes weights and diagonal
  launch_cell_weights(P, z, ws.w64.get(), mixed ? ws.w32.get() : nullptr, P.stream);
  launch_diag(P, ws.w64.get(), ws.diag.get(), P.stream);
  SolveOperator op;
  op.w64 = ws.w64.get();
  op.w32 = mixed ? ws.w32.get() : nullptr;
  op.diag_aos = ws.diag.get();
  pa_status status = solve_operator(P, op, b, x_out, o, st, false);
  if (st) st->kernel_launches += 2;
  return status;
}

// Average device time of the fused CG kernel K1 over `reps` back-to-back
// launches (state: r = 1, p_old = 0, beta = 0.5), for the roofline report.
double time_cg_apply(Problem& P, const double* z, bool fp32, int reps) {
  cudaStream_t s = P.stream;
  const int64_t n = P.ndof();
  const int grid_need = std::max(std::max(fused_apply_grid<double>(*P.mesh), fused_apply_grid<float>(*P.mesh)),
                                vec_grid(n));
  P.ws.ensure(n, P.C(), grid_need, true);
  SolverWorkspace& ws = P.ws;
  launch_cell_weights(P, z, ws.w64.get(), ws.w32.get(), s);
  launch_diag(P, ws.w64.get(), ws.t.get(), s);
  k_inv_diag<double><<<vec_grid(n), kVecThreads, 0, s>>>(P.N(), ws.t.get(), P.d_node_mask.get(), ws.dinv.get());
  k_inv_diag<float><<<vec_grid(n), kVecThreads, 0, s>>>(P.N(), ws.t.get(), P.d_node_mask.get(), ws.dinv32.get());
  launch_pack4(P.N(), ws.dinv32.get(), ws.dinv4.get(), s);
  PA_LAUNCHED();
  PcgScalars init{};
  init.beta = 0.5;
  init.rz = 1.0;
  PA_CUDA(cudaMemcpyAsync(ws.sc.get(), &init, sizeof(init), cudaMemcpyHostToDevice, s));
  const int ag = fp32 ? fused_apply_grid<float>(*P.mesh) : fused_apply_grid<double>(*P.mesh);
  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  float ms = 0.f;
  if (fp32) {
    std::vector<float> ones(n, 1.0f);
    PA_CUDA(cudaMemcpyAsync(ws.r32.get(), ones.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
    PA_CUDA(cudaMemsetAsync(ws.p32a.get(), 0, sizeof(float) * n, s));
    PA_CUDA(cudaMemsetAsync(ws.p32b.get(), 0, sizeof(float) * n, s));
    PA_CUDA(cudaMemsetAsync(ws.ap32.get(), 0, sizeof(float) * n, s));
    ApplyArgs<float> a = fused_args<float>(P, P.mesh->d_coords32_soa.get(), ws.w32.get(), ws.p32a.get(), ws.p32b.get(),
                                           ws.ap32.get(), ws.r32.get(), ws.dinv32.get(), nullptr, ws.dinv4.get());
    ApplyArgs<float> b = fused_args<float>(P, P.mesh->d_coords32_soa.get(), ws.w32.get(), ws.p32b.get(), ws.p32a.get(),
                                           ws.ap32.get(), ws.r32.get(), ws.dinv32.get(), nullptr, ws.dinv4.get());
    launch_apply_kernel<float, 1>(*P.mesh, ag, s, a);  // warm
    PA_CUDA(cudaEventRecord(P.ev0, s));
    for (int i = 0; i < reps; ++i) launch_apply_kernel<float, 1>(*P.mesh, ag, s, i % 2 ? a : b);
    PA_CUDA(cudaEventRecord(P.ev1, s));
  } else {
    std::vector<double> ones(n, 1.0);
    PA_CUDA(cudaMemcpyAsync(ws.r.get(), ones.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
    PA_CUDA(cudaMemsetAsync(ws.p0.get(), 0, sizeof(double) * n, s));
    PA_CUDA(cudaMemsetAsync(ws.p1.get(), 0, sizeof(double) * n, s));
    PA_CUDA(cudaMemsetAsync(ws.ap.get(), 0, sizeof(double) * n, s));
    ApplyArgs<double> a = fused_args<double>(P, P.mesh->d_coords_soa.get(), ws.w64.get(), ws.p0.get(), ws.p1.get(),
                                             ws.ap.get(), ws.r.get(), ws.dinv.get());
    ApplyArgs<double> b = fused_args<double>(P, P.mesh->d_coords_soa.get(), ws.w64.get(), ws.p1.get(), ws.p0.get(),
                                             ws.ap.get(), ws.r.get(), ws.dinv.get());
    launch_apply_kernel<double, 1>(*P.mesh, ag, s, a);
    PA_CUDA(cudaEventRecord(P.ev0, s));
    for (int i = 0; i < reps; ++i) launch_apply_kernel<double, 1>(*P.mesh, ag, s, i % 2 ? a : b);
    PA_CUDA(cudaEventRecord(P.ev1, s));
  }
  PA_LAUNCHED();
  PA_CUDA(cudaEventSynchronize(P.ev1));
  PA_CUDA(cudaEventElapsedTime(&ms, P.ev0, P.ev1));
  return double(ms) / reps;
}

// Average device time (ms) of the plain constrained apply y = K x (the tile
// kernel in its plain mode, as the multigrid smoother launches it) over
// `reps` back-to-back launches; y accumulates across launches (values are
// not used, only the time).
double time_apply(Problem& P, const double* z, bool fp32, int reps) {
  cudaStream_t s = P.stream;
  const int64_t n = P.ndof();
  const int grid_need = std::max(std::max(fused_apply_grid<double>(*P.mesh), fused_apply_grid<float>(*P.mesh)),
                                vec_grid(n));
  P.ws.ensure(n, P.C(), grid_need, true);
  SolverWorkspace& ws = P.ws;
  launch_cell_weights(P, z, ws.w64.get(), ws.w32.get(), s);
  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  float ms = 0.f;
  auto run = [&](auto* x, auto* y, const auto* w, const auto* coords) {
    using T = std::remove_const_t<std::remove_pointer_t<decltype(x)>>;
    std::vector<T> ones(n, T(1));
    PA_CUDA(cudaMemcpyAsync(x, ones.data(), sizeof(T) * n, cudaMemcpyHostToDevice, s));
    PA_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * n, s));
    ApplyArgs<T> a{};
    a.tv = P.mesh->tiles();
    a.tile_nodes = P.d_tile_nodes_bc.get();
    a.N = P.N();
    a.coords = coords;
    a.w = w;
    const Iso<double> i64 = P.ep.iso();
    a.iso = Iso<T>{T(i64.lam), T(i64.mu)};
    a.x = x;
    a.y = y;
    const int grid = apply_kernel_setup<T, 0>(*P.mesh);
    launch_apply_kernel<T, 0>(*P.mesh, grid, s, a);  // warm
    PA_CUDA(cudaEventRecord(P.ev0, s));
    for (int i = 0; i < reps; ++i) launch_apply_kernel<T, 0>(*P.mesh, grid, s, a);
    PA_CUDA(cudaEventRecord(P.ev1, s));
  };
  if (fp32)
    run(ws.r32.get(), ws.ap32.get(), static_cast<const float*>(ws.w32.get()), static_cast<const float*>(P.mesh->d_coords32_soa.get()));
  else
    run(ws.r.get(), ws.ap.get(), static_cast<const double*>(ws.w64.get()), static_cast<const double*>(P.mesh->d_coords_soa.get()));
  PA_LAUNCHED();
  PA_CUDA(cudaEventSynchronize(P.ev1));
  PA_CUDA(cudaEventElapsedTime(&ms, P.ev0, P.ev1));
  return double(ms) / reps;
}

}  // namespace pa
