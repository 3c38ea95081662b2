// pa_boxmg.cu -- CG preconditioned by a geometric multigrid V-cycle on
// structured boxes, every level applied by the box kernel (pa_box.cuh).
//
// The same method as pa_mg.cu (the reference's AMG-preconditioned Krylov
// solve, src/alg/AmgXLinearSolver.cpp:34-73, replaced on boxes by a
// geometric hierarchy): levels of half the hexes per axis with the mean SIMP
// weight of their children, Dirichlet dofs by injection, trilinear transfers,
// Chebyshev(2) smoothing in D^-1 K on [lmax/30, 1.1 lmax] before and after
// the coarse correction, a dense FP64 inverse on the coarsest level, and an
// FP64 outer CG whose convergence is confirmed on the true residual b - K x
// (it restarts from it otherwise).  An outer CG with the FP32 operator and
// FP64 vectors was measured on the 160x80x80 cantilever: its recursion ran
// ahead of the true residual, one restart was needed and it took 25
// iterations (12.0 ms) against 19 (10.2 ms) for the FP64 operator, so the
// outer operator stays FP64.  What changes against pa_mg.cu is the data path:
//  * every operator application is the box kernel, with the vector updates
//    of the Chebyshev steps, residuals and CG dot products fused into its
//    epilogue; one V-cycle on a level is four kernels plus the restriction:
//      pre   x = dinv (ca b - c2 K d0), d0 = dinv b / theta      (x0 = 0)
//      res   r = b - K x
//      post1 r0 = dinv (b - K xi),    xi = x + P e (prolongation formed in the input)
//      post2 x = xi + ca r0 - c2 dinv K (r0 / theta)
//    with ca = (1 + c1) / theta + c2 and (c1, c2) the degree-2 Chebyshev
//    coefficients: exactly the two-step Chebyshev recurrence of pa_mg.cu;
//  * the finest level reads the outer CG's FP64 residual and writes the FP64
//    preconditioned residual (no conversion kernels) and accumulates r . z;
//  * the outer iteration (V-cycle, p = z + beta p with K p and p . Kp in one
//    kernel, x and r updates with r . r) is one CUDA graph, launched once per
//    iteration; every scalar stays on the device;
//  * weights, diagonals and the Dirichlet masks are computed in box order from
//    the lattice (no cell permutation, no atomics), and a fine level whose six
//    tets of every hex share one weight (per-hex densities) reads one weight
//    per hex.
//  * a level with an odd hex count along an axis is coarsened to ceil(n / 2)
//    hexes: the coarse level spans one more fine hex layer, which holds no
//    fine node and counts as weight zero in the coarse weights, so every box
//    size has a hierarchy down to a few hundred dofs.
// Requirements: a box lattice (mesh_make_box, or arrays recognised by
// detect_lattice: the solver permutes b and x at its boundary), an elastic
// operator (J2 tangent solves keep pa_mg.cu), one part.
#include <algorithm>
#include <array>
#include <cmath>
#include <memory>
#include <vector>

#include "pa_box.cuh"
#include "pa_cell.cuh"
#include "pa_dense.cuh"
#include "pa_learned.cuh"
#include "pa_problem.cuh"

namespace pa {

namespace {

constexpr int kVT = 256;
int vec_blocks(int64_t n) { return int(std::min<int64_t>((n + kVT - 1) / kVT, 148 * 8)); }

// device scalars of the outer CG
// outer CG scalars on the device; kBreak and kDone adjacent (the skip flags of
// the captured iteration's launches), kRr .. kIters read by the host together
enum : int { kRz = 0, kPq, kAlpha, kBeta, kRr, kBreak, kDone, kIters, kFirst, kTol, kScalars };

// Axis paths of the six tets (pa_box.cuh): (y,x,z) (y,z,x) (z,y,x) (z,x,y)
// (x,z,y) (x,y,z), two bits per axis, tet t at bits 6t.
constexpr uint64_t kPathCode = (1ull << 0) | (0ull << 2) | (2ull << 4) |     // t0
                               (1ull << 6) | (2ull << 8) | (0ull << 10) |    // t1
                               (2ull << 12) | (1ull << 14) | (0ull << 16) |  // t2
                               (2ull << 18) | (0ull << 20) | (1ull << 22) |  // t3
                               (0ull << 24) | (2ull << 26) | (1ull << 28) |  // t4
                               (0ull << 30) | (1ull << 32) | (2ull << 34);   // t5

// m-th axis of the path of tet t
__host__ __device__ __forceinline__ int path_axis(int t, int m) { return int((kPathCode >> (6 * t + 2 * m)) & 3u); }

// corner of vertex m of path tet t (v0 = 0, v3 = 7)
__host__ __device__ __forceinline__ int path_vertex(int t, int m) {
  int c = 0;
  for (int q = 0; q < m; ++q) c |= 1 << path_axis(t, q);
  return c;
}

// ------------------------------------------------------------- functors --
// Input formers (In: load + make) and epilogues (Out: load + store) of the
// box kernel; the loads run a hex layer before their values are used.

template <typename S, typename T>
struct InVec {  // x, with the masked dofs zero (mask may be null)
  const S* x;
  const uint8_t* mask;
  int64_t N;
  struct Raw {
    S x[3];
    uint8_t mk;
  };
  __device__ Raw load(int v, bool) const {
    Raw r;
#pragma unroll
    for (int c = 0; c < 3; ++c) r.x[c] = x[c * int(N) + v];
    r.mk = mask ? mask[v] : 0;
    return r;
  }
  __device__ void make(const Raw& r, int, bool, T (&o)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) o[c] = ((r.mk >> c) & 1) ? T(0) : T(r.x[c]);
  }
};

template <typename T>
struct OutPlain {  // y = K x, masked dofs zero (mask may be null)
  T* y;
  const uint8_t* mask;
  int64_t N;
  static constexpr bool kReduce = false;
  struct Pre {
    uint8_t mk;
  };
  __device__ Pre load(int v) const { return Pre{mask ? mask[v] : uint8_t(0)}; }
  __device__ double store(const Pre& p, int v, const T (&k)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) y[c * int(N) + v] = ((p.mk >> c) & 1) ? T(0) : k[c];
    return 0.0;
  }
  __device__ void finish(double) const {}
};

template <typename B>
struct InDinvB {  // d0 = dinv b / theta
  const B* b;
  const float* dinv;
  const float* ch;  // the level's Chebyshev coefficients (1 / theta, ca, c2)
  int64_t N;
  struct Raw {
    float d[3];
    B b[3];
  };
  __device__ Raw load(int v, bool) const {
    Raw r;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r.d[c] = dinv[c * int(N) + v];
      r.b[c] = b[c * int(N) + v];
    }
    return r;
  }
  __device__ void make(const Raw& r, int, bool, float (&o)[3]) const {
    const float s = __ldg(ch);
#pragma unroll
    for (int c = 0; c < 3; ++c) o[c] = s * r.d[c] * float(r.b[c]);
  }
};

template <typename B>
struct OutPre {  // x = dinv (ca b - c2 K d0)
  float* x;
  const B* b;
  const float* dinv;
  const float* ch;
  int64_t N;
  static constexpr bool kReduce = false;
  struct Pre {
    float d[3];
    B b[3];
  };
  __device__ Pre load(int v) const {
    Pre p;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      p.d[c] = dinv[c * int(N) + v];
      p.b[c] = b[c * int(N) + v];
    }
    return p;
  }
  __device__ double store(const Pre& p, int v, const float (&k)[3]) const {
    const float ca = __ldg(ch + 1), c2 = __ldg(ch + 2);
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c * int(N) + v] = p.d[c] * (ca * float(p.b[c]) - c2 * k[c]);
    return 0.0;
  }
  __device__ void finish(double) const {}
};

template <typename B>
struct OutRes {  // r = b - K x, masked dofs zero
  float* r;
  const B* b;
  const uint8_t* mask;
  int64_t N;
  static constexpr bool kReduce = false;
  struct Pre {
    B b[3];
    uint8_t mk;
  };
  __device__ Pre load(int v) const {
    Pre p;
#pragma unroll
    for (int c = 0; c < 3; ++c) p.b[c] = b[c * int(N) + v];
    p.mk = mask[v];
    return p;
  }
  __device__ double store(const Pre& p, int v, const float (&k)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c * int(N) + v] = ((p.mk >> c) & 1) ? 0.f : float(p.b[c]) - k[c];
    return 0.0;
  }
  __device__ void finish(double) const {}
};

template <typename B>
struct OutPost1 {  // r0 = dinv (b - K xi)
  float* r0;
  const B* b;
  const float* dinv;
  int64_t N;
  static constexpr bool kReduce = false;
  struct Pre {
    float d[3];
    B b[3];
  };
  __device__ Pre load(int v) const {
    Pre p;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      p.d[c] = dinv[c * int(N) + v];
      p.b[c] = b[c * int(N) + v];
    }
    return p;
  }
  __device__ double store(const Pre& p, int v, const float (&k)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) r0[c * int(N) + v] = p.d[c] * (float(p.b[c]) - k[c]);
    return 0.0;
  }
  __device__ void finish(double) const {}
};

struct InScaled {  // d0 = r0 / theta
  const float* r;
  const float* ch;
  int64_t N;
  struct Raw {
    float r[3];
  };
  __device__ Raw load(int v, bool) const {
    Raw q;
#pragma unroll
    for (int c = 0; c < 3; ++c) q.r[c] = r[c * int(N) + v];
    return q;
  }
  __device__ void make(const Raw& q, int, bool, float (&o)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) o[c] = __ldg(ch) * q.r[c];
  }
};

// x_out = xi + ca r0 - c2 dinv K d0 (xi = x + P e, prolongated in place
// before post1; masked dofs are zero in xi, r0 and dinv); on the finest level
// (RZ) the output is the FP64 preconditioned residual z and r . z is reduced
// (finish: beta = r.z_new / r.z_old, or 0 on the first iteration).
template <typename O, bool RZ>
struct OutPost2 {
  O* xo;
  const float* x;
  const float* r0;
  const float* dinv;
  const float* ch;
  int64_t N;
  const double* rvec;  // RZ: the outer residual
  double* sc;          // RZ: the outer CG scalars
  static constexpr bool kReduce = RZ;
  struct Pre {
    float x[3], r0[3], d[3];
    double rv[RZ ? 3 : 1];
  };
  __device__ Pre load(int v) const {
    Pre p;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int q = c * int(N) + v;
      p.x[c] = x[q];
      p.r0[c] = r0[q];
      p.d[c] = dinv[q];
      if constexpr (RZ) p.rv[c] = rvec[q];
    }
    return p;
  }
  __device__ double store(const Pre& p, int v, const float (&kd)[3]) const {
    double acc = 0.0;
    const float ca = __ldg(ch + 1), c2 = __ldg(ch + 2);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float z = p.x[c] + ca * p.r0[c] - c2 * p.d[c] * kd[c];
      xo[c * int(N) + v] = O(z);
      if constexpr (RZ) acc += double(z) * p.rv[c];
    }
    return acc;
  }
  __device__ void finish(double t) const {
    if constexpr (RZ) {
      const double old = sc[kRz];
      sc[kBeta] = sc[kFirst] != 0.0 ? 0.0 : t / old;
      sc[kFirst] = 0.0;
      sc[kRz] = t;
      if (!(t > 0.0) || !isfinite(t)) sc[kBreak] = 1.0;
    }
  }
};

// power iteration: x_next = dinv K x / ||x||, ||x_next||^2 reduced
struct OutPower {
  float* xn;
  const float* dinv;
  const double* nrm_in;
  double* nrm_out;
  int64_t N;
  static constexpr bool kReduce = true;
  struct Pre {
    float d[3];
  };
  __device__ Pre load(int v) const {
    Pre p;
#pragma unroll
    for (int c = 0; c < 3; ++c) p.d[c] = dinv[c * int(N) + v];
    return p;
  }
  __device__ double store(const Pre& p, int v, const float (&k)[3]) const {
    const double q = *nrm_in;
    const float sc = (q > 0.0 && isfinite(q)) ? float(1.0 / sqrt(q)) : 1.f;
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float val = p.d[c] * k[c] * sc;
      xn[c * int(N) + v] = val;
      acc += double(val) * val;
    }
    return acc;
  }
  __device__ void finish(double t) const { *nrm_out = t; }
};

// outer CG: p = z + beta p_old formed in the input (the owner stores p_new);
// q = K p (masked), p . q reduced, alpha = r.z / p.q
struct InCgP {
  const double* z;
  const double* pold;
  double* pnew;
  const double* sc;
  int64_t N;
  struct Raw {
    double z[3], p[3];
  };
  __device__ Raw load(int v, bool) const {
    Raw r;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r.z[c] = z[c * int(N) + v];
      r.p[c] = pold[c * int(N) + v];
    }
    return r;
  }
  __device__ void make(const Raw& r, int v, bool owned, double (&o)[3]) const {
    const double beta = sc[kBeta];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o[c] = r.z[c] + beta * r.p[c];
      if (owned) pnew[c * int(N) + v] = o[c];
    }
  }
};
struct OutCgQ {
  double* q;
  const double* z;
  const double* pold;
  const uint8_t* mask;
  double* sc;
  int64_t N;
  static constexpr bool kReduce = true;
  struct Pre {
    double z[3], p[3];
    uint8_t mk;
  };
  __device__ Pre load(int v) const {
    Pre r;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r.z[c] = z[c * int(N) + v];
      r.p[c] = pold[c * int(N) + v];
    }
    r.mk = mask[v];
    return r;
  }
  __device__ double store(const Pre& r, int v, const double (&k)[3]) const {
    const double beta = sc[kBeta];
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double qv = ((r.mk >> c) & 1) ? 0.0 : k[c];
      q[c * int(N) + v] = qv;
      acc += (r.z[c] + beta * r.p[c]) * qv;
    }
    return acc;
  }
  __device__ void finish(double t) const {
    sc[kPq] = t;
    if (!(t > 0.0) || !isfinite(t)) {
      sc[kBreak] = 1.0;
      sc[kAlpha] = 0.0;
    } else {
      sc[kAlpha] = sc[kRz] / t;
    }
  }
};

// ------------------------------------------------------- vector kernels --
__device__ __forceinline__ void grid_reduce_finish(double v, double* partials, unsigned int* counter, double* out) {
  __shared__ double s_red[32];
  __shared__ bool s_last;
  const double b = block_sum_box(v, s_red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = b;
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double t = 0.0;
    for (unsigned p = threadIdx.x; p < gridDim.x; p += blockDim.x) t += __ldcg(&partials[p]);
    t = block_sum_box(t, s_red);
    if (threadIdx.x == 0) {
      *counter = 0u;
      *out = t;
    }
  }
}

// x += alpha p; r -= alpha q; r . r into sc[kRr]; the last CTA counts the
// iteration and sets kDone when r . r <= sc[kTol].  A no-op once kBreak or
// kDone is set.
__global__ void __launch_bounds__(kVT) k_bcg_update(int64_t n, double* sc, const double* __restrict__ p,
                                                    const double* __restrict__ q, double* __restrict__ x,
                                                    double* __restrict__ r, double* partials, unsigned int* counter) {
  if (sc[kBreak] != 0.0 || sc[kDone] != 0.0) return;
  const double a = sc[kAlpha];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    r[i] = ri;
    s += ri * ri;
  }
  __shared__ double s_red[32];
  __shared__ bool s_last;
  const double b = block_sum_box(s, s_red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = b;
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += __ldcg(&partials[k]);
    t = block_sum_box(t, s_red);
    if (threadIdx.x == 0) {
      *counter = 0u;
      sc[kRr] = t;
      sc[kIters] += 1.0;
      if (t <= sc[kTol]) sc[kDone] = 1.0;
    }
  }
}

// Jacobi preconditioner of the outer CG: z = dinv r (dinv zero on the masked
// dofs), r . z reduced in a fixed order, and the CG scalars updated as the
// V-cycle's last kernel does (beta, r . z, breakdown).  A no-op once kBreak or
// kDone is set.
__global__ void __launch_bounds__(kVT) k_bjacobi_z(int64_t n, const float* __restrict__ dinv,
                                                   const double* __restrict__ r, double* __restrict__ z, double* sc,
                                                   double* partials, unsigned int* counter) {
  if (sc[kBreak] != 0.0 || sc[kDone] != 0.0) return;
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double zi = double(dinv[i]) * r[i];
    z[i] = zi;
    s += zi * r[i];
  }
  __shared__ double s_red[32];
  __shared__ bool s_last;
  const double b = block_sum_box(s, s_red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = b;
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += __ldcg(&partials[k]);
    t = block_sum_box(t, s_red);
    if (threadIdx.x == 0) {
      *counter = 0u;
      const double old = sc[kRz];
      sc[kBeta] = sc[kFirst] != 0.0 ? 0.0 : t / old;
      sc[kFirst] = 0.0;
      sc[kRz] = t;
      if (!(t > 0.0) || !isfinite(t)) sc[kBreak] = 1.0;
    }
  }
}

// out = mask ? 0 : a - b (b may be null), and out . out (one thread per node,
// 32-bit node ids: 3 N < 2^31 on the box path)
__global__ void __launch_bounds__(kVT) k_bres64(int N, const double* __restrict__ a, const double* __restrict__ b,
                                                const uint8_t* __restrict__ mask, double* __restrict__ out,
                                                double* partials, unsigned int* counter, double* nrm_out) {
  double s = 0.0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
    const uint8_t mk = mask[v];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int i = d * N + v;
      const double o = ((mk >> d) & 1) ? 0.0 : a[i] - (b ? b[i] : 0.0);
      out[i] = o;
      s += o * o;
    }
  }
  grid_reduce_finish(s, partials, counter, nrm_out);
}

// (re)start of the outer CG: scalars cleared, convergence threshold tol2 on
// r . r; the executed-iteration count only at the start of a solve (full)
__global__ void k_bcg_reset(double* sc, double tol2, int full) {
  sc[kRz] = 0.0;
  sc[kPq] = 0.0;
  sc[kAlpha] = 0.0;
  sc[kBeta] = 0.0;
  sc[kBreak] = 0.0;
  sc[kDone] = 0.0;
  sc[kFirst] = 1.0;
  sc[kTol] = tol2;
  if (full) sc[kIters] = 0.0;
}

// x_soa[d N + lattice(v)] = scale * value for each Dirichlet dof (dof = 3 v + d)
__global__ void k_bscatter_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                              double scale, int64_t N, const int32_t* __restrict__ lat_of, int flip,
                              double* __restrict__ x) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nbc) return;
  const int32_t dof = dofs[i];
  const int32_t v = dof / 3, d = dof % 3;
  x[d * N + (lat_of ? lat_of[v] : v)] = (((flip >> d) & 1) ? -scale : scale) * vals[i];
}
__global__ void k_bset_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals, double scale,
                          double* __restrict__ x_aos) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nbc) return;
  x_aos[dofs[i]] = scale * vals[i];
}

// Restriction (R = P^T of trilinear interpolation), coarse masked dofs zero.
// The coarse level spans 2 c.nx fine hexes along x (and so on), at least the
// fine level's f.nx: a fine level with an odd count is padded by one hex
// layer that holds no fine node.  The 27 fine neighbours' loads are unrolled
// and predicated (a missing neighbour reads as zero), so that they are all in
// flight at once: on the small levels these launches are a few CTAs whose
// time was the chain of dependent loads.  The sum runs in the same order.
__global__ void k_brestrict(BoxDims c, BoxDims f, const float* __restrict__ fv_in, const uint8_t* __restrict__ cmask,
                            float* __restrict__ cv_out, const double* skip = nullptr) {
  if (skip && (skip[0] != 0.0 || skip[1] != 0.0)) return;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const int Nc = int(c.N), Nf = int(f.N);
  if (v >= Nc) return;
  const int I = v % c.px, J = (v / c.px) % c.py, K = v / (c.px * c.py);
  float val[27][3];
#pragma unroll
  for (int dc = 0; dc < 3; ++dc)
#pragma unroll
    for (int db = 0; db < 3; ++db)
#pragma unroll
      for (int da = 0; da < 3; ++da) {
        const int i = 2 * I + da - 1, j = 2 * J + db - 1, k = 2 * K + dc - 1;
        const bool in = i >= 0 && i < f.px && j >= 0 && j < f.py && k >= 0 && k < f.pz;
        const int fv = in ? i + f.px * (j + f.py * k) : 0;
        const int e = da + 3 * (db + 3 * dc);
#pragma unroll
        for (int d = 0; d < 3; ++d) val[e][d] = in ? __ldg(&fv_in[d * Nf + fv]) : 0.f;
      }
  float s[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int dc = 0; dc < 3; ++dc)
#pragma unroll
    for (int db = 0; db < 3; ++db)
#pragma unroll
      for (int da = 0; da < 3; ++da) {
        const float w = (dc != 1 ? 0.5f : 1.0f) * (db != 1 ? 0.5f : 1.0f) * (da != 1 ? 0.5f : 1.0f);
        const int i = 2 * I + da - 1, j = 2 * J + db - 1, k = 2 * K + dc - 1;
        const bool in = i >= 0 && i < f.px && j >= 0 && j < f.py && k >= 0 && k < f.pz;
        const int e = da + 3 * (db + 3 * dc);
        if (in)
#pragma unroll
          for (int d = 0; d < 3; ++d) s[d] += w * val[e][d];
      }
  const uint8_t mk = cmask[v];
#pragma unroll
  for (int d = 0; d < 3; ++d) cv_out[d * Nc + v] = ((mk >> d) & 1) ? 0.f : s[d];
}

// x_fine += P e (trilinear interpolation of the coarse correction), fine
// masked dofs untouched (they stay zero).  Fine node i lies at coarse
// position i / 2; every coarse node it reads exists (2 c.nx >= f.nx).  The
// (up to) eight coarse loads are unrolled and predicated, summed in order.
__global__ void k_bprolong_add(BoxDims c, BoxDims f, const float* __restrict__ e, const uint8_t* __restrict__ fmask,
                               float* __restrict__ x, const double* skip = nullptr) {
  if (skip && (skip[0] != 0.0 || skip[1] != 0.0)) return;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const int Nc = int(c.N), Nf = int(f.N);
  if (v >= Nf) return;
  const int i = v % f.px, j = (v / f.px) % f.py, k = v / (f.px * f.py);
  const int ia = i >> 1, ja = j >> 1, ka = k >> 1;
  const int ni = (i & 1) + 1, nj = (j & 1) + 1, nk = (k & 1) + 1;
  const float w = (ni == 1 ? 1.f : 0.5f) * (nj == 1 ? 1.f : 0.5f) * (nk == 1 ? 1.f : 0.5f);
  float val[8][3];
#pragma unroll
  for (int cc = 0; cc < 2; ++cc)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const bool in = a < ni && b < nj && cc < nk;
        const int cv = in ? (ia + a) + c.px * ((ja + b) + c.py * (ka + cc)) : 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) val[a + 2 * (b + 2 * cc)][d] = in ? __ldg(&e[d * Nc + cv]) : 0.f;
      }
  float s[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int cc = 0; cc < 2; ++cc)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a)
        if (a < ni && b < nj && cc < nk)
#pragma unroll
          for (int d = 0; d < 3; ++d) s[d] += val[a + 2 * (b + 2 * cc)][d];
  const uint8_t mk = fmask[v];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (!((mk >> d) & 1)) x[d * Nf + v] += w * s[d];
}

// deterministic zero-mean start vector in [-1, 1], masked; ||x||^2 reduced
__global__ void __launch_bounds__(kVT) k_bseed(int N, const uint8_t* __restrict__ mask, float* __restrict__ x,
                                               double* partials, unsigned int* counter, double* nrm_out) {
  double s = 0.0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
    const uint8_t mk = mask[v];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int i = d * N + v;
      uint32_t h = uint32_t(i) * 2654435761u + 0x9e3779b9u;
      h ^= h >> 16;
      h *= 0x85ebca6bu;
      h ^= h >> 13;
      const float val = ((mk >> d) & 1) ? 0.f : float(int(h % 2001u) - 1000) * 1e-3f;
      x[i] = val;
      s += double(val) * val;
    }
  }
  grid_reduce_finish(s, partials, counter, nrm_out);
}

// interleaved caller's order -> component-major lattice order (node_of null:
// same order; flip bit d: component d changes sign)
template <typename S, typename T>
__global__ void k_bperm_in(int N, const int32_t* __restrict__ node_of, int flip, const S* __restrict__ aos,
                           T* __restrict__ soa) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x) {
    const int64_t u = 3 * int64_t(node_of ? node_of[b] : b);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T v = T(aos[u + d]);
      soa[d * N + b] = ((flip >> d) & 1) ? -v : v;
    }
  }
}
// component-major lattice order -> interleaved caller's order
template <typename T, typename S>
__global__ void k_bperm_out(int N, const int32_t* __restrict__ node_of, int flip, const T* __restrict__ soa,
                            S* __restrict__ aos) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x) {
    const int64_t u = 3 * int64_t(node_of ? node_of[b] : b);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const S v = S(soa[d * N + b]);
      aos[u + d] = ((flip >> d) & 1) ? -v : v;
    }
  }
}
// node mask in lattice order
__global__ void k_bperm_mask(int64_t N, const int32_t* __restrict__ node_of, const uint8_t* __restrict__ in,
                             uint8_t* __restrict__ out) {
  const int64_t b = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (b < N) out[b] = in[node_of[b]];
}

// ||x||^2
__global__ void __launch_bounds__(kVT) k_bnorm2(int64_t n, const float* __restrict__ x, double* partials,
                                                unsigned int* counter, double* nrm_out) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += double(x[i]) * x[i];
  grid_reduce_finish(s, partials, counter, nrm_out);
}

// ------------------------------------------------ weights and diagonals --
// SIMP weight of every tet of the fine box from the control (per cell: user
// cell 6h + t; nodal: the mean of the tet's four nodes, src/ApplyWeighting.hpp:49-62),
// tet-major; the per-hex copy and a flag when the six tets of a hex differ.
__global__ void k_bweights(BoxDims d, const double* __restrict__ z, int layout, double p, double pmin,
                           const int32_t* __restrict__ cell_of_slot, const int32_t* __restrict__ node_of,
                           double* __restrict__ w64t, float* __restrict__ w32t, double* __restrict__ w64h,
                           float* __restrict__ w32h, unsigned int* __restrict__ differ) {
  const int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (h >= d.H) return;
  const int i = int(h % d.nx), j = int((h / d.nx) % d.ny), k = int(h / (int64_t(d.nx) * d.ny));
  double w[6];
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    double rho;
    if (layout == PA_CONTROL_CELL) {
      rho = z[cell_of_slot ? cell_of_slot[6 * h + t] : 6 * h + t];
    } else {
      rho = 0.0;
      for (int m = 0; m < 4; ++m) {
        const int c = path_vertex(t, m);
        const int64_t b = (i + (c & 1)) + int64_t(d.px) * ((j + ((c >> 1) & 1)) + int64_t(d.py) * (k + (c >> 2)));
        rho += z[node_of ? node_of[b] : b];
      }
      rho *= 0.25;
    }
    w[t] = simp(rho, p, pmin);
    w64t[t * d.H + h] = w[t];
    w32t[t * d.H + h] = float(w[t]);
  }
  bool same = true;
#pragma unroll
  for (int t = 1; t < 6; ++t) same = same && w[t] == w[0];
  w64h[h] = w[0];
  w32h[h] = float(w[0]);
  if (!same) atomicOr(differ, 1u);
}

constexpr double kDeltaScale = 0.5;

// Coarse hex weight = mean of the 48 child tets (per-hex or tet-major fine
// weights); the children in a padding layer (2 I + a >= f.nx, ...) count as
// weight zero, so a coarse hex half outside the fine box has half the weight.
// delta (may be null): a learned correction, w = mean exp(kDeltaScale
// tanh(delta[h dstride])), within exp(+-0.5) of the mean.
__global__ void k_bcoarse_w(BoxDims c, BoxDims f, const double* __restrict__ wf, int wm, double* __restrict__ w64,
                            float* __restrict__ w32, const float* __restrict__ delta, int dstride) {
  const int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (h >= c.H) return;
  const int I = int(h % c.nx), J = int((h / c.nx) % c.ny), K = int(h / (int64_t(c.nx) * c.ny));
  double s = 0.0;
  for (int cc = 0; cc < 2; ++cc)
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        if (2 * I + a >= f.nx || 2 * J + b >= f.ny || 2 * K + cc >= f.nz) continue;
        const int64_t fh = (2 * I + a) + int64_t(f.nx) * ((2 * J + b) + int64_t(f.ny) * (2 * K + cc));
        if (wm)
          for (int t = 0; t < 6; ++t) s += wf[t * f.H + fh];
        else
          s += 6.0 * wf[fh];
      }
  double w = s / 48.0;
  if (delta) w *= exp(kDeltaScale * tanh(double(delta[h * dstride])));
  w64[h] = w;
  w32[h] = float(w);
}

// Input features of the learned coarse-weight correction, per coarse hex
// (channel-last, 5 per hex) from the per-hex weights of its existing
// children (the mean of the six tets when the fine weights are per tet):
// with L(w) = 1 + log10(w) / 9 (0 at the SIMP minimum 1e-9, 1 at full
// material), L of the mean over all eight children (padding as zero, the
// weight the coarse level is given), of their geometric mean, minimum and
// maximum, and the fraction of the eight children inside the fine box.
__global__ void k_bcoarse_feat(BoxDims c, BoxDims f, const double* __restrict__ wf, int wm, float* __restrict__ feat) {
  const int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (h >= c.H) return;
  const int I = int(h % c.nx), J = int((h / c.nx) % c.ny), K = int(h / (int64_t(c.nx) * c.ny));
  double sum = 0.0, lsum = 0.0, mn = 1e300, mx = 0.0;
  int cnt = 0;
  for (int cc = 0; cc < 2; ++cc)
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        if (2 * I + a >= f.nx || 2 * J + b >= f.ny || 2 * K + cc >= f.nz) continue;
        const int64_t fh = (2 * I + a) + int64_t(f.nx) * ((2 * J + b) + int64_t(f.ny) * (2 * K + cc));
        double w = 0.0;
        if (wm)
          for (int t = 0; t < 6; ++t) w += wf[t * f.H + fh] / 6.0;
        else
          w = wf[fh];
        w = fmax(w, 1e-30);
        sum += w;
        lsum += log(w);
        mn = fmin(mn, w);
        mx = fmax(mx, w);
        ++cnt;
      }
  auto L = [](double w) { return float(1.0 + log10(fmax(w, 1e-30)) / 9.0); };
  float* o = feat + 5 * h;
  o[0] = L(sum / 8.0);
  o[1] = L(exp(lsum / cnt));
  o[2] = L(mn);
  o[3] = L(mx);
  o[4] = float(cnt) / 8.f;
}

// gw[h] += scale a^T A_h b for every hex of a level: A_h the unweighted
// stiffness of the hex's six tets, a and b FP32 component-major vectors of
// the level; a^T A_t b = vol sigma(eps(a)) . eps(b) (engineering shears).
__global__ void __launch_bounds__(256) k_bbilinear(BoxDims d, double ih0, double ih1, double ih2, double vol,
                                                   Iso<double> iso, const float* __restrict__ a,
                                                   const float* __restrict__ b, double scale, double* __restrict__ gw) {
  const int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (h >= d.H) return;
  const int i = int(h % d.nx), j = int((h / d.nx) % d.ny), k = int(h / (int64_t(d.nx) * d.ny));
  const double ih[3] = {ih0, ih1, ih2};
  const int N = int(d.N);
  double ua[8][3], ub[8][3];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int v = (i + (q & 1)) + d.px * ((j + ((q >> 1) & 1)) + d.py * (k + (q >> 2)));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ua[q][c] = a[c * N + v];
      ub[q][c] = b[c * N + v];
    }
  }
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    double ga[3][3], gb[3][3];
    int prev = 0;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int ax = path_axis(t, m), nxt = prev | (1 << ax);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ga[c][ax] = (ua[nxt][c] - ua[prev][c]) * ih[ax];
        gb[c][ax] = (ub[nxt][c] - ub[prev][c]) * ih[ax];
      }
      prev = nxt;
    }
    const double ea[6] = {ga[0][0], ga[1][1], ga[2][2], ga[1][2] + ga[2][1], ga[0][2] + ga[2][0], ga[0][1] + ga[1][0]};
    const double eb[6] = {gb[0][0], gb[1][1], gb[2][2], gb[1][2] + gb[2][1], gb[0][2] + gb[2][0], gb[0][1] + gb[1][0]};
    double sg[6];
    tet_stress(iso, vol, ea, sg);
    s += voigt_dot(sg, eb);
  }
  gw[h] += scale * s;
}

// x = 0 on the masked dofs (component-major FP32)
__global__ void k_bmask_f(int N, const uint8_t* __restrict__ mask, float* __restrict__ x) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const uint8_t mk = mask[v];
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if ((mk >> c) & 1) x[c * N + v] = 0.f;
}

// acc += 1 - (r . z + z . rho) / E: the relative energy-norm error
// ||e - z||_K^2 / E of z = M r for K e = r, E = e . r (rho = r - K z)
__global__ void __launch_bounds__(kVT) k_bcoarse_loss(int64_t n, const float* __restrict__ r,
                                                      const float* __restrict__ z, const float* __restrict__ rho,
                                                      double inv_e, double* partials, unsigned int* counter,
                                                      double* acc) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += double(z[i]) * (double(r[i]) + double(rho[i]));
  __shared__ double s_red[32];
  __shared__ bool s_last;
  const double b = block_sum_box(s, s_red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = b;
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += __ldcg(&partials[k]);
    t = block_sum_box(t, s_red);
    if (threadIdx.x == 0) {
      *counter = 0u;
      *acc += 1.0 - t * inv_e;
    }
  }
}

// dL/ddelta = w dL/dw kDeltaScale (1 - tanh^2 delta) / n (w the weight the
// level holds)
__global__ void k_bgrad_delta(int64_t H, const double* __restrict__ gw, const double* __restrict__ w,
                              const float* __restrict__ delta, double inv_n, float* __restrict__ grad) {
  const int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (h >= H) return;
  const double t = tanh(double(delta[h]));
  grad[h] = float(w[h] * gw[h] * kDeltaScale * (1.0 - t * t) * inv_n);
}

// dinv = masked ? 0 : 1 / diag(K), diag from the tets around each node:
// K_vv,dd = s [lam g_d^2 + mu g_d^2 + mu |g|^2], g the vertex's barycentric gradient.
// Diagonal of the unweighted tet stiffness, per hex corner: the tets whose
// path passes through corner q and vol ((lam + mu) g_c^2 + mu |g|^2) of the
// corner's gradient g in each (corners 0 and 7 lie on all six paths, the
// others on two).  Built on the host per level.
struct DinvTab {
  int cnt[8];
  int t[8][6];
  double coef[8][6][3];
};

DinvTab make_dinv_tab(double hx, double hy, double hz, double lam, double mu) {
  DinvTab T{};
  const double ih[3] = {1.0 / hx, 1.0 / hy, 1.0 / hz};
  const double vol = hx * hy * hz / 6.0;
  for (int q = 0; q < 8; ++q) {
    T.cnt[q] = 0;
    for (int t = 0; t < 6; ++t)
      for (int m = 0; m < 4; ++m) {
        if (path_vertex(t, m) != q) continue;
        double g[3] = {0.0, 0.0, 0.0};
        if (m >= 1) g[path_axis(t, m - 1)] += ih[path_axis(t, m - 1)];
        if (m <= 2) g[path_axis(t, m)] -= ih[path_axis(t, m)];
        const double gg = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
        const int e = T.cnt[q]++;
        T.t[q][e] = t;
        for (int c = 0; c < 3; ++c) T.coef[q][e][c] = vol * ((lam + mu) * g[c] * g[c] + mu * gg);
      }
  }
  return T;
}

// dinv = 1 / diag K per node and component (0 on masked dofs), from the
// weights (per hex or per tet) and the corner table
__global__ void k_bdinv(BoxDims d, DinvTab T, const double* __restrict__ w, int wm, const uint8_t* __restrict__ mask,
                        float* __restrict__ dinv) {
  const int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (v >= d.N) return;
  const int i = int(v % d.px), j = int((v / d.px) % d.py), k = int(v / (int64_t(d.px) * d.py));
  double dg[3] = {0.0, 0.0, 0.0};
  for (int q = 0; q < 8; ++q) {  // this node is corner q of hex (i, j, k) - offset(q)
    const int hi = i - (q & 1), hj = j - ((q >> 1) & 1), hk = k - (q >> 2);
    if (hi < 0 || hi >= d.nx || hj < 0 || hj >= d.ny || hk < 0 || hk >= d.nz) continue;
    const int64_t h = hi + int64_t(d.nx) * (hj + int64_t(d.ny) * hk);
    const double wh = wm ? 0.0 : w[h];
    for (int e = 0; e < T.cnt[q]; ++e) {
      const double s = wm ? w[T.t[q][e] * d.H + h] : wh;
#pragma unroll
      for (int c = 0; c < 3; ++c) dg[c] = fma(s, T.coef[q][e][c], dg[c]);
    }
  }
  const uint8_t mk = mask[v];
#pragma unroll
  for (int c = 0; c < 3; ++c) dinv[c * d.N + v] = ((mk >> c) & 1) || !(dg[c] > 0.0) ? 0.f : float(1.0 / dg[c]);
}

// Coarsest level: A += masked 12x12 stiffness of every tet (one thread per
// tet; component-major dofs c N + v, row stride nd).
__global__ void k_bdense_assemble(BoxDims d, double hx, double hy, double hz, Iso<double> iso,
                                  const double* __restrict__ w, const uint8_t* __restrict__ mask, int64_t nd,
                                  double* __restrict__ A) {
  const int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (e >= 6 * d.H) return;
  const int64_t h = e / 6;
  const int t = int(e % 6);
  const int i = int(h % d.nx), j = int((h / d.nx) % d.ny), k = int(h / (int64_t(d.nx) * d.ny));
  const double ih[3] = {1.0 / hx, 1.0 / hy, 1.0 / hz};
  double g[4][3];
  int64_t vv[4];
  for (int m = 0; m < 4; ++m) {
    g[m][0] = g[m][1] = g[m][2] = 0.0;
    if (m >= 1) g[m][path_axis(t, m - 1)] += ih[path_axis(t, m - 1)];
    if (m <= 2) g[m][path_axis(t, m)] -= ih[path_axis(t, m)];
    const int c = path_vertex(t, m);
    vv[m] = (i + (c & 1)) + int64_t(d.px) * ((j + ((c >> 1) & 1)) + int64_t(d.py) * (k + (c >> 2)));
  }
  const double s = hx * hy * hz / 6.0 * w[h];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      double k9[9];
      tet_kblock(iso, s, g[a], g[b], k9);
      for (int di = 0; di < 3; ++di) {
        if ((mask[vv[a]] >> di) & 1) continue;
        for (int dj = 0; dj < 3; ++dj) {
          if ((mask[vv[b]] >> dj) & 1) continue;
          atomicAdd(&A[(di * d.N + vv[a]) * nd + dj * d.N + vv[b]], k9[3 * di + dj]);
        }
      }
    }
}

// identity on Dirichlet and padding dofs; diag0 = the diagonal before elimination
__global__ void k_bdense_ident(int64_t N, int64_t nd, const uint8_t* __restrict__ mask, double* __restrict__ A,
                               double* __restrict__ diag0) {
  const int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (r >= nd) return;
  const bool fixed = r >= 3 * N || ((mask[r % N] >> (r / N)) & 1);
  if (fixed) A[r * nd + r] = 1.0;
  diag0[r] = A[r * nd + r];
}

}  // namespace

// ---------------------------------------------------------- hierarchy --
struct BoxLevel {
  BoxDims d{};
  double h[3] = {1, 1, 1};
  bool cube = true;
  int wm = 0;  // 1: tet-major weights (finest level only)
  DevBuf<double> w64;
  DevBuf<float> w32;
  DevBuf<uint8_t> own_mask;
  const uint8_t* mask = nullptr;
  DevBuf<float> dinv, x, b, r, pw0, pw1;
  float lmax = 0.f;
  bool pw_valid = false;
  // coarsest level: dense inverse
  int64_t nd = 0;
  DevBuf<double> dense, gj_c, gj_p, diag0, flag;
  DevBuf<unsigned> gj_sync;
};

struct BoxHierarchy {
  std::vector<std::unique_ptr<BoxLevel>> L;
  int fine_n[3] = {0, 0, 0};
  double fine_l[3] = {0, 0, 0};
  DevBuf<double> w64t, w64h;
  DevBuf<float> w32t, w32h;
  DevBuf<unsigned int> differ;
  DevBuf<double> partials, sc, norms;
  DevBuf<unsigned int> counter;
  DevBuf<double> p0, p1, q;  // outer CG directions (ping-pong) and K p
  DevBuf<uint8_t> mask0;     // the finest level's Dirichlet mask in lattice order (permuted meshes)
  std::vector<int32_t> mask_dofs;  // the Dirichlet set the coarse masks were built for
  bool masks_valid = false;
  DevBuf<float> cheb;  // per smoothed level: 1 / theta, ca, c2 (read by the captured iteration)
  DevBuf<double> e_partials, e_value;  // the per-cell entry points' energy reduction
  DevBuf<double> gu_k0;                // assembled K on the box: unpenalized blocks per table entry
  double gu_key[5] = {0, 0, 0, 0, 0};  // the hex sides and Lame constants they were made for
  // learned coarse-weight correction: features and network output of level 1,
  // and an explicit correction (stride 1) that overrides the network while set
  DevBuf<float> cfeat, cout3;
  const float* delta_arg = nullptr;
  // spectral estimates from the deterministic cold start (20 power steps)
  // instead of the previous solve's vector: loss evaluations then depend on
  // the control and the correction only
  bool cold_spectrum = false;
  // the captured outer iteration (two variants alternate the p buffers),
  // reused while every pointer and constant it captured is unchanged
  struct GraphKey {
    const void* ptr[6] = {};
    int wm = -1;
    double lam = 0.0, mu = 0.0;
    bool jacobi = false;
    bool operator==(const GraphKey& o) const {
      for (int k = 0; k < 6; ++k)
        if (ptr[k] != o.ptr[k]) return false;
      return wm == o.wm && lam == o.lam && mu == o.mu && jacobi == o.jacobi;
    }
  } key;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int64_t per_iter = 0;
  BoxHierarchy() = default;
  BoxHierarchy(const BoxHierarchy&) = delete;
  BoxHierarchy& operator=(const BoxHierarchy&) = delete;
  ~BoxHierarchy() { drop_graphs(); }
  void drop_graphs() {
    for (auto& e : gexec) {
      if (e) cudaGraphExecDestroy(e);
      e = nullptr;
    }
  }
};

void boxmg_release(Problem& P) {
  delete P.boxmg;
  P.boxmg = nullptr;
}

namespace {

thread_local int64_t g_box_launches = 0;

template <typename T>
BoxGeo<T> box_geo(const BoxLevel& L, const ElasticParams& ep) {
  const Iso<double> iso = ep.iso();
  const double vol = L.h[0] * L.h[1] * L.h[2] / 6.0;
  BoxGeo<T> g;
  const double s = L.cube ? 1.0 / (L.h[0] * L.h[0]) : 1.0;
  g.lam = T(iso.lam * vol * s);
  g.mu = T(iso.mu * vol * s);
  for (int a = 0; a < 3; ++a) g.ih[a] = T(1.0 / L.h[a]);
  return g;
}

// CTAs of a box launch: a brick column per (31 x 7) node block, the z range
// cut into as many chunks as fill the resident CTA slots once (a chunk may be
// one node plane: on the small coarse levels a CTA's walk along z, not the
// halo layer it recomputes, sets the launch's time; measured on 160x80x80
// with chunks of at least two planes the solve took 9.01 ms, with one 8.75).
dim3 box_grid(const BoxDims& d, int slots, int* kz_out) {
  const int gx = (d.px + kBoxX - 1) / kBoxX, gy = (d.py + kBoxY - 1) / kBoxY;
  const int gz_want = std::max(1, slots / (gx * gy));
  int kz = std::max(1, (d.pz + gz_want - 1) / gz_want);
  const int gz = (d.pz + kz - 1) / kz;
  *kz_out = kz;
  return dim3(unsigned(gx), unsigned(gy), unsigned(gz));
}

void set_dims(BoxLevel& L, int nx, int ny, int nz, double lx, double ly, double lz) {
  L.d.nx = nx;
  L.d.ny = ny;
  L.d.nz = nz;
  L.d.px = nx + 1;
  L.d.py = ny + 1;
  L.d.pz = nz + 1;
  L.d.N = int64_t(L.d.px) * L.d.py * L.d.pz;
  L.d.H = int64_t(nx) * ny * nz;
  L.h[0] = lx / nx;
  L.h[1] = ly / ny;
  L.h[2] = lz / nz;
  const double hmax = std::max(std::max(L.h[0], L.h[1]), L.h[2]);
  L.cube = std::fabs(L.h[0] - L.h[1]) <= 1e-12 * hmax && std::fabs(L.h[0] - L.h[2]) <= 1e-12 * hmax;
}

template <typename T, int WM, bool CUBE, class In, class Out>
void launch_box_t(const BoxLevel& L, const BoxGeo<T>& g, const T* w, const In& in, const Out& out, BoxRed red,
                  cudaStream_t s, double p = 0.0, double pmin = 0.0, const double* skip = nullptr) {
  static int occupancy = 0;  // resident CTAs per SM of this instance
  if (occupancy == 0) {
    int o = 0;
    PA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_box<T, WM, CUBE, In, Out>, kBoxThreads, 0));
    occupancy = std::max(1, o);
  }
  int kz = 2;
  const dim3 grid = box_grid(L.d, occupancy * num_sms(), &kz);
  k_box<T, WM, CUBE, In, Out><<<grid, kBoxThreads, 0, s>>>(L.d, g, BoxW<T, WM>{w, L.d.H, p, pmin}, kz, in, out, red,
                                                          skip);
  PA_LAUNCHED();
  g_box_launches += 1;
}

// dispatch on the level's weight layout and hex shape
template <typename T, class In, class Out>
void launch_box(const BoxLevel& L, const BoxGeo<T>& g, const T* w, const In& in, const Out& out, BoxRed red,
                cudaStream_t s, const double* skip = nullptr) {
  if (L.wm) {
    if (L.cube)
      launch_box_t<T, 1, true>(L, g, w, in, out, red, s, 0.0, 0.0, skip);
    else
      launch_box_t<T, 1, false>(L, g, w, in, out, red, s, 0.0, 0.0, skip);
  } else {
    if (L.cube)
      launch_box_t<T, 0, true>(L, g, w, in, out, red, s, 0.0, 0.0, skip);
    else
      launch_box_t<T, 0, false>(L, g, w, in, out, red, s, 0.0, 0.0, skip);
  }
}

// an upper bound on the CTAs of any box launch on the hierarchy (chunks of
// at least one plane) and of the vector kernels
int64_t max_grid_blocks(const BoxHierarchy& H) {
  int64_t m = 148 * 8;
  for (const auto& L : H.L)
    m = std::max<int64_t>(m, int64_t((L->d.px + kBoxX - 1) / kBoxX) * ((L->d.py + kBoxY - 1) / kBoxY) * L->d.pz);
  return m;
}

// coarse masks by injection (fine node (2I, 2J, 2K)); a coarse node beyond a
// padded fine level (2 I > f.nx) takes the mask of the last fine node plane
void coarse_mask(const BoxLevel& f, BoxLevel& c, const std::vector<uint8_t>& fmask, std::vector<uint8_t>& cmask) {
  cmask.assign(size_t(c.d.N), 0);
  for (int64_t K = 0; K < c.d.pz; ++K)
    for (int64_t J = 0; J < c.d.py; ++J)
      for (int64_t I = 0; I < c.d.px; ++I) {
        const int64_t i = std::min<int64_t>(2 * I, f.d.nx), j = std::min<int64_t>(2 * J, f.d.ny),
                      k = std::min<int64_t>(2 * K, f.d.nz);
        cmask[size_t(I + c.d.px * (J + c.d.py * K))] = fmask[size_t(i + f.d.px * (j + f.d.py * k))];
      }
}

// Hex counts of the multigrid levels of an nx x ny x nz box: the next level
// has ceil(n / 2) hexes per axis (an odd level is padded by one hex layer of
// weight zero), while every axis has at least 4 hexes, or at least 2 while
// the level still has more than kCoarseDofs dofs; the last level is the
// coarsest, solved by a dense inverse of at most kDenseMax dofs.
constexpr int64_t kDenseMax = 2048, kCoarseDofs = 512;
std::vector<std::array<int, 3>> box_level_counts(const int* n0) {
  std::vector<std::array<int, 3>> out;
  std::array<int, 3> n = {n0[0], n0[1], n0[2]};
  while (true) {
    out.push_back(n);
    const int mn = std::min(std::min(n[0], n[1]), n[2]);
    const int64_t dofs = 3LL * (n[0] + 1) * (n[1] + 1) * (n[2] + 1);
    if (!(mn >= 4 || (mn >= 2 && dofs > kCoarseDofs))) break;
    for (int a = 0; a < 3; ++a) n[a] = (n[a] + 1) / 2;
  }
  return out;
}

}  // namespace

// True when the box kernels can run this problem's multigrid solve: a box
// lattice (any hex counts), one part, at least one coarse level, and a
// coarsest level of at most 2048 dofs for the dense inverse.
bool boxmg_eligible(const Problem& P) {
  const Mesh& m = *P.mesh;
  if (!box_apply_eligible(P)) return false;
  const auto lv = box_level_counts(m.lat_n);
  const auto& c = lv.back();
  return lv.size() >= 2 && 3LL * (c[0] + 1) * (c[1] + 1) * (c[2] + 1) <= kDenseMax;
}

// True when the box kernel can apply this problem's operator (pa_apply).
bool box_apply_eligible(const Problem& P) {
  const Mesh& m = *P.mesh;
  return m.box_kernels && m.lat_n[0] > 0 && m.num_parts == 1 && 3 * m.N < (int64_t(1) << 31);
}

namespace {

// Build the hierarchy for the problem's box (first use or a new box), then
// refresh weights, masks, diagonals, spectral estimates and the coarsest
// inverse for control z.  False when the coarsest operator is singular (no
// dense inverse): the caller then solves with pa_mg.cu, whose coarsest
// level falls back to Chebyshev.
// The hierarchy's levels and device buffers for the problem's box.
void boxmg_setup_levels(Problem& P) {
  const Mesh& m = *P.mesh;
  cudaStream_t s = P.stream;
  boxmg_release(P);
  std::unique_ptr<BoxHierarchy> H(new BoxHierarchy());
  for (int a = 0; a < 3; ++a) {
    H->fine_n[a] = m.lat_n[a];
    H->fine_l[a] = m.lat_l[a];
  }
  const auto counts = box_level_counts(m.lat_n);
  double len[3] = {m.lat_l[0], m.lat_l[1], m.lat_l[2]};
  for (size_t l = 0; l < counts.size(); ++l) {
    const auto& n = counts[l];
    if (l > 0)  // hexes twice the size of the level above (a padded level spans more)
      for (int a = 0; a < 3; ++a) len[a] = 2.0 * H->L[l - 1]->h[a] * n[a];
    std::unique_ptr<BoxLevel> L(new BoxLevel());
    set_dims(*L, n[0], n[1], n[2], len[0], len[1], len[2]);
    const int64_t n3 = 3 * L->d.N;
    L->dinv.resize(n3);
    L->x.resize(n3);
    L->r.resize(n3);
    if (l > 0) {
      L->b.resize(n3);
      L->w64.resize(L->d.H);
      L->w32.resize(L->d.H);
      L->own_mask.resize(L->d.N);
      L->mask = L->own_mask.get();
    }
    H->L.push_back(std::move(L));
  }
  const BoxLevel& F = *H->L[0];
  H->w64t.resize(6 * F.d.H);
  H->w32t.resize(6 * F.d.H);
  H->w64h.resize(F.d.H);
  H->w32h.resize(F.d.H);
  H->differ.resize(1);
  H->partials.resize(size_t(max_grid_blocks(*H)));
  H->counter.resize(1);
  PA_CUDA(cudaMemsetAsync(H->counter.get(), 0, sizeof(unsigned int), s));
  H->sc.resize(kScalars);
  H->norms.resize(H->L.size() * 21);
  const int64_t n3 = 3 * F.d.N;
  H->p0.resize(n3);
  H->p1.resize(n3);
  H->q.resize(n3);
  P.boxmg = H.release();
}

// The problem's Dirichlet mask in lattice order (a gather on permuted meshes).
const uint8_t* lattice_mask(Problem& P) {
  const Mesh& m = *P.mesh;
  if (!m.lat_permuted) return P.d_node_mask.get();
  BoxHierarchy& H = *P.boxmg;
  H.mask0.resize(m.N);
  k_bperm_mask<<<int((m.N + kVT - 1) / kVT), kVT, 0, P.stream>>>(m.N, m.d_lat_node.get(), P.d_node_mask.get(),
                                                               H.mask0.get());
  PA_LAUNCHED();
  g_box_launches += 1;
  return H.mask0.get();
}

// True when the hierarchy must be (re)built for the problem's box.
bool boxmg_stale(const Problem& P) {
  const Mesh& m = *P.mesh;
  if (P.boxmg == nullptr) return true;
  for (int a = 0; a < 3; ++a)
    if (P.boxmg->fine_n[a] != m.lat_n[a] || P.boxmg->fine_l[a] != m.lat_l[a]) return true;
  return false;
}

bool boxmg_setup(Problem& P, const double* z) {
  cudaStream_t s = P.stream;
  if (boxmg_stale(P)) boxmg_setup_levels(P);
  PA_CHECK(P.boxmg->L.size() >= 2, "PA_SOLVER_PCG_MG needs at least one coarse level");
  BoxHierarchy& H = *P.boxmg;
  BoxLevel& F = *H.L[0];
  const Mesh& m = *P.mesh;
  F.mask = lattice_mask(P);
  // fine weights in lattice order
  PA_CUDA(cudaMemsetAsync(H.differ.get(), 0, sizeof(unsigned int), s));
  k_bweights<<<int((F.d.H + kVT - 1) / kVT), kVT, 0, s>>>(
      F.d, z, P.ep.layout, P.ep.p, P.ep.pmin, m.lat_permuted ? m.d_lat_cell.get() : nullptr,
      m.lat_permuted ? m.d_lat_node.get() : nullptr, H.w64t.get(), H.w32t.get(), H.w64h.get(), H.w32h.get(),
      H.differ.get());
  PA_LAUNCHED();
  // coarse masks by injection (host, from the problem's Dirichlet dofs),
  // rebuilt only when the Dirichlet set changed since the last solve
  if (!H.masks_valid || H.mask_dofs != P.bc_dofs) {
    std::vector<uint8_t> fmask(size_t(F.d.N), 0);
    for (int32_t dof : P.bc_dofs) {
      const int32_t v = dof / 3;
      fmask[size_t(m.lat_permuted ? m.h_lat_of_node[size_t(v)] : v)] |= uint8_t(1u << (dof % 3));
    }
    for (size_t l = 1; l < H.L.size(); ++l) {
      std::vector<uint8_t> cmask;
      coarse_mask(*H.L[l - 1], *H.L[l], fmask, cmask);
      H.L[l]->own_mask.upload(cmask.data(), cmask.size(), s);
      fmask.swap(cmask);
    }
    H.mask_dofs = P.bc_dofs;
    H.masks_valid = true;
  }
  unsigned int differ = 0;
  PA_CUDA(cudaMemcpyAsync(&differ, H.differ.get(), sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  F.wm = differ ? 1 : 0;
  const double* fw64 = F.wm ? H.w64t.get() : H.w64h.get();
  g_box_launches += 1;
  // learned correction of the level-1 weights: the explicit one of a
  // sensitivity evaluation, else the problem's coarse-weight network
  const float* delta = H.delta_arg;
  int dstride = 1;
  if (!delta && P.coarse_pc) {
    const BoxLevel& L1 = *H.L[1];
    PA_CHECK(pc_grid_points(*P.coarse_pc) == L1.d.H, "coarse-weight network: grid is not the level-1 hex grid");
    H.cfeat.resize(size_t(5 * L1.d.H));
    H.cout3.resize(size_t(3 * L1.d.H));
    k_bcoarse_feat<<<int((L1.d.H + kVT - 1) / kVT), kVT, 0, s>>>(L1.d, F.d, fw64, F.wm, H.cfeat.get());
    PA_LAUNCHED();
    pc_forward_features(*P.coarse_pc, H.cfeat.get(), H.cout3.get(), s);
    g_box_launches += 7;
    delta = H.cout3.get();
    dstride = 3;
  }
  // coarse weights of every level
  const Iso<double> iso = P.ep.iso();
  for (size_t l = 1; l < H.L.size(); ++l) {
    BoxLevel& L = *H.L[l];
    const BoxLevel& Fl = *H.L[l - 1];
    k_bcoarse_w<<<int((L.d.H + kVT - 1) / kVT), kVT, 0, s>>>(L.d, Fl.d, l == 1 ? fw64 : Fl.w64.get(),
                                                             l == 1 ? F.wm : 0, L.w64.get(), L.w32.get(),
                                                             l == 1 ? delta : nullptr, dstride);
    PA_LAUNCHED();
    g_box_launches += 1;
  }
  // coarsest level: dense inverse (eligibility guarantees at most 2048 dofs)
  BoxLevel& Lc = *H.L.back();
  {
    const int64_t n3 = 3 * Lc.d.N, nd = (n3 + kGJ - 1) / kGJ * kGJ;
    if (Lc.nd != nd) {
      Lc.dense.resize(nd * nd);
      Lc.gj_c.resize(nd * kGJ);
      Lc.gj_p.resize(2 * kGJ * kGJ);
      Lc.gj_sync.resize(1);
      Lc.diag0.resize(nd);
      Lc.flag.resize(1);
      Lc.nd = nd;
    }
    PA_CUDA(cudaMemsetAsync(Lc.dense.get(), 0, sizeof(double) * nd * nd, s));
    PA_CUDA(cudaMemsetAsync(Lc.flag.get(), 0, sizeof(double), s));
    k_bdense_assemble<<<int((6 * Lc.d.H + kVT - 1) / kVT), kVT, 0, s>>>(Lc.d, Lc.h[0], Lc.h[1], Lc.h[2], iso,
                                                                        Lc.w64.get(), Lc.mask, nd, Lc.dense.get());
    k_bdense_ident<<<int((nd + kVT - 1) / kVT), kVT, 0, s>>>(Lc.d.N, nd, Lc.mask, Lc.dense.get(), Lc.diag0.get());
    PA_LAUNCHED();
    // (on a side stream beside the other levels' set-up the median solve was
    // slower: 7.97 against 7.91 ms on 160x80x80, the cooperative launch at
    // times waiting for the power iterations' CTAs)
    gj_invert(s, nd, Lc.dense.get(), Lc.diag0.get(), Lc.gj_c.get(), Lc.gj_p.get(), Lc.gj_sync.get(), Lc.flag.get());
    g_box_launches += 3;
  }
  // every level's inverse diagonal
  for (size_t l = 0; l < H.L.size(); ++l) {
    BoxLevel& L = *H.L[l];
    const double* lw = l == 0 ? fw64 : L.w64.get();
    const DinvTab tab = make_dinv_tab(L.h[0], L.h[1], L.h[2], iso.lam, iso.mu);
    k_bdinv<<<int((L.d.N + kVT - 1) / kVT), kVT, 0, s>>>(L.d, tab, lw, l == 0 ? F.wm : 0, L.mask, L.dinv.get());
    PA_LAUNCHED();
    g_box_launches += 1;
  }
  // lmax of D^-1 K per smoothed level by power iteration, on the device
  // (the norm of each step lands in norms[level][step]); an elastic solve
  // after an elastic solve starts from the previous vector and takes 5 steps
  constexpr int kPower = 20, kPowerWarm = 5;
  const size_t NL = H.L.size();
  const size_t NS = NL - 1;  // smoothed levels (the coarsest is solved exactly)
  PA_CUDA(cudaMemsetAsync(H.norms.get(), 0, sizeof(double) * NL * (kPower + 1), s));
  BoxRed red{H.partials.get(), H.counter.get()};
  for (size_t l = 0; l < NS; ++l) {
    BoxLevel& L = *H.L[l];
    const int64_t n3 = 3 * L.d.N;
    double* nl = H.norms.get() + l * (kPower + 1);
    if (L.pw0.n != size_t(n3)) {
      L.pw0.resize(n3);
      L.pw1.resize(n3);
      L.pw_valid = false;
    }
    const bool warm = L.pw_valid && !H.cold_spectrum;
    if (!warm)
      k_bseed<<<vec_blocks(L.d.N), kVT, 0, s>>>(int(L.d.N), L.mask, L.pw0.get(), H.partials.get(), H.counter.get(), nl);
    else
      k_bnorm2<<<vec_blocks(n3), kVT, 0, s>>>(n3, L.pw0.get(), H.partials.get(), H.counter.get(), nl);
    PA_LAUNCHED();
    g_box_launches += 1;
    const int steps = warm ? kPowerWarm : kPower;
    const BoxGeo<float> g = box_geo<float>(L, P.ep);
    const float* lw32 = l == 0 ? (F.wm ? H.w32t.get() : H.w32h.get()) : L.w32.get();
    for (int it = 1; it <= steps; ++it) {
      float* xin = (it & 1) ? L.pw0.get() : L.pw1.get();
      float* xout = (it & 1) ? L.pw1.get() : L.pw0.get();
      launch_box<float>(L, g, lw32, InVec<float, float>{xin, nullptr, L.d.N},
                        OutPower{xout, L.dinv.get(), nl + it - 1, nl + it, L.d.N}, red, s);
    }
    if (steps & 1) {  // the last vector in pw0
      std::swap(L.pw0.p, L.pw1.p);
      std::swap(L.pw0.n, L.pw1.n);
    }
  }
  std::vector<double> h(NL * (kPower + 1));
  PA_CUDA(cudaMemcpyAsync(h.data(), H.norms.get(), sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
  double flag = 0.0;
  PA_CUDA(cudaMemcpyAsync(&flag, Lc.flag.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  if (flag >= 2.0) throw Error(PA_ERR_CUDA, "coarsest factorization: a grid barrier timed out");
  if (flag != 0.0) return false;
  for (size_t l = 0; l < NS; ++l) {
    BoxLevel& L = *H.L[l];
    const bool warm = L.pw_valid && !H.cold_spectrum;
    const int steps = warm ? kPowerWarm : kPower;
    PA_CHECK(h[l * (kPower + 1)] > 0.0, "multigrid level without free dofs");
    double lam = 0.0;
    for (int it = 1; it <= steps; ++it) {
      const double v = h[l * (kPower + 1) + it];
      if (std::isfinite(v)) lam = std::max(lam, std::sqrt(v));
    }
    PA_CHECK(lam > 0.0, "multigrid: no spectral estimate (zero operator?)");
    if (warm) lam = std::max(lam, 0.95 * double(L.lmax));
    L.lmax = float(lam);
    L.pw_valid = true;
  }
  return true;
}

}  // namespace
}  // namespace pa

namespace pa {
namespace {

struct ChebStep {
  float inv_theta, ca, c2;
};

// Degree-2 Chebyshev on [lmax / 30, lmax] (lmax = 1.1 x the estimate): the
// first-step coefficients of the recurrence of pa_mg.cu (cheb_coeffs).
ChebStep cheb2(float lmax_est) {
  // measured (iterations to 1e-8 on 160x80x80 / 64^3 smoothed / a 64^3 SIMP
  // design): [lmax/10, 1.15 lmax] 20 / 19 / 182, [lmax/30, 1.05 lmax] 18 / 17 /
  // 177, [lmax/5, 1.3 lmax] 23 / 21 / 205; 1.1 keeps a margin over the power
  // iteration's estimate, which approaches lmax from below
  const double lmax = 1.1 * double(lmax_est), lmin = lmax / 30.0;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
  const double rho = 1.0 / sigma;
  const double rn = 1.0 / (2.0 * sigma - rho);
  const double c1 = rn * rho, c2 = 2.0 * rn / delta;
  return ChebStep{float(1.0 / theta), float((1.0 + c1) / theta + c2), float(c2)};
}

const float* level_w32(const BoxHierarchy& H, size_t l) {
  const BoxLevel& L = *H.L[l];
  if (l > 0) return L.w32.get();
  return L.wm ? H.w32t.get() : H.w32h.get();
}
const double* level_w64(const BoxHierarchy& H, size_t l) {
  const BoxLevel& L = *H.L[l];
  if (l > 0) return L.w64.get();
  return L.wm ? H.w64t.get() : H.w64h.get();
}

// the part of the V-cycle on level l and below that reads b (B) and writes x_out (O)
// skip: the outer CG's kBreak / kDone flags (the launches become no-ops once set)
template <typename B, typename O, bool RZ>
void vcycle_level(const Problem& P, BoxHierarchy& H, size_t l, const B* b, O* xo, const double* rvec, double* sc,
                  cudaStream_t s, const double* skip);

void vcycle(const Problem& P, BoxHierarchy& H, size_t l, cudaStream_t s, const double* skip) {
  // levels >= 1: b and x in the level's FP32 buffers
  BoxLevel& L = *H.L[l];
  if (l + 1 == H.L.size()) {
    const int64_t n3 = 3 * L.d.N;
    k_mg_dense_solve<<<int((32 * n3 + kVT - 1) / kVT), kVT, 0, s>>>(n3, L.nd, L.dense.get(), L.b.get(), L.x.get(),
                                                                    skip);
    PA_LAUNCHED();
    g_box_launches += 1;
    return;
  }
  vcycle_level<float, float, false>(P, H, l, L.b.get(), L.x.get(), nullptr, nullptr, s, skip);
}

template <typename B, typename O, bool RZ>
void vcycle_level(const Problem& P, BoxHierarchy& H, size_t l, const B* b, O* xo, const double* rvec, double* sc,
                  cudaStream_t s, const double* skip) {
  BoxLevel& L = *H.L[l];
  BoxLevel& C = *H.L[l + 1];
  const float* ch = H.cheb.get() + 3 * l;
  const BoxGeo<float> g = box_geo<float>(L, P.ep);
  const float* w = level_w32(H, l);
  const BoxRed red{H.partials.get(), H.counter.get()};
  const int64_t N = L.d.N;
  // pre-smoothing from x = 0
  launch_box<float>(L, g, w, InDinvB<B>{b, L.dinv.get(), ch, N},
                    OutPre<B>{L.x.get(), b, L.dinv.get(), ch, N}, red, s, skip);
  // residual, restricted to the coarse right-hand side
  launch_box<float>(L, g, w, InVec<float, float>{L.x.get(), nullptr, N}, OutRes<B>{L.r.get(), b, L.mask, N}, red,
                    s, skip);
  k_brestrict<<<int((C.d.N + kVT - 1) / kVT), kVT, 0, s>>>(C.d, L.d, L.r.get(), C.mask, C.b.get(), skip);
  PA_LAUNCHED();
  g_box_launches += 1;
  vcycle(P, H, l + 1, s, skip);
  // post-smoothing from x + P e
  k_bprolong_add<<<int((N + kVT - 1) / kVT), kVT, 0, s>>>(C.d, L.d, C.x.get(), L.mask, L.x.get(), skip);
  PA_LAUNCHED();
  g_box_launches += 1;
  launch_box<float>(L, g, w, InVec<float, float>{L.x.get(), nullptr, N}, OutPost1<B>{L.r.get(), b, L.dinv.get(), N},
                    red, s, skip);
  launch_box<float>(L, g, w, InScaled{L.r.get(), ch, N},
                    OutPost2<O, RZ>{xo, L.x.get(), L.r.get(), L.dinv.get(), ch, N, rvec, sc}, red, s, skip);
}

// The Chebyshev coefficients of every smoothed level (from its lmax) into
// H.cheb, which the V-cycle's launches read.
void upload_cheb(BoxHierarchy& H, cudaStream_t s) {
  const size_t NS = H.L.size() - 1;
  std::vector<float> ch(3 * NS);
  for (size_t l = 0; l < NS; ++l) {
    const ChebStep c = cheb2(H.L[l]->lmax);
    ch[3 * l] = c.inv_theta;
    ch[3 * l + 1] = c.ca;
    ch[3 * l + 2] = c.c2;
  }
  if (H.cheb.n != ch.size()) H.cheb.resize(ch.size());
  PA_CUDA(cudaMemcpyAsync(H.cheb.get(), ch.data(), sizeof(float) * ch.size(), cudaMemcpyHostToDevice, s));
}

// y = K x (FP64, box kernel) with optional masks on input and output
void box_apply64(const BoxLevel& L, const ElasticParams& ep, const double* w, const double* x, double* y,
                 const uint8_t* mask, BoxRed red, cudaStream_t s) {
  launch_box<double>(L, box_geo<double>(L, ep), w, InVec<double, double>{x, mask, L.d.N},
                     OutPlain<double>{y, mask, L.d.N}, red, s);
}

// The hierarchy's levels and buffers (no device work besides allocation).
void boxmg_ensure(Problem& P) {
  if (boxmg_stale(P)) boxmg_setup_levels(P);
}

}  // namespace

// Solve K x = b with the box multigrid-preconditioned CG for control z.
// Returns false (nothing written) when the coarsest operator is singular.
bool solve_boxmg(Problem& P, const double* z, const double* b, double* x_out, const pa_solve_options& o,
                 pa_solve_stats* st, pa_status* status, bool jacobi) {
  cudaStream_t s = P.stream;
  PA_CHECK(o.rel_tol > 0.0, "rel_tol must be positive");
  g_box_launches = 0;
  if (!boxmg_setup(P, z)) return false;
  BoxHierarchy& H = *P.boxmg;
  BoxLevel& F = *H.L[0];
  const int64_t N = F.d.N, n = 3 * N;
  SolverWorkspace& ws = P.ws;
  const uint8_t* mask = F.mask;
  const double* w64 = level_w64(H, 0);
  const BoxRed red{H.partials.get(), H.counter.get()};
  double* sc = H.sc.get();
  double* bp = ws.b.get();
  double* x = ws.x.get();
  double* r = ws.r.get();
  double* t = ws.t.get();
  double* zv = ws.p0.get();
  // b' = mask(b - K x_D), component-major, and ||b'||^2
  const int64_t nbc = int64_t(P.bc_dofs.size());
  const Mesh& m = *P.mesh;
  const int32_t* node_of = m.lat_permuted ? m.d_lat_node.get() : nullptr;
  k_bperm_in<double, double><<<vec_blocks(N), kVT, 0, s>>>(int(N), node_of, m.lat_flip, b, t);
  PA_LAUNCHED();
  if (nbc) {
    PA_CUDA(cudaMemsetAsync(zv, 0, sizeof(double) * n, s));
    k_bscatter_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), 1.0, N,
                                                         m.lat_permuted ? m.d_lat_of_node.get() : nullptr,
                                                         m.lat_flip, zv);
    PA_LAUNCHED();
    box_apply64(F, P.ep, w64, zv, H.q.get(), nullptr, red, s);
    k_bres64<<<vec_blocks(N), kVT, 0, s>>>(int(N), t, H.q.get(), mask, bp, H.partials.get(), H.counter.get(), sc + kRr);
  } else {
    k_bres64<<<vec_blocks(N), kVT, 0, s>>>(int(N), t, nullptr, mask, bp, H.partials.get(), H.counter.get(), sc + kRr);
  }
  PA_LAUNCHED();
  double bb = 0.0;
  PA_CUDA(cudaMemcpyAsync(&bb, sc + kRr, sizeof(double), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  if (!(bb > 0.0)) bb = 1.0;
  const double tol2 = o.rel_tol * o.rel_tol * bb;
  const int max_iters = o.max_iters > 0 ? o.max_iters
                        : jacobi   ? int(20.0 * std::sqrt(double(n)) + 1000.0)  // as pa_solve's default
                                   : 1000;
  PA_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
  PA_CUDA(cudaMemcpyAsync(r, bp, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  PA_CUDA(cudaMemsetAsync(H.p0.get(), 0, sizeof(double) * n, s));
  k_bcg_reset<<<1, 1, 0, s>>>(sc, tol2, 1);
  PA_LAUNCHED();
  // this solve's Chebyshev coefficients, read by the captured iteration
  upload_cheb(H, s);
  // one outer iteration as a graph; two variants alternate the p buffers.
  // Captured once and relaunched by later solves while the buffers, the
  // weight layout and the material are the same.
  BoxHierarchy::GraphKey key;
  const void* ptrs[6] = {zv, r, x, mask, w64, bp};
  for (int k = 0; k < 6; ++k) key.ptr[k] = ptrs[k];
  key.wm = F.wm;
  key.lam = P.ep.iso().lam;
  key.mu = P.ep.iso().mu;
  key.jacobi = jacobi;
  if (!(H.gexec[0] && H.key == key)) {
    H.drop_graphs();
    for (int k = 0; k < 2; ++k) {
      double* pold = k == 0 ? H.p0.get() : H.p1.get();
      double* pnew = k == 0 ? H.p1.get() : H.p0.get();
      const int64_t before = g_box_launches;
      PA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        if (jacobi) {
          k_bjacobi_z<<<vec_blocks(n), kVT, 0, s>>>(n, F.dinv.get(), r, zv, sc, H.partials.get(), H.counter.get());
          g_box_launches += 1;
        } else {
          vcycle_level<double, double, true>(P, H, 0, r, zv, r, sc, s, sc + kBreak);
        }
        launch_box<double>(F, box_geo<double>(F, P.ep), w64, InCgP{zv, pold, pnew, sc, N},
                           OutCgQ{H.q.get(), zv, pold, mask, sc, N}, red, s, sc + kBreak);
        k_bcg_update<<<vec_blocks(n), kVT, 0, s>>>(n, sc, pnew, H.q.get(), x, r, H.partials.get(), H.counter.get());
      } catch (...) {
        // end the capture so that the stream is usable again, then report
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        H.drop_graphs();
        throw;
      }
      g_box_launches += 1;
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(s, &graph);
      if (ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        H.drop_graphs();
        throw Error(PA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      }
      const cudaError_t ie = cudaGraphInstantiate(&H.gexec[k], graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        H.drop_graphs();
        throw Error(PA_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
      }
      H.per_iter = g_box_launches - before;
      g_box_launches = before;
    }
    H.key = key;
  }
  const int64_t per_iter = H.per_iter;
  int iters = 0, restarts = 0;
  double rr_true = bb;
  bool converged = false, breakdown = false;
  // Iterations run in batches of captured graphs with one host read per
  // batch: the device counts the iterations it executes, marks convergence
  // (r . r <= tol2) and breakdown, and every launch after either is a no-op.
  // The batch after the first is the number of iterations the mean reduction
  // so far predicts to convergence (at most 16).
  constexpr int kFirstBatch = 4;
  const int kMaxBatch = jacobi ? 128 : 16;  // Jacobi iterations are many and short
  double h4[4];  // r . r, breakdown, done, executed iterations
  while (!converged && iters < max_iters && !breakdown) {
    const int cycle_start = iters;
    const double rr_start = iters == 0 ? bb : rr_true;
    int batch = std::min(kFirstBatch, max_iters - iters);
    while (true) {
      for (int b = 0; b < batch; ++b) {
        PA_CUDA(cudaGraphLaunch(H.gexec[(iters + b) & 1], s));
        g_box_launches += per_iter;
      }
      PA_CUDA(cudaMemcpyAsync(h4, sc + kRr, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
      PA_CUDA(cudaStreamSynchronize(s));
      iters = int(h4[3]);
      if (h4[1] != 0.0) {
        breakdown = true;
        break;
      }
      if (h4[2] != 0.0 || iters >= max_iters) break;
      const int done_in_cycle = iters - cycle_start;
      const double rate = done_in_cycle > 0 && rr_start > 0.0 ? std::pow(h4[0] / rr_start, 1.0 / done_in_cycle) : 0.0;
      int m = kFirstBatch;
      if (rate > 0.0 && rate < 1.0 && h4[0] > tol2) m = int(std::ceil(std::log(tol2 / h4[0]) / std::log(rate)));
      batch = std::max(1, std::min({m, kMaxBatch, max_iters - iters}));
    }
    if (breakdown) break;
    // confirm on the true residual r = b' - K x (p and the scalars restart)
    box_apply64(F, P.ep, w64, x, H.q.get(), mask, red, s);
    k_bres64<<<vec_blocks(N), kVT, 0, s>>>(int(N), bp, H.q.get(), mask, r, H.partials.get(), H.counter.get(), sc + kRr);
    PA_LAUNCHED();
    g_box_launches += 1;
    PA_CUDA(cudaMemcpyAsync(&rr_true, sc + kRr, sizeof(double), cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    converged = rr_true <= tol2;
    if (!converged && iters < max_iters) {
      ++restarts;
      k_bcg_reset<<<1, 1, 0, s>>>(sc, tol2, 0);
      PA_LAUNCHED();
    }
  }
  // x_out = x + x_D (interleaved, caller's order)
  k_bperm_out<double, double><<<vec_blocks(N), kVT, 0, s>>>(int(N), node_of, m.lat_flip, x, x_out);
  PA_LAUNCHED();
  if (nbc) {
    k_bset_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), 1.0, x_out);
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
    st->kernel_launches = g_box_launches + 6;
    st->fallback_iterations = 0;
  }
  *status = breakdown ? PA_ERR_BREAKDOWN : !std::isfinite(relres) ? PA_ERR_NONFINITE
                                         : converged ? PA_OK : PA_ERR_NOT_CONVERGED;
  return true;
}

// y = K(z) x on the box (interleaved x, y in the caller's node order; T =
// float or double), masked when `constrained` (masked rows and columns zero;
// the caller restores identity rows), for pa_apply.  xs, ys: 3N scratch.
template <typename T>
void box_apply(Problem& P, const double* z, const T* x, T* y, bool constrained, T* xs, T* ys) {
  cudaStream_t s = P.stream;
  boxmg_ensure(P);
  BoxHierarchy& H = *P.boxmg;
  BoxLevel& F = *H.L[0];
  const Mesh& m = *P.mesh;
  PA_CUDA(cudaMemsetAsync(H.differ.get(), 0, sizeof(unsigned int), s));
  k_bweights<<<int((F.d.H + kVT - 1) / kVT), kVT, 0, s>>>(
      F.d, z, P.ep.layout, P.ep.p, P.ep.pmin, m.lat_permuted ? m.d_lat_cell.get() : nullptr,
      m.lat_permuted ? m.d_lat_node.get() : nullptr, H.w64t.get(), H.w32t.get(), H.w64h.get(), H.w32h.get(),
      H.differ.get());
  PA_LAUNCHED();
  unsigned int differ = 0;
  PA_CUDA(cudaMemcpyAsync(&differ, H.differ.get(), sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  F.wm = differ ? 1 : 0;
  const uint8_t* mask = constrained ? lattice_mask(P) : nullptr;
  const int32_t* node_of = m.lat_permuted ? m.d_lat_node.get() : nullptr;
  k_bperm_in<T, T><<<vec_blocks(F.d.N), kVT, 0, s>>>(int(F.d.N), node_of, m.lat_flip, x, xs);
  PA_LAUNCHED();
  const BoxRed red{H.partials.get(), H.counter.get()};
  if constexpr (std::is_same<T, double>::value) {
    box_apply64(F, P.ep, level_w64(H, 0), xs, ys, mask, red, s);
  } else {
    launch_box<float>(F, box_geo<float>(F, P.ep), level_w32(H, 0), InVec<float, float>{xs, mask, F.d.N},
                      OutPlain<float>{ys, mask, F.d.N}, red, s);
  }
  k_bperm_out<T, T><<<vec_blocks(F.d.N), kVT, 0, s>>>(int(F.d.N), node_of, m.lat_flip, ys, y);
  PA_LAUNCHED();
}
template void box_apply<double>(Problem&, const double*, const double*, double*, bool, double*, double*);
template void box_apply<float>(Problem&, const double*, const float*, float*, bool, float*, float*);

// Device time of the plain FP32 (or FP64) box apply over `reps` launches
// (weights from z, random x), and its algorithmic bytes per launch: weights
// (one per hex when the tets of every hex share it), x in and y out.
double time_box_apply(Problem& P, const double* z, bool fp32, int reps, int64_t* bytes) {
  cudaStream_t s = P.stream;
  const int64_t n = P.ndof();
  DevBuf<float> x32, y32;
  DevBuf<double> x64, y64;
  DevBuf<float> s32a, s32b;
  DevBuf<double> s64a, s64b;
  if (fp32) {
    x32.resize(n);
    y32.resize(n);
    s32a.resize(n);
    s32b.resize(n);
    PA_CUDA(cudaMemsetAsync(x32.get(), 0, sizeof(float) * n, s));
    box_apply<float>(P, z, x32.get(), y32.get(), true, s32a.get(), s32b.get());
  } else {
    x64.resize(n);
    y64.resize(n);
    s64a.resize(n);
    s64b.resize(n);
    PA_CUDA(cudaMemsetAsync(x64.get(), 0, sizeof(double) * n, s));
    box_apply<double>(P, z, x64.get(), y64.get(), true, s64a.get(), s64b.get());
  }
  BoxHierarchy& H = *P.boxmg;
  BoxLevel& F = *H.L[0];
  const BoxRed red{H.partials.get(), H.counter.get()};
  const uint8_t* mask = lattice_mask(P);
  cudaEvent_t e0, e1;
  PA_CUDA(cudaEventCreate(&e0));
  PA_CUDA(cudaEventCreate(&e1));
  PA_CUDA(cudaEventRecord(e0, s));
  for (int k = 0; k < reps; ++k) {
    if (fp32)
      launch_box<float>(F, box_geo<float>(F, P.ep), level_w32(H, 0), InVec<float, float>{x32.get(), mask, F.d.N},
                        OutPlain<float>{y32.get(), mask, F.d.N}, red, s);
    else
      box_apply64(F, P.ep, level_w64(H, 0), x64.get(), y64.get(), mask, red, s);
  }
  PA_CUDA(cudaEventRecord(e1, s));
  PA_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int64_t sv = fp32 ? 4 : 8;
  if (bytes) *bytes = (F.wm ? 6 * F.d.H : F.d.H) * sv + F.d.N * (6 * sv + 1);
  return double(ms) / reps;
}


// ------------------------------------------------------ box entry points --
// The per-cell entry points (VectorFunction::value, the internal energy and
// its gradients) on a box mesh in its own numbering (pa_mesh_create_box, or
// arrays in that order): K(z) u by the box kernel with the SIMP penalty of
// the per-cell controls applied as the weights load and the interleaved
// vectors read and written in place; the energy and dF/dz by one thread per
// hex over its six tets with the lattice's edge-difference gradients.
namespace {

// x from the interleaved vector (3 per node, lattice node ids)
struct InAoS64 {
  const double* x;
  struct Raw {
    double v[3];
  };
  __device__ Raw load(int v, bool) const {
    Raw r;
#pragma unroll
    for (int c = 0; c < 3; ++c) r.v[c] = x[3 * int64_t(v) + c];
    return r;
  }
  __device__ void make(const Raw& r, int, bool, double (&o)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) o[c] = r.v[c];
  }
};

struct OutAoS64 {  // y = K x, interleaved
  double* y;
  static constexpr bool kReduce = false;
  struct Pre {};
  __device__ Pre load(int) const { return {}; }
  __device__ double store(const Pre&, int v, const double (&k)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) y[3 * int64_t(v) + c] = k[c];
    return 0.0;
  }
};

// Internal energy of every tet (1/2 V sigma(eps) . eps, unpenalized), summed
// with the SIMP weights of the per-cell controls (box slot order 6 h + t) into
// one partial per CTA, and dF/dz = dw/dz e0 per cell (grad_z may be null).
// Path tet t runs 0 -> +axis(t,0) -> +axis(t,1) -> 7, so column axis(t,m) of
// grad u is the difference of u along edge m over h[axis].
// (three CTAs per SM: 98 -> 85 registers with 36 bytes of spills, 68.8 -> 65.2 us on 160x80x80)
__global__ void __launch_bounds__(256, 3) k_benergy(BoxDims d, double ih0, double ih1, double ih2, double vol,
                                                 Iso<double> iso, double p, double pmin, const double* __restrict__ u,
                                                 const double* __restrict__ z, double* __restrict__ partials,
                                                 double* __restrict__ grad_z) {
  __shared__ double red[32];
  const int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double f = 0.0;
  if (h < d.H) {
    const int i = int(h % d.nx), j = int((h / d.nx) % d.ny), k = int(h / (int64_t(d.nx) * d.ny));
    const double ih[3] = {ih0, ih1, ih2};
    double uc[8][3];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t v = (i + (q & 1)) + int64_t(d.px) * ((j + ((q >> 1) & 1)) + int64_t(d.py) * (k + (q >> 2)));
#pragma unroll
      for (int c = 0; c < 3; ++c) uc[q][c] = u[3 * v + c];
    }
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      double du[3][3];
      int prev = 0;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const int a = path_axis(t, m), nxt = prev | (1 << a);
#pragma unroll
        for (int c = 0; c < 3; ++c) du[c][a] = (uc[nxt][c] - uc[prev][c]) * ih[a];
        prev = nxt;
      }
      const double e[6] = {du[0][0], du[1][1], du[2][2], du[1][2] + du[2][1], du[0][2] + du[2][0],
                           du[0][1] + du[1][0]};
      double sig[6];
      tet_stress(iso, vol, e, sig);
      const double e0 = 0.5 * voigt_dot(sig, e);
      const double zt = z[6 * h + t];
      f += simp(zt, p, pmin) * e0;
      if (grad_z) grad_z[6 * h + t] = simp_deriv(zt, p, pmin) * e0;
    }
  }
  const double b = block_sum_box(f, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

// VectorFunction::gradient_z with per-cell controls: dR/dz of every cell, 12
// values in the cell's own vertex order (vals[12 c + 3 n + d]): one thread per
// tet.  Cell c = 6 h + t is path tet t of hex h, whose barycentric gradients
// are g_0 = -e_a0, g_m = e_a(m-1) - e_am, g_3 = e_a2 (axes a_m of the path,
// over the hex side), so the nodal force of path vertex m is the difference
// of two stress columns.  The cell's node ids give each vertex slot's corner
// (any vertex order of a template tet).  A warp's 32 cells lie in at most 7
// hexes: the warp first loads those hexes' 8 corner displacements into shared
// memory (168 values, instead of 12 gathers per cell), and at the end stages
// its 384 outputs there and writes them as contiguous 256-byte rows.
// (six CTAs per SM: 58 -> 42 registers with 88 bytes of spills, 230 -> 219 us on 160x80x80)
__global__ void __launch_bounds__(256, 6) k_bgradient_z(BoxDims d, double ih0, double ih1, double ih2, double vol,
                                                     Iso<double> iso, double p, double pmin,
                                                     const int4* __restrict__ cells, const double* __restrict__ u,
                                                     const double* __restrict__ z, double* __restrict__ vals) {
  constexpr int kRow = 13;  // staging stride per cell (odd: two-way bank conflicts at most)
  constexpr int kHex = 7;   // hexes of a warp's 32 cells at most
  __shared__ double stage[8][32 * kRow];
  __shared__ double ucor[8][kHex * 24];  // [hex][corner][component]
  __shared__ int sb0[8][kHex];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // 32-bit indices: the box path has 3 N < 2^31, so 6 H < 2^31
  const int C = int(6 * d.H);
  const int c0 = blockIdx.x * blockDim.x + 32 * w;
  if (c0 >= C) return;  // whole warp past the end (warp-uniform)
  const int c = c0 + lane;
  const int plane = d.px * d.py;
  const int hA = c0 / 6, hB = min(c0 + 31, C - 1) / 6, nh = hB - hA + 1;
  if (lane < nh) {
    const int h = hA + lane;
    const int hy = h / d.nx, k = hy / d.ny;
    sb0[w][lane] = (h - hy * d.nx) + d.px * ((hy - k * d.ny) + d.py * k);
  }
  __syncwarp();
  for (int e = lane; e < nh * 24; e += 32) {
    const int q = e / 24, r = e - 24 * q, cr = r / 3, cc = r - 3 * cr;
    const int node = sb0[w][q] + (cr & 1) + d.px * ((cr >> 1) & 1) + plane * (cr >> 2);
    ucor[w][e] = u[3 * int64_t(node) + cc];
  }
  __syncwarp();
  double* st = stage[w] + kRow * lane;
  if (c < C) {
    const int h = c / 6;
    const int t = c - 6 * h;
    const int b0 = sb0[w][h - hA];
    const double* uc = ucor[w] + 24 * (h - hA);
    // the path's axes and corners (selects, not indexed arrays: t varies per thread)
    auto ihs = [&](int a) { return a == 0 ? ih0 : a == 1 ? ih1 : ih2; };
    int ax[3], off[4], cor[4];
    int q = 0;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (m > 0) {
        ax[m - 1] = path_axis(t, m - 1);
        q |= 1 << ax[m - 1];
      }
      cor[m] = q;
      off[m] = (q & 1) + d.px * ((q >> 1) & 1) + plane * (q >> 2);
    }
    // edge differences g[m] = (u(v_m+1) - u(v_m)) / h along axis ax[m]; column a of
    // grad u is the g[m] with ax[m] == a
    double g[3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const double s = ihs(ax[m]);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) g[m][cc] = (uc[3 * cor[m + 1] + cc] - uc[3 * cor[m] + cc]) * s;
    }
    double du[3][3];  // du[cc][a]
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) du[cc][a] = ax[0] == a ? g[0][cc] : ax[1] == a ? g[1][cc] : g[2][cc];
    const double e[6] = {du[0][0], du[1][1], du[2][2], du[1][2] + du[2][1], du[0][2] + du[2][0],
                         du[0][1] + du[1][0]};
    double sg[6];
    tet_stress(iso, vol * simp_deriv(z[c], p, pmin), e, sg);
    // stress column a (Voigt: 0 xx, 1 yy, 2 zz, 3 yz, 4 xz, 5 xy) times 1 / h_a
    auto col = [&](int a, double (&o)[3]) {
      const double s = ihs(a);
      o[0] = s * (a == 0 ? sg[0] : a == 1 ? sg[5] : sg[4]);
      o[1] = s * (a == 0 ? sg[5] : a == 1 ? sg[1] : sg[3]);
      o[2] = s * (a == 0 ? sg[4] : a == 1 ? sg[3] : sg[2]);
    };
    double f[4][3];
    {
      double s0[3], s1[3], s2[3];
      col(ax[0], s0);
      col(ax[1], s1);
      col(ax[2], s2);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        f[0][cc] = -s0[cc];
        f[1][cc] = s0[cc] - s1[cc];
        f[2][cc] = s1[cc] - s2[cc];
        f[3][cc] = s2[cc];
      }
    }
    // path vertex m goes to the cell's vertex slot n whose node is at offset
    // off[m] from the hex's base node (the four slots are the four corners)
    const int4 cv = cells[c];
    const int vs0 = cv.x - b0, vs1 = cv.y - b0, vs2 = cv.z - b0;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int n = vs0 == off[m] ? 0 : vs1 == off[m] ? 1 : vs2 == off[m] ? 2 : 3;
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) st[3 * n + cc] = f[m][cc];
    }
  }
  __syncwarp();
  const int64_t base = 12 * int64_t(c0), end = 12 * int64_t(C);
#pragma unroll
  for (int r = 0; r < 12; ++r) {
    const int e = 32 * r + lane;
    if (base + e < end) vals[base + e] = stage[w][kRow * (e / 12) + e % 12];
  }
}

__global__ void k_bsum_partials(int n, const double* __restrict__ partials, double* __restrict__ out) {
  __shared__ double red[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
  v = block_sum_box(v, red);
  if (threadIdx.x == 0) *out = v;
}

}  // namespace

bool box_entry_eligible(const Problem& P) {
  const Mesh& m = *P.mesh;
  return box_apply_eligible(P) && !m.lat_permuted && m.lat_flip == 0 && P.ep.layout == PA_CONTROL_CELL;
}

void box_entry_apply(Problem& P, const double* z, const double* u, double* y) {
  boxmg_ensure(P);
  BoxHierarchy& H = *P.boxmg;
  const BoxLevel& F = *H.L[0];
  const BoxRed red{H.partials.get(), H.counter.get()};
  const BoxGeo<double> g = box_geo<double>(F, P.ep);
  if (F.cube)
    launch_box_t<double, 2, true>(F, g, z, InAoS64{u}, OutAoS64{y}, red, P.stream, P.ep.p, P.ep.pmin);
  else
    launch_box_t<double, 2, false>(F, g, z, InAoS64{u}, OutAoS64{y}, red, P.stream, P.ep.p, P.ep.pmin);
}

// ------------------------------------------- learned coarse-level weights --
// The level-1 weights of the box multigrid may carry a learned correction
// w1 = mean exp(0.5 tanh(delta)) (k_bcoarse_w), delta from a network on the
// level-1 hex grid (pa_learned.cu) fed with k_bcoarse_feat.  Training needs
// dL/ddelta of the V-cycle's energy-norm error on residual/error pairs
// (K e = r, E = e . r): with z = V r, L = ||e - z||_K^2 / E = 1 - (r.z + z.rho) / E
// (rho = r - K z), and for the two-grid cycle with exact coarse solve
// x_c = A^-1 R (r - K S r) (A the level-1 operator, R = P^T, S the symmetric
// Chebyshev smoother),
//   dL/dw_h = 2 a^T A_h x_c / E,  a = A^-1 R (I - K S) rho,
// A_h the unweighted stiffness of coarse hex h.  A^-1 is applied by the
// level-1 V-cycle (exact when level 1 is the coarsest), and the dependence
// of deeper levels and of level 1's smoother on w1 is not followed.

bool boxmg_coarse_grid(const Problem& P, int dims[3]) {
  if (!boxmg_eligible(P)) return false;
  const auto lv = box_level_counts(P.mesh->lat_n);
  for (int a = 0; a < 3; ++a) dims[a] = lv[1][a];
  return true;
}

void boxmg_coarse_features(Problem& P, const double* z, float* feat) {
  PA_CHECK(boxmg_eligible(P), "the problem's mesh has no box multigrid");
  const LearnedPC* keep = P.coarse_pc;
  P.coarse_pc = nullptr;  // the set-up below only needs the fine weights
  bool ok = false;
  try {
    ok = boxmg_setup(P, z);
  } catch (...) {
    P.coarse_pc = const_cast<LearnedPC*>(keep);
    throw;
  }
  P.coarse_pc = const_cast<LearnedPC*>(keep);
  PA_CHECK(ok, "singular coarsest operator");
  BoxHierarchy& H = *P.boxmg;
  const BoxLevel& F = *H.L[0];
  const BoxLevel& L1 = *H.L[1];
  const double* fw64 = F.wm ? H.w64t.get() : H.w64h.get();
  k_bcoarse_feat<<<int((L1.d.H + kVT - 1) / kVT), kVT, 0, P.stream>>>(L1.d, F.d, fw64, F.wm, feat);
  PA_LAUNCHED();
}

void boxmg_coarse_sensitivity(Problem& P, const double* z, const float* delta, int nres, const double* res,
                              const double* energies, double* loss, float* grad) {
  PA_CHECK(boxmg_eligible(P), "the problem's mesh has no box multigrid");
  PA_CHECK(nres > 0, "no residuals");
  boxmg_ensure(P);
  BoxHierarchy& H = *P.boxmg;
  H.delta_arg = delta;
  H.cold_spectrum = true;
  bool ok = false;
  try {
    ok = boxmg_setup(P, z);
  } catch (...) {
    H.delta_arg = nullptr;
    H.cold_spectrum = false;
    throw;
  }
  H.delta_arg = nullptr;
  H.cold_spectrum = false;
  PA_CHECK(ok, "singular coarsest operator");
  cudaStream_t s = P.stream;
  upload_cheb(H, s);
  BoxLevel& F = *H.L[0];
  BoxLevel& C = *H.L[1];
  const int64_t N = F.d.N, n = 3 * N, N1 = C.d.N;
  const Mesh& m = *P.mesh;
  const int32_t* node_of = m.lat_permuted ? m.d_lat_node.get() : nullptr;
  DevBuf<float> r32(n), z32(n), rho(n), sr(n), zeta(n), xc(3 * N1);
  DevBuf<double> gw(size_t(C.d.H)), acc(1);
  PA_CUDA(cudaMemsetAsync(gw.get(), 0, sizeof(double) * C.d.H, s));
  PA_CUDA(cudaMemsetAsync(acc.get(), 0, sizeof(double), s));
  const BoxGeo<float> g = box_geo<float>(F, P.ep);
  const float* w0 = level_w32(H, 0);
  const float* ch0 = H.cheb.get();
  const BoxRed red{H.partials.get(), H.counter.get()};
  const double vol1 = C.h[0] * C.h[1] * C.h[2] / 6.0;
  for (int k = 0; k < nres; ++k) {
    const double E = energies[k];
    PA_CHECK(E > 0.0, "residual energies must be positive");
    k_bperm_in<double, float><<<vec_blocks(N), kVT, 0, s>>>(int(N), node_of, m.lat_flip, res + int64_t(k) * n,
                                                            r32.get());
    k_bmask_f<<<int((N + kVT - 1) / kVT), kVT, 0, s>>>(int(N), F.mask, r32.get());
    PA_LAUNCHED();
    // z = V r; x_c = the level-1 correction of this cycle
    vcycle_level<float, float, false>(P, H, 0, r32.get(), z32.get(), nullptr, nullptr, s, nullptr);
    PA_CUDA(cudaMemcpyAsync(xc.get(), C.x.get(), sizeof(float) * 3 * N1, cudaMemcpyDeviceToDevice, s));
    // rho = r - K z; the loss
    launch_box<float>(F, g, w0, InVec<float, float>{z32.get(), nullptr, N}, OutRes<float>{rho.get(), r32.get(), F.mask, N},
                      red, s);
    k_bcoarse_loss<<<vec_blocks(n), kVT, 0, s>>>(n, r32.get(), z32.get(), rho.get(), 1.0 / E, H.partials.get(),
                                                 H.counter.get(), acc.get());
    PA_LAUNCHED();
    // zeta = (I - K S) rho, a = A^-1 R zeta
    launch_box<float>(F, g, w0, InDinvB<float>{rho.get(), F.dinv.get(), ch0, N},
                      OutPre<float>{sr.get(), rho.get(), F.dinv.get(), ch0, N}, red, s);
    launch_box<float>(F, g, w0, InVec<float, float>{sr.get(), nullptr, N},
                      OutRes<float>{zeta.get(), rho.get(), F.mask, N}, red, s);
    k_brestrict<<<int((N1 + kVT - 1) / kVT), kVT, 0, s>>>(C.d, F.d, zeta.get(), C.mask, C.b.get(), nullptr);
    PA_LAUNCHED();
    vcycle(P, H, 1, s, nullptr);
    k_bbilinear<<<int((C.d.H + 255) / 256), 256, 0, s>>>(C.d, 1.0 / C.h[0], 1.0 / C.h[1], 1.0 / C.h[2], vol1,
                                                        P.ep.iso(), C.x.get(), xc.get(), 2.0 / E, gw.get());
    PA_LAUNCHED();
  }
  k_bgrad_delta<<<int((C.d.H + kVT - 1) / kVT), kVT, 0, s>>>(C.d.H, gw.get(), C.w64.get(), delta, 1.0 / nres, grad);
  PA_LAUNCHED();
  double a = 0.0;
  PA_CUDA(cudaMemcpyAsync(&a, acc.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  *loss = a / nres;
}

void box_entry_gradient_z(Problem& P, const double* z, const double* u, double* vals) {
  boxmg_ensure(P);
  const BoxLevel& F = *P.boxmg->L[0];
  const double vol = F.h[0] * F.h[1] * F.h[2] / 6.0;
  const int64_t C = 6 * F.d.H;
  k_bgradient_z<<<int((C + 255) / 256), 256, 0, P.stream>>>(
      F.d, 1.0 / F.h[0], 1.0 / F.h[1], 1.0 / F.h[2], vol, P.ep.iso(), P.ep.p, P.ep.pmin,
      reinterpret_cast<const int4*>(P.mesh->d_cells.get()), u, z, vals);
  PA_LAUNCHED();
}

void box_entry_energy(Problem& P, const double* z, const double* u, double* value, double* grad_z) {
  boxmg_ensure(P);
  BoxHierarchy& H = *P.boxmg;
  const BoxLevel& F = *H.L[0];
  const int blocks = int((F.d.H + 255) / 256);
  if (H.e_partials.n < size_t(blocks)) H.e_partials.resize(blocks);
  const double vol = F.h[0] * F.h[1] * F.h[2] / 6.0;
  k_benergy<<<blocks, 256, 0, P.stream>>>(F.d, 1.0 / F.h[0], 1.0 / F.h[1], 1.0 / F.h[2], vol, P.ep.iso(), P.ep.p,
                                          P.ep.pmin, u, z, H.e_partials.get(), grad_z);
  PA_LAUNCHED();
  if (value) {
    k_bsum_partials<<<1, 1024, 0, P.stream>>>(blocks, H.e_partials.get(), value);
    PA_LAUNCHED();
  }
}


// ----------------------------------------------- assembled K on the box --
// VectorFunction::gradient_u as the block-CRS matrix on a box mesh in its own
// numbering with the mesh's sorted columns: one thread per (neighbour slot,
// node) block, which sums the tets around that edge and writes its 3 x 3
// block once (no atomics, no zeroing).  In the six-tet split every tet is a
// monotone path 0 -> e_a -> e_a + e_b -> (1,1,1) through its hex, so the
// neighbours of node v are v +- e_S for the seven non-empty axis sets S, and
// in node-id order they are the fifteen slots of BoxEdges (px, py >= 2).
// A CTA takes 32 consecutive nodes, one node per lane, and its four warps
// split the fifteen slots into groups of equal tet counts (the node itself has
// 24 tets, every neighbour 4 or 6: 96 in all), so the loops over the hexes and
// tets of an edge are uniform in a warp, their table entries (kernel
// parameters) broadcast, and the warps reach the barrier before the rows'
// write-back together; the CTA writes its rows from shared memory as one
// contiguous range.
namespace {

struct BoxEdges {
  int8_t off[15][3];      // neighbour offset of each slot, in node-id order
  uint8_t count[15][8];   // tets of the edge in the hex at origin v - corner(o)
  uint8_t tet[15][8][6];  // t | m_v << 3 | m_w << 5
  int8_t grad[6][4][3];   // gradient of vertex m of tet t on a unit hex (-1, 0, 1 per axis)
  uint8_t group[4][6];    // slots of each warp of a CTA, 24 tets per warp
  uint8_t group_n[4];
};

BoxEdges make_box_edges() {
  static const int8_t kOff[15][3] = {{-1, -1, -1}, {0, -1, -1}, {-1, 0, -1}, {0, 0, -1}, {-1, -1, 0},
                                     {0, -1, 0},   {-1, 0, 0},  {0, 0, 0},   {1, 0, 0},  {0, 1, 0},
                                     {1, 1, 0},    {0, 0, 1},   {1, 0, 1},   {0, 1, 1},  {1, 1, 1}};
  BoxEdges E{};
  for (int t = 0; t < 6; ++t)
    for (int m = 0; m < 4; ++m) {
      for (int d = 0; d < 3; ++d) E.grad[t][m][d] = 0;
      if (m >= 1) E.grad[t][m][path_axis(t, m - 1)] += 1;
      if (m <= 2) E.grad[t][m][path_axis(t, m)] -= 1;
    }
  for (int sl = 0; sl < 15; ++sl) {
    for (int d = 0; d < 3; ++d) E.off[sl][d] = kOff[sl][d];
    for (int o = 0; o < 8; ++o) {  // v is corner o of the hex
      const int wi = (o & 1) + kOff[sl][0], wj = ((o >> 1) & 1) + kOff[sl][1], wk = (o >> 2) + kOff[sl][2];
      E.count[sl][o] = 0;
      if (wi < 0 || wi > 1 || wj < 0 || wj > 1 || wk < 0 || wk > 1) continue;
      const int qw = wi + 2 * wj + 4 * wk;
      for (int t = 0; t < 6; ++t) {
        int mv = -1, mw = -1;
        for (int m = 0; m < 4; ++m) {
          if (path_vertex(t, m) == o) mv = m;
          if (path_vertex(t, m) == qw) mw = m;
        }
        if (mv >= 0 && mw >= 0) E.tet[sl][o][E.count[sl][o]++] = uint8_t(t | (mv << 3) | (mw << 5));
      }
    }
  }
  // warp groups: the node itself (24 tets), four six-tet slots, four
  // six-tet slots, six four-tet slots
  static const int kGroup[4][6] = {{7}, {0, 3, 5, 6}, {8, 9, 11, 14}, {1, 2, 4, 10, 12, 13}};
  static const int kGroupN[4] = {1, 4, 4, 6};
  for (int g = 0; g < 4; ++g) {
    E.group_n[g] = uint8_t(kGroupN[g]);
    int tets = 0;
    for (int q = 0; q < kGroupN[g]; ++q) {
      E.group[g][q] = uint8_t(kGroup[g][q]);
      for (int o = 0; o < 8; ++o) tets += E.count[kGroup[g][q]][o];
    }
    PA_CHECK(tets == 24, "unbalanced slot groups");
  }
  return E;
}

constexpr int kGuNodes = 32;  // nodes per CTA of k_bgradient_u and k_bgradient_x (15 slots each)
constexpr int kGuWarps = 4;   // warps per CTA, one slot group each

__global__ void __launch_bounds__(32 * kGuWarps) k_bgradient_u(BoxDims d, double vol, double p, double pmin,
                                                             int layout, BoxEdges E, const double* __restrict__ k0,
                                                             const double* __restrict__ z,
                                                             const int32_t* __restrict__ rowmap,
                                                             double* __restrict__ vals) {
  // thread (group, node) = (warp, lane): a warp takes its group's slots of 32
  // consecutive nodes; the CTA's blocks are staged in shared memory and its
  // rows written as one contiguous range
  __shared__ double stage[15 * kGuNodes * 9];
  const int64_t v0 = int64_t(blockIdx.x) * kGuNodes;
  const int64_t v1 = v0 + kGuNodes < d.N ? v0 + kGuNodes : d.N;
  const int grp = int(threadIdx.x) / 32;
  const int64_t v = v0 + int(threadIdx.x) % 32;
  const int64_t base = rowmap[v0];
  if (v < v1) {
    const int vi = int(v % d.px), vj = int((v / d.px) % d.py), vk = int(v / (int64_t(d.px) * d.py));
    auto inside = [&](int i, int j, int k) {
      return i >= 0 && i <= d.nx && j >= 0 && j <= d.ny && k >= 0 && k <= d.nz;
    };
    for (int gq = 0; gq < E.group_n[grp]; ++gq) {
      const int sl = E.group[grp][gq];
      if (inside(vi + E.off[sl][0], vj + E.off[sl][1], vk + E.off[sl][2])) {
        // the block's position in the row: its slot for an interior node (every
        // neighbour exists), else the count of existing neighbours before it
        int rank = sl;
        if (vi == 0 || vj == 0 || vk == 0 || vi == d.nx || vj == d.ny || vk == d.nz) {
          rank = 0;
          for (int q = 0; q < sl; ++q) rank += inside(vi + E.off[q][0], vj + E.off[q][1], vk + E.off[q][2]) ? 1 : 0;
        }
        double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int o = 0; o < 8; ++o) {
          const int n = E.count[sl][o];
          if (n == 0) continue;
          const int oi = vi - (o & 1), oj = vj - ((o >> 1) & 1), ok = vk - (o >> 2);
          if (oi < 0 || oj < 0 || ok < 0 || oi >= d.nx || oj >= d.ny || ok >= d.nz) continue;
          const int64_t h = oi + int64_t(d.nx) * (oj + int64_t(d.ny) * ok);
          for (int e = 0; e < n; ++e) {
            const int t = E.tet[sl][o][e] & 7;
            double rho;
            if (layout == PA_CONTROL_CELL) {
              rho = z[6 * h + t];
            } else {
              rho = 0.0;
              for (int m = 0; m < 4; ++m) {
                const int c = path_vertex(t, m);
                rho += 0.25 * z[(oi + (c & 1)) +
                                int64_t(d.px) * ((oj + ((c >> 1) & 1)) + int64_t(d.py) * (ok + (c >> 2)))];
              }
            }
            const double w = vol * simp(rho, p, pmin);
            const double* kb = k0 + 9 * ((sl * 8 + o) * 6 + e);
#pragma unroll
            for (int q = 0; q < 9; ++q) K[q] = fma(w, __ldg(kb + q), K[q]);
          }
        }
        double* dst = stage + 9 * (int64_t(rowmap[v]) - base + rank);
#pragma unroll
        for (int q = 0; q < 9; ++q) dst[q] = K[q];
      }
    }
  }
  __syncthreads();
  const int64_t count = 9 * (int64_t(rowmap[v1]) - base);
  for (int64_t e = threadIdx.x; e < count; e += blockDim.x) vals[9 * base + e] = stage[e];
}

// barycentric gradients of the six path tets' vertices on the box's hexes
// (the BoxEdges unit-hex pattern scaled by 1 / h per axis)
struct TetGrads {
  double g[6][4][3];
};

// VectorFunction::gradient_x on a box mesh in its own numbering with sorted
// columns, by the same (slot group, node) threads as k_bgradient_u: the block at row
// v, column w holds d R_w / d x_v ([k][j] = d R_w,j / d x_v,k), summed over the
// tets of the edge.  For a linear tet with barycentric gradients g, volume V,
// displacement gradient H = sum_m u_m g_m^T and stress S = w sigma(sym H), the
// nodal force is R_a = V S g_a, and moving vertex b along e_k gives
// dV = V g_b,k, dg_a = -g_a,k g_b, dH = -H e_k g_b^T (= D), dS = w sigma(sym D):
//   d R_a / d x_b,k = V (g_b,k S g_a + dS g_a - g_a,k S g_b),
// with tr D = -(H^T g_b)_k and dS g_a = w (lam tr D g_a - mu (g_b . g_a) H e_k
// - mu (H^T g_a)_k g_b).  u is read at the tet's four lattice corners.
__global__ void __launch_bounds__(32 * kGuWarps) k_bgradient_x(BoxDims d, double vol, double p, double pmin,
                                                             int layout, BoxEdges E, Iso<double> iso, TetGrads G,
                                                             const double* __restrict__ u,
                                                             const double* __restrict__ z,
                                                             const int32_t* __restrict__ rowmap,
                                                             double* __restrict__ vals) {
  __shared__ double stage[15 * kGuNodes * 9];
  const int64_t v0 = int64_t(blockIdx.x) * kGuNodes;
  const int64_t v1 = v0 + kGuNodes < d.N ? v0 + kGuNodes : d.N;
  const int grp = int(threadIdx.x) / 32;
  const int64_t v = v0 + int(threadIdx.x) % 32;
  const int64_t base = rowmap[v0];
  if (v < v1) {
    const int vi = int(v % d.px), vj = int((v / d.px) % d.py), vk = int(v / (int64_t(d.px) * d.py));
    auto inside = [&](int i, int j, int k) {
      return i >= 0 && i <= d.nx && j >= 0 && j <= d.ny && k >= 0 && k <= d.nz;
    };
    for (int gq = 0; gq < E.group_n[grp]; ++gq) {
      const int sl = E.group[grp][gq];
      if (inside(vi + E.off[sl][0], vj + E.off[sl][1], vk + E.off[sl][2])) {
        int rank = sl;
        if (vi == 0 || vj == 0 || vk == 0 || vi == d.nx || vj == d.ny || vk == d.nz) {
          rank = 0;
          for (int q = 0; q < sl; ++q) rank += inside(vi + E.off[q][0], vj + E.off[q][1], vk + E.off[q][2]) ? 1 : 0;
        }
        double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int o = 0; o < 8; ++o) {
          const int n = E.count[sl][o];
          if (n == 0) continue;
          const int oi = vi - (o & 1), oj = vj - ((o >> 1) & 1), ok = vk - (o >> 2);
          if (oi < 0 || oj < 0 || ok < 0 || oi >= d.nx || oj >= d.ny || ok >= d.nz) continue;
          const int64_t h = oi + int64_t(d.nx) * (oj + int64_t(d.ny) * ok);
          for (int e = 0; e < n; ++e) {
            const int code = E.tet[sl][o][e], t = code & 7, mv = (code >> 3) & 3, mw = code >> 5;
            double rho;
            if (layout == PA_CONTROL_CELL) {
              rho = z[6 * h + t];
            } else {
              rho = 0.0;
              for (int m = 0; m < 4; ++m) {
                const int c = path_vertex(t, m);
                rho += 0.25 * z[(oi + (c & 1)) +
                                int64_t(d.px) * ((oj + ((c >> 1) & 1)) + int64_t(d.py) * (ok + (c >> 2)))];
              }
            }
            const double w = simp(rho, p, pmin);
            // H = sum_m u_m g_m^T over the tet's path vertices
            double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int m = 0; m < 4; ++m) {
              const int c = path_vertex(t, m);
              const int64_t node = (oi + (c & 1)) + int64_t(d.px) * ((oj + ((c >> 1) & 1)) + int64_t(d.py) * (ok + (c >> 2)));
              double gm[3];
#pragma unroll
              for (int a = 0; a < 3; ++a) gm[a] = G.g[t][m][a];
#pragma unroll
              for (int i = 0; i < 3; ++i) {
                const double ui = u[3 * node + i];
#pragma unroll
                for (int a = 0; a < 3; ++a) H[i][a] = fma(ui, gm[a], H[i][a]);
              }
            }
            const double tr = H[0][0] + H[1][1] + H[2][2];
            double S[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
              for (int j = 0; j < 3; ++j)
                S[i][j] = w * ((i == j ? iso.lam * tr : 0.0) + iso.mu * (H[i][j] + H[j][i]));
            double gv[3], gw[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              gv[a] = G.g[t][mv][a];
              gw[a] = G.g[t][mw][a];
            }
            double Sgw[3], Sgv[3], Htv[3], Htw[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
              Sgw[i] = S[i][0] * gw[0] + S[i][1] * gw[1] + S[i][2] * gw[2];
              Sgv[i] = S[i][0] * gv[0] + S[i][1] * gv[1] + S[i][2] * gv[2];
              Htv[i] = H[0][i] * gv[0] + H[1][i] * gv[1] + H[2][i] * gv[2];
              Htw[i] = H[0][i] * gw[0] + H[1][i] * gw[1] + H[2][i] * gw[2];
            }
            const double gvgw = gv[0] * gw[0] + gv[1] * gw[1] + gv[2] * gw[2];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              const double trD = -Htv[k];
#pragma unroll
              for (int j = 0; j < 3; ++j) {
                const double dSgw = w * (iso.lam * trD * gw[j] - iso.mu * (H[j][k] * gvgw + gv[j] * Htw[k]));
                K[3 * k + j] += vol * (gv[k] * Sgw[j] + dSgw - gw[k] * Sgv[j]);
              }
            }
          }
        }
        double* dst = stage + 9 * (int64_t(rowmap[v]) - base + rank);
#pragma unroll
        for (int q = 0; q < 9; ++q) dst[q] = K[q];
      }
    }
  }
  __syncthreads();
  const int64_t count = 9 * (int64_t(rowmap[v1]) - base);
  for (int64_t e = threadIdx.x; e < count; e += blockDim.x) vals[9 * base + e] = stage[e];
}

}  // namespace

bool box_gradient_u(Problem& P, const double* z, double* entries) {
  const Mesh& m = *P.mesh;
  if (!(m.box_kernels && m.lat_n[0] > 0 && !m.lat_permuted && m.lat_flip == 0 && m.cols_sorted && m.d_rowmap.n))
    return false;
  static const BoxEdges edges = make_box_edges();
  boxmg_ensure(P);
  BoxHierarchy& H = *P.boxmg;
  const BoxLevel& F = *H.L[0];
  // the unpenalized 3 x 3 block of every (slot, hex corner, tet) entry: on a
  // uniform box it depends only on the hex sides and the Lame constants
  const Iso<double> iso = P.ep.iso();
  const double key[5] = {F.h[0], F.h[1], F.h[2], iso.lam, iso.mu};
  if (!H.gu_k0.n || !std::equal(key, key + 5, H.gu_key)) {
    std::vector<double> k0(size_t(15 * 8 * 6 * 9), 0.0);
    const double ih[3] = {1.0 / F.h[0], 1.0 / F.h[1], 1.0 / F.h[2]};
    for (int sl = 0; sl < 15; ++sl)
      for (int o = 0; o < 8; ++o)
        for (int e = 0; e < edges.count[sl][o]; ++e) {
          const int code = edges.tet[sl][o][e], t = code & 7, mv = (code >> 3) & 3, mw = code >> 5;
          double ga[3], gb[3];
          for (int c = 0; c < 3; ++c) {
            ga[c] = ih[c] * edges.grad[t][mv][c];
            gb[c] = ih[c] * edges.grad[t][mw][c];
          }
          const double dd = iso.mu * (ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]);
          double* kb = &k0[size_t(9 * ((sl * 8 + o) * 6 + e))];
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) kb[3 * i + j] = iso.lam * ga[i] * gb[j] + iso.mu * ga[j] * gb[i] + (i == j ? dd : 0.0);
        }
    H.gu_k0.upload(k0.data(), k0.size(), P.stream);
    std::copy(key, key + 5, H.gu_key);
  }
  k_bgradient_u<<<int((F.d.N + kGuNodes - 1) / kGuNodes), 32 * kGuWarps, 0, P.stream>>>(
      F.d, F.h[0] * F.h[1] * F.h[2] / 6.0, P.ep.p, P.ep.pmin, P.ep.layout, edges, H.gu_k0.get(), z,
      m.d_rowmap.get(), entries);
  PA_LAUNCHED();
  return true;
}

// VectorFunction::gradient_x on a box mesh (the volume term; the caller adds
// the surface loads): false (nothing launched) on any other mesh.
bool box_gradient_x(Problem& P, const double* u, const double* z, double* entries) {
  const Mesh& m = *P.mesh;
  if (!(m.box_kernels && m.lat_n[0] > 0 && !m.lat_permuted && m.lat_flip == 0 && m.cols_sorted && m.d_rowmap.n))
    return false;
  static const BoxEdges edges = make_box_edges();
  boxmg_ensure(P);
  const BoxLevel& F = *P.boxmg->L[0];
  TetGrads G;
  for (int t = 0; t < 6; ++t)
    for (int mm = 0; mm < 4; ++mm)
      for (int a = 0; a < 3; ++a) G.g[t][mm][a] = edges.grad[t][mm][a] / F.h[a];
  k_bgradient_x<<<int((F.d.N + kGuNodes - 1) / kGuNodes), 32 * kGuWarps, 0, P.stream>>>(
      F.d, F.h[0] * F.h[1] * F.h[2] / 6.0, P.ep.p, P.ep.pmin, P.ep.layout, edges, P.ep.iso(), G, u, z,
      m.d_rowmap.get(), entries);
  PA_LAUNCHED();
  return true;
}

}  // namespace pa
