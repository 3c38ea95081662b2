// pa_dense.cuh -- dense FP64 inverse of a small symmetric positive definite
// matrix on the GPU (the coarsest multigrid level): blocked Gauss-Jordan
// elimination in place, without pivoting, in 64-wide blocks, and the
// matrix-vector product with the inverse.  Each TU that includes this gets
// its own copy of the kernels (anonymous namespace).
#pragma once

#include <cstdint>

#include "pa_internal.cuh"

namespace pa {
namespace {

constexpr int kGJ = 64, kGJc = 32;

// In-place Gauss-Jordan of the pivot block A[K,K] -> P^-1 (one CTA of 256
// threads).  Thread t keeps the 4 x 4 sub-block (rows 4 (t / 16) + i, columns
// 4 (t % 16) + j) in registers; for each pivot p the owners of row p and
// column p publish them in shared memory (double-buffered, one barrier per
// pivot) and every thread updates its sub-block.  A pivot that is not above
// 1e-12 of its row's original diagonal marks the matrix as (numerically)
// singular in *flag, checked once after the loop.
__global__ void __launch_bounds__(256) k_gj_pivot(int64_t nd, int64_t k0, const double* __restrict__ A,
                                                  const double* __restrict__ diag0, double* __restrict__ piv,
                                                  double* __restrict__ flag) {
  __shared__ double rowb[2][kGJ], colb[2][kGJ], pivots[kGJ];
  const int a = threadIdx.x >> 4, b = threadIdx.x & 15;
  double R[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) R[i][j] = A[(k0 + 4 * a + i) * nd + k0 + 4 * b + j];
  for (int p = 0; p < kGJ; ++p) {
    const int q = p & 1, pr = p >> 2, pc = p & 3;
    if (b == pr) {  // this thread holds column p for its four rows
#pragma unroll
      for (int i = 0; i < 4; ++i) colb[q][4 * a + i] = pc == 0 ? R[i][0] : pc == 1 ? R[i][1] : pc == 2 ? R[i][2] : R[i][3];
    }
    if (a == pr) {  // and row p for its four columns
#pragma unroll
      for (int j = 0; j < 4; ++j) rowb[q][4 * b + j] = pc == 0 ? R[0][j] : pc == 1 ? R[1][j] : pc == 2 ? R[2][j] : R[3][j];
    }
    __syncthreads();
    const double pv = rowb[q][p];
    if (threadIdx.x == 0) pivots[p] = pv;
    const double ip = 1.0 / pv;
    double cr[4], rc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      cr[i] = colb[q][4 * a + i] * ip;
      rc[i] = rowb[q][4 * b + i];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const bool rp = 4 * a + i == p, cp = 4 * b + j == p;
        const double gen = R[i][j] - cr[i] * rc[j];
        R[i][j] = rp ? (cp ? ip : rc[j] * ip) : (cp ? -cr[i] : gen);
      }
  }
  __syncthreads();
  if (threadIdx.x < kGJ && !(pivots[threadIdx.x] > 1e-12 * diag0[k0 + threadIdx.x])) *flag = 1.0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) piv[(4 * a + i) * kGJ + 4 * b + j] = R[i][j];
}

// acc (this thread's 4x4 outputs of a 64x64 tile) += L[64 x 64] R[64 x 64];
// thread t owns rows t/16 + 16p and columns t%16 + 16q.
__device__ __forceinline__ void gj_tile_mma(const double* __restrict__ L, int64_t ldl, const double* __restrict__ R,
                                            int64_t ldr, double acc[4][4]) {
  __shared__ double Ls[kGJ][kGJc + 1];
  __shared__ double Rs[kGJc][kGJ];
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
  for (int k0 = 0; k0 < kGJ; k0 += kGJc) {
    for (int e = threadIdx.x; e < kGJ * kGJc; e += blockDim.x) {
      Ls[e / kGJc][e % kGJc] = L[(e / kGJc) * ldl + k0 + e % kGJc];
      Rs[e / kGJ][e % kGJ] = R[(k0 + e / kGJ) * ldr + e % kGJ];
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kGJc; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = Ls[tr + 16 * q][k];
        b[q] = Rs[k][tc + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
    }
    __syncthreads();
  }
}

// Row panel W = P^-1 A[K, :] and a copy of the column panel Cp = A[:, K]
// (both read before k_gj_update overwrites them); block j covers columns /
// rows j*64 .. j*64+63.
__global__ void __launch_bounds__(256) k_gj_panels(int64_t nd, int64_t k0, const double* __restrict__ A,
                                                   const double* __restrict__ piv, double* __restrict__ W,
                                                   double* __restrict__ Cp) {
  const int64_t j0 = int64_t(blockIdx.x) * kGJ;
  double acc[4][4] = {};
  gj_tile_mma(piv, kGJ, A + k0 * nd + j0, nd, acc);
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) W[(tr + 16 * p) * nd + j0 + tc + 16 * q] = acc[p][q];
  for (int e = threadIdx.x; e < kGJ * kGJ; e += blockDim.x)
    Cp[(j0 + e / kGJ) * kGJ + e % kGJ] = A[(j0 + e / kGJ) * nd + k0 + e % kGJ];
}

// One Gauss-Jordan block step on tile (I, J):
//   I = K, J = K: P^-1;  I = K: W;  J = K: -Cp P^-1;  else A - Cp W.
__global__ void __launch_bounds__(256) k_gj_update(int64_t nd, int64_t k0, double* __restrict__ A,
                                                   const double* __restrict__ piv, const double* __restrict__ W,
                                                   const double* __restrict__ Cp) {
  const int64_t j0 = int64_t(blockIdx.x) * kGJ, i0 = int64_t(blockIdx.y) * kGJ;
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
  const bool ik = i0 == k0, jk = j0 == k0;
  if (ik) {  // block-uniform
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = tr + 16 * p, c = tc + 16 * q;
        A[(i0 + r) * nd + j0 + c] = jk ? piv[r * kGJ + c] : W[r * nd + j0 + c];
      }
    return;
  }
  double acc[4][4] = {};
  gj_tile_mma(Cp + i0 * kGJ, kGJ, jk ? piv : W + j0, jk ? kGJ : nd, acc);
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double* a = &A[(i0 + tr + 16 * p) * nd + j0 + tc + 16 * q];
      *a = jk ? -acc[p][q] : *a - acc[p][q];
    }
}

// x = A^-1 b on the coarsest level: one warp per row, FP64 sums
__global__ void k_mg_dense_solve(int64_t n3, int64_t nd, const double* __restrict__ Ainv, const float* __restrict__ b,
                                 float* __restrict__ x) {
  const int64_t r = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n3) return;
  double s = 0.0;
  for (int64_t c = lane; c < n3; c += 32) s = fma(Ainv[r * nd + c], double(b[c]), s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[r] = float(s);
}


// Invert the nd x nd matrix A in place (nd a multiple of 64); w (64 x nd),
// cp (nd x 64), piv (64 x 64) are scratch; *flag (zeroed by the caller) is
// set when a pivot is not above 1e-12 of its original diagonal (diag0).
inline void gj_invert(cudaStream_t s, int64_t nd, double* A, const double* diag0, double* w, double* cp, double* piv,
                      double* flag) {
  for (int64_t k0 = 0; k0 < nd; k0 += kGJ) {
    k_gj_pivot<<<1, 256, 0, s>>>(nd, k0, A, diag0, piv, flag);
    k_gj_panels<<<int(nd / kGJ), 256, 0, s>>>(nd, k0, A, piv, w, cp);
    k_gj_update<<<dim3(unsigned(nd / kGJ), unsigned(nd / kGJ)), 256, 0, s>>>(nd, k0, A, piv, w, cp);
    PA_LAUNCHED();
  }
}

}  // namespace
}  // namespace pa
