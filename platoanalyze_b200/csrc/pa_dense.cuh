// pa_dense.cuh -- dense FP64 inverse of a small symmetric positive definite
// matrix on the GPU (the coarsest multigrid level): blocked Gauss-Jordan
// elimination in place, without pivoting, in 64-wide blocks, and the
// matrix-vector product with the inverse.  Each TU that includes this gets
// its own copy of the kernels (anonymous namespace).
#pragma once

#include <algorithm>
#include <cstdint>

#include "pa_internal.cuh"

namespace pa {
namespace {

constexpr int kGJ = 64, kGJc = 32;
// polls of a grid barrier before it gives up (about a quarter of a second)
constexpr int kGJSpin = 1 << 22;

// Marks the factorization as failed: 1 = a pivot not above 1e-12 of its
// original diagonal (numerically singular), 2 = a grid barrier timed out.
// Non-negative doubles order like their bit patterns, so the larger code wins.
__device__ __forceinline__ void gj_fail(double* flag, double code) {
  atomicMax(reinterpret_cast<unsigned long long*>(flag), static_cast<unsigned long long>(__double_as_longlong(code)));
}

// In-place Gauss-Jordan of the 64 x 64 pivot tile at T (leading dimension
// ldt) -> piv = T^-1 (row-major 64 x 64), by the 256 threads of one CTA.
// Thread t keeps the 4 x 4 sub-block (rows 4 (t / 16) + i, columns
// 4 (t % 16) + j) in registers; for each pivot p the owners of row p and
// column p publish them in shared memory (double-buffered, one barrier per
// pivot) and every thread updates its sub-block.  Pivots are checked against
// the original diagonal (diag0) once after the loop.  Loads bypass L1: other
// CTAs wrote T since this CTA last read it.
__device__ void gj_pivot_tile(const double* T, int64_t ldt, const double* __restrict__ diag0, double* __restrict__ piv,
                              double* flag) {
  __shared__ double rowb[2][kGJ], colb[2][kGJ], pivots[kGJ];
  const int a = threadIdx.x >> 4, b = threadIdx.x & 15;
  double R[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) R[i][j] = __ldcg(&T[(4 * a + i) * ldt + 4 * b + j]);
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
  if (threadIdx.x < kGJ && !(pivots[threadIdx.x] > 1e-12 * diag0[threadIdx.x])) gj_fail(flag, 1.0);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) piv[(4 * a + i) * kGJ + 4 * b + j] = R[i][j];
}

// acc (this thread's 4x4 outputs of a 64x64 tile) = L[64 x 64] R[64 x 64];
// thread t owns rows t/16 + 16p and columns t%16 + 16q.  Every global read
// of L and R is complete when it returns.
__device__ __forceinline__ void gj_tile_mma(const double* L, int64_t ldl, const double* R, int64_t ldr,
                                            double acc[4][4]) {
  __shared__ double Ls[kGJ][kGJc + 1];
  __shared__ double Rs[kGJc][kGJ];
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = 0.0;
  for (int k0 = 0; k0 < kGJ; k0 += kGJc) {
    for (int e = threadIdx.x; e < kGJ * kGJc; e += blockDim.x) {
      Ls[e / kGJc][e % kGJc] = __ldcg(&L[(e / kGJc) * ldl + k0 + e % kGJc]);
      Rs[e / kGJ][e % kGJ] = __ldcg(&R[(k0 + e / kGJ) * ldr + e % kGJ]);
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

__device__ __forceinline__ unsigned gj_ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Barrier over all CTAs of the cooperative launch: the n-th barrier waits for
// n x gridDim.x arrivals on *count.  The wait is bounded: after kGJSpin polls
// the CTA marks the factorization failed (code 2) and goes on; the caller
// returns when the flag is set.  False when the factorization has failed.
__device__ __forceinline__ bool gj_grid_sync(unsigned* count, unsigned target, double* flag) {
  __shared__ int failed;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(count, 1u);
    int it = 0;
    while (gj_ld_acquire(count) < target) {
      if (++it > kGJSpin) {
        gj_fail(flag, 2.0);
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    failed = *reinterpret_cast<volatile double*>(flag) >= 2.0;
  }
  __syncthreads();
  return !failed;
}

// The whole blocked Gauss-Jordan inverse of the nd x nd matrix A (nd = 64 nb,
// row-major, symmetric positive definite, no pivoting) in one cooperative
// launch.  Block step k with the pivot inverse Pk = A_kk^-1 (in piv[k & 1]):
//   phase 1: A_kj <- Pk A_kj (j != k), A_kk <- Pk, Cp_i <- A_ik (i != k);
//   phase 2: A_ij <- A_ij - Cp_i A_kj (i, j != k), A_ik <- -Cp_i Pk.
// A grid barrier separates the phases.  CTA 0 updates tile (k+1, k+1) first
// in phase 2 and inverts it into piv[(k+1) & 1] while the other CTAs update
// the rest, so the pivot inversion is off the critical path.  Every tile is
// read and written by one CTA per phase; the column panel is read from its
// copy Cp, so no tile is read by one CTA while another writes it.
__global__ void __launch_bounds__(256) k_gj_invert(int nd, double* A, const double* __restrict__ diag0,
                                                   double* __restrict__ piv, double* __restrict__ Cp,
                                                   unsigned* count, double* flag) {
  const int nb = nd / kGJ, G = int(gridDim.x), cta = int(blockIdx.x);
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
  unsigned barriers = 0;
  if (cta == 0) gj_pivot_tile(A, nd, diag0, piv, flag);
  if (!gj_grid_sync(count, ++barriers * unsigned(G), flag)) return;
  for (int k = 0; k < nb; ++k) {
    const int64_t k0 = int64_t(k) * kGJ;
    const double* Pk = piv + (k & 1) * kGJ * kGJ;
    // phase 1: the row panel (tasks 0 .. nb-1) and the column-panel copy (nb .. 2nb-1)
    for (int t = cta; t < 2 * nb; t += G) {
      double acc[4][4];
      if (t < nb) {
        const int64_t j0 = int64_t(t) * kGJ;
        if (t == k) {
          for (int e = threadIdx.x; e < kGJ * kGJ; e += blockDim.x)
            A[(k0 + e / kGJ) * nd + k0 + e % kGJ] = __ldcg(&Pk[e]);
          continue;
        }
        gj_tile_mma(Pk, kGJ, A + k0 * nd + j0, nd, acc);
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) A[(k0 + tr + 16 * p) * nd + j0 + tc + 16 * q] = acc[p][q];
      } else if (t - nb != k) {
        const int64_t i0 = int64_t(t - nb) * kGJ;
        for (int e = threadIdx.x; e < kGJ * kGJ; e += blockDim.x)
          Cp[(i0 + e / kGJ) * kGJ + e % kGJ] = __ldcg(&A[(i0 + e / kGJ) * nd + k0 + e % kGJ]);
      }
    }
    if (!gj_grid_sync(count, ++barriers * unsigned(G), flag)) return;
    // phase 2: tiles (i, j), i != k, enumerated row by row over the other rows
    const bool look = k + 1 < nb;
    auto update = [&](int i, int j) {
      const int64_t i0 = int64_t(i) * kGJ, j0 = int64_t(j) * kGJ;
      double acc[4][4];
      const bool jk = j == k;
      gj_tile_mma(Cp + i0 * kGJ, kGJ, jk ? Pk : A + k0 * nd + j0, jk ? kGJ : nd, acc);
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          double* a = &A[(i0 + tr + 16 * p) * nd + j0 + tc + 16 * q];
          *a = jk ? -acc[p][q] : __ldcg(a) - acc[p][q];
        }
    };
    if (cta == 0 && look) {
      update(k + 1, k + 1);
      __syncthreads();
      gj_pivot_tile(A + (k0 + kGJ) * nd + k0 + kGJ, nd, diag0 + k0 + kGJ, piv + ((k + 1) & 1) * kGJ * kGJ, flag);
    }
    if (cta > 0 || G == 1) {
      const int workers = G > 1 ? G - 1 : 1, me = G > 1 ? cta - 1 : 0;
      for (int t = me; t < (nb - 1) * nb; t += workers) {
        const int ir = t / nb, j = t % nb, i = ir < k ? ir : ir + 1;
        if (look && i == k + 1 && j == k + 1) continue;  // done by CTA 0
        update(i, j);
      }
    }
    if (k + 1 < nb && !gj_grid_sync(count, ++barriers * unsigned(G), flag)) return;
  }
}

// x = A^-1 b on the coarsest level: one warp per row, FP64 sums
// skip (may be null): two flags; the launch is a no-op when either is set.
__global__ void k_mg_dense_solve(int64_t n3, int64_t nd, const double* __restrict__ Ainv, const float* __restrict__ b,
                                 float* __restrict__ x, const double* skip = nullptr) {
  if (skip && (skip[0] != 0.0 || skip[1] != 0.0)) return;
  const int64_t r = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n3) return;
  double s = 0.0;
  for (int64_t c = lane; c < n3; c += 32) s = fma(Ainv[r * nd + c], double(b[c]), s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[r] = float(s);
}


// Invert the nd x nd matrix A in place (nd a multiple of 64) with one
// cooperative launch of k_gj_invert over every co-resident CTA.  cp (nd x 64),
// piv (2 x 64 x 64) and sync (one unsigned, the barrier count) are scratch;
// *flag (zeroed by the caller) becomes 1 when a pivot is not above 1e-12 of
// its original diagonal (diag0) and 2 when a grid barrier timed out.
inline void gj_invert(cudaStream_t s, int64_t nd, double* A, const double* diag0, double* cp, double* piv,
                      unsigned* sync, double* flag) {
  static int grid = 0;  // co-resident CTAs of k_gj_invert on this device
  if (grid == 0) {
    int dev = 0, sms = 0, occ = 0, coop = 0;
    PA_CUDA(cudaGetDevice(&dev));
    PA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PA_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    PA_CHECK(coop != 0, "the device does not support cooperative launches");
    PA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gj_invert, 256, 0));
    PA_CHECK(occ > 0, "k_gj_invert does not fit on a multiprocessor");
    grid = sms * std::min(occ, 2);
  }
  // no more CTAs than the largest phase has tiles (fewer CTAs also make the
  // grid barriers cheaper): phase 2 updates (nb - 1) nb tiles, one CTA more
  // inverts the next pivot tile
  const int nb = int(nd / kGJ);
  const int g = std::max(1, std::min(grid, std::max(2 * nb, (nb - 1) * nb + 1)));
  PA_CUDA(cudaMemsetAsync(sync, 0, sizeof(unsigned), s));
  int ndi = int(nd);
  void* args[] = {&ndi, &A, &diag0, &piv, &cp, &sync, &flag};
  PA_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_gj_invert), dim3(unsigned(g)), dim3(256),
                                      args, 0, s));
}

}  // namespace
}  // namespace pa
