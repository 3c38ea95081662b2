// pa_learned.cu -- learned preconditioner: a four-layer 3x3x3 convolutional
// network on the nodal grid of a structured box, run on the sm_100a tensor
// cores (forward) and trained by the library's own FP32 backward kernels.
//
// Preconditioner (for the Dirichlet-constrained operator K, Jacobi diagonal D):
//   M r = D^-1 r + s D^-1/2 f(x),  x = (D^-1/2 r / s, stiffness, Dirichlet),
//   s = sqrt(r.D^-1 r / n_free),
// with f the network (5 -> 32 -> 32 -> 32 -> 3 channels, ReLU after layers 1-3,
// zero padding at the grid boundary).  The last layer starts at zero, so a new
// network is exactly Jacobi.  Training minimises, per residual/error pair
// (r, e) with K e = r, the relative energy-norm error of one correction:
//   L = ||e - M r||_K^2 / ||e||_K^2 = (z.Kz - 2 z.r) / (e.r) + 1,  z = M r,
// whose gradient in z is 2 (K z - r) / (e.r); K z is the matrix-free apply.
//
// Data layout: activations are channel-last BF16, act[v * C + c], v the node
// index i + gx (j + gy k) (the box mesh's numbering).  Convolution weights in
// the tensor-core layout [tap][Cin/8][Cout][8] BF16 (K-major 8x16-byte core
// matrices); tap t = dx + 3 dy + 9 dz for offset (dx-1, dy-1, dz-1).
//
// Forward kernel (k_conv3_tc): persistent CTAs of 128 threads; a tile is
// 8 x 16 x 2 output nodes = two layers of the M = 128 rows of a tcgen05.mma.
// The CTA keeps all 27 taps of the weights in shared memory, stages the tile's
// 10 x 18 x 4 input halo channel-group-major ([Cin/8][720 nodes][8]) so that
// every tap's A operand is the same halo viewed at a shifted start address
// (rows 16 B apart, row groups 160 B apart, layers 2880 B apart), and one
// thread issues 2 x 27 x Cin/16 MMAs of 128 x Cout x 16 into two TMEM
// accumulators that share each B operand.  The epilogue (tcgen05.ld, bias,
// ReLU, BF16) writes 64 contiguous bytes per node.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "pa_learned.cuh"
#include "pa_tc.cuh"
#include "pa_tiled.cuh"

namespace pa {

namespace {

constexpr int kCin[kPcLayers] = {5, 32, 32, 32};
constexpr int kCout[kPcLayers] = {32, 32, 32, 3};
constexpr int kCinP[kPcLayers] = {16, 32, 32, 32};
constexpr int kCoutP[kPcLayers] = {32, 32, 32, 16};
constexpr int kFeatures = 5;

int64_t w_offset(int l) {
  int64_t o = 0;
  for (int k = 0; k < l; ++k) o += int64_t(kCout[k]) * kCin[k] * 27 + kCout[k];
  return o;
}
int64_t b_offset(int l) { return w_offset(l) + int64_t(kCout[l]) * kCin[l] * 27; }

constexpr int kTX = 8, kTY = 16, kTZ = 2;
constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = kTZ + 2;
constexpr int kHalo = kHX * kHY * kHZ;  // 720
constexpr int kConvThreads = 128;
constexpr int kTmemCols = 64;  // two 128 x Cout accumulators (Cout <= 32)

__device__ __forceinline__ void cp16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tc::smem_u32(smem)), "l"(gmem) : "memory");
}

struct ConvArgs {
  const __nv_bfloat16* in;  // [G][CIN]
  const __nv_bfloat16* w;   // [27][CIN/8][COUT][8]
  const float* bias;        // [COUT]
  __nv_bfloat16* out_bf;    // [G][COUT] or null
  float* out_f32;           // [G][4] (channels 0..3) or null
  const int32_t* done;      // skip the launch when *done != 0 (null: never)
  int* err;                 // set to 1 if a tensor-core wait ran out
  int gx, gy, gz;
};

template <int CIN, int COUT>
struct ConvSmem {
  __nv_bfloat16 w[27 * CIN * COUT];  // B operands of all taps
  __nv_bfloat16 halo[CIN * kHalo];   // A operand source, [CIN/8][kHalo][8]
  float bias[COUT];
  uint64_t mbar;
  uint32_t tmem_base;
  int32_t pad;
};

template <int CIN, int COUT, bool RELU>
__global__ void __launch_bounds__(kConvThreads) k_conv3_tc(ConvArgs a) {
  static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "tile shapes");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  ConvSmem<CIN, COUT>& S = *reinterpret_cast<ConvSmem<CIN, COUT>*>(smem_raw);
  if (a.done && *a.done) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntx = (a.gx + kTX - 1) / kTX, nty = (a.gy + kTY - 1) / kTY, ntz = (a.gz + kTZ - 1) / kTZ;
  const int ntiles = ntx * nty * ntz;

  constexpr int kWChunks = 27 * CIN * COUT / 8;
  for (int i = tid; i < kWChunks; i += kConvThreads) cp16(&S.w[8 * i], a.w + 8 * i);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  if (tid < COUT) S.bias[tid] = a.bias[tid];
  if (tid == 0) tc::mbar_init(&S.mbar, 1);
  if (warp == 0) tc::tmem_alloc(&S.tmem_base, kTmemCols);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  tc::fence_proxy_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = S.tmem_base;
  const uint32_t hb = tc::smem_u32(S.halo), wb = tc::smem_u32(S.w);
  constexpr uint32_t idesc = tc::instr_desc_bf16(128, COUT);
  uint32_t phase = 0;
  bool ok = true;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    const int x0 = tx * kTX, y0 = ty * kTY, z0 = tz * kTZ;
    // halo: node (x0 + hx - 1, y0 + hy - 1, z0 + hz - 1), zero outside the grid;
    // the channel group runs fastest so that consecutive threads read one
    // node's contiguous channels
    for (int i = tid; i < (CIN / 8) * kHalo; i += kConvThreads) {
      const int cg = i % (CIN / 8), hv = i / (CIN / 8);
      const int hx = hv % kHX, hy = (hv / kHX) % kHY, hz = hv / (kHX * kHY);
      const int x = x0 + hx - 1, y = y0 + hy - 1, z = z0 + hz - 1;
      __nv_bfloat16* dst = &S.halo[(cg * kHalo + hv) * 8];
      if (x >= 0 && x < a.gx && y >= 0 && y < a.gy && z >= 0 && z < a.gz) {
        const int64_t v = x + int64_t(a.gx) * (y + int64_t(a.gy) * z);
        cp16(dst, a.in + v * CIN + cg * 8);
      } else {
        *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll 1
      for (int t = 0; t < 27; ++t) {
        const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
        const uint32_t aoff = uint32_t(((dz * kHY + dy) * kHX + dx) * 16);
#pragma unroll
        for (int j = 0; j < CIN / 16; ++j) {
          const uint32_t a0 = hb + uint32_t(2 * j * kHalo * 16) + aoff;
          const uint64_t bd = tc::smem_desc(wb + uint32_t((t * (CIN / 8) + 2 * j) * COUT * 16), COUT * 16, 128);
          const uint32_t acc = (t | j) != 0 ? 1u : 0u;
          // output layer z0 into columns [0, COUT), layer z0 + 1 into [COUT, 2 COUT)
          tc::mma_bf16(tmem, tc::smem_desc(a0, kHalo * 16, kHX * 16), bd, idesc, acc);
          tc::mma_bf16(tmem + COUT, tc::smem_desc(a0 + kHY * kHX * 16, kHalo * 16, kHX * 16), bd, idesc, acc);
        }
      }
      tc::commit(&S.mbar);
    }
    // the issuing thread waits for the accumulator; the others wait at the barrier
    const bool got = tid == 0 ? tc::mbar_wait(&S.mbar, phase) : true;
    phase ^= 1u;
    if (__syncthreads_or(got ? 0 : 1)) {
      ok = false;
      break;
    }
    tc::fence_after_sync();
    // epilogue: row m = 32 warp + lane of accumulator h is node (x0 + m % 8, y0 + m / 8, z0 + h)
    const int m = warp * 32 + lane;
    const int x = x0 + (m & 7), y = y0 + (m >> 3);
#pragma unroll
    for (int h = 0; h < kTZ; ++h) {
      const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(h * COUT);
      float vals[COUT];
      if constexpr (COUT == 32) {
        uint32_t r[32];
        tc::tmem_ld32(taddr, r);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 32; ++c) vals[c] = __uint_as_float(r[c]);
      } else {
        uint32_t r[16];
        tc::tmem_ld16(taddr, r);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 16; ++c) vals[c] = __uint_as_float(r[c]);
      }
      const int z = z0 + h;
      if (x < a.gx && y < a.gy && z < a.gz) {
        const int64_t v = x + int64_t(a.gx) * (y + int64_t(a.gy) * z);
#pragma unroll
        for (int c = 0; c < COUT; ++c) {
          vals[c] += S.bias[c];
          if (RELU) vals[c] = fmaxf(vals[c], 0.0f);
        }
        if (a.out_bf) {
          uint32_t pk[COUT / 2];
#pragma unroll
          for (int c = 0; c < COUT / 2; ++c) {
            __nv_bfloat162 hh = __floats2bfloat162_rn(vals[2 * c], vals[2 * c + 1]);
            pk[c] = *reinterpret_cast<uint32_t*>(&hh);
          }
          uint4* dst = reinterpret_cast<uint4*>(a.out_bf + v * COUT);
#pragma unroll
          for (int q = 0; q < COUT / 8; ++q) dst[q] = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
        }
        if (a.out_f32)
          reinterpret_cast<float4*>(a.out_f32)[v] = make_float4(vals[0], vals[1], vals[2], vals[3]);
      }
    }
    tc::fence_before_sync();
  }
  if (!ok) {
    // the accumulator may still be in use: wait once more (bounded) before freeing it
    if (tid == 0) {
      atomicExch(a.err, 1);
      tc::mbar_wait(&S.mbar, phase ^ 1u);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

template <int CIN, int COUT, bool RELU>
void launch_conv_instance(const ConvArgs& a, cudaStream_t s) {
  // CTAs per SM from the shared-memory footprint (228 KB per SM, 1 KB reserved
  // per CTA), at most 4 (4 x 64 of the 512 tensor-memory columns)
  static int grid_per_sm = 0;
  const size_t smem = sizeof(ConvSmem<CIN, COUT>);
  if (!grid_per_sm) {
    PA_CUDA(cudaFuncSetAttribute(k_conv3_tc<CIN, COUT, RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    grid_per_sm = std::max(1, std::min(4, int((228 * 1024) / (smem + 1024))));
  }
  const int ntiles = ((a.gx + kTX - 1) / kTX) * ((a.gy + kTY - 1) / kTY) * ((a.gz + kTZ - 1) / kTZ);
  const int grid = std::max(1, std::min(ntiles, grid_per_sm * num_sms()));
  k_conv3_tc<CIN, COUT, RELU><<<grid, kConvThreads, smem, s>>>(a);
  PA_LAUNCHED();
}

// ------------------------------------------------------ FP32 backward --
// gin[u][ci] = [act_in[u][ci] > 0] * sum_t sum_co W[co][ci][t] gout[u - off_t][co]
// (the ReLU mask of the layer that produced act_in; act_in of layer 1 is not needed).
template <int CIN_P, int COUT_R, int COUT_P>
__global__ void __launch_bounds__(256) k_conv_bwd_data(const float* __restrict__ gout, const float* __restrict__ W,
                                                       int cin_r, const __nv_bfloat16* __restrict__ act_in, int gx,
                                                       int gy, int gz, float* __restrict__ gin) {
  extern __shared__ float wsm[];  // [27][COUT_R][CIN_P]
  for (int i = threadIdx.x; i < 27 * COUT_R * CIN_P; i += blockDim.x) {
    const int ci = i % CIN_P, co = (i / CIN_P) % COUT_R, t = i / (CIN_P * COUT_R);
    wsm[i] = ci < cin_r ? W[(int64_t(co) * cin_r + ci) * 27 + t] : 0.0f;
  }
  __syncthreads();
  const int64_t G = int64_t(gx) * gy * gz;
  for (int64_t u = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; u < G; u += int64_t(gridDim.x) * blockDim.x) {
    const int x = int(u % gx), y = int((u / gx) % gy), z = int(u / (int64_t(gx) * gy));
    float acc[CIN_P];
#pragma unroll
    for (int c = 0; c < CIN_P; ++c) acc[c] = 0.0f;
    for (int t = 0; t < 27; ++t) {
      const int vx = x - (t % 3 - 1), vy = y - ((t / 3) % 3 - 1), vz = z - (t / 9 - 1);
      if (vx < 0 || vx >= gx || vy < 0 || vy >= gy || vz < 0 || vz >= gz) continue;
      const float* gr = gout + (vx + int64_t(gx) * (vy + int64_t(gy) * vz)) * COUT_P;
#pragma unroll 4
      for (int co = 0; co < COUT_R; ++co) {
        const float g = gr[co];
        const float* wr = wsm + (t * COUT_R + co) * CIN_P;
#pragma unroll
        for (int c = 0; c < CIN_P; ++c) acc[c] = fmaf(wr[c], g, acc[c]);
      }
    }
    const __nv_bfloat16* ar = act_in + u * CIN_P;
#pragma unroll
    for (int c = 0; c < CIN_P; ++c)
      gin[u * CIN_P + c] = (c < cin_r && __bfloat162float(ar[c]) > 0.0f) ? acc[c] : 0.0f;
  }
}

// dW[co][ci][t] += sum_v gout[v][co] act_in[v + off_t][ci]; db[co] += sum_v gout[v][co].
// blockIdx.y = tap; thread = (co = tid / 8, ci = 4 (tid % 8) .. + 3); a CTA sums `chunk` nodes.
template <int CIN_P, int COUT_P>
__global__ void __launch_bounds__(256) k_conv_bwd_weight(const float* __restrict__ gout,
                                                         const __nv_bfloat16* __restrict__ act_in, int cin_r,
                                                         int cout_r, int gx, int gy, int gz, int chunk,
                                                         float* __restrict__ dW, float* __restrict__ db) {
  const int t = blockIdx.y;
  const int ox = t % 3 - 1, oy = (t / 3) % 3 - 1, oz = t / 9 - 1;
  const int co = threadIdx.x >> 3, ci0 = (threadIdx.x & 7) * 4;
  if (co >= cout_r || ci0 >= cin_r || ci0 >= CIN_P) return;
  const int64_t G = int64_t(gx) * gy * gz;
  const int64_t v0 = int64_t(blockIdx.x) * chunk, v1 = (v0 + chunk < G) ? v0 + chunk : G;
  if (v0 >= v1) return;
  float acc[4] = {0.f, 0.f, 0.f, 0.f}, bacc = 0.f;
  int x = int(v0 % gx), y = int((v0 / gx) % gy), z = int(v0 / (int64_t(gx) * gy));
  const bool bias_thread = (t == 0 && ci0 == 0);
  for (int64_t v = v0; v < v1; ++v) {
    const float g = gout[v * COUT_P + co];
    if (bias_thread) bacc += g;
    const int ux = x + ox, uy = y + oy, uz = z + oz;
    if (ux >= 0 && ux < gx && uy >= 0 && uy < gy && uz >= 0 && uz < gz) {
      const int64_t u = ux + int64_t(gx) * (uy + int64_t(gy) * uz);
      const uint2 raw = *reinterpret_cast<const uint2*>(act_in + u * CIN_P + ci0);
      const __nv_bfloat162 lo = *reinterpret_cast<const __nv_bfloat162*>(&raw.x);
      const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162*>(&raw.y);
      acc[0] = fmaf(g, __low2float(lo), acc[0]);
      acc[1] = fmaf(g, __high2float(lo), acc[1]);
      acc[2] = fmaf(g, __low2float(hi), acc[2]);
      acc[3] = fmaf(g, __high2float(hi), acc[3]);
    }
    if (++x == gx) {
      x = 0;
      if (++y == gy) {
        y = 0;
        ++z;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (ci0 + k < cin_r) atomicAdd(&dW[(int64_t(co) * cin_r + ci0 + k) * 27 + t], acc[k]);
  if (bias_thread) atomicAdd(&db[co], bacc);
}

__global__ void k_adam(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2,
                       float gscale) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// FP32 master weights [co][ci][t] (real sizes) -> BF16 [t][cin_p/8][cout_p][8], padded with zeros.
__global__ void k_pack_weights(const float* __restrict__ W, const float* __restrict__ b, int cin_r, int cout_r,
                               int cin_p, int cout_p, __nv_bfloat16* __restrict__ wpk, float* __restrict__ bpad) {
  const int n = 27 * cin_p * cout_p;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = i % 8, co = (i / 8) % cout_p, cg = (i / (8 * cout_p)) % (cin_p / 8), t = i / (cout_p * cin_p);
    const int ci = cg * 8 + k;
    const float val = (co < cout_r && ci < cin_r) ? W[(int64_t(co) * cin_r + ci) * 27 + t] : 0.0f;
    wpk[i] = __float2bfloat16_rn(val);
  }
  if (blockIdx.x == 0)
    for (int c = threadIdx.x; c < cout_p; c += blockDim.x) bpad[c] = c < cout_r ? b[c] : 0.0f;
}

// Caller features (G x 5 FP32) -> layer-1 input (G x 16 BF16).
__global__ void k_feat_to_a0(int64_t G, const float* __restrict__ f, __nv_bfloat16* __restrict__ a0) {
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < G; v += int64_t(gridDim.x) * blockDim.x) {
    float c[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) c[k] = k < kFeatures ? f[v * kFeatures + k] : 0.0f;
    uint32_t pk[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      __nv_bfloat162 h = __floats2bfloat162_rn(c[2 * k], c[2 * k + 1]);
      pk[k] = *reinterpret_cast<uint32_t*>(&h);
    }
    uint4* dst = reinterpret_cast<uint4*>(a0 + v * 16);
    dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  }
}

// Residual (SoA) -> layer-1 input: scaled residual, stiffness and Dirichlet features.
template <typename T>
__global__ void k_pc_pack(int64_t N, const T* __restrict__ r, const float* __restrict__ dsq,
                          const float2* __restrict__ feat, const double* __restrict__ rdr, double inv_nfree,
                          const int32_t* __restrict__ done, __nv_bfloat16* __restrict__ a0) {
  if (done && *done) return;
  const double s2 = *rdr * inv_nfree;
  const float inv = s2 > 0.0 ? float(1.0 / sqrt(s2)) : 0.0f;
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < N; v += int64_t(gridDim.x) * blockDim.x) {
    const float2 f = feat[v];
    const float c0 = float(r[v]) * dsq[v] * inv;
    const float c1 = float(r[N + v]) * dsq[N + v] * inv;
    const float c2 = float(r[2 * N + v]) * dsq[2 * N + v] * inv;
    __nv_bfloat162 h0 = __floats2bfloat162_rn(c0, c1), h1 = __floats2bfloat162_rn(c2, f.x),
                   h2 = __floats2bfloat162_rn(f.y, 0.0f);
    uint4* dst = reinterpret_cast<uint4*>(a0 + v * 16);
    dst[0] = make_uint4(*reinterpret_cast<uint32_t*>(&h0), *reinterpret_cast<uint32_t*>(&h1),
                        *reinterpret_cast<uint32_t*>(&h2), 0u);
    dst[1] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// max over nodes of the mean diagonal (positive floats compare as their bit patterns)
__global__ void k_diag_max(int64_t N, const double* __restrict__ diag, unsigned int* __restrict__ out) {
  unsigned int best = 0u;
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < N; v += int64_t(gridDim.x) * blockDim.x) {
    const float m = float((diag[3 * v] + diag[3 * v + 1] + diag[3 * v + 2]) * (1.0 / 3.0));
    if (m > 0.0f) best = max(best, __float_as_uint(m));
  }
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

// D^-1 and D^-1/2 (SoA, zero on constrained dofs) and the node features.
__global__ void k_pc_features(int64_t N, const double* __restrict__ diag, const uint8_t* __restrict__ mask,
                              const unsigned int* __restrict__ dmax_bits, float* __restrict__ dinv,
                              float* __restrict__ dsq, float2* __restrict__ feat) {
  const float dmax = __uint_as_float(*dmax_bits);
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < N; v += int64_t(gridDim.x) * blockDim.x) {
    const unsigned mk = mask ? mask[v] : 0u;
    float msum = 0.0f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double g = diag[3 * v + d];
      msum += float(g);
      const bool c = (mk >> d) & 1u;
      const float di = (c || !(g > 0.0)) ? 0.0f : float(1.0 / g);
      dinv[d * N + v] = di;
      dsq[d * N + v] = sqrtf(di);
    }
    const float m = msum * (1.0f / 3.0f);
    float s = (m > 0.0f && dmax > 0.0f) ? 1.0f + log10f(m / dmax) * (1.0f / 9.0f) : 0.0f;
    s = fminf(fmaxf(s, 0.0f), 1.0f);
    feat[v] = make_float2(s, float(__popc(mk & 7u)) * (1.0f / 3.0f));
  }
}

// r.D^-1 r (SoA) into *out (zeroed by the caller).
__global__ void k_pc_rdr(int64_t n, const float* __restrict__ r, const float* __restrict__ dinv, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += double(r[i]) * double(dinv[i]) * double(r[i]);
  s = block_sum(s, red);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

// z = D^-1 r + s D^-1/2 f   (SoA)
__global__ void k_pc_combine(int64_t N, const float* __restrict__ r, const float* __restrict__ dinv,
                             const float* __restrict__ dsq, const float* __restrict__ out,
                             const double* __restrict__ rdr, double inv_nfree, float* __restrict__ z) {
  const double s2 = *rdr * inv_nfree;
  const float sig = s2 > 0.0 ? float(sqrt(s2)) : 0.0f;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    z[i] = dinv[i] * r[i] + sig * dsq[i] * out[4 * v + d];
  }
}

// Loss terms (z.Kz - 2 z.r) / E into *loss and the gradient of the loss with
// respect to the network output: s D^-1/2 2 (Kz - r) / E, as G x 16 (channels 0..2).
__global__ void k_pc_loss_grad(int64_t N, const float* __restrict__ z, const float* __restrict__ q,
                               const float* __restrict__ r, const float* __restrict__ dsq,
                               const double* __restrict__ rdr, double inv_nfree, double E, double* loss,
                               float* __restrict__ gout) {
  __shared__ double red[32];
  const double s2 = *rdr * inv_nfree;
  const float sig = s2 > 0.0 ? float(sqrt(s2)) : 0.0f;
  const float gs = float(2.0 / E);
  double acc = 0.0;
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < N; v += int64_t(gridDim.x) * blockDim.x) {
    float g[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int64_t i = d * N + v;
      acc += double(z[i]) * (double(q[i]) - 2.0 * double(r[i]));
      g[d] = sig * dsq[i] * gs * (q[i] - r[i]);
    }
    float4* dst = reinterpret_cast<float4*>(gout + 16 * v);
    dst[0] = make_float4(g[0], g[1], g[2], 0.0f);
    dst[1] = dst[2] = dst[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) atomicAdd(loss, acc / E);
}

// G x 3 -> G x 16 (zero padded)
__global__ void k_pad_gout(int64_t G, const float* __restrict__ g3, float* __restrict__ g16) {
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < G; v += int64_t(gridDim.x) * blockDim.x) {
    float4* dst = reinterpret_cast<float4*>(g16 + 16 * v);
    dst[0] = make_float4(g3[3 * v], g3[3 * v + 1], g3[3 * v + 2], 0.0f);
    dst[1] = dst[2] = dst[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
}

// G x 4 -> G x 3
__global__ void k_take3(int64_t G, const float* __restrict__ o4, float* __restrict__ o3) {
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < G; v += int64_t(gridDim.x) * blockDim.x) {
    o3[3 * v] = o4[4 * v];
    o3[3 * v + 1] = o4[4 * v + 1];
    o3[3 * v + 2] = o4[4 * v + 2];
  }
}

int grid_for(int64_t n, int threads = 256) {
  const int64_t want = (n + threads - 1) / threads;
  return int(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(num_sms()) * 8)));
}

}  // namespace

struct LearnedPC {
  int device = 0;
  int gx = 0, gy = 0, gz = 0;
  int64_t G = 0;
  cudaStream_t stream = nullptr;
  DevBuf<float> params, grads, adam_m, adam_v;
  DevBuf<__nv_bfloat16> wpk[kPcLayers];
  DevBuf<float> bpad[kPcLayers];
  DevBuf<__nv_bfloat16> act[kPcLayers];  // inputs of layers 1..4
  DevBuf<float> out;                     // G x 4, network output (channels 0..2)
  DevBuf<float> g_a, g_b;                // G x 32 backward buffers
  DevBuf<float> dsq, dinv, r32, z32, q32;
  DevBuf<float2> feat;
  DevBuf<double> scal;          // [0] r.D^-1 r, [1] loss accumulator
  DevBuf<unsigned int> dmax;
  DevBuf<int> err;
  int64_t adam_t = 0;
  ~LearnedPC() {
    if (stream) cudaStreamDestroy(stream);
  }
};

int64_t pc_num_params() { return w_offset(kPcLayers); }
int pc_device(const LearnedPC& pc) { return pc.device; }
int64_t pc_grid_points(const LearnedPC& pc) { return pc.G; }
cudaStream_t pc_stream(const LearnedPC& pc) { return pc.stream; }

namespace {

void pack_all(LearnedPC& pc, cudaStream_t s) {
  for (int l = 0; l < kPcLayers; ++l) {
    const int n = 27 * kCinP[l] * kCoutP[l];
    k_pack_weights<<<(n + 255) / 256, 256, 0, s>>>(pc.params.get() + w_offset(l), pc.params.get() + b_offset(l),
                                                   kCin[l], kCout[l], kCinP[l], kCoutP[l], pc.wpk[l].get(),
                                                   pc.bpad[l].get());
    PA_LAUNCHED();
  }
}

// Layers 1..4 on pc.act[0]; outputs into act[1..3] and pc.out.
void run_layers(LearnedPC& pc, const int32_t* done, cudaStream_t s) {
  ConvArgs a{};
  a.done = done;
  a.err = pc.err.get();
  a.gx = pc.gx;
  a.gy = pc.gy;
  a.gz = pc.gz;
  for (int l = 0; l < kPcLayers; ++l) {
    a.in = pc.act[l].get();
    a.w = pc.wpk[l].get();
    a.bias = pc.bpad[l].get();
    a.out_bf = l + 1 < kPcLayers ? pc.act[l + 1].get() : nullptr;
    a.out_f32 = l + 1 < kPcLayers ? nullptr : pc.out.get();
    if (l == 0)
      launch_conv_instance<16, 32, true>(a, s);
    else if (l < 3)
      launch_conv_instance<32, 32, true>(a, s);
    else
      launch_conv_instance<32, 16, false>(a, s);
  }
}

template <int CIN_P, int COUT_R, int COUT_P>
void launch_bwd_data(LearnedPC& pc, int l, const float* gout, const __nv_bfloat16* act_in, float* gin, cudaStream_t s) {
  const size_t smem = sizeof(float) * 27 * COUT_R * CIN_P;
  static bool configured = false;
  if (!configured) {
    PA_CUDA(cudaFuncSetAttribute(k_conv_bwd_data<CIN_P, COUT_R, COUT_P>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    configured = true;
  }
  const int grid = int(std::min<int64_t>((pc.G + 255) / 256, int64_t(num_sms()) * 2));
  k_conv_bwd_data<CIN_P, COUT_R, COUT_P><<<grid, 256, smem, s>>>(gout, pc.params.get() + w_offset(l), kCin[l],
                                                                  act_in, pc.gx, pc.gy, pc.gz, gin);
  PA_LAUNCHED();
}

template <int CIN_P, int COUT_P>
void launch_bwd_weight(LearnedPC& pc, int l, const float* gout, const __nv_bfloat16* act_in, cudaStream_t s) {
  constexpr int kChunk = 1024;
  const dim3 grid(unsigned((pc.G + kChunk - 1) / kChunk), 27);
  k_conv_bwd_weight<CIN_P, COUT_P><<<grid, 256, 0, s>>>(gout, act_in, kCin[l], kCout[l], pc.gx, pc.gy, pc.gz, kChunk,
                                                        pc.grads.get() + w_offset(l), pc.grads.get() + b_offset(l));
  PA_LAUNCHED();
}

// Accumulate d(loss)/d(params) into pc.grads from gout4 = d(loss)/d(layer-4 output), G x 16.
void backward(LearnedPC& pc, const float* gout4, cudaStream_t s) {
  launch_bwd_weight<32, 16>(pc, 3, gout4, pc.act[3].get(), s);
  launch_bwd_data<32, 3, 16>(pc, 3, gout4, pc.act[3].get(), pc.g_a.get(), s);
  launch_bwd_weight<32, 32>(pc, 2, pc.g_a.get(), pc.act[2].get(), s);
  launch_bwd_data<32, 32, 32>(pc, 2, pc.g_a.get(), pc.act[2].get(), pc.g_b.get(), s);
  launch_bwd_weight<32, 32>(pc, 1, pc.g_b.get(), pc.act[1].get(), s);
  launch_bwd_data<32, 32, 32>(pc, 1, pc.g_b.get(), pc.act[1].get(), pc.g_a.get(), s);
  launch_bwd_weight<16, 32>(pc, 0, pc.g_a.get(), pc.act[0].get(), s);
}

void check_err(LearnedPC& pc, cudaStream_t s) {
  int h = 0;
  PA_CUDA(cudaMemcpyAsync(&h, pc.err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  if (h) throw Error(PA_ERR_CUDA, "learned preconditioner: a tensor-core wait timed out");
}

}  // namespace

LearnedPC* pc_new(int gx, int gy, int gz, uint64_t seed) {
  PA_CHECK(gx >= 1 && gy >= 1 && gz >= 1, "grid dimensions must be positive");
  PA_CHECK(int64_t(gx) * gy * gz < (int64_t(1) << 31), "grid too large");
  std::unique_ptr<LearnedPC> pc(new LearnedPC());
  PA_CUDA(cudaGetDevice(&pc->device));
  pc->gx = gx;
  pc->gy = gy;
  pc->gz = gz;
  pc->G = int64_t(gx) * gy * gz;
  PA_CUDA(cudaStreamCreateWithFlags(&pc->stream, cudaStreamDefault));  // ordered against the legacy default stream
  const int64_t np = pc_num_params();
  std::vector<float> h(np, 0.0f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l + 1 < kPcLayers; ++l) {
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / float(27 * kCin[l])));
    for (int64_t i = 0; i < int64_t(kCout[l]) * kCin[l] * 27; ++i) h[w_offset(l) + i] = nd(rng);
  }
  pc->params.upload(h.data(), np, pc->stream);
  pc->grads.resize(np);
  pc->adam_m.resize(np);
  pc->adam_v.resize(np);
  PA_CUDA(cudaMemsetAsync(pc->adam_m.get(), 0, sizeof(float) * np, pc->stream));
  PA_CUDA(cudaMemsetAsync(pc->adam_v.get(), 0, sizeof(float) * np, pc->stream));
  for (int l = 0; l < kPcLayers; ++l) {
    pc->wpk[l].resize(size_t(27) * kCinP[l] * kCoutP[l]);
    pc->bpad[l].resize(kCoutP[l]);
    pc->act[l].resize(size_t(pc->G) * kCinP[l]);
  }
  pc->out.resize(size_t(pc->G) * 4);
  pc->scal.resize(4);
  pc->dmax.resize(1);
  pc->err.resize(1);
  PA_CUDA(cudaMemsetAsync(pc->err.get(), 0, sizeof(int), pc->stream));
  pack_all(*pc, pc->stream);
  PA_CUDA(cudaStreamSynchronize(pc->stream));
  return pc.release();
}

void pc_delete(LearnedPC* pc) { delete pc; }

void pc_check_grid(const LearnedPC& pc, const Mesh& m) {
  PA_CHECK(m.N == pc.G, "mesh node count differs from the network's grid");
  // nodes on the grid, x fastest: coordinates affine in (i, j, k)
  const double* X = m.coords.data();
  const int64_t sx = 1, sy = pc.gx, sz = int64_t(pc.gx) * pc.gy;
  double h[3] = {X[3 * sx] - X[0], X[3 * sy + 1] - X[1], X[3 * sz + 2] - X[2]};
  PA_CHECK(h[0] > 0 && h[1] > 0 && h[2] > 0, "mesh is not the network's grid (spacing)");
  const double tol = 1e-6 * std::min(h[0], std::min(h[1], h[2]));
  for (int64_t v = 0; v < m.N; ++v) {
    const int64_t i = v % pc.gx, j = (v / pc.gx) % pc.gy, k = v / sz;
    const double e[3] = {X[0] + i * h[0], X[1] + j * h[1], X[2] + k * h[2]};
    for (int d = 0; d < 3; ++d)
      PA_CHECK(std::fabs(X[3 * v + d] - e[d]) <= tol, "mesh nodes are not the network's grid in x-fastest order");
  }
}

void pc_set_params(LearnedPC& pc, const float* d_params, cudaStream_t s) {
  PA_CUDA(cudaMemcpyAsync(pc.params.get(), d_params, sizeof(float) * pc_num_params(), cudaMemcpyDeviceToDevice, s));
  pack_all(pc, s);
}

void pc_get_params(const LearnedPC& pc, float* d_params, cudaStream_t s) {
  PA_CUDA(cudaMemcpyAsync(d_params, pc.params.get(), sizeof(float) * pc_num_params(), cudaMemcpyDeviceToDevice, s));
}

void pc_forward_features(LearnedPC& pc, const float* d_feat, float* d_out, cudaStream_t s) {
  k_feat_to_a0<<<grid_for(pc.G), 256, 0, s>>>(pc.G, d_feat, pc.act[0].get());
  PA_LAUNCHED();
  run_layers(pc, nullptr, s);
  k_take3<<<grid_for(pc.G), 256, 0, s>>>(pc.G, pc.out.get(), d_out);
  PA_LAUNCHED();
  check_err(pc, s);
}

double pc_time_forward(LearnedPC& pc, int reps) {
  cudaStream_t s = pc.stream;
  cudaEvent_t e0, e1;
  PA_CUDA(cudaEventCreate(&e0));
  PA_CUDA(cudaEventCreate(&e1));
  run_layers(pc, nullptr, s);  // warm
  PA_CUDA(cudaEventRecord(e0, s));
  for (int i = 0; i < reps; ++i) run_layers(pc, nullptr, s);
  PA_CUDA(cudaEventRecord(e1, s));
  PA_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  check_err(pc, s);
  return double(ms) / reps;
}

int64_t pc_forward_flops(const LearnedPC& pc) {
  int64_t f = 0;
  for (int l = 0; l < kPcLayers; ++l) f += 2LL * 27 * kCin[l] * kCout[l];
  return f * pc.G;
}

void pc_backward_features(LearnedPC& pc, const float* d_feat, const float* d_gout, float* d_gparams, cudaStream_t s) {
  k_feat_to_a0<<<grid_for(pc.G), 256, 0, s>>>(pc.G, d_feat, pc.act[0].get());
  PA_LAUNCHED();
  run_layers(pc, nullptr, s);
  pc.g_a.resize(size_t(pc.G) * 32);
  pc.g_b.resize(size_t(pc.G) * 32);
  DevBuf<float> g16(size_t(pc.G) * 16);
  k_pad_gout<<<grid_for(pc.G), 256, 0, s>>>(pc.G, d_gout, g16.get());
  PA_LAUNCHED();
  PA_CUDA(cudaMemsetAsync(pc.grads.get(), 0, sizeof(float) * pc_num_params(), s));
  backward(pc, g16.get(), s);
  PA_CUDA(cudaMemcpyAsync(d_gparams, pc.grads.get(), sizeof(float) * pc_num_params(), cudaMemcpyDeviceToDevice, s));
  check_err(pc, s);
}

// ------------------------------------------------ solver-facing pieces --
void pc_prepare_operator(LearnedPC& pc, Problem& P, const double* diag_aos, float* dinv_out, cudaStream_t s) {
  const int64_t N = P.N();
  pc.dsq.resize(3 * N);
  pc.feat.resize(N);
  PA_CUDA(cudaMemsetAsync(pc.dmax.get(), 0, sizeof(unsigned int), s));
  k_diag_max<<<grid_for(N), 256, 0, s>>>(N, diag_aos, pc.dmax.get());
  PA_LAUNCHED();
  k_pc_features<<<grid_for(N), 256, 0, s>>>(N, diag_aos, P.d_node_mask.get(), pc.dmax.get(), dinv_out, pc.dsq.get(),
                                           pc.feat.get());
  PA_LAUNCHED();
}

template <typename T>
void pc_launch_network(LearnedPC& pc, const T* r, const double* rdr, double inv_nfree, const int32_t* done,
                       cudaStream_t s) {
  k_pc_pack<T><<<grid_for(pc.G), 256, 0, s>>>(pc.G, r, pc.dsq.get(), pc.feat.get(), rdr, inv_nfree, done,
                                              pc.act[0].get());
  PA_LAUNCHED();
  run_layers(pc, done, s);
}
template void pc_launch_network<float>(LearnedPC&, const float*, const double*, double, const int32_t*, cudaStream_t);

const float* pc_output(const LearnedPC& pc) { return pc.out.get(); }
const float* pc_dsq(const LearnedPC& pc) { return pc.dsq.get(); }
int* pc_error_flag(LearnedPC& pc) { return pc.err.get(); }
void pc_check_error(LearnedPC& pc, cudaStream_t s) { check_err(pc, s); }

int64_t free_dofs(const Problem& P) {
  std::vector<uint8_t> seen(size_t(P.ndof()), 0);
  int64_t c = 0;
  for (int32_t d : P.bc_dofs)
    if (!seen[d]) {
      seen[d] = 1;
      ++c;
    }
  return std::max<int64_t>(1, P.ndof() - c);
}

void pc_apply(LearnedPC& pc, Problem& P, const double* z, const double* r_aos, double* out_aos) {
  cudaStream_t s = P.stream;
  const int64_t N = P.N(), n = 3 * N;
  DevBuf<double> w64(P.C()), diag(n);
  DevBuf<float> w32(P.C());
  launch_cell_weights(P, z, w64.get(), w32.get(), s);
  launch_diag(P, w64.get(), diag.get(), s);
  pc.dinv.resize(n);
  pc.r32.resize(n);
  pc.z32.resize(n);
  pc_prepare_operator(pc, P, diag.get(), pc.dinv.get(), s);
  launch_aos_to_soa<double, float>(r_aos, pc.r32.get(), N, s);
  PA_CUDA(cudaMemsetAsync(pc.scal.get(), 0, sizeof(double), s));
  k_pc_rdr<<<grid_for(n), 256, 0, s>>>(n, pc.r32.get(), pc.dinv.get(), pc.scal.get());
  PA_LAUNCHED();
  const double inv_nfree = 1.0 / double(free_dofs(P));
  pc_launch_network<float>(pc, pc.r32.get(), pc.scal.get(), inv_nfree, nullptr, s);
  k_pc_combine<<<grid_for(n), 256, 0, s>>>(N, pc.r32.get(), pc.dinv.get(), pc.dsq.get(), pc.out.get(), pc.scal.get(),
                                           inv_nfree, pc.z32.get());
  PA_LAUNCHED();
  launch_soa_to_aos<float, double>(pc.z32.get(), out_aos, N, s);
  check_err(pc, s);
}

void pc_train(LearnedPC& pc, Problem& P, const PcTrainSet& set, const pa_pc_train_options& o, pa_pc_train_stats* st) {
  PA_CHECK(set.num_samples > 0 && set.num_densities > 0, "empty training set");
  PA_CHECK(o.steps > 0 && o.batch > 0 && o.learning_rate > 0.0, "bad training options");
  for (int i = 0; i < set.num_samples; ++i) {
    PA_CHECK(set.sample_density[i] >= 0 && set.sample_density[i] < set.num_densities, "sample density index");
    PA_CHECK(set.sample_energy[i] > 0.0 && std::isfinite(set.sample_energy[i]), "sample energies must be positive");
  }
  cudaStream_t s = P.stream;
  const int64_t N = P.N(), n = 3 * N, C = P.C();
  DevBuf<double> w64(C), diag(n);
  DevBuf<float> w32(C), g16(size_t(pc.G) * 16);
  pc.dinv.resize(n);
  pc.r32.resize(n);
  pc.z32.resize(n);
  pc.q32.resize(n);
  pc.g_a.resize(size_t(pc.G) * 32);
  pc.g_b.resize(size_t(pc.G) * 32);
  const double inv_nfree = 1.0 / double(free_dofs(P));
  cudaEvent_t e0, e1;
  PA_CUDA(cudaEventCreate(&e0));
  PA_CUDA(cudaEventCreate(&e1));
  PA_CUDA(cudaEventRecord(e0, s));
  std::mt19937_64 rng(o.seed);
  std::vector<double> losses(o.steps);
  DevBuf<double> loss_dev(o.steps);
  PA_CUDA(cudaMemsetAsync(loss_dev.get(), 0, sizeof(double) * o.steps, s));
  int cur_density = -1;
  int64_t launches = 0;
  const int64_t np = pc_num_params();
  for (int step = 0; step < o.steps; ++step) {
    PA_CUDA(cudaMemsetAsync(pc.grads.get(), 0, sizeof(float) * np, s));
    for (int b = 0; b < o.batch; ++b) {
      const int smp = int(rng() % uint64_t(set.num_samples));
      const int d = set.sample_density[smp];
      if (d != cur_density) {
        launch_cell_weights(P, set.densities + int64_t(d) * P.nz(), w64.get(), w32.get(), s);
        launch_diag(P, w64.get(), diag.get(), s);
        pc_prepare_operator(pc, P, diag.get(), pc.dinv.get(), s);
        cur_density = d;
        launches += 4;
      }
      launch_aos_to_soa<double, float>(set.residuals + int64_t(smp) * n, pc.r32.get(), N, s);
      PA_CUDA(cudaMemsetAsync(pc.scal.get(), 0, sizeof(double), s));
      k_pc_rdr<<<grid_for(n), 256, 0, s>>>(n, pc.r32.get(), pc.dinv.get(), pc.scal.get());
      PA_LAUNCHED();
      pc_launch_network<float>(pc, pc.r32.get(), pc.scal.get(), inv_nfree, nullptr, s);
      k_pc_combine<<<grid_for(n), 256, 0, s>>>(N, pc.r32.get(), pc.dinv.get(), pc.dsq.get(), pc.out.get(),
                                               pc.scal.get(), inv_nfree, pc.z32.get());
      PA_LAUNCHED();
      launch_apply_tiled<float>(P, w32.get(), pc.z32.get(), pc.q32.get(), true, s);
      k_pc_loss_grad<<<grid_for(N), 256, 0, s>>>(N, pc.z32.get(), pc.q32.get(), pc.r32.get(), pc.dsq.get(),
                                                 pc.scal.get(), inv_nfree, set.sample_energy[smp],
                                                 loss_dev.get() + step, g16.get());
      PA_LAUNCHED();
      backward(pc, g16.get(), s);
      launches += 19;
    }
    // Adam with a cosine-decayed step size, gradients averaged over the batch
    ++pc.adam_t;
    const double frac = o.steps > 1 ? double(step) / double(o.steps - 1) : 1.0;
    const double lr = o.learning_rate * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * frac)));
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = float(1.0 - std::pow(double(b1), double(pc.adam_t)));
    const float bc2 = float(1.0 - std::pow(double(b2), double(pc.adam_t)));
    k_adam<<<grid_for(np), 256, 0, s>>>(np, pc.params.get(), pc.grads.get(), pc.adam_m.get(), pc.adam_v.get(),
                                        float(lr), b1, b2, 1e-8f, bc1, bc2, 1.0f / float(o.batch));
    PA_LAUNCHED();
    pack_all(pc, s);
    launches += 1 + kPcLayers;
  }
  PA_CUDA(cudaEventRecord(e1, s));
  PA_CUDA(cudaMemcpyAsync(losses.data(), loss_dev.get(), sizeof(double) * o.steps, cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaEventSynchronize(e1));
  PA_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  check_err(pc, s);
  for (double& l : losses) l = l / o.batch + 1.0;
  if (st) {
    st->initial_loss = losses.front();
    const int k = std::min(10, o.steps);
    double f = 0.0;
    for (int i = o.steps - k; i < o.steps; ++i) f += losses[i];
    st->final_loss = f / k;
    st->seconds = ms * 1e-3;
    st->steps = o.steps;
    st->kernel_launches = launches;
  }
}

}  // namespace pa
