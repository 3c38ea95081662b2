// pa_noalloc.cu -- the compliance ("Internal Elastic Energy") value without
// any allocation by the library.
//
// Who needs it: callers that must not allocate device memory while they run.
// Examples are a host framework that owns every device byte through its own
// pool, a real-time or timed loop where cudaMalloc's implicit device
// synchronisation is not acceptable, and an embedding that cannot create
// library handles (pa_mesh_create / pa_problem_create allocate).  They pass
// raw device arrays in and a device scalar out, and the library uses only
// the fixed scratch array below.
//
// Scratch: one file-scope __device__ array of kNoAllocBlocks doubles (256 KB)
// holding the per-block partial sums of the energy.  Every GPU that loads the
// library holds it until the process exits.  It bounds the mesh size: at most
// kNoAllocBlocks * kNoAllocThreads = 8,388,608 cells per call; larger meshes are
// rejected with PA_ERR_INVALID_ARG.  All calls share the array and it keeps the
// last call's contents; each call overwrites every slot it later reads (one
// per block it launches), so nothing needs clearing, but two calls whose
// kernels overlap on the GPU (different streams, or different host threads)
// race on it.  Serialise such calls on one stream.
//
// Inputs live on the device, so the host cannot validate them: a node id in
// cells2nodes outside [0, num_nodes) is caught in the kernel (that cell reads
// nothing through it and the value comes out NaN), but the lengths of coords,
// u and z (N or C per the control layout) cannot be checked; arrays shorter
// than the stated sizes are undefined behaviour.
//
// Host code must not pass `g_noalloc_partials` to a kernel: in host code that
// name is a host-side stand-in, not the device address.  The address is
// obtained with cudaGetSymbolAddress once per device, the first time the entry
// point runs on that device (with that device current); that first call
// should therefore come before any stream capture.
#include <mutex>

#include "pa_cell.cuh"

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocBlocks = 32768;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocBlocks];

std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

struct NoAllocMat {
  pa::Iso<double> iso;
  double p, pmin;
  int layout;
};

__device__ __forceinline__ double noalloc_block_sum(double v, double* smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? smem[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// Per-cell 1/2 vol p(rho) eps:C:eps (src/elliptic/InternalElasticEnergy.hpp:100-158),
// one partial sum per block into the scratch array.
// A cell with a node id outside [0, N) reads nothing through it and
// contributes NaN, so the value comes out NaN instead of an out-of-bounds read.
__global__ void __launch_bounds__(kNoAllocThreads) k_energy_noalloc(const int32_t* __restrict__ cells,
                                                                    const double* __restrict__ coords, int64_t C,
                                                                    int64_t N, NoAllocMat m,
                                                                    const double* __restrict__ u,
                                                                    const double* __restrict__ z,
                                                                    double* __restrict__ partials) {
  __shared__ double s_red[32];
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double f = 0.0;
  int v[4] = {0, 0, 0, 0};
  bool in_range = false;
  if (c < C) {
    const int4 q = reinterpret_cast<const int4*>(cells)[c];
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    in_range = true;
#pragma unroll
    for (int n = 0; n < 4; ++n) in_range = in_range && v[n] >= 0 && int64_t(v[n]) < N;
    if (!in_range) f = __longlong_as_double(0x7ff8000000000000LL);  // quiet NaN
  }
  if (in_range) {
    double x[4][3], ue[12], g[4][3], vol, e[6], sig[6];
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        x[n][d] = coords[3 * int64_t(v[n]) + d];
        ue[3 * n + d] = u[3 * int64_t(v[n]) + d];
      }
    pa::tet_geometry(x, g, vol);
    pa::tet_strain(g, ue, e);
    const double rho = m.layout == PA_CONTROL_CELL ? z[c] : 0.25 * (z[v[0]] + z[v[1]] + z[v[2]] + z[v[3]]);
    pa::tet_stress(m.iso, vol * pa::simp(rho, m.p, m.pmin), e, sig);
    f = 0.5 * pa::voigt_dot(sig, e);
  }
  const double b = noalloc_block_sum(f, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

__global__ void __launch_bounds__(1024) k_sum_noalloc(const double* __restrict__ partials, int n,
                                                      double* __restrict__ out) {
  __shared__ double s_red[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
  v = noalloc_block_sum(v, s_red);
  if (threadIdx.x == 0) *out = v;
}

// True for memory of device `dev` (or managed memory).  A pointer that
// cudaPointerGetAttributes rejects is reported as not on the device; that
// error is its own (the call returns it synchronously) and is cleared.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    if (cudaPeekAtLastError() == e) cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" pa_status pa_sf_value_noalloc(const int32_t* cells2nodes, int64_t num_cells, const double* coords,
                                         int64_t num_nodes, const double* u, const double* z,
                                         const pa_elastic_params* params, double* value, void* stream) {
  try {
    if (!cells2nodes || !coords || !u || !z || !params || !value) throw pa::Error(PA_ERR_INVALID_ARG, "null argument");
    if (num_cells <= 0 || num_nodes <= 0) throw pa::Error(PA_ERR_INVALID_ARG, "empty mesh");
    if (num_cells > int64_t(kNoAllocBlocks) * kNoAllocThreads)
      throw pa::Error(PA_ERR_INVALID_ARG, "pa_sf_value_noalloc: at most 8388608 cells per call (fixed scratch of "
                                          "32768 block sums); got " + std::to_string(num_cells));
    if (params->control_layout != PA_CONTROL_NODAL && params->control_layout != PA_CONTROL_CELL)
      throw pa::Error(PA_ERR_INVALID_ARG, "unknown control layout");
    if (reinterpret_cast<uintptr_t>(cells2nodes) % 16 != 0)
      throw pa::Error(PA_ERR_INVALID_ARG, "cells2nodes must be 16-byte aligned");
    int dev = 0;
    PA_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) throw pa::Error(PA_ERR_UNSUPPORTED, "device ordinal too large");
    const void* arrays[] = {cells2nodes, coords, u, z, value};
    for (const void* a : arrays)
      if (!on_device(a, dev))
        throw pa::Error(PA_ERR_INVALID_ARG, "pa_sf_value_noalloc takes device pointers of the current device only");
    double* scratch = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_noalloc_mutex);
      if (!g_noalloc_ptr[dev]) {
        void* addr = nullptr;
        PA_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_partials));
        g_noalloc_ptr[dev] = static_cast<double*>(addr);
      }
      scratch = g_noalloc_ptr[dev];
    }
    const double c = params->youngs_modulus / ((1.0 + params->poissons_ratio) * (1.0 - 2.0 * params->poissons_ratio));
    NoAllocMat m{pa::Iso<double>{c * params->poissons_ratio, 0.5 * c * (1.0 - 2.0 * params->poissons_ratio)},
                 params->simp_exponent, params->simp_min, params->control_layout};
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int blocks = int((num_cells + kNoAllocThreads - 1) / kNoAllocThreads);
    k_energy_noalloc<<<blocks, kNoAllocThreads, 0, s>>>(cells2nodes, coords, num_cells, num_nodes, m, u, z,
                                                        scratch);
    PA_LAUNCHED();
    k_sum_noalloc<<<1, 1024, 0, s>>>(scratch, blocks, value);
    PA_LAUNCHED();
    return PA_OK;
  } catch (const pa::Error& e) {
    pa::set_last_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    pa::set_last_error(e.what());
    return PA_ERR_INVALID_ARG;
  }
}
