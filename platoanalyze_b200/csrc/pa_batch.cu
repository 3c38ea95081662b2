// pa_batch.cu -- batched solves: one independent Jacobi-PCG per mesh part,
// all parts advanced together by the same kernels.
//
// A parted mesh (pa_mesh_set_parts) is the disjoint union of independent
// problems (e.g. 64 boxes of different sizes, each with its own density field
// and load).  Its tiles never mix parts, so the fused apply (tile kernel, mode
// 2) can take each tile's beta from its part, sum p.Kp into its part and skip
// the tiles of parts that have converged; the update kernel sums r.z and r.r
// per part.  Every part has its own alpha, beta, stopping test and iteration
// count, so the result of each part is the result of solving it alone, and a
// chunk of iterations for all parts is one CUDA graph replay.  A part that
// stops inside a chunk keeps its direction (its tiles copy p forward) and
// resumes with it if the FP64 residual check sends it back.
//
// Precision as the mixed solver (pa_solver.cu): FP32 vectors and operator,
// FP64 dots, FP64 iterate, FP64 true residual per part once per chunk.
#include <algorithm>
#include <cmath>

#include "pa_problem.cuh"
#include "pa_tiled.cuh"

namespace pa {

namespace {

constexpr int kBT = 256;

int bgrid(int64_t n) {
  const int64_t want = (n + kBT - 1) / kBT;
  return int(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(num_sms()) * 8)));
}

// Per-part sums of a block-contiguous range of the SoA index space: each
// thread keeps a running sum for the part it is in and flushes it to shared
// memory when the part changes (parts are node ranges, so that is rare).
struct PartRun {
  int cur = -1;
  double a = 0.0, b = 0.0;
  __device__ __forceinline__ void flush(double* sacc) {
    if (cur >= 0) {
      atomicAdd(&sacc[2 * cur], a);
      atomicAdd(&sacc[2 * cur + 1], b);
    }
    a = b = 0.0;
  }
};

__device__ __forceinline__ void block_range(int64_t n, int64_t& i0, int64_t& i1) {
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  i0 = blockIdx.x * per;
  i1 = i0 + per < n ? i0 + per : n;
}

__device__ __forceinline__ void flush_block(double* sacc, int P, double* pacc) {
  __syncthreads();
  for (int q = threadIdx.x; q < P; q += blockDim.x) {
    const double a = sacc[2 * q], b = sacc[2 * q + 1];
    if (a != 0.0 || b != 0.0) {
      atomicAdd(&pacc[2 * q], a);
      atomicAdd(&pacc[2 * q + 1], b);
    }
  }
}

// x += alpha_p p, r -= alpha_p Ap, Ap = 0, per-part r.z and r.r; the last CTA
// sets every active part's beta, iteration count and stopping flag, and the
// global done flag once all parts have stopped.
__global__ void __launch_bounds__(kBT) k_batch_update(int64_t N, float* __restrict__ x, float* __restrict__ r,
                                                      const float* __restrict__ p, float* __restrict__ ap,
                                                      const float* __restrict__ dinv,
                                                      const uint16_t* __restrict__ node_part,
                                                      PartScalars* __restrict__ psc, int P, double* __restrict__ pacc,
                                                      unsigned int* counter, PcgScalars* __restrict__ sc) {
  extern __shared__ double sacc[];  // 2P
  if (sc->done) return;
  for (int i = threadIdx.x; i < 2 * P; i += blockDim.x) sacc[i] = 0.0;
  __syncthreads();
  int64_t i0, i1;
  block_range(3 * N, i0, i1);
  PartRun run;
  bool active = false;
  float alpha = 0.0f;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int64_t v = i % N;
    const int part = node_part[v];
    if (part != run.cur) {
      run.flush(sacc);
      run.cur = part;
      active = psc[part].done == 0;
      alpha = float(psc[part].alpha);
    }
    if (!active) continue;
    x[i] += alpha * p[i];
    const float ri = r[i] - alpha * ap[i];
    r[i] = ri;
    ap[i] = 0.0f;
    run.a += double(ri) * double(dinv[i] * ri);
    run.b += double(ri) * double(ri);
  }
  run.flush(sacc);
  flush_block(sacc, P, pacc);
  if (last_block_arrive(counter)) {
    int all = 1;
    for (int q = threadIdx.x; q < P; q += blockDim.x) {
      PartScalars& ps = psc[q];
      const double t0 = __ldcg(&pacc[2 * q]), t1 = __ldcg(&pacc[2 * q + 1]);
      pacc[2 * q] = pacc[2 * q + 1] = 0.0;
      if (!ps.done) {
        ps.beta = t0 / ps.rz;
        ps.rz = t0;
        ps.rr = t1;
        ps.iters += 1;
        if (!isfinite(t0) || !isfinite(t1)) { ps.breakdown = 1; ps.done = 1; }
        if (t1 <= ps.stop2) ps.done = 1;
      }
      if (!ps.done) all = 0;
    }
    all = __syncthreads_and(all);
    if (threadIdx.x == 0) {
      sc->iters += 1;
      if (all) sc->done = 1;
      *counter = 0u;
    }
  }
}

// Per-part r.z and r.r of a fresh residual; parts at or below their stop2 stop.
__global__ void __launch_bounds__(kBT) k_batch_init(int64_t N, const float* __restrict__ r,
                                                    const float* __restrict__ dinv,
                                                    const uint16_t* __restrict__ node_part,
                                                    PartScalars* __restrict__ psc, int P, double* __restrict__ pacc,
                                                    unsigned int* counter, PcgScalars* __restrict__ sc) {
  extern __shared__ double sacc[];
  for (int i = threadIdx.x; i < 2 * P; i += blockDim.x) sacc[i] = 0.0;
  __syncthreads();
  int64_t i0, i1;
  block_range(3 * N, i0, i1);
  PartRun run;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int part = node_part[i % N];
    if (part != run.cur) {
      run.flush(sacc);
      run.cur = part;
    }
    const double ri = double(r[i]);
    run.a += ri * double(dinv[i]) * ri;
    run.b += ri * ri;
  }
  run.flush(sacc);
  flush_block(sacc, P, pacc);
  if (last_block_arrive(counter)) {
    int all = 1;
    for (int q = threadIdx.x; q < P; q += blockDim.x) {
      PartScalars& ps = psc[q];
      const double t0 = __ldcg(&pacc[2 * q]), t1 = __ldcg(&pacc[2 * q + 1]);
      pacc[2 * q] = pacc[2 * q + 1] = 0.0;
      if (!ps.done) {
        ps.rz = t0;
        ps.rr = t1;
        if (t1 <= ps.stop2) ps.done = 1;
      }
      if (!ps.done) all = 0;
    }
    all = __syncthreads_and(all);
    if (threadIdx.x == 0) {
      sc->done = all;
      *counter = 0u;
    }
  }
}

// out[p] += sum over part p of v^2 (FP64, SoA vector of 3N)
__global__ void __launch_bounds__(kBT) k_part_norm2(int64_t N, const double* __restrict__ v,
                                                    const uint16_t* __restrict__ node_part, int P,
                                                    double* __restrict__ out /*2P*/) {
  extern __shared__ double sacc[];
  for (int i = threadIdx.x; i < 2 * P; i += blockDim.x) sacc[i] = 0.0;
  __syncthreads();
  int64_t i0, i1;
  block_range(3 * N, i0, i1);
  PartRun run;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int part = node_part[i % N];
    if (part != run.cur) {
      run.flush(sacc);
      run.cur = part;
    }
    run.a += v[i] * v[i];
  }
  run.flush(sacc);
  flush_block(sacc, P, out);
}

// out_soa = mask ? 0 : a_aos - t_soa (t may be null); x += dx, dx = 0; f32 copy
__global__ void k_b_aos_minus_soa(int64_t N, const double* __restrict__ a, const double* __restrict__ t,
                                  const uint8_t* __restrict__ mask, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    const bool c = mask && ((mask[v] >> d) & 1);
    out[i] = c ? 0.0 : a[3 * v + d] - (t ? t[i] : 0.0);
  }
}
__global__ void k_b_sub_masked(int64_t N, const double* __restrict__ a, const double* __restrict__ b,
                               const uint8_t* __restrict__ mask, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    const bool c = mask && ((mask[v] >> d) & 1);
    out[i] = c ? 0.0 : a[i] - b[i];
  }
}
__global__ void k_b_fold(int64_t n, double* __restrict__ x, float* __restrict__ dx) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += double(dx[i]);
    dx[i] = 0.0f;
  }
}
__global__ void k_b_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(a[i]);
}
template <typename T>
__global__ void k_b_inv_diag(int64_t N, const double* __restrict__ diag_aos, const uint8_t* __restrict__ mask,
                             T* __restrict__ dinv) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 3 * N; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t d = i / N, v = i - d * N;
    const bool c = mask && ((mask[v] >> d) & 1);
    const double g = diag_aos[3 * v + d];
    dinv[i] = (c || g == 0.0) ? T(0) : T(1.0 / g);
  }
}
__global__ void k_b_scatter_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                               int64_t N, double* __restrict__ xd) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < nbc) xd[(dofs[i] % 3) * N + dofs[i] / 3] = vals[i];
}
__global__ void k_b_set_bc(int64_t nbc, const int32_t* __restrict__ dofs, const double* __restrict__ vals,
                           double* __restrict__ x) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < nbc) x[dofs[i]] = vals[i];
}

}  // namespace

// Batched mixed-precision Jacobi-PCG on a parted mesh; b and x_out interleaved.
pa_status solve_batched(Problem& P, const SolveOperator& op, const double* b, double* x_out,
                        const pa_solve_options& o, pa_solve_stats* st) {
  Mesh& m = *P.mesh;
  const int NP = m.num_parts;
  PA_CHECK(NP > 1 && NP <= kMaxParts, "batched solve needs a mesh with 2.." + std::to_string(kMaxParts) + " parts");
  PA_CHECK(o.method == PA_SOLVER_PCG_MIXED, "batched solves run in mixed precision (PA_SOLVER_PCG_MIXED)");
  PA_CHECK(o.rel_tol > 0.0, "rel_tol must be positive");
  PA_CHECK(op.w32 != nullptr && op.plas32 == nullptr, "batched solves serve the elastic operator");
  cudaStream_t s = P.stream;
  const int64_t n = P.ndof(), N = P.N();
  const int ag = apply_kernel_setup<float, 2>(m);
  const int grid_need = std::max(std::max(apply_kernel_setup<float, 1>(m), apply_kernel_setup<double, 1>(m)),
                                 bgrid(n));
  P.ws.ensure(n, P.C(), grid_need, true);
  SolverWorkspace& ws = P.ws;
  const int max_iters = o.max_iters > 0 ? o.max_iters : int(20.0 * std::sqrt(double(n)) + 1000);
  int chunk = o.check_every > 0 ? o.check_every : 64;
  chunk += chunk % 2;
  const double tol2 = o.rel_tol * o.rel_tol;
  const int vg = bgrid(n);
  const size_t sacc_bytes = sizeof(double) * 2 * NP;
  const uint8_t* mask = P.d_node_mask.get();
  const uint16_t* npart = m.d_node_part.get();
  const int64_t nbc = op.homogeneous_bc ? 0 : int64_t(P.bc_dofs.size());
  int64_t launches = 0;
  if (!P.ev0) { PA_CUDA(cudaEventCreate(&P.ev0)); PA_CUDA(cudaEventCreate(&P.ev1)); }
  cudaEvent_t t0;
  PA_CUDA(cudaEventCreate(&t0));
  PA_CUDA(cudaEventRecord(t0, s));

  DevBuf<PartScalars> psc(NP);
  DevBuf<double> pacc(2 * NP), norms(2 * NP);
  PA_CUDA(cudaMemsetAsync(pacc.get(), 0, sizeof(double) * 2 * NP, s));
  auto part_norm2 = [&](const double* v, std::vector<double>& outv) {
    PA_CUDA(cudaMemsetAsync(norms.get(), 0, sizeof(double) * 2 * NP, s));
    k_part_norm2<<<vg, kBT, sacc_bytes, s>>>(N, v, npart, NP, norms.get());
    PA_LAUNCHED();
    std::vector<double> h(2 * NP);
    PA_CUDA(cudaMemcpyAsync(h.data(), norms.get(), sizeof(double) * 2 * NP, cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    outv.resize(NP);
    for (int q = 0; q < NP; ++q) outv[q] = h[2 * q];
    launches += 1;
  };

  k_b_inv_diag<double><<<vg, kBT, 0, s>>>(N, op.diag_aos, mask, ws.dinv.get());
  k_b_inv_diag<float><<<vg, kBT, 0, s>>>(N, op.diag_aos, mask, ws.dinv32.get());
  PA_LAUNCHED();
  launch_pack4(N, ws.dinv32.get(), ws.dinv4.get(), s);
  launches += 2;
  double* bprime = ws.b.get();
  if (nbc) {
    PA_CUDA(cudaMemsetAsync(ws.p0.get(), 0, sizeof(double) * n, s));
    k_b_scatter_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), N, ws.p0.get());
    PA_LAUNCHED();
    launch_apply_tiled<double>(P, op.w64, ws.p0.get(), ws.t.get(), false, s);
    k_b_aos_minus_soa<<<vg, kBT, 0, s>>>(N, b, ws.t.get(), mask, bprime);
    launches += 3;
  } else {
    k_b_aos_minus_soa<<<vg, kBT, 0, s>>>(N, b, nullptr, nullptr, bprime);
    launches += 1;
  }
  PA_LAUNCHED();
  if (o.use_initial_guess) {
    k_b_aos_minus_soa<<<vg, kBT, 0, s>>>(N, x_out, nullptr, mask, ws.x.get());
    PA_LAUNCHED();
    launches += 1;
  } else {
    PA_CUDA(cudaMemsetAsync(ws.x.get(), 0, sizeof(double) * n, s));
  }
  std::vector<double> bb, rr;
  part_norm2(bprime, bb);
  for (double& v : bb)
    if (!(v > 0.0)) v = 1.0;
  auto true_residual = [&]() {
    launch_apply_tiled<double>(P, op.w64, ws.x.get(), ws.t.get(), true, s);
    k_b_sub_masked<<<vg, kBT, 0, s>>>(N, bprime, ws.t.get(), mask, ws.r.get());
    PA_LAUNCHED();
    launches += 3;
    part_norm2(ws.r.get(), rr);
  };
  true_residual();

  PA_CUDA(cudaMemsetAsync(ws.dx32.get(), 0, sizeof(float) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.p32a.get(), 0, sizeof(float) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.p32b.get(), 0, sizeof(float) * n, s));
  PA_CUDA(cudaMemsetAsync(ws.ap32.get(), 0, sizeof(float) * n, s));

  // graph: chunk x (fused apply in batched mode, batched update)
  auto args = [&](float* p_old, float* p_new) {
    ApplyArgs<float> a{};
    a.tv = m.tiles();
    a.N = N;
    a.coords = m.d_coords32_soa.get();
    a.coords4 = m.d_coords32_aos4.get();
    a.w = op.w32;
    a.tile_nodes = P.d_tile_nodes_bc.get();
    Iso<double> i64 = P.ep.iso();
    a.iso = Iso<float>{float(i64.lam), float(i64.mu)};
    a.x = p_old;
    a.y = ws.ap32.get();
    a.r = ws.r32.get();
    a.dinv = ws.dinv32.get();
    a.dinv4 = ws.dinv4.get();
    a.p_new = p_new;
    a.sc = ws.sc.get();
    a.partials = ws.partials.get();
    a.counter = ws.counters.get();
    a.tile_part = m.d_tile_part.get();
    a.psc = psc.get();
    a.pacc = pacc.get();
    a.num_parts = NP;
    return a;
  };
  const ApplyArgs<float> a_even = args(ws.p32a.get(), ws.p32b.get()), a_odd = args(ws.p32b.get(), ws.p32a.get());
  DevBuf<double> pacc2(2 * NP);
  PA_CUDA(cudaMemsetAsync(pacc2.get(), 0, sizeof(double) * 2 * NP, s));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  PA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < chunk; ++k) {
    launch_apply_kernel<float, 2>(m, ag, s, k % 2 == 0 ? a_even : a_odd);
    const float* pnew = (k % 2 == 0) ? ws.p32b.get() : ws.p32a.get();
    k_batch_update<<<vg, kBT, sacc_bytes, s>>>(N, ws.dx32.get(), ws.r32.get(), pnew, ws.ap32.get(), ws.dinv32.get(),
                                               npart, psc.get(), NP, pacc2.get(), ws.counters.get() + 1, ws.sc.get());
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

  const double hint = 0.25;
  std::vector<PartScalars> hp(NP);
  for (auto& q : hp) q = PartScalars{};
  std::vector<uint8_t> conv(NP, 0);
  int replacements = 0, global_iters = 0;
  bool first = true;
  while (true) {
    bool all = true;
    for (int q = 0; q < NP; ++q) {
      conv[q] = rr[q] <= tol2 * bb[q];
      all = all && conv[q];
    }
    if (all) break;
    int most = 0;
    for (int q = 0; q < NP; ++q) most = std::max(most, hp[q].iters);
    if (most >= max_iters) break;
    k_b_to_f32<<<vg, kBT, 0, s>>>(n, ws.r.get(), ws.r32.get());
    PA_LAUNCHED();
    for (int q = 0; q < NP; ++q) {
      PartScalars& ps = hp[q];
      ps.stop2 = hint * tol2 * bb[q];
      if (first || ps.breakdown) ps.beta = 0.0;  // (re)start the part's direction
      ps.done = conv[q] ? 1 : 0;
      ps.breakdown = 0;
    }
    PA_CUDA(cudaMemcpyAsync(psc.get(), hp.data(), sizeof(PartScalars) * NP, cudaMemcpyHostToDevice, s));
    PcgScalars gsc{};
    gsc.iters = global_iters;
    PA_CUDA(cudaMemcpyAsync(ws.sc.get(), &gsc, sizeof(gsc), cudaMemcpyHostToDevice, s));
    k_batch_init<<<vg, kBT, sacc_bytes, s>>>(N, ws.r32.get(), ws.dinv32.get(), npart, psc.get(), NP, pacc2.get(),
                                             ws.counters.get() + 1, ws.sc.get());
    PA_LAUNCHED();
    PA_CUDA(cudaGraphLaunch(exec, s));
    PcgScalars hs{};
    PA_CUDA(cudaMemcpyAsync(&hs, ws.sc.get(), sizeof(hs), cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaMemcpyAsync(hp.data(), psc.get(), sizeof(PartScalars) * NP, cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
    launches += 2 + 2LL * chunk;
    // newest p sits in p32b after an odd number of executed iterations
    if ((hs.iters - global_iters) % 2)
      PA_CUDA(cudaMemcpyAsync(ws.p32a.get(), ws.p32b.get(), sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    global_iters = hs.iters;
    k_b_fold<<<vg, kBT, 0, s>>>(n, ws.x.get(), ws.dx32.get());
    PA_LAUNCHED();
    first = false;
    true_residual();
    ++replacements;
  }

  launch_soa_to_aos<double, double>(ws.x.get(), x_out, N, s);
  launches += 1;
  if (nbc) {
    k_b_set_bc<<<int((nbc + 255) / 256), 256, 0, s>>>(nbc, P.d_bc_dofs.get(), P.d_bc_vals.get(), x_out);
    PA_LAUNCHED();
    launches += 1;
  }
  PA_CUDA(cudaEventRecord(P.ev1, s));
  PA_CUDA(cudaEventSynchronize(P.ev1));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, t0, P.ev1));
  cudaEventDestroy(t0);
  P.part_iterations.assign(NP, 0);
  P.part_rel_residual.assign(NP, 0.0);
  int most = 0;
  double worst = 0.0;
  bool all = true;
  for (int q = 0; q < NP; ++q) {
    P.part_iterations[q] = hp[q].iters;
    P.part_rel_residual[q] = std::sqrt(rr[q] / bb[q]);
    most = std::max(most, hp[q].iters);
    worst = std::max(worst, P.part_rel_residual[q]);
    all = all && rr[q] <= tol2 * bb[q];
  }
  if (st) {
    st->iterations = most;
    st->replacements = replacements;
    st->rel_residual = worst;
    st->seconds = ms * 1e-3;
    st->converged = all ? 1 : 0;
    st->kernel_launches = launches;
    st->fallback_iterations = 0;
  }
  if (!std::isfinite(worst)) return PA_ERR_NONFINITE;
  return all ? PA_OK : PA_ERR_NOT_CONVERGED;
}

}  // namespace pa
