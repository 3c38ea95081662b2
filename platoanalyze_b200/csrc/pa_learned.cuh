// pa_learned.cuh -- the learned preconditioner behind pa_pc* (not part of the ABI).
#pragma once
#include "pa_problem.cuh"

namespace pa {

struct LearnedPC;

// Network: four 3x3x3 convolutions on the nodal grid of a structured box,
// 5 -> 32 -> 32 -> 32 -> 3 channels, ReLU after the first three.
constexpr int kPcLayers = 4;
int64_t pc_num_params();

LearnedPC* pc_new(int gx, int gy, int gz, uint64_t seed);
void pc_delete(LearnedPC* pc);
int pc_device(const LearnedPC& pc);
int64_t pc_grid_points(const LearnedPC& pc);
cudaStream_t pc_stream(const LearnedPC& pc);
// Throws unless the mesh's nodes are the grid points in x-fastest order.
void pc_check_grid(const LearnedPC& pc, const Mesh& m);

void pc_set_params(LearnedPC& pc, const float* d_params, cudaStream_t s);
void pc_get_params(const LearnedPC& pc, float* d_params, cudaStream_t s);
// Network on caller features (G x 5 FP32, rounded to BF16 at the input) -> G x 3 FP32.
void pc_forward_features(LearnedPC& pc, const float* d_feat, float* d_out, cudaStream_t s);
// Average device time of the four convolutions (ms) on the current layer-1
// input, and their algorithmic FLOPs (real channel counts).
double pc_time_forward(LearnedPC& pc, int reps);
int64_t pc_forward_flops(const LearnedPC& pc);
// d(sum gout . out)/d(params) for the same features (forward included).
void pc_backward_features(LearnedPC& pc, const float* d_feat, const float* d_gout, float* d_gparams, cudaStream_t s);
// out = M r for density z (interleaved vectors, device).
void pc_apply(LearnedPC& pc, Problem& P, const double* z, const double* r_aos, double* out_aos);

struct PcTrainSet {
  int32_t num_densities = 0, num_samples = 0;
  const double* densities = nullptr;      // device, num_densities x nz
  const double* residuals = nullptr;      // device, num_samples x 3N interleaved
  std::vector<int32_t> sample_density;    // host
  std::vector<double> sample_energy;      // host, e . r per sample
};
void pc_train(LearnedPC& pc, Problem& P, const PcTrainSet& set, const pa_pc_train_options& o, pa_pc_train_stats* st);

// Pieces the flexible-CG solver uses: D^-1 (SoA, into dinv_out), D^-1/2 and
// the node features from the interleaved diagonal; the network on residual r
// (SoA) with r.D^-1 r at *rdr, output G x 4 at pc_output (skipped while *done).
void pc_prepare_operator(LearnedPC& pc, Problem& P, const double* diag_aos, float* dinv_out, cudaStream_t s);
template <typename T>
void pc_launch_network(LearnedPC& pc, const T* r, const double* rdr, double inv_nfree, const int32_t* done,
                       cudaStream_t s);
constexpr int kPcNetworkLaunches = 1 + kPcLayers;
const float* pc_output(const LearnedPC& pc);
const float* pc_dsq(const LearnedPC& pc);
void pc_check_error(LearnedPC& pc, cudaStream_t s);
int64_t free_dofs(const Problem& P);

pa_status solve_fcg(Problem& P, const SolveOperator& op, LearnedPC& pc, const double* b, double* x_out,
                    const pa_solve_options& o, pa_solve_stats* st);

}  // namespace pa
