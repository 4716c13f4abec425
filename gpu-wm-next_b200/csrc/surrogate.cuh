// surrogate.cuh — the learned warm-rain microphysics: an MLP (T, p, rho_d, qv, qc, qr, dt)
// -> (f_cond, f_auto, f_evap, dtheta, dqv) with three 64-wide GELU hidden layers, trained
// on cell samples of the plain scheme by the kernels of surrogate.cu and run with BF16
// tensor-core inference inside the warm-rain column sweep.  The first three outputs are
// the condensation, autoconversion and rain-evaporation amounts as fractions of what
// bounds them (rain_fractions); the amounts move water between vapour, cloud and rain,
// so the water budget closes by construction.  dtheta and dqv are redundant outputs
// that the inference checks against the latent heating and the vapour change the
// amounts imply.
#pragma once

#include "physics.cuh"
#include "rain_cell.cuh"

namespace gwmb {

// Parameter vector (FP32): W1 (64x7) b1 (64) W2 (64x64) b2 (64) W3 (64x64) b3 (64)
// W4 (5x64) b4 (5), weights row-major as [out][in].
constexpr int kMlpIn = 7, kMlpHid = 64, kMlpOut = 5;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpHid * kMlpIn, kOffW2 = kOffB1 + kMlpHid,
              kOffB2 = kOffW2 + kMlpHid * kMlpHid, kOffW3 = kOffB2 + kMlpHid,
              kOffB3 = kOffW3 + kMlpHid * kMlpHid, kOffW4 = kOffB3 + kMlpHid,
              kOffB4 = kOffW4 + kMlpOut * kMlpHid, kMlpParams = kOffB4 + kMlpOut;
// Normalisation vector: x_mean (7) x_std (7) y_mean (5) y_std (5); input range x_min (7) x_max (7).
constexpr int kMlpNorm = 2 * kMlpIn + 2 * kMlpOut, kMlpRange = 2 * kMlpIn;

// Training samples of the plain scheme at the cells of one state.
struct RecordArgs {
  RainArgs r;                       // the state and the warm-rain configuration
  float* x;                         // (capacity, 7) features
  float* y;                         // (capacity, 5) targets: f_cond, f_auto, f_evap, dtheta, dqv
  unsigned long long* count;
  long long capacity;
  unsigned long long seed;
  float p_active, p_inactive;       // keep probabilities of active / inactive cells
};
cudaError_t launch_rain_record(const RecordArgs& a, cudaStream_t s);

// Statistics (FP64, fixed order) of an (n, d) array: out[2*d] = mean (d), std (d);
// rng[2*d] = min (d), max (d) (null: skipped).
cudaError_t mlp_column_stats(const float* a, long long n, int d, double* out, double* rng, cudaStream_t s);

struct MlpBatch {
  const float* params;   // device, kMlpParams
  const float* norm;     // device, kMlpNorm
  const float* x;        // device (n, 7) raw features
  const float* y;        // device (n, 5) raw targets
  const int* index;      // device sample indices of the batch (null: 0..n-1)
  int n;
  float* scratch;        // device: activations and deltas, mlp_scratch_floats(n)
  float* partial;        // device: mlp_partial_floats(n)
  float* grad;           // device, kMlpParams: gradient of the mean loss
  double* loss;          // device, 1 value: mean squared error of the normalised targets
};
size_t mlp_scratch_floats(int n);
size_t mlp_partial_floats(int n);
cudaError_t mlp_loss_grad(const MlpBatch& b, cudaStream_t s);
// Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on params with moments m, v.
cudaError_t mlp_adam(float* params, const float* grad, float* m, float* v, float lr, int t, cudaStream_t s);

}  // namespace gwmb
