// surrogate_rain.cuh — launch interface of the warm-rain kernel with the learned
// microphysics (surrogate_rain.cu).
#pragma once

#include <cstdint>

#include "dycore.cuh"
#include "surrogate.cuh"

namespace gwmb {

// Weights in the tensor cores' shared-memory operand layout (BF16, K-major, no swizzle):
// W1 [64 x 16], W2 and W3 [64 x 64], W4 [16 x 64] (5 outputs padded), 20480 bytes.
constexpr int kSurWeightBytes = 20480;
// Biases: b1 (64) b2 (64) b3 (64) b4 (5, padded to 8).
constexpr int kSurBias = 3 * kMlpHid + 8;

struct SurrogateArgs {
  const unsigned char* weights;  // kSurWeightBytes, 16-byte aligned
  const float* bias;             // kSurBias
  const float* norm;             // kMlpNorm: x mean/std, y mean/std
  const float* range;            // kMlpRange: x min/max of the training data
  float tol_water;               // fraction margin; |dqv_net - (e - c)| <= tol_water (|c| + |e| + dqv spread)
  float tol_energy;              // |dtheta_net - L/(cp pi)(c - e)| <= tol_energy (L/(cp pi)|c - e| + dtheta spread)
  // accumulated counters (kSurStats): cells that took the plain scheme after the network
  // ran, cells the network ran on, and per check the cells that failed it (input range,
  // fraction range, water, energy; a cell can fail several)
  unsigned long long* stats;
  int* work;                     // unit counter of the network kernel (zeroed before each launch)
  int* err;                      // error word: set to 1 when a bounded wait gave up
  // feature evaluation (launch_rain_net_eval): n rows of kMlpIn features in, the network's
  // kMlpOut outputs in physical units out (device arrays); unused by the warm-rain launch
  const float* eval_x;
  float* eval_y;
  long long eval_n;
};
constexpr int kSurStats = 6;

cudaError_t launch_warm_rain_surrogate(const RainArgs& a, const SurrogateArgs& s, cudaStream_t st);
// The same tensor-core network on s.eval_n feature rows (no gate, no checks, no cells):
// s.eval_y[row * kMlpOut + q] = output q of row, de-normalised.
cudaError_t launch_rain_net_eval(const SurrogateArgs& s, cudaStream_t st);

// Host: weights (FP32 parameter vector) -> the BF16 operand blob and FP32 biases.
void surrogate_operands(const float* params, unsigned char* weights, float* bias);

}  // namespace gwmb
