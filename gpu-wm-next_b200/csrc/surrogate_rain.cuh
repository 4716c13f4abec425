// surrogate_rain.cuh — launch interface of the warm-rain kernel with the learned
// microphysics (surrogate_rain.cu).
#pragma once

#include <cstdint>

#include "dycore.cuh"
#include "surrogate.cuh"

namespace gwmb {

// Weights as mma.sync B fragments, per lane: layer 1 (8), layers 2 and 3 (32 each),
// output layer (4) fragments of 32 lanes x (b0, b1) BF16 pairs.
constexpr int kSurFrags = 8 + 32 + 32 + 4;
// Biases: b1 (64) b2 (64) b3 (64) b4 (5, padded to 8).
constexpr int kSurBias = 3 * kMlpHid + 8;

struct SurrogateArgs {
  const uint2* frags;            // kSurFrags * 32
  const float* bias;             // kSurBias
  const float* norm;             // kMlpNorm: x mean/std, y mean/std
  const float* range;            // kMlpRange: x min/max of the training data
  float tol_water;               // fraction margin; |dqv_net - (e - c)| <= tol_water (|c| + |e| + dqv spread)
  float tol_energy;              // |dtheta_net - L/(cp pi)(c - e)| <= tol_energy (L/(cp pi)|c - e| + dtheta spread)
  // accumulated counters (kSurStats): cells that took the plain scheme after the network
  // ran, cells the network ran on, and per check the cells that failed it (input range,
  // fraction range, water, energy; a cell can fail several)
  unsigned long long* stats;
  int* work;                     // row counter of the network kernel (zeroed before each launch)
};
constexpr int kSurStats = 6;

cudaError_t launch_warm_rain_surrogate(const RainArgs& a, const SurrogateArgs& s, cudaStream_t st);

// Host: weights (FP32 parameter vector) -> BF16 B fragments and FP32 biases.
void surrogate_fragments(const float* params, uint2* frags, float* bias);

}  // namespace gwmb
