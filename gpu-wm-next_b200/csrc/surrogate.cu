// surrogate.cu — training side of the learned warm-rain microphysics.
//
//  * k_rain_record_*: cell samples of the plain scheme (warm_rain.cu:36-120 through
//    rain_cell.cuh): features (T, p, rho_d, qv, qc, qr, dt) of a state and the targets
//    (the three process fractions, dtheta, dqv), written in cell order.
//  * mlp_loss_grad: mean squared error of the normalised targets and its exact gradient,
//    deterministic: one thread per sample for the forward and backward sweeps, then the
//    weight gradients as tiled products over fixed chunks of samples reduced in a
//    fixed order (no floating-point atomics).
//  * mlp_adam: the optimiser step.
// FP32 throughout; the inference kernel (surrogate_rain.cu) runs the same network in
// BF16 on the tensor cores.  GELU is the tanh form 0.5 z (1 + tanh(c (z + 0.044715 z^3))).
#include <algorithm>
#include <cstdint>

#include "surrogate.cuh"

namespace gwmb {
namespace {

constexpr int kChunk = 1024;  // samples per gradient partial

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Samples are written in cell order, whatever the thread schedule: pass 1 counts the
// kept cells of each block's contiguous cell range, a single thread turns the counts
// into offsets, and pass 2 writes each block's kept cells at its offset in order (a
// block-wide scan per 256 cells).  The training data, and so the trained network, are
// therefore reproducible run to run.
constexpr int kRecThreads = 256, kRecIters = 16, kRecCells = kRecThreads * kRecIters;

// The sample of cell q (global C order); returns whether it is kept.
__device__ __forceinline__ bool record_cell(const RecordArgs& a, long long q, float* x, float* t) {
  const RainArgs& r = a.r;
  const Geom& g = r.g;
  const MicroParams mp{r.dt, r.relax, r.thr, r.rate, r.evap, r.latent};
  const int i = (int)(q % g.nx);
  const long long rest = q / g.nx;
  const int j = (int)(rest % g.ny), k = (int)(rest / g.ny);
  const int o = gidx(g, i, j, k);
  const float rho_d = r.rho[o];
  const MicroCell c0 = micro_state(rho_d, r.rt[o], r.qv[o], r.qc[o], r.qr[o]);
  MicroCell c1 = c0;
  MicroRates pr;
  micro_step(c1, mp, &pr);
  rain_fractions(c0, pr, mp, t);
  t[3] = c1.th - c0.th;
  t[4] = c1.qv - c0.qv;
  const bool active = pr.cond != 0.0f || pr.autoconv != 0.0f || pr.rain_evap != 0.0f || t[3] != 0.0f || t[4] != 0.0f;
  const double u = (double)(mix64(a.seed ^ mix64((unsigned long long)q)) >> 11) * (1.0 / 9007199254740992.0);
  rain_features(c0, rho_d, r.dt, x);
  return u < (active ? a.p_active : a.p_inactive);
}

__global__ void __launch_bounds__(kRecThreads) k_rain_record_count(const RecordArgs a, long long n,
                                                                   unsigned* __restrict__ counts) {
  const long long q0 = (long long)blockIdx.x * kRecCells;
  unsigned c = 0;
  for (int it = 0; it < kRecIters; ++it) {
    const long long q = q0 + (long long)it * kRecThreads + threadIdx.x;
    float x[kMlpIn], t[kMlpOut];
    const bool keep = q < n && record_cell(a, q, x, t);
    c += (unsigned)__syncthreads_count(keep);
  }
  if (threadIdx.x == 0) counts[blockIdx.x] = c;
}

// Exclusive scan of the block counts (one block of 1024 threads, each over a
// contiguous segment); *total = all kept samples.
__global__ void __launch_bounds__(1024) k_rain_record_scan(const unsigned* __restrict__ counts, int nb,
                                                           unsigned long long* __restrict__ offsets,
                                                           unsigned long long* total) {
  __shared__ unsigned long long s[1024];
  const int per = (nb + 1023) / 1024;
  const int b0 = min(nb, (int)threadIdx.x * per), b1 = min(nb, b0 + per);
  unsigned long long sum = 0;
  for (int b = b0; b < b1; ++b) sum += counts[b];
  s[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (int q = 0; q < 1024; ++q) {
      const unsigned long long v = s[q];
      s[q] = run;
      run += v;
    }
    *total = run;
  }
  __syncthreads();
  unsigned long long run = s[threadIdx.x];
  for (int b = b0; b < b1; ++b) {
    offsets[b] = run;
    run += counts[b];
  }
}

__global__ void __launch_bounds__(kRecThreads) k_rain_record_write(const RecordArgs a, long long n,
                                                                   const unsigned long long* __restrict__ offsets) {
  __shared__ unsigned s_w[kRecThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long q0 = (long long)blockIdx.x * kRecCells;
  unsigned long long base = offsets[blockIdx.x];
  for (int it = 0; it < kRecIters; ++it) {
    const long long q = q0 + (long long)it * kRecThreads + threadIdx.x;
    float x[kMlpIn], t[kMlpOut];
    const bool keep = q < n && record_cell(a, q, x, t);
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) s_w[wid] = __popc(m);
    __syncthreads();
    unsigned before = __popc(m & ((1u << lane) - 1u)), all = 0;
    for (int w = 0; w < kRecThreads / 32; ++w) {
      const unsigned c = s_w[w];
      before += w < wid ? c : 0u;
      all += c;
    }
    const unsigned long long at = base + before;
    if (keep && (long long)at < a.capacity) {
#pragma unroll
      for (int f = 0; f < kMlpIn; ++f) a.x[at * kMlpIn + f] = x[f];
#pragma unroll
      for (int f = 0; f < kMlpOut; ++f) a.y[at * kMlpOut + f] = t[f];
    }
    base += all;
    __syncthreads();
  }
}

// ---- column statistics, FP64, fixed order
constexpr int kStatBlocks = 256;
__global__ void k_stats1(const float* __restrict__ a, long long n, int d, double* __restrict__ part) {
  // part[block][d][4]: sum, sum of squares, min, max
  __shared__ double s[256][4];
  for (int f = 0; f < d; ++f) {
    double sum = 0.0, sq = 0.0, mn = 1e300, mx = -1e300;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
      const double v = a[r * d + f];
      sum += v; sq += v * v; mn = fmin(mn, v); mx = fmax(mx, v);
    }
    s[threadIdx.x][0] = sum; s[threadIdx.x][1] = sq; s[threadIdx.x][2] = mn; s[threadIdx.x][3] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t0 = 0.0, t1 = 0.0, t2 = 1e300, t3 = -1e300;
      for (int q = 0; q < (int)blockDim.x; ++q) {
        t0 += s[q][0]; t1 += s[q][1]; t2 = fmin(t2, s[q][2]); t3 = fmax(t3, s[q][3]);
      }
      double* p = part + ((size_t)blockIdx.x * d + f) * 4;
      p[0] = t0; p[1] = t1; p[2] = t2; p[3] = t3;
    }
    __syncthreads();
  }
}
__global__ void k_stats2(const double* __restrict__ part, int nb, long long n, int d, double* out, double* rng) {
  for (int f = threadIdx.x; f < d; f += blockDim.x) {
    double t0 = 0.0, t1 = 0.0, t2 = 1e300, t3 = -1e300;
    for (int b = 0; b < nb; ++b) {
      const double* p = part + ((size_t)b * d + f) * 4;
      t0 += p[0]; t1 += p[1]; t2 = fmin(t2, p[2]); t3 = fmax(t3, p[3]);
    }
    const double mean = t0 / (double)n;
    const double var = fmax(t1 / (double)n - mean * mean, 0.0);
    out[f] = mean;
    out[d + f] = sqrt(var);
    if (rng) { rng[f] = t2; rng[d + f] = t3; }
  }
}

// ---- forward and backward sweeps, one thread per sample
constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2/pi)
__device__ __forceinline__ float gelu_t(float z, float& dg) {
  const float u = kGeluC * (z + 0.044715f * z * z * z);
  const float t = tanhf(u);
  dg = 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * 0.044715f * z * z);
  return 0.5f * z * (1.0f + t);
}

// scratch (feature-major, n samples): X0 (7) Z1 A1 Z2 A2 Z3 A3 (64 each) D1 D2 D3 (64 each)
// D4 (5), then the per-block loss partials
constexpr int kScrX0 = 0, kScrZ1 = kScrX0 + kMlpIn, kScrA1 = kScrZ1 + kMlpHid, kScrZ2 = kScrA1 + kMlpHid,
              kScrA2 = kScrZ2 + kMlpHid, kScrZ3 = kScrA2 + kMlpHid, kScrA3 = kScrZ3 + kMlpHid,
              kScrD1 = kScrA3 + kMlpHid, kScrD2 = kScrD1 + kMlpHid, kScrD3 = kScrD2 + kMlpHid,
              kScrD4 = kScrD3 + kMlpHid, kScrRows = kScrD4 + kMlpOut;
constexpr int kFbThreads = 128;

__global__ void __launch_bounds__(kFbThreads) k_mlp_fwd_bwd(const MlpBatch bt, double* loss_part) {
  __shared__ float w[kMlpParams];
  __shared__ float nrm[kMlpNorm];
  __shared__ double s_loss[kFbThreads];
  for (int q = threadIdx.x; q < kMlpParams; q += blockDim.x) w[q] = bt.params[q];
  for (int q = threadIdx.x; q < kMlpNorm; q += blockDim.x) nrm[q] = bt.norm[q];
  __syncthreads();
  const int n = bt.n;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (b < n) {
    float* S = bt.scratch;
    auto at = [&](int row) -> float& { return S[(size_t)row * n + b]; };
    const long long src = bt.index ? bt.index[b] : b;
    float in[kMlpHid];
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) {
      in[f] = (bt.x[src * kMlpIn + f] - nrm[f]) / nrm[kMlpIn + f];
      at(kScrX0 + f) = in[f];
    }
    // layer 1 (7 -> 64)
    for (int j = 0; j < kMlpHid; ++j) {
      float z = w[kOffB1 + j];
#pragma unroll
      for (int f = 0; f < kMlpIn; ++f) z += w[kOffW1 + j * kMlpIn + f] * in[f];
      float dg;
      at(kScrZ1 + j) = z;
      at(kScrA1 + j) = gelu_t(z, dg);
    }
    // layers 2 and 3 (64 -> 64)
    const int offw[2] = {kOffW2, kOffW3}, offb[2] = {kOffB2, kOffB3};
    const int rin[2] = {kScrA1, kScrA2}, rz[2] = {kScrZ2, kScrZ3}, ra[2] = {kScrA2, kScrA3};
    for (int L = 0; L < 2; ++L) {
#pragma unroll
      for (int f = 0; f < kMlpHid; ++f) in[f] = at(rin[L] + f);
      for (int j = 0; j < kMlpHid; ++j) {
        float z = w[offb[L] + j];
#pragma unroll
        for (int f = 0; f < kMlpHid; ++f) z += w[offw[L] + j * kMlpHid + f] * in[f];
        float dg;
        at(rz[L] + j) = z;
        at(ra[L] + j) = gelu_t(z, dg);
      }
    }
    // output layer (64 -> 5) and the loss gradient
#pragma unroll
    for (int f = 0; f < kMlpHid; ++f) in[f] = at(kScrA3 + f);
    float d4[kMlpOut];
#pragma unroll
    for (int o = 0; o < kMlpOut; ++o) {
      float y = w[kOffB4 + o];
#pragma unroll
      for (int f = 0; f < kMlpHid; ++f) y += w[kOffW4 + o * kMlpHid + f] * in[f];
      const float sd = nrm[2 * kMlpIn + kMlpOut + o];  // 0: a constant target, normalised to 0
      const float t = sd > 0.0f ? (bt.y[src * kMlpOut + o] - nrm[2 * kMlpIn + o]) / sd : 0.0f;
      const float e = y - t;
      l += (double)e * (double)e;
      d4[o] = 2.0f * e / ((float)n * (float)kMlpOut);
      at(kScrD4 + o) = d4[o];
    }
    // backward: delta3 = (W4^T d4) * gelu'(z3)
    float dnext[kMlpHid];
#pragma unroll
    for (int f = 0; f < kMlpHid; ++f) {
      float s = 0.0f;
#pragma unroll
      for (int o = 0; o < kMlpOut; ++o) s += w[kOffW4 + o * kMlpHid + f] * d4[o];
      float dg;
      gelu_t(at(kScrZ3 + f), dg);
      dnext[f] = s * dg;
      at(kScrD3 + f) = dnext[f];
    }
    // delta2 = (W3^T delta3) * gelu'(z2); delta1 = (W2^T delta2) * gelu'(z1)
    const int bw[2] = {kOffW3, kOffW2}, bz[2] = {kScrZ2, kScrZ1}, bd[2] = {kScrD2, kScrD1};
    for (int L = 0; L < 2; ++L) {
      float dcur[kMlpHid];
      for (int f = 0; f < kMlpHid; ++f) {
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < kMlpHid; ++j) s += w[bw[L] + j * kMlpHid + f] * dnext[j];
        float dg;
        gelu_t(at(bz[L] + f), dg);
        dcur[f] = s * dg;
        at(bd[L] + f) = dcur[f];
      }
#pragma unroll
      for (int f = 0; f < kMlpHid; ++f) dnext[f] = dcur[f];
    }
  }
  s_loss[threadIdx.x] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)blockDim.x; ++q) t += s_loss[q];
    loss_part[blockIdx.x] = t;
  }
}

// Gradient of one layer over one chunk of samples: part[o][i] = sum_b D[o][b] A[i][b]
// (i < I) and part[o][I] = sum_b D[o][b], for O <= 64 outputs and I <= 64 inputs.
__global__ void __launch_bounds__(256) k_mlp_grad_chunk(const float* __restrict__ S, int n, int rowD, int O,
                                                       int rowA, int I, int off_w, int off_b,
                                                       float* __restrict__ partial) {
  __shared__ float Ds[64][33], As[65][33];
  const int c = blockIdx.x;
  const int b0 = c * kChunk, b1 = min(n, b0 + kChunk);
  const int t = threadIdx.x, o = t & 63, jg = t >> 6;  // 4 groups of input columns
  float acc[17];
#pragma unroll
  for (int q = 0; q < 17; ++q) acc[q] = 0.0f;
  for (int s0 = b0; s0 < b1; s0 += 32) {
    const int m = min(32, b1 - s0);
    for (int q = t; q < 64 * 32; q += 256) {
      const int r = q >> 5, sidx = q & 31;
      Ds[r][sidx] = (r < O && sidx < m) ? S[(size_t)(rowD + r) * n + s0 + sidx] : 0.0f;
    }
    for (int q = t; q < 65 * 32; q += 256) {
      const int r = q >> 5, sidx = q & 31;
      float v = 0.0f;
      if (sidx < m) v = r < I ? S[(size_t)(rowA + r) * n + s0 + sidx] : (r == I ? 1.0f : 0.0f);
      As[r][sidx] = v;
    }
    __syncthreads();
    for (int sidx = 0; sidx < 32; ++sidx) {
      const float d = Ds[o][sidx];
#pragma unroll
      for (int q = 0; q < 17; ++q) {
        const int i = jg * 17 + q;
        if (i <= 64) acc[q] += d * As[i][sidx];
      }
    }
    __syncthreads();
  }
  if (o < O) {
#pragma unroll
    for (int q = 0; q < 17; ++q) {
      const int i = jg * 17 + q;
      if (i < I) partial[(size_t)c * kMlpParams + off_w + o * I + i] = acc[q];
      else if (i == I) partial[(size_t)c * kMlpParams + off_b + o] = acc[q];
    }
  }
}

__global__ void k_mlp_grad_reduce(const float* __restrict__ partial, int chunks, float* __restrict__ grad,
                                  const double* __restrict__ loss_part, int nlb, double* loss, double inv) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) {
    float s = 0.0f;
    for (int c = 0; c < chunks; ++c) s += partial[(size_t)c * kMlpParams + p];
    grad[p] = s;
  }
  if (p == 0 && loss) {
    double t = 0.0;
    for (int q = 0; q < nlb; ++q) t += loss_part[q];
    *loss = t * inv;
  }
}

__global__ void k_mlp_adam(float* params, const float* grad, float* m, float* v, float lr, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const float g = grad[p];
  const float mm = 0.9f * m[p] + 0.1f * g;
  const float vv = 0.999f * v[p] + 0.001f * g * g;
  m[p] = mm;
  v[p] = vv;
  params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + 1.0e-8f);
}

}  // namespace

cudaError_t launch_rain_record(const RecordArgs& a, cudaStream_t s) {
  const long long n = (long long)a.r.g.nx * a.r.g.ny * a.r.g.nz;
  const long long nb = (n + kRecCells - 1) / kRecCells;
  if (nb > (1LL << 30)) return cudaErrorInvalidValue;
  unsigned* counts = nullptr;
  unsigned long long* offsets = nullptr;
  cudaError_t e = cudaMallocAsync(&counts, (size_t)nb * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  e = cudaMallocAsync(&offsets, (size_t)nb * sizeof(unsigned long long), s);
  if (e != cudaSuccess) { cudaFreeAsync(counts, s); return e; }
  k_rain_record_count<<<(unsigned)nb, kRecThreads, 0, s>>>(a, n, counts);
  k_rain_record_scan<<<1, 1024, 0, s>>>(counts, (int)nb, offsets, a.count);
  k_rain_record_write<<<(unsigned)nb, kRecThreads, 0, s>>>(a, n, offsets);
  e = cudaGetLastError();
  cudaFreeAsync(offsets, s);
  cudaFreeAsync(counts, s);
  return e;
}

cudaError_t mlp_column_stats(const float* a, long long n, int d, double* out, double* rng, cudaStream_t s) {
  double* part = nullptr;
  cudaError_t e = cudaMallocAsync(&part, (size_t)kStatBlocks * d * 4 * sizeof(double), s);
  if (e != cudaSuccess) return e;
  k_stats1<<<kStatBlocks, 256, 0, s>>>(a, n, d, part);
  k_stats2<<<1, 32, 0, s>>>(part, kStatBlocks, n, d, out, rng);
  e = cudaGetLastError();
  cudaFreeAsync(part, s);
  return e;
}

size_t mlp_scratch_floats(int n) { return (size_t)kScrRows * n; }
size_t mlp_partial_floats(int n) {
  const size_t chunks = (size_t)(n + kChunk - 1) / kChunk;
  return chunks * kMlpParams + 2 * ((size_t)(n + kFbThreads - 1) / kFbThreads) + 16;
}

cudaError_t mlp_loss_grad(const MlpBatch& bt, cudaStream_t s) {
  if (bt.n <= 0) return cudaErrorInvalidValue;
  const int chunks = (bt.n + kChunk - 1) / kChunk;
  const int nlb = (bt.n + kFbThreads - 1) / kFbThreads;
  // loss partials live after the gradient partials (8-byte aligned: chunks*kMlpParams + pad)
  size_t off = (size_t)chunks * kMlpParams;
  off = (off + 1) & ~size_t(1);
  double* loss_part = reinterpret_cast<double*>(bt.partial + off);
  k_mlp_fwd_bwd<<<nlb, kFbThreads, 0, s>>>(bt, loss_part);
  // (layer: delta rows, outputs, activation rows, inputs, weight and bias offsets)
  k_mlp_grad_chunk<<<chunks, 256, 0, s>>>(bt.scratch, bt.n, kScrD1, kMlpHid, kScrX0, kMlpIn, kOffW1, kOffB1, bt.partial);
  k_mlp_grad_chunk<<<chunks, 256, 0, s>>>(bt.scratch, bt.n, kScrD2, kMlpHid, kScrA1, kMlpHid, kOffW2, kOffB2, bt.partial);
  k_mlp_grad_chunk<<<chunks, 256, 0, s>>>(bt.scratch, bt.n, kScrD3, kMlpHid, kScrA2, kMlpHid, kOffW3, kOffB3, bt.partial);
  k_mlp_grad_chunk<<<chunks, 256, 0, s>>>(bt.scratch, bt.n, kScrD4, kMlpOut, kScrA3, kMlpHid, kOffW4, kOffB4, bt.partial);
  k_mlp_grad_reduce<<<(kMlpParams + 255) / 256, 256, 0, s>>>(bt.partial, chunks, bt.grad, loss_part, nlb, bt.loss,
                                                              1.0 / ((double)bt.n * kMlpOut));
  return cudaGetLastError();
}

cudaError_t mlp_adam(float* params, const float* grad, float* m, float* v, float lr, int t, cudaStream_t s) {
  const float c1 = 1.0f - powf(0.9f, (float)t), c2 = 1.0f - powf(0.999f, (float)t);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, c1, c2);
  return cudaGetLastError();
}

}  // namespace gwmb
