// scalar.cu — advance_scalar_ssprk3 (src/dycore/dry_transport.cu:285-325): SSPRK3 of a
// scalar field under a constant advection velocity with first-order upwind differences
// (upwind_stage_kernel, :13-37), on the global owned array (nz, ny, nx) in device memory.
//
// One kernel per stage with the stage's blend fused in (blend_stage_kernel, :39-46):
//   stage 1: q1 = L(q)
//   stage 2: q2 = 0.75 q + 0.25 L(q1)
//   stage 3: q  = 1/3 q + 2/3 L(q2)        (in place: each cell reads only its own q)
// with L(x) = x - dt (u dx/dx + v dx/dy).  The roundings are the reference build's: the
// divisions, fma(-dt, fma(u, dqx, v*dqy), q) for the stage and fma(wa, a, wb*b) for the
// blend (the contractions its compiler makes of the written expressions, identified on
// its golden vectors), written out so that no compiler choice can change them.  The
// stencil's halo is the periodic image, or zero beyond an open side: what the
// reference's halo exchange gives its virtual ranks (an absent neighbour sends zeros).
#include "../../include/gwm_b200.h"
#include "common.cuh"

namespace gwmb {
namespace {

struct ScalarStage {
  int nx, ny, nz, px, py;
  float u, v, dt, dx, dy;
  const float* in;
  const float* q0;  // blend partner (null: no blend)
  float* out;
  float wa, wb;
};

constexpr int kSX = 32, kSY = 8;

__global__ void __launch_bounds__(kSX * kSY) k_scalar_stage(const ScalarStage a) {
  const int i = blockIdx.x * kSX + threadIdx.x, j = blockIdx.y * kSY + threadIdx.y, k = blockIdx.z;
  if (i >= a.nx || j >= a.ny) return;
  const size_t plane = (size_t)a.nx * a.ny;
  const float* in = a.in + (size_t)k * plane;
  auto at = [&](int ii, int jj) -> float {
    if (ii < 0 || ii >= a.nx) {
      if (!a.px) return 0.0f;
      ii = ii < 0 ? ii + a.nx : ii - a.nx;
    }
    if (jj < 0 || jj >= a.ny) {
      if (!a.py) return 0.0f;
      jj = jj < 0 ? jj + a.ny : jj - a.ny;
    }
    return __ldg(in + (size_t)jj * a.nx + ii);
  };
  const float q = at(i, j);
  const float dqx = (a.u >= 0.0f) ? (q - at(i - 1, j)) / a.dx : (at(i + 1, j) - q) / a.dx;
  const float dqy = (a.v >= 0.0f) ? (q - at(i, j - 1)) / a.dy : (at(i, j + 1) - q) / a.dy;
  // the reference build's contractions of q - dt*(u*dqx + v*dqy) and wa*a + wb*b
  const float t = __fmaf_rn(-a.dt, __fmaf_rn(a.u, dqx, __fmul_rn(a.v, dqy)), q);
  const size_t o = (size_t)k * plane + (size_t)j * a.nx + i;
  a.out[o] = a.q0 ? __fmaf_rn(a.wa, a.q0[o], __fmul_rn(a.wb, t)) : t;
}

}  // namespace
}  // namespace gwmb

extern "C" int gwm_b200_scalar_ssprk3(const gwm_b200_scalar_desc* d, float* q, int nsteps, void* stream) {
  using namespace gwmb;
  if (!d || !q || d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || nsteps < 0 || d->nz > 65535 || !(d->dx > 0.0f) ||
      !(d->dy > 0.0f))
    return GWM_B200_ERR_ARG;
  if (nsteps == 0) return GWM_B200_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t n = (size_t)d->nx * d->ny * d->nz;
  float *q1 = nullptr, *q2 = nullptr;
  if (cudaMallocAsync(&q1, n * sizeof(float), s) != cudaSuccess) return GWM_B200_ERR_CUDA;
  if (cudaMallocAsync(&q2, n * sizeof(float), s) != cudaSuccess) {
    cudaFreeAsync(q1, s);
    return GWM_B200_ERR_CUDA;
  }
  ScalarStage a{d->nx, d->ny, d->nz, d->periodic_x, d->periodic_y, d->u_adv, d->v_adv, d->dt, d->dx, d->dy,
                nullptr, nullptr, nullptr, 0.0f, 0.0f};
  const dim3 block(kSX, kSY), grid((d->nx + kSX - 1) / kSX, (d->ny + kSY - 1) / kSY, d->nz);
  cudaError_t e = cudaSuccess;
  for (int step = 0; step < nsteps && e == cudaSuccess; ++step) {
    a.in = q; a.q0 = nullptr; a.out = q1;
    k_scalar_stage<<<grid, block, 0, s>>>(a);
    a.in = q1; a.q0 = q; a.out = q2; a.wa = 0.75f; a.wb = 0.25f;
    k_scalar_stage<<<grid, block, 0, s>>>(a);
    a.in = q2; a.q0 = q; a.out = q; a.wa = 1.0f / 3.0f; a.wb = 2.0f / 3.0f;
    k_scalar_stage<<<grid, block, 0, s>>>(a);
    e = cudaGetLastError();
  }
  cudaFreeAsync(q2, s);
  cudaFreeAsync(q1, s);
  if (e != cudaSuccess) return GWM_B200_ERR_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? GWM_B200_OK : GWM_B200_ERR_CUDA;
}
