// halo.cu — owned<->padded packing, the reference's virtual-rank halo exchange
// as device kernels, EOS pressure and deterministic FP64 reductions.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <mutex>

#include <cuda.h>

#include "../../include/gwm_b200.h"
#include "halo.cuh"

namespace gwmb {
namespace {

__device__ __forceinline__ void owned_shape(const Geom& g, int o, int& fx, int& fy, int& fz) {
  fx = g.nx + (o == kFaceX);
  fy = g.ny + (o == kFaceY);
  fz = g.nz + (o == kFaceZ);
}

__global__ void k_pack(const Geom g, int o, const float* __restrict__ src, float* __restrict__ dst) {
  int fx, fy, fz;
  owned_shape(g, o, fx, fy, fz);
  const long long n = (long long)fx * fy * fz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % fx);
    const long long r = q / fx;
    const int j = (int)(r % fy);
    const int k = (int)(r / fy);
    float v = src[q];
    if (o == kFaceX && g.per_x && (i == 0 || i == g.nx)) {
      const long long row = q - i;
      v = 0.5f * (src[row] + src[row + g.nx]);
    }
    if (o == kFaceY && g.per_y && (j == 0 || j == g.ny)) {
      const long long col = q - (long long)j * fx;
      v = 0.5f * (src[col] + src[col + (long long)g.ny * fx]);
    }
    store_mirrored(dst, g, o, i, j, k, v);
  }
}

// Boundary strips.  Compact index q of a field with owned shape (fx, fy, fz):
// west/east strips hold (j, k) at q = side*fy*fz + k*fy + j, south/north strips hold
// (i, k) at q = 2*fy*fz + (side-2)*fx*fz + k*fx + i.
__device__ __forceinline__ void strip_pos(const Geom& g, int o, long long q, int& side, int& i, int& j,
                                          int& k) {
  int fx, fy, fz;
  owned_shape(g, o, fx, fy, fz);
  const long long ew = (long long)fy * fz;
  if (q < 2 * ew) {
    side = (int)(q / ew);
    const long long r = q - side * ew;
    k = (int)(r / fy);
    j = (int)(r - (long long)k * fy);
    i = side == 0 ? 0 : fx - 1;
  } else {
    const long long ns = (long long)fx * fz;
    const long long r0 = q - 2 * ew;
    side = 2 + (int)(r0 / ns);
    const long long r = r0 - (side - 2) * ns;
    k = (int)(r / fx);
    i = (int)(r - (long long)k * fx);
    j = side == 2 ? 0 : fy - 1;
  }
}

__global__ void k_strips(const Geom g, const StripJobs jobs) {
  const StripJob& jb = jobs.j[blockIdx.y];
  const int o = jb.orient;
  int fx, fy, fz;
  owned_shape(g, o, fx, fy, fz);
  const long long n = 2LL * fz * (fx + fy);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    int side, i, j, k;
    strip_pos(g, o, q, side, i, j, k);
    const bool open = side < 2 ? !g.per_x : !g.per_y;
    switch (jb.mode) {
      case 0:
        if (open) store_mirrored(jb.padded, g, o, i, j, k, jb.compact[q]);
        break;
      case 1:
        jb.compact[q] = jb.padded[gidx(g, i, j, k)];
        break;
      case 2: {
        const long long at = ((long long)k * fy + j) * fx + i;
        float v = jb.aux[at];
        if (o == kFaceX && g.per_x && (i == 0 || i == g.nx)) v = 0.5f * (jb.aux[at - i] + jb.aux[at - i + g.nx]);
        if (o == kFaceY && g.per_y && (j == 0 || j == g.ny)) {
          const long long col = at - (long long)j * fx;
          v = 0.5f * (jb.aux[col] + jb.aux[col + (long long)g.ny * fx]);
        }
        jb.compact[q] = v;
        break;
      }
      case 3:
        if (open) store_mirrored(jb.padded, g, o, i, j, k, theta_of(jb.aux[q], jb.compact[q]));
        break;
      case 4:
        if (open) store_mirrored(jb.padded, g, o, i, j, k, 0.0f);
        break;
    }
  }
}

__global__ void k_unpack(const Geom g, int o, const float* __restrict__ src, float* __restrict__ dst) {
  int fx, fy, fz;
  owned_shape(g, o, fx, fy, fz);
  const long long n = (long long)fx * fy * fz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % fx);
    const long long r = q / fx;
    const int j = (int)(r % fy);
    const int k = (int)(r / fy);
    dst[q] = src[gidx(g, i, j, k)];
  }
}

// Reference per-rank storage index: field3d.hpp:49-54
struct RankView {
  int ox, oy, oz, h;  // owned extents of this orientation, halo
  float* d;
  __device__ __forceinline__ float& at(int i, int j, int k) const {
    return d[((long long)k * (oy + 2 * h) + (j + h)) * (ox + 2 * h) + (i + h)];
  }
};

__device__ __forceinline__ RankView view(const RankTable& t, int r) {
  RankView v;
  v.ox = t.r[r].nxl + (t.orient == kFaceX);
  v.oy = t.r[r].nyl + (t.orient == kFaceY);
  v.oz = t.nz + (t.orient == kFaceZ);
  v.h = t.halo;
  v.d = t.r[r].data;
  return v;
}

// x phase: pack_face_x_faces_impl / pack_scalar_x_faces + unpack (halo_exchange.cpp:32-73, 313-342)
__global__ void k_rank_x(const RankTable t) {
  const int r = blockIdx.y;
  const RankView me = view(t, r);
  const int h = t.halo;
  const long long n = (long long)me.oz * me.oy * h * 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int side = (int)(q & 1);
    long long rr = q >> 1;
    const int hh = (int)(rr % h);
    rr /= h;
    const int j = (int)(rr % me.oy);
    const int k = (int)(rr / me.oy);
    if (side == 0) {  // west halo <- west neighbour's east send
      const int w = t.r[r].west;
      float v = 0.0f;
      if (w >= 0) {
        const RankView nb = view(t, w);
        const int ei = (t.orient == kFaceX) ? t.r[w].nxl - h + hh : nb.ox - h + hh;
        v = nb.at(ei, j, k);
      }
      me.at(-h + hh, j, k) = v;
    } else {  // east halo <- east neighbour's west send
      const int e = t.r[r].east;
      float v = 0.0f;
      if (e >= 0) {
        const RankView nb = view(t, e);
        const int wi = (t.orient == kFaceX) ? 1 + hh : hh;
        v = nb.at(wi, j, k);
      }
      me.at(me.ox + hh, j, k) = v;
    }
  }
}

// y phase over i in [-h, ox+h): pack_face_y_faces_impl / pack_scalar_y_faces + unpack
// (halo_exchange.cpp:75-116, 344-373)
__global__ void k_rank_y(const RankTable t) {
  const int r = blockIdx.y;
  const RankView me = view(t, r);
  const int h = t.halo;
  const int wx = me.ox + 2 * h;
  const long long n = (long long)me.oz * h * wx * 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int side = (int)(q & 1);
    long long rr = q >> 1;
    const int i = (int)(rr % wx) - h;
    rr /= wx;
    const int hh = (int)(rr % h);
    const int k = (int)(rr / h);
    if (side == 0) {
      const int s = t.r[r].south;
      float v = 0.0f;
      if (s >= 0) {
        const RankView nb = view(t, s);
        const int nj = (t.orient == kFaceY) ? t.r[s].nyl - h + hh : nb.oy - h + hh;
        v = nb.at(i, nj, k);
      }
      me.at(i, -h + hh, k) = v;
    } else {
      const int nn = t.r[r].north;
      float v = 0.0f;
      if (nn >= 0) {
        const RankView nb = view(t, nn);
        const int sj = (t.orient == kFaceY) ? 1 + hh : hh;
        v = nb.at(i, sj, k);
      }
      me.at(i, me.oy + hh, k) = v;
    }
  }
}

// synchronize_face_owned_interfaces_impl (halo_exchange.cpp:249-284)
__global__ void k_rank_sync(const RankTable t) {
  const int r = blockIdx.y;
  const RankView me = view(t, r);
  if (t.orient == kFaceX) {
    const int e = t.r[r].east;
    if (!(e >= 0 && (r < e || e == r))) return;
    const RankView nb = view(t, e);
    const int nyl = t.r[r].nyl, nxl = t.r[r].nxl;
    const long long n = (long long)me.oz * nyl;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
      const int j = (int)(q % nyl), k = (int)(q / nyl);
      const float avg = 0.5f * (me.at(nxl, j, k) + nb.at(0, j, k));
      me.at(nxl, j, k) = avg;
      nb.at(0, j, k) = avg;
    }
  } else if (t.orient == kFaceY) {
    const int nn = t.r[r].north;
    if (!(nn >= 0 && (r < nn || nn == r))) return;
    const RankView nb = view(t, nn);
    const int nyl = t.r[r].nyl, nxl = t.r[r].nxl;
    const long long n = (long long)me.oz * nxl;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
      const int i = (int)(q % nxl), k = (int)(q / nxl);
      const float avg = 0.5f * (me.at(i, nyl, k) + nb.at(i, 0, k));
      me.at(i, nyl, k) = avg;
      nb.at(i, 0, k) = avg;
    }
  }
}

__global__ void k_pressure(const float* rho, const float* rt, float* p, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    p[q] = eos_pressure(rho[q], rt[q]);
}

__device__ __forceinline__ void block_reduce3(double& s, double& mn, double& mx) {
  __shared__ double sh[3][32];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (l == 0) { sh[0][w] = s; sh[1][w] = mn; sh[2][w] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    s = 0.0; mn = DBL_MAX; mx = -DBL_MAX;
    for (int q = 0; q < nw; ++q) { s += sh[0][q]; mn = fmin(mn, sh[1][q]); mx = fmax(mx, sh[2][q]); }
  }
}

__global__ void __launch_bounds__(256) k_reduce_pass1(const Geom g, int o, int mode, const float* f,
                                                      const float* rho, const float* idz,
                                                      int idz_terrain, double* part) {
  int fx, fy, fz;
  owned_shape(g, o, fx, fy, fz);
  const long long n = (long long)fx * fy * fz;
  double s = 0.0, mn = DBL_MAX, mx = -DBL_MAX;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % fx);
    const long long r = q / fx;
    const int j = (int)(r % fy);
    const int k = (int)(r / fy);
    const int a = gidx(g, i, j, k);
    double v = (double)f[a];
    if (mode == 1) v = v / fmax((double)rho[a], 1.0e-12);
    if (mode == 2) v = v * (1.0 / (double)(idz_terrain ? idz[a] : idz[k]));
    s += v;
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  block_reduce3(s, mn, mx);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s;
    part[gridDim.x + blockIdx.x] = mn;
    part[2 * gridDim.x + blockIdx.x] = mx;
  }
}

// mode 0: the value a + b; 1: 1 where a + b > 0, else 0 (a count of positive cells)
__global__ void k_reduce_2d_pass1(const double* a, const double* b, long long n, double* part, int mode) {
  double s = 0.0, mn = DBL_MAX, mx = -DBL_MAX;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    double v = a[q] + (b ? b[q] : 0.0);
    if (mode == 1) v = v > 0.0 ? 1.0 : 0.0;
    s += v;
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  block_reduce3(s, mn, mx);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s;
    part[gridDim.x + blockIdx.x] = mn;
    part[2 * gridDim.x + blockIdx.x] = mx;
  }
}

__global__ void k_reduce_pass2(const double* part, int nb, ReduceOut* out) {
  double s = 0.0, mn = DBL_MAX, mx = -DBL_MAX;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) {
    s += part[q];
    mn = fmin(mn, part[nb + q]);
    mx = fmax(mx, part[2 * nb + q]);
  }
  block_reduce3(s, mn, mx);
  if (threadIdx.x == 0) { out->sum = s; out->mn = mn; out->mx = mx; }
}

// Allocation-free field statistics: the per-block partials live in a fixed
// device array of this file instead of caller- or context-allocated memory.
constexpr int kNoAllocBlocks = 1024;  // 3 x 1024 doubles = 24 KiB per device
static __device__ __align__(256) double g_noalloc_partials[3 * kNoAllocBlocks];

__global__ void __launch_bounds__(256) k_stats_pass1(const float* __restrict__ x, long long n,
                                                     double* part) {
  double s = 0.0, mn = DBL_MAX, mx = -DBL_MAX;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const double v = (double)x[q];
    s += v;
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  block_reduce3(s, mn, mx);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s;
    part[gridDim.x + blockIdx.x] = mn;
    part[2 * gridDim.x + blockIdx.x] = mx;
  }
}

inline int blocks_for(long long n, int per) {
  long long b = (n + per - 1) / per;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

}  // namespace

cudaError_t launch_pack(const Geom& g, int orient, const float* src, float* dst, cudaStream_t s) {
  const long long n = (long long)(g.nx + (orient == kFaceX)) * (g.ny + (orient == kFaceY)) *
                      (g.nz + (orient == kFaceZ));
  k_pack<<<blocks_for(n, 256), 256, 0, s>>>(g, orient, src, dst);
  return cudaGetLastError();
}

long long strip_len(const Geom& g, int orient) {
  const long long fx = g.nx + (orient == kFaceX), fy = g.ny + (orient == kFaceY), fz = g.nz + (orient == kFaceZ);
  return 2 * fz * (fx + fy);
}

cudaError_t launch_strips(const Geom& g, const StripJobs& jobs, cudaStream_t s) {
  if (jobs.n <= 0) return cudaSuccess;
  if (jobs.n > kMaxStripJobs) return cudaErrorInvalidValue;
  long long n = 0;
  for (int t = 0; t < jobs.n; ++t) n = std::max(n, strip_len(g, jobs.j[t].orient));
  const int bx = (int)std::min<long long>((n + 255) / 256, 1024);
  k_strips<<<dim3(bx, jobs.n), 256, 0, s>>>(g, jobs);
  return cudaGetLastError();
}

// BoundaryCacheIR::bracket (include/gwm/ingest/boundary_cache.hpp:52-76) and the
// weight of interpolate_boundary_snapshot (src/ingest/runtime_case.cpp:205-221) for the
// three updater calls of a step, then the next step's start time.
__global__ void k_boundary_clock(BoundaryClock* c, const int* __restrict__ off, int n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const float t0 = c->t_start, dt = c->dt;
  const float sim[3] = {0.0f, dt, 0.5f * dt};  // dry_core.cu:568, 591, 620
  for (int s = 0; s < 3; ++s) {
    const int t = (int)lroundf(t0 + sim[s]);  // prepared_case_init.cpp:403-404
    int lo = -1, hi = -1;
    for (int q = 0; q < n; ++q) {
      if (off[q] <= t) lo = q;
      if (off[q] >= t) { hi = q; break; }
    }
    if (lo < 0) lo = 0;
    if (hi < 0) hi = n - 1;
    float a = 0.0f;
    if (lo != hi && off[lo] != off[hi]) a = (float)(t - off[lo]) / (float)(off[hi] - off[lo]);
    else hi = lo;  // the lower snapshot itself
    c->lo[s] = lo;
    c->hi[s] = hi;
    c->alpha[s] = a;
  }
  c->t_start = t0 + dt;
}

// (1 - alpha) lower + alpha upper as interpolate_bundle writes it (runtime_case.cpp:113),
// without contraction; tracer strips become rho_d * q (prepared_case_init.cpp:590).
__global__ void k_boundary_interp(const float* __restrict__ cache, long long per_snap, long long dry_len,
                                  long long cell_len, int ntr, const BoundaryClock* __restrict__ c, int stage,
                                  float* __restrict__ out) {
  const int lo = c->lo[stage], hi = c->hi[stage];
  const float a = c->alpha[stage], b = 1.0f - a;
  const float* L = cache + lo * per_snap;
  const float* H = cache + hi * per_snap;
  auto lerp = [&](long long e) { return lo == hi ? L[e] : __fadd_rn(__fmul_rn(b, L[e]), __fmul_rn(a, H[e])); };
  const long long n = dry_len + (long long)ntr * cell_len;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    if (e < dry_len) {
      out[e] = lerp(e);
    } else {
      const long long r = (e - dry_len) % cell_len;  // same position of the density strip
      out[e] = __fmul_rn(lerp(r), lerp(e));
    }
  }
}

cudaError_t launch_boundary_clock(BoundaryClock* clock, const int* offsets, int n, cudaStream_t s) {
  if (n <= 0) return cudaErrorInvalidValue;
  k_boundary_clock<<<1, 32, 0, s>>>(clock, offsets, n);
  return cudaGetLastError();
}

cudaError_t launch_boundary_interp(const float* cache, long long per_snap, long long dry_len, long long cell_len,
                                   int ntr, const BoundaryClock* clock, int stage, float* out, cudaStream_t s) {
  if (stage < 0 || stage > 2 || cell_len <= 0) return cudaErrorInvalidValue;
  const long long n = dry_len + (long long)ntr * cell_len;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 1184);
  k_boundary_interp<<<blocks, 256, 0, s>>>(cache, per_snap, dry_len, cell_len, ntr, clock, stage, out);
  return cudaGetLastError();
}

cudaError_t launch_unpack(const Geom& g, int orient, const float* src, float* dst, cudaStream_t s) {
  const long long n = (long long)(g.nx + (orient == kFaceX)) * (g.ny + (orient == kFaceY)) *
                      (g.nz + (orient == kFaceZ));
  k_unpack<<<blocks_for(n, 256), 256, 0, s>>>(g, orient, src, dst);
  return cudaGetLastError();
}

cudaError_t launch_rank_halo(const RankTable& t, int op, cudaStream_t s) {
  if (t.n <= 0 || t.n > kMaxRanks) return cudaErrorInvalidValue;
  if (op == 0) {
    if (t.halo <= 0) return cudaSuccess;
    k_rank_x<<<dim3(64, t.n), 256, 0, s>>>(t);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_rank_y<<<dim3(64, t.n), 256, 0, s>>>(t);
    return cudaGetLastError();
  }
  if (t.orient != kFaceX && t.orient != kFaceY) return cudaSuccess;
  k_rank_sync<<<dim3(64, t.n), 256, 0, s>>>(t);
  return cudaGetLastError();
}

cudaError_t launch_pressure(const float* rho, const float* rt, float* p, long long n, cudaStream_t s) {
  k_pressure<<<blocks_for(n, 256), 256, 0, s>>>(rho, rt, p, n);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const Geom& g, int orient, int mode, const float* f, const float* rho,
                          const float* idz, int idz_terrain, double* partials, ReduceOut* out,
                          cudaStream_t s) {
  k_reduce_pass1<<<kReduceBlocks, 256, 0, s>>>(g, orient, mode, f, rho, idz, idz_terrain, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_reduce_pass2<<<1, 256, 0, s>>>(partials, kReduceBlocks, out);
  return cudaGetLastError();
}

cudaError_t launch_reduce_2d(const double* a, const double* b, long long n, double* partials,
                             ReduceOut* out, cudaStream_t s, int mode) {
  k_reduce_2d_pass1<<<kReduceBlocks, 256, 0, s>>>(a, b, n, partials, mode);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_reduce_pass2<<<1, 256, 0, s>>>(partials, kReduceBlocks, out);
  return cudaGetLastError();
}

}  // namespace gwmb

// ---------------------------------------------------------------------------
// Allocation-free entry point (see include/gwm_b200.h).  The device address of
// g_noalloc_partials is resolved with the device current and cached together with the
// context it belongs to.  A module's globals live in one context: if the device's
// current context is a different one (after cudaDeviceReset, or a context torn down
// and created again), the address is resolved again before use.
using namespace gwmb;

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoAllocSlot {
  void* ctx = nullptr;   // CUcontext the address was resolved in
  double* addr = nullptr;
};
NoAllocSlot g_noalloc[kMaxDevices];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {  // driver entry point: no libcuda link needed
  static CtxGetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  });
  return fn;
}
}  // namespace

extern "C" int gwm_b200_field_stats_noalloc(const float* x, long long n, double* out, void* stream) {
  if (!x || !out || n <= 0 || n > (long long)INT_MAX) return GWM_B200_ERR_ARG;
  // an error left pending by other code is the caller's to see: return without clearing it
  if (cudaPeekAtLastError() != cudaSuccess) return GWM_B200_ERR_CUDA;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return GWM_B200_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return GWM_B200_ERR_ARG;
  double* part = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    CUcontext ctx = nullptr;
    const CtxGetCurrentFn get = ctx_get_current();
    if (get && get(&ctx) != CUDA_SUCCESS) ctx = nullptr;
    NoAllocSlot& slot = g_noalloc[dev];
    if (!slot.addr || slot.ctx != (void*)ctx) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return GWM_B200_ERR_CUDA;
      if (!ctx && get) get(&ctx);  // the runtime made the primary context current just now
      slot.addr = static_cast<double*>(p);
      slot.ctx = (void*)ctx;
    }
    part = slot.addr;
  }
  cudaStream_t s = (cudaStream_t)stream;
  long long nb = (n + 256LL * 8 - 1) / (256LL * 8);
  if (nb > kNoAllocBlocks) nb = kNoAllocBlocks;
  // every partial the second pass reads is written by the first: nothing to clear
  k_stats_pass1<<<(int)nb, 256, 0, s>>>(x, n, part);
  if (cudaGetLastError() != cudaSuccess) return GWM_B200_ERR_CUDA;
  k_reduce_pass2<<<1, 256, 0, s>>>(part, (int)nb, reinterpret_cast<ReduceOut*>(out));
  if (cudaGetLastError() != cudaSuccess) return GWM_B200_ERR_CUDA;
  if (!stream && cudaStreamSynchronize(s) != cudaSuccess) return GWM_B200_ERR_CUDA;
  return GWM_B200_OK;
}
