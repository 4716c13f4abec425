// capi.cu — the C-ABI of libgwm_b200.so: context, device buffer plan, step
// sequencing, state I/O, budgets and the halo operators.
//
// Buffer plan of one member (all fields share one padded geometry, see common.cuh):
//   Q[5]        step state: rho_d, rho_theta_m, mom_u, mom_v, mom_w
//   R[2]        density during a step (ping-pong between kernels)
//   P[2]        pressure perturbation p'(R) handed from one acoustic substep to the next
//   TH[2]       theta frozen for an RK stage (ping-pong between stages)
//   B[2][3]     stage base momenta written by the slow kernel
//   D[2][3]     acoustic momentum increments m - m_base (ping-pong between substeps)
//   T0/T1/T2    tracer masses (state and two stage buffers), moist members
//   precip      FP64 surface accumulation + Neumaier compensation
//   acc         ring of three fixed-point level-sum slots (theta, or rho and p)
// A kernel at ring position n reads slot n%3, accumulates into (n+1)%3 and clears
// (n+2)%3; a dry step launches 3*(1+ns) ring kernels, a multiple of three, so the
// slot pattern of every step is the same and one captured graph replays any step.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <iomanip>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include <cuda.h>

#include "../../include/gwm_b200.h"
#include "common.cuh"
#include "dycore.cuh"
#include "halo.cuh"
#include "physics.cuh"
#include "plan_view.cuh"
#include "surrogate.cuh"
#include "surrogate_rain.cuh"

using namespace gwmb;

namespace {

constexpr int kSlot = 2 * kMaxNz;  // ulls per ring slot (a, b)

struct Member {
  gwm_b200_grid_desc gd{};
  gwm_b200_member_desc md{};
  std::vector<float> terrain;
  std::vector<double> eta;
  Geom g{};
  bool terrain_active = false;
  size_t field_elems = 0;
  char* block = nullptr;
  float* Q[5]{};
  float* R[2]{};
  float* P[2]{};
  float* TH[2]{};
  float* B[2][3]{};
  float* D[2][3]{};
  float* T0[3]{};
  float* T1[3]{};
  float* T2[3]{};
  // TracerRegistry + TracerState (include/gwm/state/tracer_registry.hpp:23-49,
  // tracer_state.hpp:12-119): the tracers in registry order, each with its mass field
  // rho*q and the two SSPRK3 stage buffers.  A moist member registers the warm-rain triple
  // first (T0/T1/T2: specific humidity, cloud water, rain water); tracers added later get
  // their own device block (extra).
  struct Tracer {
    std::string name, units;
    bool positive = true;
    float* f[3]{};
  };
  std::vector<Tracer> reg;
  std::vector<char*> extra;
  float *zc = nullptr, *idc = nullptr, *idf = nullptr;
  float* colref[2]{};                // terrain: the substep input's column reference (K11)
  double *precip = nullptr, *pcomp = nullptr;
  unsigned long long* acc = nullptr;
  double* base = nullptr;            // FP64 base state of the perturbation EOS
  bool base_valid = false;
  float* staging = nullptr;
  float* io_stage = nullptr;         // host-to-host stepping: one staging buffer per field
  double* red_part = nullptr;
  ReduceOut* red_out = nullptr;
  int ring = 0;
  bool theta_valid = false;
  int* err = nullptr;                // device error word (bounded waits that gave up)
  unsigned* gbar = nullptr;          // grid-barrier words of the persistent acoustic launch
  // reference boundary state (apply_reference_boundaries at every stage start): compact
  // strips of rho, rho*theta, u, v, w and the three tracers; bsave holds the stage-1
  // input's own strips, which the blends of stages 2 and 3 need unchanged
  float* bstrip = nullptr;
  float* bsave = nullptr;
  long long boff[9]{};
  bool has_boundary = false, has_tracer_boundary = false;
  // prepared-case boundary cache: n snapshots of strips laid out like bstrip (tracer strips
  // hold mixing ratios), their forecast offsets (s) and the device clock
  char* bcache_block = nullptr;
  float* bcache = nullptr;
  int* bcache_off = nullptr;
  BoundaryClock* bclock = nullptr;
  int bcache_n = 0;
  // Rayleigh damping layer (extension): [tau_c(nz) | tau_f(nz+1) | u_ref(nz) | v_ref(nz)]
  float* damp = nullptr;
  bool damping = false;
  // learned warm-rain microphysics: fragments | bias | norm | range | fallback counter
  char* sur = nullptr;
  bool use_surrogate = false;
  float sur_tol_water = 0.0f, sur_tol_energy = 0.0f;
  // TMA descriptors of the substep's buffers: (buffer, box kind 0 cell / 1 face / 2 own, map)
  std::vector<std::tuple<const float*, int, CUtensorMap>> tmaps;
  const CUtensorMap* tmap(const float* buf, int kind) const {
    for (const auto& t : tmaps)
      if (std::get<0>(t) == buf && std::get<1>(t) == kind) return &std::get<2>(t);
    return nullptr;
  }

  unsigned long long* slot(int s) { return acc + (size_t)(((s % 3) + 3) % 3) * kSlot; }
};

}  // namespace

// Per-kernel CUDA-event timing (profiling mode, direct launches only).
enum KernelKind { kKSlow = 0, kKFast, kKTracer, kKRain, kKColumn, kKOther, kKinds };
const char* const kKindNames[kKinds] = {"k_slow_stage", "k_fast_substep", "k_tracer_stage",
                                        "k_warm_rain", "k_column_reference", "other"};

struct gwm_b200_ctx {
  std::vector<Member> m;
  bool profile = false;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_events;
  double prof_ms[kKinds] = {};
  long long prof_n[kKinds] = {};
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  bool use_graph = false;
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0;
  int fast_tile_rows = 0;  // acoustic substep: 0 owned-tile flat kernel, 8/16 overlapped tiles
  int slow_tile_rows = 16;    // slow stage: overlapped tiles of 8 or 16 rows
  int tracer_tile_rows = 16;  // tracer stage: overlapped tiles of 8 or 16 rows
  long long launches = 0;
  long long cur_launches = 0;
  // members advance on their own streams, forked from and joined back to `stream`
  // (one graph with a branch per member when captured)
  bool concurrent = true;
  std::vector<cudaStream_t> mstreams;
  std::vector<cudaEvent_t> mjoin;
  cudaEvent_t mfork = nullptr;
  // host-to-host stepping: copy-in and copy-out streams, and their events (the fields in,
  // the end of the dry step, the end of the step)
  cudaStream_t cin = nullptr, cout = nullptr;
  std::vector<cudaEvent_t> io_ev;
};

namespace {

int fail(gwm_b200_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(c, GWM_B200_ERR_CUDA,                                                    \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

// ---------------------------------------------------------------------------
// Hybrid-height metrics, FP64 compute and FP32 store: grid_metrics.hpp:87-239.
struct HostMetrics {
  std::vector<float> zc, idc, idf;  // unpadded (k, j, i)
};

double terrain_weight(double eta, double taper) {  // grid_metrics.hpp:126-144
  if (eta <= 0.0) return 1.0;
  if (eta >= 1.0) return 0.0;
  if (taper <= 0.0) {
    const double s = std::clamp(eta, 0.0, 1.0);
    return 1.0 - s * s * (3.0 - 2.0 * s);
  }
  if (eta <= taper) return 1.0;
  const double s = std::clamp((eta - taper) / std::max(1.0e-9, 1.0 - taper), 0.0, 1.0);
  return 1.0 - s * s * (3.0 - 2.0 * s);
}

HostMetrics build_metrics(const Member& M) {
  const int nx = M.gd.nx, ny = M.gd.ny, nz = M.gd.nz;
  const double zt = M.gd.z_top, taper = M.gd.terrain_taper_eta;
  std::vector<double> ei(nz + 1), ec(nz), bi(nz + 1), bc(nz), zi(nz + 1), zcc(nz);
  for (int k = 0; k <= nz; ++k) {
    ei[k] = M.eta.empty() ? (double)k / (double)nz : M.eta[k];
    bi[k] = terrain_weight(ei[k], taper);
    zi[k] = ei[k] * zt;
  }
  for (int k = 0; k < nz; ++k) {
    ec[k] = M.eta.empty() ? ((double)k + 0.5) / (double)nz : 0.5 * (M.eta[k] + M.eta[k + 1]);
    bc[k] = terrain_weight(ec[k], taper);
    zcc[k] = ec[k] * zt;
  }
  HostMetrics H;
  const size_t plane = (size_t)nx * ny;
  H.zc.resize(plane * nz);
  H.idc.resize(plane * nz);
  H.idf.resize(plane * (nz + 1));
  std::vector<float> zim(nz + 1);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const double th = M.terrain.empty() ? 0.0 : (double)M.terrain[(size_t)j * nx + i];
      for (int k = 0; k <= nz; ++k) {
        zim[k] = (float)(zi[k] + bi[k] * th);
        float f = 0.0f;
        if (k > 0 && k < nz) {
          const double dzf = (zcc[k] + bc[k] * th) - (zcc[k - 1] + bc[k - 1] * th);
          f = (float)(1.0 / std::max(dzf, 1.0e-6));
        }
        H.idf[((size_t)k * ny + j) * nx + i] = f;
      }
      for (int k = 0; k < nz; ++k) {
        H.zc[((size_t)k * ny + j) * nx + i] = (float)(zcc[k] + bc[k] * th);
        const double dzc = (double)zim[k + 1] - (double)zim[k];
        H.idc[((size_t)k * ny + j) * nx + i] = (float)(1.0 / std::max(dzc, 1.0e-6));
      }
    }
  return H;
}

// Pad an unpadded metric field into the field geometry; halo columns take the
// periodically wrapped values (the reference indexes metrics with
// wrap_metric_index, dry_fast_modes.cu:24-30) or the clamped edge on open axes.
std::vector<float> pad_metric(const Member& M, const std::vector<float>& src, int levels) {
  const Geom& g = M.g;
  std::vector<float> out((size_t)g.plane * (g.nz + 1), 0.0f);
  auto wrap = [](int v, int n, bool per) {
    if (per) { int m = v % n; return m < 0 ? m + n : m; }
    return std::clamp(v, 0, n - 1);
  };
  for (int k = 0; k < levels; ++k)
    for (int j = -1; j <= g.ny + 1; ++j)
      for (int i = -1; i <= g.nx + 1; ++i) {
        const int si = wrap(i, g.nx, g.per_x), sj = wrap(j, g.ny, g.per_y);
        out[gidx(g, i, j, k)] = src[((size_t)k * g.ny + sj) * g.nx + si];
      }
  return out;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 3-D map over one padded field (pitch x rows x (nz+1) FP32) with an (bx, by, 1) box.
bool encode_field_map(CUtensorMap* out, const float* base, const Geom& g, int bx, int by) {
  const EncodeTiledFn fn = tensor_map_encoder();
  if (!fn || (reinterpret_cast<uintptr_t>(base) & 15) || (g.pitch * 4) % 16) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)g.pitch, (cuuint64_t)g.rows, (cuuint64_t)(g.nz + 1)};
  const cuuint64_t strides[2] = {(cuuint64_t)g.pitch * 4, (cuuint64_t)g.plane * 4};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Maps of every buffer the flat-terrain TMA substep may read (false if unavailable).
bool build_substep_maps(Member& M) {
  M.tmaps.clear();
  const int* boxes[4] = {kTmaCellBox, kTmaFaceBox, kTmaOwnBox, kTmaYFaceBox};
  auto add = [&](const float* buf, int kind) {
    CUtensorMap m;
    if (!encode_field_map(&m, buf, M.g, boxes[kind][0], boxes[kind][1])) return false;
    M.tmaps.emplace_back(buf, kind, m);
    return true;
  };
  bool ok = true;
  for (int i = 0; i < 2; ++i) {
    ok = ok && add(M.R[i], 0) && add(M.TH[i], 0) && add(M.P[i], 0) && add(M.R[i], 2) && add(M.TH[i], 2);
    ok = ok && add(M.D[i][0], 1) && add(M.D[i][1], 1) && add(M.D[i][2], 2);
    for (int f = 0; f < 3; ++f) ok = ok && add(M.B[i][f], 2);
  }
  for (int f = 2; f < 5; ++f) ok = ok && add(M.Q[f], 2);  // bases of the stand-alone fast modes
  // slow stage: inputs with 40 x 18 boxes (kind 0) and Y faces with 40 x 19 (kind 3)
  for (int f : {0, 1, 2, 4}) ok = ok && add(M.Q[f], 0);
  ok = ok && add(M.Q[3], 3);
  for (int i = 0; i < 2; ++i) {
    ok = ok && add(M.B[i][0], 0) && add(M.B[i][2], 0) && add(M.B[i][1], 3);
    ok = ok && add(M.D[i][0], 0) && add(M.D[i][2], 0) && add(M.D[i][1], 3);
  }
  // tracer stage: the three tracer generations (cells) and the frozen X/Y fluxes
  if (M.md.moist)
    for (int t = 0; t < 3; ++t) ok = ok && add(M.T0[t], 0) && add(M.T1[t], 0) && add(M.T2[t], 0);
  ok = ok && add(M.Q[2], 1) && add(M.Q[3], 1);
  if (!ok) M.tmaps.clear();
  return ok;
}

// Maps of every buffer the terrain TMA substep may read (false if unavailable).
bool build_terrain_substep_maps(Member& M) {
  M.tmaps.clear();
  const int* boxes[4] = {kTmaCellBox, kTmaFaceBox, kTmaOwnBox, kTmaYFaceBox};
  auto add = [&](const float* buf, int kind) {
    CUtensorMap m;
    if (!encode_field_map(&m, buf, M.g, boxes[kind][0], boxes[kind][1])) return false;
    M.tmaps.emplace_back(buf, kind, m);
    return true;
  };
  bool ok = add(M.zc, 0);
  for (int i = 0; i < 2; ++i) {
    ok = ok && add(M.R[i], 0) && add(M.TH[i], 0) && add(M.P[i], 0) && add(M.R[i], 2) && add(M.TH[i], 2);
    ok = ok && add(M.D[i][0], 1) && add(M.D[i][1], 1) && add(M.D[i][2], 2);
  }
  // slow stage: inputs with 40 x 18 boxes (kind 0) and Y faces with 40 x 19 (kind 3)
  for (int f : {0, 1, 2, 4}) ok = ok && add(M.Q[f], 0);
  ok = ok && add(M.Q[3], 3);
  for (int i = 0; i < 2; ++i) {
    ok = ok && add(M.B[i][0], 0) && add(M.B[i][2], 0) && add(M.B[i][1], 3);
    ok = ok && add(M.D[i][0], 0) && add(M.D[i][2], 0) && add(M.D[i][1], 3);
  }
  // tracer stage: the three tracer generations (cells), the frozen X/Y fluxes and Z faces
  if (M.md.moist)
    for (int t = 0; t < 3; ++t) ok = ok && add(M.T0[t], 0) && add(M.T1[t], 0) && add(M.T2[t], 0);
  ok = ok && add(M.Q[2], 1) && add(M.Q[3], 1) && add(M.Q[4], 2);
  if (!ok) M.tmaps.clear();
  return ok;
}

int alloc_member(gwm_b200_ctx* c, Member& M) {
  const gwm_b200_grid_desc& d = M.gd;
  Geom& g = M.g;
  g.nx = d.nx; g.ny = d.ny; g.nz = d.nz;
  g.pitch = ((kXOff + d.nx + 2 + 31) / 32) * 32;
  g.rows = d.ny + 3;
  g.plane = g.pitch * g.rows;
  g.per_x = d.periodic_x ? 1 : 0;
  g.per_y = d.periodic_y ? 1 : 0;
  g.dx = (float)d.dx;
  g.dy = (float)d.dy;
  g.inv_dx = 1.0f / g.dx;
  g.inv_dy = 1.0f / g.dy;
  M.field_elems = (size_t)g.plane * (g.nz + 1);
  const size_t fbytes = ((M.field_elems * sizeof(float) + 255) / 256) * 256;
  const bool moist = M.md.moist != 0;
  const int nfields = 5 + 2 + 2 + 2 + 6 + 6 + (moist ? 9 : 0) + (M.terrain_active ? 5 : 0);
  const size_t owned_max = (size_t)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
  const size_t plane2 = (size_t)d.nx * d.ny;
  const size_t extra = ((2 * plane2 * sizeof(double) + 255) / 256) * 256 +
                       3 * kSlot * sizeof(unsigned long long) + owned_max * sizeof(float) +
                       3 * kReduceBlocks * sizeof(double) + 32 * sizeof(ReduceOut) + 4096 +
                       3 * 4 * (kMaxNz + 1) * sizeof(float) + 3 * kMaxNz * sizeof(double) + 512 +
                       4 * (kMaxNz + 1) * sizeof(float) + 256 + 256;
  const size_t total = nfields * fbytes + extra;
  CK(cudaMalloc(&M.block, total));
  CK(cudaMemsetAsync(M.block, 0, total, c->stream));
  char* p = M.block;
  auto take = [&](size_t bytes) { char* r = p; p += ((bytes + 255) / 256) * 256; return r; };
  for (auto& q : M.Q) q = (float*)take(fbytes);
  for (auto& q : M.R) q = (float*)take(fbytes);
  for (auto& q : M.P) q = (float*)take(fbytes);
  for (auto& q : M.TH) q = (float*)take(fbytes);
  for (auto& b : M.B) for (auto& q : b) q = (float*)take(fbytes);
  for (auto& b : M.D) for (auto& q : b) q = (float*)take(fbytes);
  if (moist) {
    for (auto& q : M.T0) q = (float*)take(fbytes);
    for (auto& q : M.T1) q = (float*)take(fbytes);
    for (auto& q : M.T2) q = (float*)take(fbytes);
    // make_warm_rain_registry (tracer_registry.hpp:56-62)
    const char* names[3] = {"specific_humidity", "cloud_water_mixing_ratio", "rain_water_mixing_ratio"};
    M.reg.clear();
    for (int t = 0; t < 3; ++t) {
      Member::Tracer tr;
      tr.name = names[t];
      tr.units = "kg/kg";
      tr.f[0] = M.T0[t]; tr.f[1] = M.T1[t]; tr.f[2] = M.T2[t];
      M.reg.push_back(tr);
    }
  }
  M.precip = (double*)take(plane2 * sizeof(double));
  M.pcomp = (double*)take(plane2 * sizeof(double));
  M.acc = (unsigned long long*)take(3 * kSlot * sizeof(unsigned long long));
  M.base = (double*)take(3 * kMaxNz * sizeof(double));
  M.staging = (float*)take(owned_max * sizeof(float));
  M.red_part = (double*)take(3 * kReduceBlocks * sizeof(double));
  M.red_out = (ReduceOut*)take(32 * sizeof(ReduceOut));
  M.err = (int*)take(sizeof(int));
  M.gbar = (unsigned*)take(2 * sizeof(unsigned));
  M.damp = (float*)take(4 * (kMaxNz + 1) * sizeof(float));
  // metrics
  const HostMetrics H = build_metrics(M);
  if (M.terrain_active) {
    M.colref[0] = (float*)take(fbytes);  // column hydrostatic reference: pressure, density
    M.colref[1] = (float*)take(fbytes);
    M.zc = (float*)take(fbytes);
    M.idc = (float*)take(fbytes);
    M.idf = (float*)take(fbytes);
    const auto zc = pad_metric(M, H.zc, d.nz), idc = pad_metric(M, H.idc, d.nz),
               idf = pad_metric(M, H.idf, d.nz + 1);
    CK(cudaMemcpy(M.zc, zc.data(), zc.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(M.idc, idc.data(), idc.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(M.idf, idf.data(), idf.size() * sizeof(float), cudaMemcpyHostToDevice));
  } else {  // horizontally uniform: one value per level
    M.zc = (float*)take((kMaxNz + 1) * sizeof(float));
    M.idc = (float*)take((kMaxNz + 1) * sizeof(float));
    M.idf = (float*)take((kMaxNz + 1) * sizeof(float));
    std::vector<float> zc(d.nz), idc(d.nz), idf(d.nz + 1);
    const size_t plane = (size_t)d.nx * d.ny;
    for (int k = 0; k < d.nz; ++k) { zc[k] = H.zc[k * plane]; idc[k] = H.idc[k * plane]; }
    for (int k = 0; k <= d.nz; ++k) idf[k] = H.idf[k * plane];
    CK(cudaMemcpy(M.zc, zc.data(), zc.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(M.idc, idc.data(), idc.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(M.idf, idf.data(), idf.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  if ((size_t)(p - M.block) > total) return fail(c, GWM_B200_ERR_ARG, "internal: buffer plan overflow");
  // empty when TMA descriptors are unavailable
  if (M.terrain_active) build_terrain_substep_maps(M);
  else build_substep_maps(M);
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

constexpr int kFastTma = 3;  // fast_tile_rows value selecting the TMA-fed substep
// fast_tile_rows value selecting the TMA-fed substeps of a stage in one persistent launch
constexpr int kFastStage = 4;
bool fast_tma_path(const gwm_b200_ctx* c) { return c->fast_tile_rows == kFastTma || c->fast_tile_rows == kFastStage; }
constexpr int kSlowTma = 3;  // slow_tile_rows value selecting the TMA-fed slow stage
constexpr int kTracerTma = 3;  // tracer_tile_rows value selecting the TMA-fed tracer stage

// One tracer stage: the TMA-fed kernel when selected, else overlapped tiles.
cudaError_t launch_tracers(gwm_b200_ctx* c, const Member& M, const TracerArgs& a) {
  if (c->tracer_tile_rows == kTracerTma) {
    TracerMaps m{};
    const CUtensorMap* rho = M.tmap(a.rho, 0);
    const CUtensorMap* u = M.tmap(a.u, 1);
    const CUtensorMap* v = M.tmap(a.v, 1);
    const CUtensorMap* w = M.tmap(a.w, 2);
    if (!rho || !u || !v || !w) return cudaErrorInvalidValue;
    for (int t = 0; t < a.ntracers; ++t) {
      const CUtensorMap* q = M.tmap(a.q_in[t], 0);
      if (!q) return cudaErrorInvalidValue;
      m.q[t] = *q;
    }
    m.rho = *rho; m.u = *u; m.v = *v; m.w = *w;
    return launch_tracer_tma(a, m, c->stream);
  }
  return launch_tracer_stage(a, c->stream, c->tracer_tile_rows == kTracerTma ? 16 : c->tracer_tile_rows);
}

// One slow stage: the TMA-fed kernels when selected (flat terrain, or terrain without the
// p' level sums), else overlapped tiles.
cudaError_t launch_stage(gwm_b200_ctx* c, const Member& M, const SlowArgs& a, bool terr) {
  if (!a.tend_only && c->slow_tile_rows == kSlowTma && (!terr || a.acc_mode != 1)) {
    SlowMaps m{};
    const CUtensorMap* p[8] = {M.tmap(a.rho, 0), M.tmap(a.th, 0), M.tmap(a.u, 0), M.tmap(a.v, 3),
                               M.tmap(a.w, 0), a.du ? M.tmap(a.du, 0) : nullptr,
                               a.du ? M.tmap(a.dv, 3) : nullptr, a.du ? M.tmap(a.dw, 0) : nullptr};
    for (int i = 0; i < 5; ++i)
      if (!p[i]) return cudaErrorInvalidValue;
    if (a.du && (!p[5] || !p[6] || !p[7] || !a.dv || !a.dw)) return cudaErrorInvalidValue;
    m.rho = *p[0]; m.th = *p[1]; m.u = *p[2]; m.v = *p[3]; m.w = *p[4];
    if (a.du) { m.du = *p[5]; m.dv = *p[6]; m.dw = *p[7]; }
    if (terr) {
      const CUtensorMap* z = M.tmap(a.zc, 0);
      if (!z) return cudaErrorInvalidValue;
      m.z = *z;
      return launch_slow_terrain_tma(a, m, c->stream);
    }
    return launch_slow_tma(a, m, c->stream);
  }
  return launch_slow(a, terr, c->stream, c->slow_tile_rows == kSlowTma ? 16 : c->slow_tile_rows);
}

// One acoustic substep: the TMA-fed kernels when selected (flat terrain or terrain),
// else the owned-tile or overlapped-tile kernels.
// p_ready: the first substep's p' (with its halo) is in f.p_in, written by the slow stage
// TMA descriptors of one substep's inputs (k_fast_tma); false when one is missing
bool fast_maps(const Member& M, const FastArgs& f, bool first, bool p_ready, FastMaps& m) {
  const bool fin = f.final_kind == 2;
  const bool pin = !first || p_ready;  // p' loaded with its ring, not derived
  // rho and theta with the halo ring where p' is derived from them, owned boxes otherwise
  const CUtensorMap* rho = M.tmap(f.rho_in, pin ? 2 : 0);
  const CUtensorMap* th = M.tmap(f.th, pin ? 2 : 0);
  const CUtensorMap* du = first ? nullptr : M.tmap(f.du_in, 1);
  const CUtensorMap* dv = first ? nullptr : M.tmap(f.dv_in, 1);
  const CUtensorMap* dw = first ? nullptr : M.tmap(f.dw_in, 2);
  const CUtensorMap* bu = fin ? M.tmap(f.bu, 2) : nullptr;
  const CUtensorMap* bv = fin ? M.tmap(f.bv, 2) : nullptr;
  const CUtensorMap* bw = fin ? M.tmap(f.bw, 2) : nullptr;
  const CUtensorMap* pm = pin ? M.tmap(f.p_in, 0) : nullptr;
  if (!rho || !th || (!first && (!du || !dv || !dw)) || (pin && !pm) || (fin && (!bu || !bv || !bw)) ||
      (f.final_kind == 0 && !f.p_out))
    return false;
  m.rho = *rho; m.th = *th;
  if (!first) { m.du = *du; m.dv = *dv; m.dw = *dw; }
  if (pin) m.p = *pm;
  if (fin) { m.bu = *bu; m.bv = *bv; m.bw = *bw; }
  return true;
}

// TMA descriptors of one terrain substep's inputs (k_fast_terrain_tma); false when one is missing
bool fast_terrain_maps(const Member& M, const FastArgs& f, bool first, FastTerrainMaps& m) {
  const CUtensorMap* rho = M.tmap(f.rho_in, first ? 0 : 2);
  const CUtensorMap* th = M.tmap(f.th, first ? 0 : 2);
  const CUtensorMap* z = M.tmap(f.zc, 0);
  const CUtensorMap* pm = first ? nullptr : M.tmap(f.p_in, 0);
  const CUtensorMap* du = first ? nullptr : M.tmap(f.du_in, 1);
  const CUtensorMap* dv = first ? nullptr : M.tmap(f.dv_in, 1);
  const CUtensorMap* dw = first ? nullptr : M.tmap(f.dw_in, 2);
  if (!rho || !th || !z || (!first && (!pm || !du || !dv || !dw))) return false;
  m.rho = *rho; m.th = *th; m.z = *z;
  if (!first) { m.p = *pm; m.du = *du; m.dv = *dv; m.dw = *dw; }
  return true;
}

cudaError_t launch_substep(gwm_b200_ctx* c, const Member& M, const FastArgs& f, bool first, bool terr,
                           bool p_ready = false) {
  if (terr && fast_tma_path(c)) {
    FastTerrainMaps m{};
    if (!fast_terrain_maps(M, f, first, m)) return cudaErrorInvalidValue;
    return launch_fast_terrain_tma(f, m, first, c->stream);
  }
  if (!terr && fast_tma_path(c)) {
    FastMaps m{};
    if (!fast_maps(M, f, first, p_ready, m)) return cudaErrorInvalidValue;
    return launch_fast_tma(f, m, first, p_ready, c->stream);
  }
  return launch_fast(f, first, terr, c->stream, c->fast_tile_rows);
}

// The first n substeps of a stage (flat terrain) in one persistent launch; f[0] is the
// stage's first substep.
cudaError_t launch_substeps_persistent(gwm_b200_ctx* c, const Member& M, const FastArgs* f, int n, bool p_ready) {
  FastStage st{};
  st.n = n;
  st.count = M.gbar;
  st.gen = M.gbar + 1;
  for (int q = 0; q < n; ++q) {
    st.a[q] = f[q];
    if (!fast_maps(M, f[q], q == 0, p_ready, st.m[q])) return cudaErrorInvalidValue;
  }
  return launch_fast_stage_tma(st, p_ready, c->stream);
}

constexpr int kStripOrient[8] = {kCell, kCell, kFaceX, kFaceY, kFaceZ, kCell, kCell, kCell};

StripJob strip_job(float* padded, float* compact, const float* aux, int orient, int mode) {
  StripJob j{};
  j.padded = padded; j.compact = compact; j.aux = aux; j.orient = orient; j.mode = mode;
  return j;
}

// theta level sums of a stage input into slot(ring), replacing those of the state
// before the boundary strips were written (mode 0: rho*theta stored, 2: theta stored)
int recompute_theta_sums(gwm_b200_ctx* c, Member& M, const float* rho, const float* th, int mode);

// Reads and clears the device error words; call after the stream has drained.
int check_device_errors(gwm_b200_ctx* c) {
  for (auto& M : c->m) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, M.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (e) {
      CK(cudaMemsetAsync(M.err, 0, sizeof(int), c->stream));
      return fail(c, GWM_B200_ERR_TIMEOUT, "a bounded wait in the acoustic substep gave up (tile load did not complete)");
    }
  }
  return GWM_B200_OK;
}

int count_launch(gwm_b200_ctx* c, cudaError_t e, const char* what) {
  ++c->cur_launches;
  if (e != cudaSuccess) return fail(c, GWM_B200_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return GWM_B200_OK;
}

int kind_of(const char* name) {
  const std::string n(name);
  if (n == "slow stage") return kKSlow;
  if (n == "fast substep") return kKFast;
  if (n == "tracer stage") return kKTracer;
  if (n == "warm rain") return kKRain;
  if (n == "column reference") return kKColumn;
  return kKOther;
}

void prof_begin(gwm_b200_ctx* c, cudaEvent_t* e0) {
  *e0 = nullptr;
  if (!c->profile) return;
  cudaEventCreate(e0);
  cudaEventRecord(*e0, c->stream);
}
void prof_end(gwm_b200_ctx* c, cudaEvent_t e0, const char* name) {
  if (!c->profile || !e0) return;
  cudaEvent_t e1;
  cudaEventCreate(&e1);
  cudaEventRecord(e1, c->stream);
  c->prof_events.push_back({kind_of(name), {e0, e1}});
}

#define LAUNCH(expr, name)                          \
  do {                                              \
    cudaEvent_t e0_;                                \
    prof_begin(c, &e0_);                            \
    int rc_ = count_launch(c, (expr), name);        \
    prof_end(c, e0_, name);                         \
    if (rc_ != GWM_B200_OK) return rc_;             \
  } while (0)

double inv_count(const Member& M) { return 1.0 / ((double)M.g.nx * (double)M.g.ny); }

// FP64 base state of the pressure-perturbation EOS from the current rho_theta
int ensure_base(gwm_b200_ctx* c, Member& M) {
  if (M.base_valid) return GWM_B200_OK;
  LAUNCH(launch_base_state(M.g, M.Q[1], M.base, c->stream), "base state");
  M.base_valid = true;
  return GWM_B200_OK;
}

// theta level sums of the step state into slot(ring) (dry_core.cu:462-490)
int enqueue_theta(gwm_b200_ctx* c, Member& M) {
  CK(cudaMemsetAsync(M.slot(M.ring), 0, kSlot * sizeof(unsigned long long), c->stream));
  LevelSumArgs a{};
  a.g = M.g; a.rho = M.Q[0]; a.rt = M.Q[1]; a.mode = 0;
  a.acc_a = M.slot(M.ring); a.acc_b = M.slot(M.ring) + kMaxNz;
  a.clr_a = M.slot(M.ring + 1); a.clr_b = M.slot(M.ring + 1) + kMaxNz;
  LAUNCH(launch_level_sums(a, c->stream), "level sums");
  M.theta_valid = true;
  return GWM_B200_OK;
}

bool rain_feeds_theta(const Member& M) { return M.md.moist && M.md.enable_warm_rain; }

int recompute_theta_sums(gwm_b200_ctx* c, Member& M, const float* rho, const float* th, int mode) {
  CK(cudaMemsetAsync(M.slot(M.ring), 0, kMaxNz * sizeof(unsigned long long), c->stream));
  LevelSumArgs a{};
  a.g = M.g; a.rho = rho; a.rt = th; a.mode = mode;
  a.acc_a = M.slot(M.ring); a.acc_b = M.slot(M.ring) + kMaxNz;
  LAUNCH(launch_level_sums(a, c->stream), "level sums");
  return GWM_B200_OK;
}

// BoundaryUpdater::apply at a stage start (dry_core.cu:568, 591, 620) with the reference
// boundary state: the stage input is (rho, rho*theta or theta, B + D).
int enqueue_dry_boundary(gwm_b200_ctx* c, Member& M, int s, const float* rho, const float* th,
                         float* const* base, float* const* inc) {
  StripJobs J{};
  auto push = [&](const StripJob& j) { J.j[J.n++] = j; };
  if (s == 0) {  // keep q0 intact: save the input's strips, write the boundary's
    StripJobs S{};
    for (int f = 0; f < 5; ++f) S.j[S.n++] = strip_job(M.Q[f], M.bsave + M.boff[f], nullptr, kStripOrient[f], 1);
    LAUNCH(launch_strips(M.g, S, c->stream), "boundary strips");
    for (int f = 0; f < 5; ++f) push(strip_job(M.Q[f], M.bstrip + M.boff[f], nullptr, kStripOrient[f], 0));
  } else {
    push(strip_job(const_cast<float*>(rho), M.bstrip + M.boff[0], nullptr, kCell, 0));
    push(strip_job(const_cast<float*>(th), M.bstrip + M.boff[1], M.bstrip + M.boff[0], kCell, 3));
    for (int f = 0; f < 3; ++f) {
      push(strip_job(base[f], M.bstrip + M.boff[2 + f], nullptr, kStripOrient[2 + f], 0));
      if (inc) push(strip_job(inc[f], nullptr, nullptr, kStripOrient[2 + f], 4));
    }
  }
  LAUNCH(launch_strips(M.g, J, c->stream), "boundary strips");
  return recompute_theta_sums(c, M, rho, th, s == 0 ? 0 : 2);
}

// Put back the stage-1 input's own strips once the first slow stage has read them.
int restore_stage1_strips(gwm_b200_ctx* c, Member& M, int first, int count, float* const* fields) {
  StripJobs J{};
  for (int f = 0; f < count; ++f)
    J.j[J.n++] = strip_job(fields[f], M.bsave + M.boff[first + f], nullptr, kStripOrient[first + f], 0);
  LAUNCH(launch_strips(M.g, J, c->stream), "boundary strips");
  return GWM_B200_OK;
}

// Strips of the boundary cache interpolated at RK stage s of the current step (the
// clock kernel of the step filled the stage's bracket and weight).
int enqueue_boundary_interp(gwm_b200_ctx* c, Member& M, int s) {
  const int ntr = M.has_tracer_boundary ? 3 : 0;
  LAUNCH(launch_boundary_interp(M.bcache, M.boff[8], M.boff[5], M.boff[1] - M.boff[0], ntr, M.bclock, s, M.bstrip,
                                c->stream),
         "boundary interpolation");
  return GWM_B200_OK;
}

// One advance_dry_state_ssprk3 (dry_core.cu:541-651).
int enqueue_dry(gwm_b200_ctx* c, Member& M) {
  const gwm_b200_step_config& sc = M.md.step;
  const bool fast = sc.enable_fast_modes != 0;
  const int ns = std::max(1, sc.fast_substeps);
  const float dt = sc.dt;
  const float dtf = dt / (float)ns;
  const bool terr = M.terrain_active;
  const bool rain_theta = rain_feeds_theta(M);
  int rcur = 0, dcur = -1;
  const float wa[3] = {0.0f, 0.75f, 1.0f / 3.0f}, wb[3] = {1.0f, 0.25f, 2.0f / 3.0f};
  for (int s = 0; s < 3; ++s) {
    SlowArgs a{};
    a.g = M.g;
    if (s == 0) {
      a.rho = M.Q[0]; a.th = M.Q[1]; a.th_is_rt = 1;
      a.u = M.Q[2]; a.v = M.Q[3]; a.w = M.Q[4];
    } else {
      a.rho = M.R[rcur]; a.th = M.TH[(s - 1) & 1]; a.th_is_rt = 0;
      a.u = M.B[(s - 1) & 1][0]; a.v = M.B[(s - 1) & 1][1]; a.w = M.B[(s - 1) & 1][2];
      if (fast && dcur >= 0) { a.du = M.D[dcur][0]; a.dv = M.D[dcur][1]; a.dw = M.D[dcur][2]; }
      a.rho0 = M.Q[0]; a.rt0 = M.Q[1]; a.u0 = M.Q[2]; a.v0 = M.Q[3]; a.w0 = M.Q[4];
    }
    a.wa = wa[s]; a.wb = wb[s];
    a.dt = dt; a.gravity = sc.gravity;
    const int rnext = (s == 0) ? 0 : (rcur ^ 1);
    if (fast || s < 2) {
      a.o_rho = M.R[rnext]; a.o_th = M.TH[s & 1]; a.out_rt = 0;
      a.o_u = M.B[s & 1][0]; a.o_v = M.B[s & 1][1]; a.o_w = M.B[s & 1][2];
    } else {
      a.o_rho = M.Q[0]; a.o_th = M.Q[1]; a.out_rt = 1;
      a.o_u = M.Q[2]; a.o_v = M.Q[3]; a.o_w = M.Q[4];
    }
    a.th_acc = M.slot(M.ring);
    a.acc_a = M.slot(M.ring + 1); a.acc_b = M.slot(M.ring + 1) + kMaxNz;
    a.clr_a = M.slot(M.ring + 2); a.clr_b = M.slot(M.ring + 2) + kMaxNz;
    a.acc_mode = fast ? (terr ? 0 : 1) : ((s == 2 && rain_theta) ? 0 : 2);
    // the TMA slow stage stores the p' it evaluates for the level sums, and the first
    // substep (TMA too) loads it with its ring instead of deriving it again
    const bool p_handoff = fast && !terr && a.acc_mode == 1 && c->slow_tile_rows == kSlowTma && fast_tma_path(c);
    if (p_handoff) a.p_out = M.P[rnext];
    a.inv_count = inv_count(M);
    a.zc = M.zc; a.idz_c = M.idc; a.idz_f = M.idf; a.base = M.base;
    a.err = M.err;
    if (M.damping) {
      a.damp_c = M.damp; a.damp_f = M.damp + (kMaxNz + 1);
      a.uref = M.damp + 2 * (kMaxNz + 1); a.vref = M.damp + 3 * (kMaxNz + 1);
    }
    if (M.has_boundary) {
      if (M.bcache_n > 0) {  // PreparedCaseBoundaryUpdater::apply at sim_time 0, dt, dt/2
        if (s == 0) LAUNCH(launch_boundary_clock(M.bclock, M.bcache_off, M.bcache_n, c->stream), "boundary clock");
        const int rc = enqueue_boundary_interp(c, M, s);
        if (rc) return rc;
      }
      float* base[3] = {const_cast<float*>(a.u), const_cast<float*>(a.v), const_cast<float*>(a.w)};
      float* inc[3] = {const_cast<float*>(a.du), const_cast<float*>(a.dv), const_cast<float*>(a.dw)};
      const int rc = enqueue_dry_boundary(c, M, s, a.rho, a.th, base, a.du ? inc : nullptr);
      if (rc) return rc;
    }
    LAUNCH(launch_stage(c, M, a, terr), "slow stage");
    if (M.has_boundary && s == 0) {
      const int rc = restore_stage1_strips(c, M, 0, 5, M.Q);
      if (rc) return rc;
    }
    M.ring = (M.ring + 1) % 3;
    rcur = rnext;
    if (!fast) continue;
    dcur = -1;
    // persistent mode: the stage's substeps are collected and launched together (the
    // step's very last substep, with its longer ring, keeps its own launch)
    const bool persistent = !terr && c->fast_tile_rows == kFastStage && ns <= kFastStageMax + 1;
    FastArgs pend[kFastStageMax];
    int npend = 0;
    for (int n = 0; n < ns; ++n) {
      FastArgs f{};
      f.g = M.g;
      f.rho_in = M.R[rcur]; f.rho_out = M.R[rcur ^ 1];
      f.p_in = M.P[rcur]; f.p_out = M.P[rcur ^ 1];
      f.th = M.TH[s & 1];
      const int dout = (n == 0) ? 0 : (dcur ^ 1);
      if (n > 0) { f.du_in = M.D[dcur][0]; f.dv_in = M.D[dcur][1]; f.dw_in = M.D[dcur][2]; }
      f.du_out = M.D[dout][0]; f.dv_out = M.D[dout][1]; f.dw_out = M.D[dout][2];
      f.final_kind = (n == ns - 1) ? (s == 2 ? 2 : 1) : 0;
      f.acc_off = (f.final_kind == 2 && rain_theta) ? 1 : 0;
      f.bu = M.B[s & 1][0]; f.bv = M.B[s & 1][1]; f.bw = M.B[s & 1][2];
      f.f_rho = M.Q[0]; f.f_rt = M.Q[1]; f.f_u = M.Q[2]; f.f_v = M.Q[3]; f.f_w = M.Q[4];
      f.dtf = dtf; f.gravity = sc.gravity;
      f.hmom = sc.fast_update_horizontal_momentum; f.dens = sc.fast_update_density;
      f.ref_a = M.slot(M.ring); f.ref_b = M.slot(M.ring) + kMaxNz;
      f.inv_count = inv_count(M);
      f.acc_a = M.slot(M.ring + 1); f.acc_b = M.slot(M.ring + 1) + kMaxNz;
      f.clr_a = M.slot(M.ring + 2); f.clr_b = M.slot(M.ring + 2) + kMaxNz;
      f.zc = M.zc; f.idz_c = M.idc; f.idz_f = M.idf; f.base = M.base;
      f.err = M.err;
      if (persistent && f.final_kind != 2 && npend < kFastStageMax) {
        pend[npend++] = f;
      } else {
        if (npend > 0) {
          LAUNCH(launch_substeps_persistent(c, M, pend, npend, p_handoff), "fast substep");
          npend = 0;
        }
        if (terr) {  // the substep input's column reference, then the substep
          f.col_pref = M.colref[0]; f.col_rref = M.colref[1];
          LAUNCH(launch_column_reference(f, c->stream), "column reference");
        }
        LAUNCH(launch_substep(c, M, f, n == 0, terr, n == 0 && p_handoff), "fast substep");
      }
      M.ring = (M.ring + 1) % 3;
      rcur ^= 1;
      dcur = dout;
    }
    if (npend > 0) LAUNCH(launch_substeps_persistent(c, M, pend, npend, p_handoff), "fast substep");
  }
  return GWM_B200_OK;
}

// advance_passive_tracers_ssprk3 (dry_transport.cu:440-518) over every registered tracer,
// three tracers per kernel pass.  Each tracer is advanced on its own (the reference loops
// over tracers), so grouping does not change any result.  The reference boundary state
// covers the warm-rain triple; tracers added later take the Null tracer updater.
int enqueue_tracers(gwm_b200_ctx* c, Member& M) {
  const float wa[3] = {0.0f, 0.75f, 1.0f / 3.0f}, wb[3] = {1.0f, 0.25f, 2.0f / 3.0f};
  const int nt = (int)M.reg.size();
  for (int g0 = 0; g0 < nt; g0 += 3) {
    const int ng = std::min(3, nt - g0);
    const bool bnd = M.has_tracer_boundary && M.md.moist && g0 == 0;
    for (int s = 0; s < 3; ++s) {
      TracerArgs a{};
      a.g = M.g;
      a.rho = M.Q[0]; a.u = M.Q[2]; a.v = M.Q[3]; a.w = M.Q[4];
      for (int t = 0; t < ng; ++t) {
        const Member::Tracer& T = M.reg[g0 + t];
        a.q_in[t] = T.f[s];
        a.q0[t] = s == 0 ? nullptr : T.f[0];
        a.q_out[t] = T.f[(s + 1) % 3];
      }
      a.wa = wa[s]; a.wb = wb[s]; a.dt = M.md.step.dt;
      a.ntracers = ng;
      a.idz_c = M.idc; a.terrain = M.terrain_active;
      a.err = M.err;
      if (bnd) {  // TracerBoundaryUpdater::apply on the stage input
        if (M.bcache_n > 0) {  // PreparedCaseTracerBoundaryUpdater at sim_time 0, dt, dt/2
          const int rc = enqueue_boundary_interp(c, M, s);
          if (rc) return rc;
        }
        if (s == 0) {
          StripJobs J{};
          for (int t = 0; t < 3; ++t) J.j[J.n++] = strip_job(M.T0[t], M.bsave + M.boff[5 + t], nullptr, kCell, 1);
          LAUNCH(launch_strips(M.g, J, c->stream), "boundary strips");
        }
        StripJobs A{};
        for (int t = 0; t < 3; ++t)
          A.j[A.n++] = strip_job(const_cast<float*>(a.q_in[t]), M.bstrip + M.boff[5 + t], nullptr, kCell, 0);
        LAUNCH(launch_strips(M.g, A, c->stream), "boundary strips");
      }
      LAUNCH(launch_tracers(c, M, a), "tracer stage");
      if (bnd && s == 0) {
        const int rc = restore_stage1_strips(c, M, 5, 3, M.T0);
        if (rc) return rc;
      }
    }
  }
  return GWM_B200_OK;
}

// apply_warm_rain_microphysics (warm_rain.cu:214-353)
int enqueue_rain(gwm_b200_ctx* c, Member& M, int fallout) {
  const gwm_b200_warm_rain_config& r = M.md.rain;
  RainArgs a{};
  a.g = M.g;
  a.rho = M.Q[0]; a.rt = M.Q[1];
  a.qv = M.T0[0]; a.qc = M.T0[1]; a.qr = M.T0[2];
  a.precip = M.precip; a.precip_comp = M.pcomp;
  a.dt = r.dt; a.relax = r.condensation_relaxation; a.thr = r.cloud_autoconversion_threshold;
  a.rate = r.cloud_autoconversion_rate; a.evap = r.rain_evaporation_rate;
  a.vt = r.rain_terminal_velocity; a.layer_depth = r.sedimentation_layer_depth_m;
  a.latent = r.enable_latent_heating;
  int mode = 0;
  if (fallout == 1 && r.rain_terminal_velocity > 0.0f) mode = 1;
  if (fallout == 2 && r.rain_terminal_velocity > 0.0f && r.sedimentation_layer_depth_m > 0.0f) mode = 2;
  a.fallout_mode = mode;
  a.idz_c = M.idc; a.terrain = M.terrain_active;
  a.th_acc = M.slot(M.ring);
  a.inv_count = inv_count(M);
  if (M.use_surrogate) {
    SurrogateArgs sa{};
    sa.weights = (const unsigned char*)M.sur;
    sa.bias = (const float*)(M.sur + kSurWeightBytes);
    sa.norm = sa.bias + kSurBias;
    sa.range = sa.norm + kMlpNorm;
    sa.stats = (unsigned long long*)(M.sur + 65536);
    sa.work = (int*)(M.sur + 65536 + 128);
    sa.err = M.err;
    sa.tol_water = M.sur_tol_water;
    sa.tol_energy = M.sur_tol_energy;
    LAUNCH(launch_warm_rain_surrogate(a, sa, c->stream), "warm rain");
  } else {
    LAUNCH(launch_warm_rain(a, c->stream), "warm rain");
  }
  return GWM_B200_OK;
}

int enqueue_full_step(gwm_b200_ctx* c, Member& M) {
  int rc = enqueue_dry(c, M);
  if (rc) return rc;
  if (M.md.enable_tracer_transport && !M.reg.empty()) {
    rc = enqueue_tracers(c, M);
    if (rc) return rc;
  }
  if (M.md.moist && M.md.enable_warm_rain) {
    // the rain kernel accumulates the theta sums the next step's first stage reads
    rc = enqueue_rain(c, M, 1);
    if (rc) return rc;
  }
  return GWM_B200_OK;
}

int check_member(gwm_b200_ctx* c, int member) {
  if (!c) return GWM_B200_ERR_ARG;
  if (member < 0 || member >= (int)c->m.size()) return fail(c, GWM_B200_ERR_ARG, "member index out of range");
  return GWM_B200_OK;
}

void drop_graph(gwm_b200_ctx* c) {
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
}

}  // namespace

// ===========================================================================
extern "C" {

int gwm_b200_create(const gwm_b200_grid_desc* grids, const gwm_b200_member_desc* members,
                    int n_members, gwm_b200_ctx** out) {
  if (!out || !grids || !members || n_members <= 0) return GWM_B200_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GWM_B200_ERR_NO_DEVICE;
  auto* c = new gwm_b200_ctx();
  if (const char* t = std::getenv("GWM_B200_FAST_TILE_ROWS")) { const int r = std::atoi(t); c->fast_tile_rows = (r == 8 || r == 16) ? r : 0; }
  cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return GWM_B200_ERR_CUDA; }
  c->stream = c->own_stream;
  if (init_fast_tma() != cudaSuccess || init_fast_terrain_tma() != cudaSuccess || init_slow_tma() != cudaSuccess ||
      init_slow_terrain_tma() != cudaSuccess || init_tracer_tma() != cudaSuccess) {
    cudaStreamDestroy(c->own_stream);
    delete c;
    return GWM_B200_ERR_CUDA;
  }
  c->m.resize(n_members);
  for (int i = 0; i < n_members; ++i) {
    Member& M = c->m[i];
    M.gd = grids[i];
    M.md = members[i];
    const gwm_b200_grid_desc& d = M.gd;
    std::string why;
    if (d.nx <= 0 || d.ny <= 0 || d.nz <= 0) why = "grid dimensions must be positive";
    else if (d.halo != 1) why = "halo must be 1 (every stencil of the step reaches one cell)";
    else if (d.nz > kMaxNz) why = "nz exceeds the supported maximum (256)";
    else if (!(d.dx > 0 && d.dy > 0 && d.z_top > 0)) why = "dx, dy and z_top must be positive";
    else if ((double)(((kXOff + d.nx + 2 + 31) / 32) * 32) * (d.ny + 3) * (d.nz + 1) >= 2147483647.0)
      why = "grid too large for 32-bit field indexing";
    else if (M.md.step.fast_substeps < 1 && M.md.step.enable_fast_modes) why = "fast_substeps must be >= 1";
    if (!why.empty()) {
      gwm_b200_destroy(c);
      static thread_local std::string last;
      last = why;
      return GWM_B200_ERR_ARG;
    }
    if (d.terrain) {
      M.terrain.assign(d.terrain, d.terrain + (size_t)d.nx * d.ny);
      for (float h : M.terrain)  // terrain_active: dry_fast_modes.cu:484-492
        if (std::abs((double)h) > 1.0e-6) { M.terrain_active = true; break; }
    }
    if (d.eta_interfaces) M.eta.assign(d.eta_interfaces, d.eta_interfaces + d.nz + 1);
    M.gd.terrain = nullptr;
    M.gd.eta_interfaces = nullptr;
    int rc = alloc_member(c, M);
    if (rc != GWM_B200_OK) {
      std::fprintf(stderr, "gwm_b200_create: %s\n", c->err.c_str());
      gwm_b200_destroy(c);
      return rc;
    }
  }
  *out = c;
  return GWM_B200_OK;
}

void gwm_b200_destroy(gwm_b200_ctx* c) {
  if (!c) return;
  drop_graph(c);
  for (auto& M : c->m) {
    if (M.block) cudaFree(M.block);
    if (M.bstrip) cudaFree(M.bstrip);
    if (M.sur) cudaFree(M.sur);
    for (char* b : M.extra) cudaFree(b);
    if (M.bcache_block) cudaFree(M.bcache_block);
    if (M.io_stage) cudaFree(M.io_stage);
  }
  if (c->cin) cudaStreamDestroy(c->cin);
  if (c->cout) cudaStreamDestroy(c->cout);
  for (auto ev : c->io_ev) cudaEventDestroy(ev);
  for (auto st : c->mstreams) cudaStreamDestroy(st);
  for (auto ev : c->mjoin) cudaEventDestroy(ev);
  if (c->mfork) cudaEventDestroy(c->mfork);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

int gwm_b200_set_concurrent(gwm_b200_ctx* c, int enable) {
  if (!c) return GWM_B200_ERR_ARG;
  c->concurrent = enable != 0;
  drop_graph(c);
  return GWM_B200_OK;
}

const char* gwm_b200_last_error(const gwm_b200_ctx* c) { return c ? c->err.c_str() : "null context"; }

int gwm_b200_set_stream(gwm_b200_ctx* c, void* stream) {
  if (!c) return GWM_B200_ERR_ARG;
  drop_graph(c);
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return GWM_B200_OK;
}

int gwm_b200_synchronize(gwm_b200_ctx* c) {
  if (!c) return GWM_B200_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  return check_device_errors(c);
}

int gwm_b200_use_graph(gwm_b200_ctx* c, int enable) {
  if (!c) return GWM_B200_ERR_ARG;
  c->use_graph = enable != 0;
  if (!c->use_graph) drop_graph(c);
  return GWM_B200_OK;
}

long long gwm_b200_launch_count(const gwm_b200_ctx* c) { return c ? c->launches : -1; }

int gwm_b200_set_tile(gwm_b200_ctx* c, int kernel, int rows) {
  if (!c) return GWM_B200_ERR_ARG;
  const bool ok = kernel == 1   ? (rows == 0 || rows == kFastTma || rows == kFastStage || rows == 8 || rows == 16)
                  : kernel == 0 ? (rows == kSlowTma || rows == 8 || rows == 16)
                                : kernel == 2 && (rows == kTracerTma || rows == 8 || rows == 16);
  if (!ok) return GWM_B200_ERR_ARG;
  if ((kernel == 1 && (rows == kFastTma || rows == kFastStage)) || (kernel == 0 && rows == kSlowTma) ||
      (kernel == 2 && rows == kTracerTma))
    for (const auto& M : c->m)
      if (M.tmaps.empty())
        return fail(c, GWM_B200_ERR_ARG, "TMA substep unavailable (tensor-map encoder not found)");
  drop_graph(c);
  (kernel == 0 ? c->slow_tile_rows : kernel == 1 ? c->fast_tile_rows : c->tracer_tile_rows) = rows;
  return GWM_B200_OK;
}

int gwm_b200_get_tile(const gwm_b200_ctx* c, int kernel) {
  if (!c) return GWM_B200_ERR_ARG;
  if (kernel == 0) return c->slow_tile_rows;
  if (kernel == 1) return c->fast_tile_rows;
  if (kernel == 2) return c->tracer_tile_rows;
  return GWM_B200_ERR_ARG;
}

int gwm_b200_upload(gwm_b200_ctx* c, int member, const gwm_b200_fields* h) {
  int rc = check_member(c, member);
  if (rc) return rc;
  if (!h) return fail(c, GWM_B200_ERR_ARG, "null field set");
  Member& M = c->m[member];
  const Geom& g = M.g;
  struct F { const float* src; float* dst; int o; };
  std::vector<F> list = {{h->rho_d, M.Q[0], kCell}, {h->rho_theta_m, M.Q[1], kCell},
                         {h->mom_u, M.Q[2], kFaceX}, {h->mom_v, M.Q[3], kFaceY},
                         {h->mom_w, M.Q[4], kFaceZ}};
  if (M.md.moist) {
    list.push_back({h->qv, M.T0[0], kCell});
    list.push_back({h->qc, M.T0[1], kCell});
    list.push_back({h->qr, M.T0[2], kCell});
  } else if (h->qv || h->qc || h->qr || h->precip) {
    return fail(c, GWM_B200_ERR_ARG, "tracer fields given to a dry member");
  }
  for (const auto& f : list) {
    if (!f.src) continue;
    const size_t n = (size_t)(g.nx + (f.o == kFaceX)) * (g.ny + (f.o == kFaceY)) * (g.nz + (f.o == kFaceZ));
    CK(cudaMemcpyAsync(M.staging, f.src, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(launch_pack(g, f.o, M.staging, f.dst, c->stream));
  }
  if (M.md.moist && h->precip) {
    const size_t n = (size_t)g.nx * g.ny;
    CK(cudaMemcpyAsync(M.precip, h->precip, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(M.pcomp, 0, n * sizeof(double), c->stream));
  }
  if (h->rho_d || h->rho_theta_m) M.theta_valid = false;
  if (h->rho_theta_m) M.base_valid = false;
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_set_boundary_state(gwm_b200_ctx* c, int member, const gwm_b200_fields* h) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  drop_graph(c);
  M.bcache_n = 0;  // a fixed boundary state replaces a boundary cache
  if (!h) {
    M.has_boundary = M.has_tracer_boundary = false;
    return GWM_B200_OK;
  }
  if (!h->rho_d || !h->rho_theta_m || !h->mom_u || !h->mom_v || !h->mom_w)
    return fail(c, GWM_B200_ERR_ARG, "boundary state needs rho_d, rho_theta_m and the three momenta");
  const bool tracers = M.md.moist && h->qv && h->qc && h->qr;
  if (!M.bstrip) {
    long long off = 0;
    for (int f = 0; f < 8; ++f) { M.boff[f] = off; off += strip_len(M.g, kStripOrient[f]); }
    M.boff[8] = off;
    CK(cudaMalloc(&M.bstrip, 2 * off * sizeof(float)));
    CK(cudaMemsetAsync(M.bstrip, 0, 2 * off * sizeof(float), c->stream));
    M.bsave = M.bstrip + off;
  }
  const float* src[8] = {h->rho_d, h->rho_theta_m, h->mom_u, h->mom_v, h->mom_w, h->qv, h->qc, h->qr};
  const Geom& g = M.g;
  for (int f = 0; f < (tracers ? 8 : 5); ++f) {
    const int o = kStripOrient[f];
    const size_t n = (size_t)(g.nx + (o == kFaceX)) * (g.ny + (o == kFaceY)) * (g.nz + (o == kFaceZ));
    CK(cudaMemcpyAsync(M.staging, src[f], n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    StripJobs J{};
    J.j[J.n++] = strip_job(nullptr, M.bstrip + M.boff[f], M.staging, o, 2);
    CK(launch_strips(g, J, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  M.has_boundary = true;
  M.has_tracer_boundary = tracers;
  return GWM_B200_OK;
}

int gwm_b200_set_boundary_cache(gwm_b200_ctx* c, int member, int n, const int* offsets,
                                const gwm_b200_fields* snapshots) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  drop_graph(c);
  if (n <= 0 || !offsets || !snapshots) {
    M.bcache_n = 0;
    M.has_boundary = M.has_tracer_boundary = false;
    return n == 0 ? GWM_B200_OK : fail(c, GWM_B200_ERR_ARG, "boundary cache needs snapshots and offsets");
  }
  for (int q = 1; q < n; ++q)  // validate_runtime_boundary_cache (runtime_case.cpp:260-262)
    if (offsets[q] <= offsets[q - 1]) return fail(c, GWM_B200_ERR_ARG, "Boundary cache offsets must be strictly monotonic");
  bool tracers = M.md.moist != 0;
  for (int q = 0; q < n; ++q) {
    const gwm_b200_fields& h = snapshots[q];
    if (!h.rho_d || !h.rho_theta_m || !h.mom_u || !h.mom_v || !h.mom_w)
      return fail(c, GWM_B200_ERR_ARG, "boundary snapshots need rho_d, rho_theta_m and the three momenta");
    tracers = tracers && h.qv && h.qc && h.qr;
  }
  if (!M.bstrip) {
    long long off = 0;
    for (int f = 0; f < 8; ++f) { M.boff[f] = off; off += strip_len(M.g, kStripOrient[f]); }
    M.boff[8] = off;
    CK(cudaMalloc(&M.bstrip, 2 * off * sizeof(float)));
    CK(cudaMemsetAsync(M.bstrip, 0, 2 * off * sizeof(float), c->stream));
    M.bsave = M.bstrip + off;
  }
  if (M.bcache_block) { CK(cudaFree(M.bcache_block)); M.bcache_block = nullptr; }
  const size_t snap_bytes = ((size_t)n * M.boff[8] * sizeof(float) + 255) / 256 * 256;
  const size_t off_bytes = ((size_t)n * sizeof(int) + 255) / 256 * 256;
  CK(cudaMalloc(&M.bcache_block, snap_bytes + off_bytes + sizeof(BoundaryClock)));
  M.bcache = (float*)M.bcache_block;
  M.bcache_off = (int*)(M.bcache_block + snap_bytes);
  M.bclock = (BoundaryClock*)(M.bcache_block + snap_bytes + off_bytes);
  const Geom& g = M.g;
  for (int q = 0; q < n; ++q) {
    const gwm_b200_fields& h = snapshots[q];
    const float* src[8] = {h.rho_d, h.rho_theta_m, h.mom_u, h.mom_v, h.mom_w, h.qv, h.qc, h.qr};
    for (int f = 0; f < (tracers ? 8 : 5); ++f) {
      const int o = kStripOrient[f];
      const size_t cnt = (size_t)(g.nx + (o == kFaceX)) * (g.ny + (o == kFaceY)) * (g.nz + (o == kFaceZ));
      CK(cudaMemcpyAsync(M.staging, src[f], cnt * sizeof(float), cudaMemcpyHostToDevice, c->stream));
      StripJobs J{};
      J.j[J.n++] = strip_job(nullptr, M.bcache + (size_t)q * M.boff[8] + M.boff[f], M.staging, o, 2);
      CK(launch_strips(g, J, c->stream));
      CK(cudaStreamSynchronize(c->stream));  // the staging buffer is reused by the next copy
    }
  }
  CK(cudaMemcpyAsync(M.bcache_off, offsets, n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  BoundaryClock clk{};
  clk.t_start = 0.0f;
  clk.dt = M.md.step.dt;
  CK(cudaMemcpyAsync(M.bclock, &clk, sizeof(clk), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  M.bcache_n = n;
  M.has_boundary = true;
  M.has_tracer_boundary = tracers;
  return GWM_B200_OK;
}

int gwm_b200_set_step_start_time(gwm_b200_ctx* c, int member, float t) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  if (M.bcache_n <= 0) return fail(c, GWM_B200_ERR_ARG, "no boundary cache is set");
  const float t0 = std::max(t, 0.0f);  // set_step_start_time (prepared_case_init.cpp:1006-1009)
  CK(cudaMemcpyAsync(&M.bclock->t_start, &t0, sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_get_step_start_time(gwm_b200_ctx* c, int member, float* t) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  if (!t) return fail(c, GWM_B200_ERR_ARG, "null output");
  if (M.bcache_n <= 0) return fail(c, GWM_B200_ERR_ARG, "no boundary cache is set");
  CK(cudaMemcpyAsync(t, &M.bclock->t_start, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

// Rayleigh damping rate tau(z) = rate * sin^2(pi/2 (z - z_d)/(z_top - z_d)) above z_d at a
// level's terrain-free height eta * z_top (an extension: the reference has no damping layer).
static double rayleigh_rate(double z, double z_d, double z_top, double rate) {
  if (rate <= 0.0 || z <= z_d || z_top <= z_d) return 0.0;
  const double s = std::sin(0.5 * 3.14159265358979323846 * std::min(1.0, (z - z_d) / (z_top - z_d)));
  return rate * s * s;
}

int gwm_b200_set_damping(gwm_b200_ctx* c, int member, double z_bottom, double rate, const double* u_ref,
                         const double* v_ref) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  drop_graph(c);
  if (rate <= 0.0) { M.damping = false; return GWM_B200_OK; }
  const int nz = M.g.nz;
  const double zt = M.gd.z_top;
  std::vector<float> h(4 * (kMaxNz + 1), 0.0f);
  for (int k = 0; k < nz; ++k) {
    const double ec = M.eta.empty() ? ((double)k + 0.5) / nz : 0.5 * (M.eta[k] + M.eta[k + 1]);
    h[k] = (float)rayleigh_rate(ec * zt, z_bottom, zt, rate);
    h[2 * (kMaxNz + 1) + k] = u_ref ? (float)u_ref[k] : 0.0f;
    h[3 * (kMaxNz + 1) + k] = v_ref ? (float)v_ref[k] : 0.0f;
  }
  for (int k = 0; k <= nz; ++k) {
    const double ei = M.eta.empty() ? (double)k / nz : M.eta[k];
    h[(kMaxNz + 1) + k] = (float)rayleigh_rate(ei * zt, z_bottom, zt, rate);
  }
  CK(cudaMemcpy(M.damp, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
  M.damping = true;
  return GWM_B200_OK;
}

int gwm_b200_apply_reference_boundaries(gwm_b200_ctx* c, int member) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  if (!M.has_boundary) return fail(c, GWM_B200_ERR_ARG, "no boundary state set");
  StripJobs J{};
  for (int f = 0; f < 5; ++f) J.j[J.n++] = strip_job(M.Q[f], M.bstrip + M.boff[f], nullptr, kStripOrient[f], 0);
  if (M.has_tracer_boundary)
    for (int t = 0; t < 3; ++t) J.j[J.n++] = strip_job(M.T0[t], M.bstrip + M.boff[5 + t], nullptr, kCell, 0);
  CK(launch_strips(M.g, J, c->stream));
  M.theta_valid = false;
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

// ---------------------------------------------------------------------------
// Learned warm-rain microphysics: samples, training, gradient.
namespace {
RainArgs rain_args(const Member& M, int fallout) {
  const gwm_b200_warm_rain_config& r = M.md.rain;
  RainArgs a{};
  a.g = M.g;
  a.rho = M.Q[0]; a.rt = M.Q[1];
  a.qv = M.T0[0]; a.qc = M.T0[1]; a.qr = M.T0[2];
  a.dt = r.dt; a.relax = r.condensation_relaxation; a.thr = r.cloud_autoconversion_threshold;
  a.rate = r.cloud_autoconversion_rate; a.evap = r.rain_evaporation_rate;
  a.vt = r.rain_terminal_velocity; a.layer_depth = r.sedimentation_layer_depth_m;
  a.latent = r.enable_latent_heating;
  int mode = 0;
  if (fallout == 1 && r.rain_terminal_velocity > 0.0f) mode = 1;
  if (fallout == 2 && r.rain_terminal_velocity > 0.0f && r.sedimentation_layer_depth_m > 0.0f) mode = 2;
  a.fallout_mode = mode;
  a.idz_c = M.idc; a.terrain = M.terrain_active;
  return a;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
}  // namespace

int gwm_b200_rain_record(gwm_b200_ctx* c, int member, float* x, float* y, long long capacity,
                         unsigned long long seed, float p_active, float p_inactive, long long* n_out) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  if (!M.md.moist) return fail(c, GWM_B200_ERR_ARG, "warm-rain samples need a moist member");
  if (!x || !y || capacity <= 0 || !n_out) return fail(c, GWM_B200_ERR_ARG, "bad sample buffers");
  RecordArgs a{};
  a.r = rain_args(M, 1);
  a.x = x; a.y = y; a.capacity = capacity; a.seed = seed;
  a.p_active = p_active; a.p_inactive = p_inactive;
  unsigned long long* count = nullptr;
  CK(cudaMallocAsync(&count, sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(count, 0, sizeof(unsigned long long), c->stream));
  a.count = count;
  CK(launch_rain_record(a, c->stream));
  unsigned long long h = 0;
  CK(cudaMemcpyAsync(&h, count, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(count, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *n_out = (long long)std::min<unsigned long long>(h, (unsigned long long)capacity);
  return GWM_B200_OK;
}

int gwm_b200_mlp_loss_grad(const float* params, const float* norm, const float* x, const float* y, int n,
                           float* grad, double* loss) {
  if (!params || !norm || !x || !y || n <= 0 || !grad || !loss) return GWM_B200_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GWM_B200_ERR_NO_DEVICE;
  cudaStream_t s = nullptr;
  float *dp = nullptr, *dn = nullptr, *dx = nullptr, *dy = nullptr, *scr = nullptr, *part = nullptr, *dg = nullptr;
  double* dl = nullptr;
  auto bad = [&](cudaError_t e) { return e != cudaSuccess; };
  int rc = GWM_B200_OK;
  if (bad(cudaMalloc(&dp, kMlpParams * 4)) || bad(cudaMalloc(&dn, kMlpNorm * 4)) ||
      bad(cudaMalloc(&dx, (size_t)n * kMlpIn * 4)) || bad(cudaMalloc(&dy, (size_t)n * kMlpOut * 4)) ||
      bad(cudaMalloc(&scr, mlp_scratch_floats(n) * 4)) || bad(cudaMalloc(&part, mlp_partial_floats(n) * 4)) ||
      bad(cudaMalloc(&dg, kMlpParams * 4)) || bad(cudaMalloc(&dl, sizeof(double)))) {
    rc = GWM_B200_ERR_CUDA;
  } else {
    cudaMemcpy(dp, params, kMlpParams * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dn, norm, kMlpNorm * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dx, x, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dy, y, (size_t)n * kMlpOut * 4, cudaMemcpyHostToDevice);
    MlpBatch b{dp, dn, dx, dy, nullptr, n, scr, part, dg, dl};
    if (bad(mlp_loss_grad(b, s)) || bad(cudaMemcpy(grad, dg, kMlpParams * 4, cudaMemcpyDeviceToHost)) ||
        bad(cudaMemcpy(loss, dl, sizeof(double), cudaMemcpyDeviceToHost)))
      rc = GWM_B200_ERR_CUDA;
  }
  for (void* p : {(void*)dp, (void*)dn, (void*)dx, (void*)dy, (void*)scr, (void*)part, (void*)dg, (void*)dl})
    if (p) cudaFree(p);
  return rc;
}

int gwm_b200_mlp_train(const float* x, const float* y, long long n, const gwm_b200_mlp_train_config* cfg,
                       float* params, float* norm, float* range, double* loss_per_epoch) {
  if (!x || !y || n <= 0 || !cfg || !params || !norm || cfg->epochs <= 0 || cfg->batch <= 0) return GWM_B200_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GWM_B200_ERR_NO_DEVICE;
  const int batch = (int)std::min<long long>(cfg->batch, n);
  cudaStream_t s = nullptr;
  std::vector<void*> owned;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return p;
  };
  auto cleanup = [&](int rc) {
    for (void* p : owned) cudaFree(p);
    return rc;
  };
  double* stats = (double*)alloc((2 * kMlpIn + 2 * kMlpIn + 2 * kMlpOut) * sizeof(double));
  float* dp = (float*)alloc(kMlpParams * 4);
  float* dn = (float*)alloc(kMlpNorm * 4);
  float* dg = (float*)alloc(kMlpParams * 4);
  float* dm = (float*)alloc(kMlpParams * 4);
  float* dv = (float*)alloc(kMlpParams * 4);
  float* scr = (float*)alloc(mlp_scratch_floats(batch) * 4);
  float* part = (float*)alloc(mlp_partial_floats(batch) * 4);
  double* dl = (double*)alloc(sizeof(double));
  int* didx = (int*)alloc((size_t)n * sizeof(int));
  if (!stats || !dp || !dn || !dg || !dm || !dv || !scr || !part || !dl || !didx) return cleanup(GWM_B200_ERR_CUDA);
  // normalisation: FP64 means and standard deviations of inputs and targets; input range
  if (mlp_column_stats(x, n, kMlpIn, stats, stats + 2 * kMlpIn, s) != cudaSuccess ||
      mlp_column_stats(y, n, kMlpOut, stats + 4 * kMlpIn, nullptr, s) != cudaSuccess)
    return cleanup(GWM_B200_ERR_CUDA);
  double hs[4 * kMlpIn + 2 * kMlpOut];
  if (cudaMemcpy(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost) != cudaSuccess) return cleanup(GWM_B200_ERR_CUDA);
  for (int f = 0; f < kMlpIn; ++f) {
    norm[f] = (float)hs[f];
    norm[kMlpIn + f] = hs[kMlpIn + f] > 1e-30 ? (float)hs[kMlpIn + f] : 1.0f;  // constant input (dt)
    if (range) { range[f] = (float)hs[2 * kMlpIn + f]; range[kMlpIn + f] = (float)hs[3 * kMlpIn + f]; }
  }
  for (int o = 0; o < kMlpOut; ++o) {
    norm[2 * kMlpIn + o] = (float)hs[4 * kMlpIn + o];
    const double sd = hs[4 * kMlpIn + kMlpOut + o];
    // a target that never varies gets scale 0: inference reproduces its mean exactly
    norm[2 * kMlpIn + kMlpOut + o] = sd > 1e-30 ? (float)sd : 0.0f;
  }
  uint64_t rng = cfg->seed ? cfg->seed : 0x5EED5EEDull;
  if (cfg->init) {  // Xavier-uniform weights, zero biases
    auto uni = [&]() { return (double)(splitmix(rng) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0; };
    auto fill_w = [&](int off, int nout, int nin) {
      const double lim = std::sqrt(6.0 / (nin + nout));
      for (int q = 0; q < nout * nin; ++q) params[off + q] = (float)(lim * uni());
    };
    std::fill(params, params + kMlpParams, 0.0f);
    fill_w(kOffW1, kMlpHid, kMlpIn);
    fill_w(kOffW2, kMlpHid, kMlpHid);
    fill_w(kOffW3, kMlpHid, kMlpHid);
    fill_w(kOffW4, kMlpOut, kMlpHid);
  }
  cudaMemcpy(dp, params, kMlpParams * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dn, norm, kMlpNorm * 4, cudaMemcpyHostToDevice);
  cudaMemset(dm, 0, kMlpParams * 4);
  cudaMemset(dv, 0, kMlpParams * 4);
  std::vector<int> perm((size_t)n);
  for (long long q = 0; q < n; ++q) perm[(size_t)q] = (int)q;
  int t = 0;
  for (int ep = 0; ep < cfg->epochs; ++ep) {
    for (long long q = n - 1; q > 0; --q) std::swap(perm[(size_t)q], perm[(size_t)(splitmix(rng) % (uint64_t)(q + 1))]);
    if (cudaMemcpy(didx, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      return cleanup(GWM_B200_ERR_CUDA);
    double ep_loss = 0.0;
    long long seen = 0;
    for (long long b0 = 0; b0 + batch <= n; b0 += batch) {
      MlpBatch b{dp, dn, x, y, didx + b0, batch, scr, part, dg, dl};
      if (mlp_loss_grad(b, s) != cudaSuccess || mlp_adam(dp, dg, dm, dv, cfg->lr, ++t, s) != cudaSuccess)
        return cleanup(GWM_B200_ERR_CUDA);
      double l = 0.0;
      if (cudaMemcpy(&l, dl, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return cleanup(GWM_B200_ERR_CUDA);
      ep_loss += l * batch;
      seen += batch;
    }
    if (loss_per_epoch) loss_per_epoch[ep] = seen ? ep_loss / (double)seen : 0.0;
  }
  if (cudaMemcpy(params, dp, kMlpParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return cleanup(GWM_B200_ERR_CUDA);
  return cleanup(GWM_B200_OK);
}

int gwm_b200_mlp_infer(const float* params, const float* norm, const float* x, float* y, long long n, void* stream) {
  if (!params || !norm || !x || !y || n <= 0 || n > 0x7fffff00LL) return GWM_B200_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GWM_B200_ERR_NO_DEVICE;
  std::vector<unsigned char> fr(kSurWeightBytes);
  std::vector<float> tail(kSurBias + kMlpNorm + kMlpRange, 0.0f);
  surrogate_operands(params, fr.data(), tail.data());
  std::copy(norm, norm + kMlpNorm, tail.begin() + kSurBias);
  char* buf = nullptr;
  if (cudaMalloc(&buf, 65536 + 256) != cudaSuccess) return GWM_B200_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  bool ok = cudaMemsetAsync(buf + 65536, 0, 256, s) == cudaSuccess &&
            cudaMemcpyAsync(buf, fr.data(), fr.size(), cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(buf + fr.size(), tail.data(), tail.size() * sizeof(float), cudaMemcpyHostToDevice, s) ==
                cudaSuccess;
  SurrogateArgs sa{};
  sa.weights = (const unsigned char*)buf;
  sa.bias = (const float*)(buf + kSurWeightBytes);
  sa.norm = sa.bias + kSurBias;
  sa.range = sa.norm + kMlpNorm;
  sa.stats = nullptr;
  sa.work = (int*)(buf + 65536 + 128);
  sa.err = (int*)(buf + 65536 + 192);
  sa.eval_x = x;
  sa.eval_y = y;
  sa.eval_n = n;
  int err = 0;
  ok = ok && launch_rain_net_eval(sa, s) == cudaSuccess &&
       cudaMemcpyAsync(&err, sa.err, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
       cudaStreamSynchronize(s) == cudaSuccess;
  cudaFree(buf);
  if (!ok) return GWM_B200_ERR_CUDA;
  return err ? GWM_B200_ERR_TIMEOUT : GWM_B200_OK;
}

int gwm_b200_set_rain_surrogate(gwm_b200_ctx* c, int member, const float* params, const float* norm,
                                const float* range, float tol_water, float tol_energy) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  drop_graph(c);
  if (!params) { M.use_surrogate = false; return GWM_B200_OK; }
  if (!norm || !range || !M.md.moist) return fail(c, GWM_B200_ERR_ARG, "surrogate needs norm, range and a moist member");
  if (!M.sur) {
    CK(cudaMalloc(&M.sur, 65536 + 256));
    CK(cudaMemset(M.sur + 65536, 0, 256));
  }
  static_assert(kSurWeightBytes + (kSurBias + kMlpNorm + kMlpRange) * sizeof(float) <= 65536, "surrogate buffer");
  std::vector<unsigned char> fr(kSurWeightBytes);
  std::vector<float> tail(kSurBias + kMlpNorm + kMlpRange);
  surrogate_operands(params, fr.data(), tail.data());
  std::copy(norm, norm + kMlpNorm, tail.begin() + kSurBias);
  std::copy(range, range + kMlpRange, tail.begin() + kSurBias + kMlpNorm);
  CK(cudaMemcpy(M.sur, fr.data(), fr.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(M.sur + fr.size(), tail.data(), tail.size() * sizeof(float), cudaMemcpyHostToDevice));
  M.use_surrogate = true;
  M.sur_tol_water = tol_water;
  M.sur_tol_energy = tol_energy;
  return GWM_B200_OK;
}

int gwm_b200_surrogate_stats(gwm_b200_ctx* c, int member, long long* stats, int reset) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  if (!stats) return GWM_B200_ERR_ARG;
  std::fill(stats, stats + GWM_B200_SURROGATE_STATS, 0LL);
  if (!M.sur) return GWM_B200_OK;
  static_assert(GWM_B200_SURROGATE_STATS == kSurStats, "surrogate counters");
  unsigned long long h[kSurStats] = {};
  CK(cudaMemcpyAsync(h, M.sur + 65536, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  if (reset) CK(cudaMemsetAsync(M.sur + 65536, 0, sizeof(h), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int q = 0; q < kSurStats; ++q) stats[q] = (long long)h[q];
  return GWM_B200_OK;
}

int gwm_b200_test_stall_tile_load(gwm_b200_ctx* c, int member, int plane) {
  const int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  if (plane < 0 || plane > M.g.nz) return fail(c, GWM_B200_ERR_ARG, "plane out of range");
  const int word = plane + 1;  // err[1]: 0 = no request
  CK(cudaMemcpyAsync(M.err + 1, &word, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_surrogate_fallbacks(gwm_b200_ctx* c, int member, long long* count, int reset) {
  if (!count) return GWM_B200_ERR_ARG;
  long long st[GWM_B200_SURROGATE_STATS];
  int rc = gwm_b200_surrogate_stats(c, member, st, reset);
  *count = rc ? 0 : st[0];
  return rc;
}

// ---- tracer registry ----------------------------------------------------------
int gwm_b200_tracer_add(gwm_b200_ctx* c, int member, const char* name, const char* units, int positive) {
  int rc = check_member(c, member);
  if (rc) return rc;
  if (!name || !*name) return fail(c, GWM_B200_ERR_ARG, "tracer name must not be empty");
  Member& M = c->m[member];
  for (const auto& t : M.reg)
    if (t.name == name) return fail(c, GWM_B200_ERR_ARG, "Tracer already exists in registry");
  const size_t fbytes = ((M.field_elems * sizeof(float) + 255) / 256) * 256;
  char* blk = nullptr;
  CK(cudaMalloc(&blk, 3 * fbytes));
  M.extra.push_back(blk);
  CK(cudaMemsetAsync(blk, 0, 3 * fbytes, c->stream));
  Member::Tracer tr;
  tr.name = name;
  tr.units = units ? units : "";
  tr.positive = positive != 0;
  for (int q = 0; q < 3; ++q) tr.f[q] = (float*)(blk + q * fbytes);
  if (!M.tmaps.empty()) {  // TMA maps of the tracer stage (cells with the ring)
    for (int q = 0; q < 3; ++q) {
      CUtensorMap m;
      if (!encode_field_map(&m, tr.f[q], M.g, kTmaCellBox[0], kTmaCellBox[1]))
        return fail(c, GWM_B200_ERR_CUDA, "tensor map of an added tracer");
      M.tmaps.emplace_back(tr.f[q], 0, m);
    }
  }
  M.reg.push_back(tr);
  drop_graph(c);  // the step now launches more tracer passes
  CK(cudaStreamSynchronize(c->stream));
  return (int)M.reg.size() - 1;
}

int gwm_b200_tracer_find(const gwm_b200_ctx* c, int member, const char* name) {
  if (!c || member < 0 || member >= (int)c->m.size() || !name) return GWM_B200_ERR_ARG;
  const auto& reg = c->m[member].reg;
  for (size_t t = 0; t < reg.size(); ++t)
    if (reg[t].name == name) return (int)t;
  return GWM_B200_ERR_ARG;
}

int gwm_b200_tracer_count(const gwm_b200_ctx* c, int member) {
  if (!c || member < 0 || member >= (int)c->m.size()) return GWM_B200_ERR_ARG;
  return (int)c->m[member].reg.size();
}

const char* gwm_b200_tracer_name(const gwm_b200_ctx* c, int member, int index) {
  if (!c || member < 0 || member >= (int)c->m.size()) return nullptr;
  const auto& reg = c->m[member].reg;
  if (index < 0 || index >= (int)reg.size()) return nullptr;
  return reg[index].name.c_str();
}

static int tracer_index(gwm_b200_ctx* c, int member, int index) {
  const int rc = check_member(c, member);
  if (rc) return rc;
  if (index < 0 || index >= (int)c->m[member].reg.size()) return fail(c, GWM_B200_ERR_ARG, "tracer index out of range");
  return GWM_B200_OK;
}

int gwm_b200_tracer_upload(gwm_b200_ctx* c, int member, int index, const float* host) {
  int rc = tracer_index(c, member, index);
  if (rc) return rc;
  if (!host) return fail(c, GWM_B200_ERR_ARG, "null tracer field");
  Member& M = c->m[member];
  const size_t n = (size_t)M.g.nx * M.g.ny * M.g.nz;
  CK(cudaMemcpyAsync(M.staging, host, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CK(launch_pack(M.g, kCell, M.staging, M.reg[index].f[0], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_tracer_download(gwm_b200_ctx* c, int member, int index, float* host) {
  int rc = tracer_index(c, member, index);
  if (rc) return rc;
  if (!host) return fail(c, GWM_B200_ERR_ARG, "null tracer field");
  Member& M = c->m[member];
  const size_t n = (size_t)M.g.nx * M.g.ny * M.g.nz;
  CK(launch_unpack(M.g, kCell, M.reg[index].f[0], M.staging, c->stream));
  CK(cudaMemcpyAsync(host, M.staging, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_tracer_total(gwm_b200_ctx* c, int member, int index, double* total) {
  int rc = tracer_index(c, member, index);
  if (rc) return rc;
  if (!total) return fail(c, GWM_B200_ERR_ARG, "null output");
  Member& M = c->m[member];
  CK(launch_reduce(M.g, kCell, 0, M.reg[index].f[0], nullptr, nullptr, 0, M.red_part, M.red_out + 20, c->stream));
  ReduceOut r;
  CK(cudaMemcpyAsync(&r, M.red_out + 20, sizeof(ReduceOut), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *total = r.sum;
  return GWM_B200_OK;
}

int gwm_b200_download(gwm_b200_ctx* c, int member, gwm_b200_fields* h) {
  int rc = check_member(c, member);
  if (rc) return rc;
  if (!h) return fail(c, GWM_B200_ERR_ARG, "null field set");
  Member& M = c->m[member];
  const Geom& g = M.g;
  struct F { float* dst; const float* src; int o; };
  std::vector<F> list = {{h->rho_d, M.Q[0], kCell}, {h->rho_theta_m, M.Q[1], kCell},
                         {h->mom_u, M.Q[2], kFaceX}, {h->mom_v, M.Q[3], kFaceY},
                         {h->mom_w, M.Q[4], kFaceZ}};
  if (M.md.moist) {
    list.push_back({h->qv, M.T0[0], kCell});
    list.push_back({h->qc, M.T0[1], kCell});
    list.push_back({h->qr, M.T0[2], kCell});
  }
  for (const auto& f : list) {
    if (!f.dst) continue;
    const size_t n = (size_t)(g.nx + (f.o == kFaceX)) * (g.ny + (f.o == kFaceY)) * (g.nz + (f.o == kFaceZ));
    CK(launch_unpack(g, f.o, f.src, M.staging, c->stream));
    CK(cudaMemcpyAsync(f.dst, M.staging, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  }
  if (M.md.moist && h->precip) {
    const size_t n = (size_t)g.nx * g.ny;
    std::vector<double> comp(n);
    CK(cudaMemcpyAsync(h->precip, M.precip, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(comp.data(), M.pcomp, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t q = 0; q < n; ++q) h->precip[q] += comp[q];
  }
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

// One pass of `one` over all members: concurrently on per-member streams (fork/join
// around the context stream) when there are several, else in order on the stream.
static int enqueue_members(gwm_b200_ctx* c, int (*one)(gwm_b200_ctx*, Member&)) {
  const size_t n = c->m.size();
  if (n <= 1 || !c->concurrent || c->profile) {
    for (auto& M : c->m) {
      const int rc = one(c, M);
      if (rc) return rc;
    }
    return GWM_B200_OK;
  }
  if (c->mstreams.size() != n) {
    for (size_t i = c->mstreams.size(); i < n; ++i) {
      cudaStream_t st;
      cudaEvent_t ev;
      CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      c->mstreams.push_back(st);
      c->mjoin.push_back(ev);
    }
    if (!c->mfork) CK(cudaEventCreateWithFlags(&c->mfork, cudaEventDisableTiming));
  }
  cudaStream_t main = c->stream;
  CK(cudaEventRecord(c->mfork, main));
  int rc = GWM_B200_OK;
  for (size_t i = 0; i < n && !rc; ++i) {
    CK(cudaStreamWaitEvent(c->mstreams[i], c->mfork, 0));
    c->stream = c->mstreams[i];
    rc = one(c, c->m[i]);
    c->stream = main;
    CK(cudaEventRecord(c->mjoin[i], c->mstreams[i]));
    CK(cudaStreamWaitEvent(main, c->mjoin[i], 0));
  }
  return rc;
}

static int run_steps(gwm_b200_ctx* c, int nsteps, int (*one)(gwm_b200_ctx*, Member&)) {
  c->cur_launches = 0;
  for (auto& M : c->m) {
    int rc = ensure_base(c, M);
    if (rc) return rc;
    if (!M.theta_valid) {
      rc = enqueue_theta(c, M);
      if (rc) return rc;
    }
  }
  if (c->use_graph && !c->profile && nsteps > 0 && one == enqueue_full_step) {
    if (!c->graph) {
      const long long before = c->cur_launches;
      std::vector<int> rings;
      for (auto& M : c->m) rings.push_back(M.ring);
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue_members(c, one);
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
      if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
      if (e != cudaSuccess) return fail(c, GWM_B200_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&c->graph, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return fail(c, GWM_B200_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      c->graph_launches = c->cur_launches - before;
      // a step advances every ring by a multiple of three: restore the positions
      for (size_t i = 0; i < c->m.size(); ++i) c->m[i].ring = rings[i];
      c->cur_launches = before;
    }
    for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(c->graph, c->stream));
    c->cur_launches += c->graph_launches * nsteps;
  } else {
    for (int s = 0; s < nsteps; ++s) {
      const int rc = enqueue_members(c, one);
      if (rc) return rc;
    }
  }
  c->launches = c->cur_launches;
  if (c->stream == c->own_stream || c->profile) {
    CK(cudaStreamSynchronize(c->stream));
    const int rc = check_device_errors(c);
    if (rc) return rc;
  }
  if (c->profile) {
    for (auto& pe : c->prof_events) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
      c->prof_ms[pe.first] += ms;
      c->prof_n[pe.first] += 1;
      cudaEventDestroy(pe.second.first);
      cudaEventDestroy(pe.second.second);
    }
    c->prof_events.clear();
  }
  return GWM_B200_OK;
}

int gwm_b200_profile(gwm_b200_ctx* c, int enable) {
  if (!c) return GWM_B200_ERR_ARG;
  c->profile = enable != 0;
  if (c->profile) drop_graph(c);
  for (int k = 0; k < kKinds; ++k) { c->prof_ms[k] = 0; c->prof_n[k] = 0; }
  return GWM_B200_OK;
}

int gwm_b200_profile_read(const gwm_b200_ctx* c, int kind, double* total_ms, long long* launches,
                          const char** name) {
  if (!c || kind < 0 || kind >= kKinds) return GWM_B200_ERR_ARG;
  if (total_ms) *total_ms = c->prof_ms[kind];
  if (launches) *launches = c->prof_n[kind];
  if (name) *name = kKindNames[kind];
  return kKinds;
}

int gwm_b200_step(gwm_b200_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return GWM_B200_ERR_ARG;
  return run_steps(c, nsteps, enqueue_full_step);
}

// One full step of a single-member context from host buffers to host buffers: the state
// is copied in from `in`, advanced as gwm_b200_step does, and copied out to `out` (the
// same buffers may be given for both).  The copies overlap the step's phases on two copy
// streams.  The moisture fields and the precipitation go up while the dry step runs (it
// does not read them), and rho and the momenta, which neither the tracers nor the warm
// rain change, come down while those run.  Results equal upload + step + download.
int gwm_b200_step_host(gwm_b200_ctx* c, const gwm_b200_fields* in, gwm_b200_fields* out) {
  if (!c || !in || !out) return GWM_B200_ERR_ARG;
  if (c->m.size() != 1) return fail(c, GWM_B200_ERR_ARG, "host-to-host stepping takes a single-member context");
  Member& M = c->m[0];
  const Geom& g = M.g;
  const bool moist = M.md.moist != 0;
  const float* src[8] = {in->rho_d, in->rho_theta_m, in->mom_u, in->mom_v, in->mom_w, in->qv, in->qc, in->qr};
  float* dst[8] = {out->rho_d, out->rho_theta_m, out->mom_u, out->mom_v, out->mom_w, out->qv, out->qc, out->qr};
  float* dev[8] = {M.Q[0], M.Q[1], M.Q[2], M.Q[3], M.Q[4], M.T0[0], M.T0[1], M.T0[2]};
  constexpr int orient[8] = {kCell, kCell, kFaceX, kFaceY, kFaceZ, kCell, kCell, kCell};
  const int nf = moist ? 8 : 5;
  for (int f = 0; f < nf; ++f)
    if (!src[f] || !dst[f]) return fail(c, GWM_B200_ERR_ARG, "host-to-host stepping needs every field of the state");
  if (moist && (!in->precip || !out->precip))
    return fail(c, GWM_B200_ERR_ARG, "host-to-host stepping of a moist member needs the precipitation");
  if (!moist && (in->qv || in->qc || in->qr || in->precip))
    return fail(c, GWM_B200_ERR_ARG, "tracer fields given to a dry member");
  const size_t owned_max = (size_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  if (!c->cin) {
    CK(cudaStreamCreateWithFlags(&c->cin, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->cout, cudaStreamNonBlocking));
    c->io_ev.assign(11, nullptr);
    for (auto& ev : c->io_ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  if (!M.io_stage) CK(cudaMalloc(&M.io_stage, 8 * owned_max * sizeof(float)));
  auto stage = [&](int f) { return M.io_stage + (size_t)f * owned_max; };
  auto count = [&](int f) {
    const int o = orient[f];
    return (size_t)(g.nx + (o == kFaceX)) * (g.ny + (o == kFaceY)) * (g.nz + (o == kFaceZ));
  };
  cudaEvent_t* ev_in = c->io_ev.data();  // [0..8]: field f (8: precipitation) is on the device
  cudaEvent_t ev_dry = c->io_ev[9], ev_end = c->io_ev[10];
  const size_t n2 = (size_t)g.nx * g.ny;
  c->cur_launches = 0;
  // the dry fields up, each packed as soon as it lands; rho and rho*theta first, so the
  // EOS base state and the theta level sums of the new state run while the momenta land
  M.theta_valid = false;
  M.base_valid = false;
  for (int f = 0; f < 5; ++f) {
    CK(cudaMemcpyAsync(stage(f), src[f], count(f) * sizeof(float), cudaMemcpyHostToDevice, c->cin));
    CK(cudaEventRecord(ev_in[f], c->cin));
    CK(cudaStreamWaitEvent(c->stream, ev_in[f], 0));
    CK(launch_pack(g, orient[f], stage(f), dev[f], c->stream));
    if (f == 1) {
      int rb = ensure_base(c, M);
      if (rb) return rb;
      rb = enqueue_theta(c, M);
      if (rb) return rb;
    }
  }
  // the moisture fields up behind them, during the dry step
  if (moist) {
    for (int f = 5; f < 8; ++f) {
      CK(cudaMemcpyAsync(stage(f), src[f], count(f) * sizeof(float), cudaMemcpyHostToDevice, c->cin));
      CK(cudaEventRecord(ev_in[f], c->cin));
    }
    CK(cudaMemcpyAsync(M.precip, in->precip, n2 * sizeof(double), cudaMemcpyHostToDevice, c->cin));
    CK(cudaMemsetAsync(M.pcomp, 0, n2 * sizeof(double), c->cin));
    CK(cudaEventRecord(ev_in[8], c->cin));
  }
  int rc = enqueue_dry(c, M);
  if (rc) return rc;
  CK(cudaEventRecord(ev_dry, c->stream));
  // rho and the momenta down while the tracers and the warm rain run
  CK(cudaStreamWaitEvent(c->cout, ev_dry, 0));
  for (int f : {0, 2, 3, 4}) {
    CK(launch_unpack(g, orient[f], dev[f], stage(f), c->cout));
    CK(cudaMemcpyAsync(dst[f], stage(f), count(f) * sizeof(float), cudaMemcpyDeviceToHost, c->cout));
  }
  if (moist) {
    for (int f = 5; f < 9; ++f) CK(cudaStreamWaitEvent(c->stream, ev_in[f], 0));
    for (int f = 5; f < 8; ++f) CK(launch_pack(g, orient[f], stage(f), dev[f], c->stream));
  }
  if (M.md.enable_tracer_transport && !M.reg.empty()) {
    rc = enqueue_tracers(c, M);
    if (rc) return rc;
  }
  if (moist && M.md.enable_warm_rain) {
    rc = enqueue_rain(c, M, 1);
    if (rc) return rc;
  }
  CK(cudaEventRecord(ev_end, c->stream));
  // the rest down after the step
  CK(cudaStreamWaitEvent(c->cout, ev_end, 0));
  std::vector<double> comp;
  for (int f = 1; f < nf; f += (f == 1 ? 4 : 1)) {  // rho*theta, then the tracers
    CK(launch_unpack(g, orient[f], dev[f], stage(f), c->cout));
    CK(cudaMemcpyAsync(dst[f], stage(f), count(f) * sizeof(float), cudaMemcpyDeviceToHost, c->cout));
  }
  if (moist) {
    comp.resize(n2);
    CK(cudaMemcpyAsync(out->precip, M.precip, n2 * sizeof(double), cudaMemcpyDeviceToHost, c->cout));
    CK(cudaMemcpyAsync(comp.data(), M.pcomp, n2 * sizeof(double), cudaMemcpyDeviceToHost, c->cout));
  }
  CK(cudaStreamSynchronize(c->cout));
  CK(cudaStreamSynchronize(c->stream));
  c->launches = c->cur_launches;
  rc = check_device_errors(c);
  if (rc) return rc;
  for (size_t q = 0; q < comp.size(); ++q) out->precip[q] += comp[q];
  return GWM_B200_OK;
}

int gwm_b200_advance_dry(gwm_b200_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return GWM_B200_ERR_ARG;
  // a dry-only call must leave theta sums of the dry result: treat rain as absent
  std::vector<int> saved;
  for (auto& M : c->m) { saved.push_back(M.md.enable_warm_rain); M.md.enable_warm_rain = 0; }
  const int rc = run_steps(c, nsteps, enqueue_dry);
  for (size_t i = 0; i < c->m.size(); ++i) c->m[i].md.enable_warm_rain = saved[i];
  return rc;
}

int gwm_b200_advance_tracers(gwm_b200_ctx* c) {
  if (!c) return GWM_B200_ERR_ARG;
  c->cur_launches = 0;
  for (auto& M : c->m) {
    if (M.reg.empty()) continue;
    int rc = enqueue_tracers(c, M);
    if (rc) return rc;
  }
  c->launches = c->cur_launches;
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_warm_rain(gwm_b200_ctx* c, int fallout) {
  if (!c || fallout < 0 || fallout > 2) return GWM_B200_ERR_ARG;
  c->cur_launches = 0;
  for (auto& M : c->m) {
    if (!M.md.moist) continue;
    // fresh theta sums of the post-microphysics state
    CK(cudaMemsetAsync(M.slot(M.ring), 0, kSlot * sizeof(unsigned long long), c->stream));
    int rc = enqueue_rain(c, M, fallout);
    if (rc) return rc;
    M.theta_valid = true;
  }
  c->launches = c->cur_launches;
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_fast_modes(gwm_b200_ctx* c) {
  if (!c) return GWM_B200_ERR_ARG;
  c->cur_launches = 0;
  for (auto& M : c->m) {
    const gwm_b200_step_config& sc = M.md.step;
    const int ns = std::max(1, sc.fast_substeps);
    const bool terr = M.terrain_active;
    // theta frozen from the state, base momenta = the state's momenta,
    // density copied so the first substep never reads what it writes
    LAUNCH(launch_theta_field(M.g, M.Q[0], M.Q[1], M.TH[0], c->stream), "theta field");
    CK(cudaMemcpyAsync(M.R[0], M.Q[0], M.field_elems * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
    // rho and p level sums of the state (flat-terrain reference) into slot(ring)
    CK(cudaMemsetAsync(M.slot(M.ring), 0, kSlot * sizeof(unsigned long long), c->stream));
    int rcb = ensure_base(c, M);
    if (rcb) return rcb;
    LevelSumArgs ls{};
    ls.g = M.g; ls.rho = M.Q[0]; ls.rt = M.Q[1]; ls.mode = 1; ls.base = M.base;
    ls.acc_a = M.slot(M.ring); ls.acc_b = M.slot(M.ring) + kMaxNz;
    ls.clr_a = M.slot(M.ring + 1); ls.clr_b = M.slot(M.ring + 1) + kMaxNz;
    LAUNCH(launch_level_sums(ls, c->stream), "level sums");
    int rcur = 0, dcur = -1;
    for (int n = 0; n < ns; ++n) {
      FastArgs f{};
      f.g = M.g;
      f.rho_in = M.R[rcur]; f.rho_out = M.R[rcur ^ 1];
      f.p_in = M.P[rcur]; f.p_out = M.P[rcur ^ 1];
      f.th = M.TH[0];
      const int dout = (n == 0) ? 0 : (dcur ^ 1);
      if (n > 0) { f.du_in = M.D[dcur][0]; f.dv_in = M.D[dcur][1]; f.dw_in = M.D[dcur][2]; }
      f.du_out = M.D[dout][0]; f.dv_out = M.D[dout][1]; f.dw_out = M.D[dout][2];
      f.final_kind = (n == ns - 1) ? 2 : 0;
      f.bu = M.Q[2]; f.bv = M.Q[3]; f.bw = M.Q[4];
      f.f_rho = M.Q[0]; f.f_rt = M.Q[1]; f.f_u = M.Q[2]; f.f_v = M.Q[3]; f.f_w = M.Q[4];
      f.dtf = sc.dt / (float)ns; f.gravity = sc.gravity;
      f.hmom = sc.fast_update_horizontal_momentum; f.dens = sc.fast_update_density;
      f.ref_a = M.slot(M.ring); f.ref_b = M.slot(M.ring) + kMaxNz;
      f.inv_count = inv_count(M);
      f.acc_a = M.slot(M.ring + 1); f.acc_b = M.slot(M.ring + 1) + kMaxNz;
      f.clr_a = M.slot(M.ring + 2); f.clr_b = M.slot(M.ring + 2) + kMaxNz;
      f.zc = M.zc; f.idz_c = M.idc; f.idz_f = M.idf; f.base = M.base;
      f.err = M.err;
      if (terr) {
        f.col_pref = M.colref[0]; f.col_rref = M.colref[1];
        LAUNCH(launch_column_reference(f, c->stream), "column reference");
      }
      LAUNCH(launch_substep(c, M, f, n == 0, terr), "fast substep");
      M.ring = (M.ring + 1) % 3;
      rcur ^= 1;
      dcur = dout;
    }
    M.theta_valid = true;  // the final substep left theta sums of the result in slot(ring)
  }
  c->launches = c->cur_launches;
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_slow_tendencies(gwm_b200_ctx* c, int member, gwm_b200_fields* h) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  rc = ensure_base(c, M);
  if (rc) return rc;
  if (!M.theta_valid) {
    rc = enqueue_theta(c, M);
    if (rc) return rc;
  }
  SlowArgs a{};
  a.g = M.g;
  a.rho = M.Q[0]; a.th = M.Q[1]; a.th_is_rt = 1;
  a.u = M.Q[2]; a.v = M.Q[3]; a.w = M.Q[4];
  a.dt = M.md.step.dt; a.gravity = M.md.step.gravity;
  a.o_rho = M.R[0]; a.o_th = M.TH[0]; a.o_u = M.B[0][0]; a.o_v = M.B[0][1]; a.o_w = M.B[0][2];
  a.tend_only = 1;
  a.th_acc = M.slot(M.ring);
  a.acc_mode = 0;
  a.inv_count = inv_count(M);
  a.zc = M.zc; a.idz_c = M.idc; a.idz_f = M.idf; a.base = M.base;
  if (M.damping) {
    a.damp_c = M.damp; a.damp_f = M.damp + (kMaxNz + 1);
    a.uref = M.damp + 2 * (kMaxNz + 1); a.vref = M.damp + 3 * (kMaxNz + 1);
  }
  CK(launch_slow(a, M.terrain_active, c->stream, c->slow_tile_rows == kSlowTma ? 16 : c->slow_tile_rows));
  gwm_b200_fields tmp{};
  tmp.rho_d = h->rho_d; tmp.rho_theta_m = h->rho_theta_m;
  tmp.mom_u = h->mom_u; tmp.mom_v = h->mom_v; tmp.mom_w = h->mom_w;
  const Geom& g = M.g;
  struct F { float* dst; const float* src; int o; };
  const F list[5] = {{tmp.rho_d, M.R[0], kCell}, {tmp.rho_theta_m, M.TH[0], kCell},
                     {tmp.mom_u, M.B[0][0], kFaceX}, {tmp.mom_v, M.B[0][1], kFaceY},
                     {tmp.mom_w, M.B[0][2], kFaceZ}};
  for (const auto& f : list) {
    if (!f.dst) continue;
    const size_t n = (size_t)(g.nx + (f.o == kFaceX)) * (g.ny + (f.o == kFaceY)) * (g.nz + (f.o == kFaceZ));
    CK(launch_unpack(g, f.o, f.src, M.staging, c->stream));
    CK(cudaMemcpyAsync(f.dst, M.staging, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return GWM_B200_OK;
}

int gwm_b200_budgets(gwm_b200_ctx* c, int member, gwm_b200_budget* out) {
  int rc = check_member(c, member);
  if (rc) return rc;
  if (!out) return fail(c, GWM_B200_ERR_ARG, "null budget");
  Member& M = c->m[member];
  const Geom& g = M.g;
  cudaStream_t s = c->stream;
  CK(launch_reduce(g, kCell, 0, M.Q[0], nullptr, nullptr, 0, M.red_part, M.red_out + 0, s));
  CK(launch_reduce(g, kCell, 0, M.Q[1], nullptr, nullptr, 0, M.red_part, M.red_out + 1, s));
  CK(launch_reduce(g, kFaceX, 0, M.Q[2], nullptr, nullptr, 0, M.red_part, M.red_out + 2, s));
  CK(launch_reduce(g, kFaceY, 0, M.Q[3], nullptr, nullptr, 0, M.red_part, M.red_out + 3, s));
  CK(launch_reduce(g, kFaceZ, 0, M.Q[4], nullptr, nullptr, 0, M.red_part, M.red_out + 4, s));
  CK(launch_reduce(g, kCell, 1, M.Q[1], M.Q[0], nullptr, 0, M.red_part, M.red_out + 5, s));
  int nout = 6;
  if (M.md.moist) {
    for (int t = 0; t < 3; ++t)
      CK(launch_reduce(g, kCell, 2, M.T0[t], nullptr, M.idc, M.terrain_active, M.red_part, M.red_out + 6 + t, s));
    CK(launch_reduce_2d(M.precip, M.pcomp, (long long)g.nx * g.ny, M.red_part, M.red_out + 9, s));
    nout = 10;
  }
  ReduceOut r[10];
  CK(cudaMemcpyAsync(r, M.red_out, nout * sizeof(ReduceOut), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  gwm_b200_budget& b = *out;
  std::memset(&b, 0, sizeof(b));
  b.total_dry_mass = r[0].sum; b.rho_min = r[0].mn; b.rho_max = r[0].mx;
  b.total_rho_theta_m = r[1].sum;
  b.total_horizontal_momentum_x = r[2].sum; b.u_min = r[2].mn; b.u_max = r[2].mx;
  b.total_horizontal_momentum_y = r[3].sum; b.v_min = r[3].mn; b.v_max = r[3].mx;
  b.total_vertical_momentum = r[4].sum; b.w_min = r[4].mn; b.w_max = r[4].mx;
  b.theta_min = r[5].mn; b.theta_max = r[5].mx;
  if (M.md.moist) {
    b.vapor_water_path_sum_kg_m2 = r[6].sum;
    b.cloud_water_path_sum_kg_m2 = r[7].sum;
    b.rain_water_path_sum_kg_m2 = r[8].sum;
    b.accumulated_surface_precipitation_sum_mm = r[9].sum;
    b.mean_surface_precipitation_mm = r[9].sum / ((double)g.nx * g.ny);
    b.max_surface_precipitation_mm = r[9].mx;
  }
  if (!std::isfinite(b.total_dry_mass) || !std::isfinite(b.total_rho_theta_m) || !(b.rho_min > 0.0))
    return fail(c, GWM_B200_ERR_STATE, "non-finite or non-positive density in the state");
  return GWM_B200_OK;
}

// summarize_runtime_state + runtime_state_summary_to_json (src/core/runtime_summary.cpp:
// 27-178, 180-247) from FP64 device reductions over the member's global fields.
namespace {
// runtime_state_summary_to_json (runtime_summary.cpp:180-251) of a member's state; the
// return value is the budget's state status (GWM_B200_ERR_STATE for a non-finite or
// non-positive density) or an error of the reductions.
int runtime_summary_text(gwm_b200_ctx* c, int member, const char* indent, std::string& js) {
  Member& M = c->m[member];
  gwm_b200_budget b{};
  const int state_rc = gwm_b200_budgets(c, member, &b);
  if (state_rc != GWM_B200_OK && state_rc != GWM_B200_ERR_STATE) return state_rc;
  const Geom& g = M.g;
  cudaStream_t s = c->stream;
  const int nt = (int)M.reg.size();
  std::vector<ReduceOut> col(nt), mix(nt);
  for (int t = 0; t < nt; ++t) {
    CK(launch_reduce(g, kCell, 2, M.reg[t].f[0], nullptr, M.idc, M.terrain_active, M.red_part, M.red_out + 20, s));
    CK(launch_reduce(g, kCell, 1, M.reg[t].f[0], M.Q[0], nullptr, 0, M.red_part, M.red_out + 21, s));
    ReduceOut r[2];
    CK(cudaMemcpyAsync(r, M.red_out + 20, sizeof(r), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    col[t] = r[0];
    mix[t] = r[1];
  }
  // moisture budget: water paths from the warm-rain tracers, surface precipitation from
  // the accumulation (moist members)
  auto path = [&](const char* name) {
    for (int t = 0; t < nt; ++t)
      if (M.reg[t].name == name) return col[t].sum;
    return 0.0;
  };
  const double vap = path("specific_humidity"), cld = path("cloud_water_mixing_ratio"),
               rain = path("rain_water_mixing_ratio");
  double psum = 0.0, pmean = 0.0, pmax = 0.0, pfrac = 0.0, pmean_wet = 0.0;
  long long ncell = 0, nwet = 0;
  if (M.md.moist) {
    const long long n2 = (long long)g.nx * g.ny;
    CK(launch_reduce_2d(M.precip, M.pcomp, n2, M.red_part, M.red_out + 20, s, 0));
    CK(launch_reduce_2d(M.precip, M.pcomp, n2, M.red_part, M.red_out + 21, s, 1));
    ReduceOut r[2];
    CK(cudaMemcpyAsync(r, M.red_out + 20, sizeof(r), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    psum = r[0].sum;
    pmean = r[0].sum / (double)n2;
    pmax = r[0].mx;
    ncell = n2;
    nwet = (long long)r[1].sum;
    pfrac = (double)nwet / (double)n2;
    // every accumulated value is >= 0, so the precipitating cells hold the whole sum
    if (nwet > 0) pmean_wet = r[0].sum / (double)nwet;
  }
  const std::string in = indent ? indent : "  ";
  std::ostringstream o;
  o << std::setprecision(17);
  o << "{\n";
  o << in << "\"total_dry_mass\": " << b.total_dry_mass << ",\n";
  o << in << "\"total_rho_theta_m\": " << b.total_rho_theta_m << ",\n";
  o << in << "\"total_horizontal_momentum_x\": " << b.total_horizontal_momentum_x << ",\n";
  o << in << "\"total_horizontal_momentum_y\": " << b.total_horizontal_momentum_y << ",\n";
  o << in << "\"total_vertical_momentum\": " << b.total_vertical_momentum << ",\n";
  o << in << "\"rho_d\": {\"min\": " << b.rho_min << ", \"max\": " << b.rho_max << "},\n";
  o << in << "\"theta_m\": {\"min\": " << b.theta_min << ", \"max\": " << b.theta_max << "},\n";
  o << in << "\"u_face\": {\"min\": " << b.u_min << ", \"max\": " << b.u_max << "},\n";
  o << in << "\"v_face\": {\"min\": " << b.v_min << ", \"max\": " << b.v_max << "},\n";
  o << in << "\"w_face\": {\"min\": " << b.w_min << ", \"max\": " << b.w_max << "},\n";
  o << in << "\"moisture\": {\n";
  o << in << "  \"vapor_water_path_sum_kg_m2\": " << vap << ",\n";
  o << in << "  \"cloud_water_path_sum_kg_m2\": " << cld << ",\n";
  o << in << "  \"rain_water_path_sum_kg_m2\": " << rain << ",\n";
  o << in << "  \"condensed_water_path_sum_kg_m2\": " << cld + rain << ",\n";
  o << in << "  \"total_water_path_sum_kg_m2\": " << vap + (cld + rain) << ",\n";
  o << in << "  \"accumulated_surface_precipitation_sum_mm\": " << psum << ",\n";
  o << in << "  \"mean_surface_precipitation_mm\": " << pmean << ",\n";
  o << in << "  \"max_surface_precipitation_mm\": " << pmax << ",\n";
  o << in << "  \"total_surface_cell_count\": " << ncell << ",\n";
  o << in << "  \"precipitating_surface_cell_count\": " << nwet << ",\n";
  o << in << "  \"precipitating_surface_fraction\": " << pfrac << ",\n";
  o << in << "  \"mean_precipitating_surface_precipitation_mm\": " << pmean_wet << "\n";
  o << in << "},\n";
  o << in << "\"tracers\": {\n";
  for (int t = 0; t < nt; ++t) {
    const auto& T = M.reg[t];
    o << in << "  \"" << T.name << "\": {\n";
    o << in << "    \"units\": \"" << T.units << "\",\n";
    o << in << "    \"positive\": " << (T.positive ? "true" : "false") << ",\n";
    o << in << "    \"column_integrated_sum_kg_m2\": " << col[t].sum << ",\n";
    o << in << "    \"mixing_ratio\": {\"min\": " << mix[t].mn << ", \"max\": " << mix[t].mx << "}\n";
    o << in << "  }" << (t + 1 != nt ? "," : "") << "\n";
  }
  o << in << "}\n";
  o << "}";
  js = o.str();
  return state_rc;
}

// text into the caller's buffer (cap bytes, NUL-terminated); *len receives the bytes needed
int put_text(gwm_b200_ctx* c, const std::string& js, char* buf, long long cap, long long* len) {
  if (len) *len = (long long)js.size() + 1;
  if (buf && cap > 0) {
    const size_t n = std::min<size_t>(js.size(), (size_t)cap - 1);
    std::memcpy(buf, js.data(), n);
    buf[n] = 0;
    if ((long long)js.size() + 1 > cap) return fail(c, GWM_B200_ERR_ARG, "output buffer too small");
  }
  return GWM_B200_OK;
}

// one phase of enqueue_full_step (the same enqueues in the same order)
int enqueue_phase_tracers(gwm_b200_ctx* c, Member& M) {
  return (M.md.enable_tracer_transport && !M.reg.empty()) ? enqueue_tracers(c, M) : GWM_B200_OK;
}
int enqueue_phase_rain(gwm_b200_ctx* c, Member& M) {
  return (M.md.moist && M.md.enable_warm_rain) ? enqueue_rain(c, M, 1) : GWM_B200_OK;
}

// maybe_write_phase_summary's document (gwm_prepared_case_driver.cpp:97-131)
int phase_summary_text(gwm_b200_ctx* c, int member, int step, float t, const char* phase, std::string& js) {
  std::string summary;
  const int rc = runtime_summary_text(c, member, "    ", summary);
  if (rc != GWM_B200_OK && rc != GWM_B200_ERR_STATE) return rc;
  std::ostringstream o;
  o << "{\n  \"step\": " << step << ",\n  \"step_start_seconds\": " << t << ",\n  \"phase\": \""
    << (phase ? phase : "") << "\",\n  \"summary\": " << summary << "\n}\n";
  js = o.str();
  return rc;
}
}  // namespace

int gwm_b200_runtime_summary_json(gwm_b200_ctx* c, int member, const char* indent, char* buf, long long cap,
                                  long long* len) {
  int rc = check_member(c, member);
  if (rc) return rc;
  std::string js;
  const int state_rc = runtime_summary_text(c, member, indent, js);
  if (state_rc != GWM_B200_OK && state_rc != GWM_B200_ERR_STATE) return state_rc;
  rc = put_text(c, js, buf, cap, len);
  return rc ? rc : state_rc;
}

int gwm_b200_phase_summary_json(gwm_b200_ctx* c, int member, int step, float step_start_seconds,
                                const char* phase, char* buf, long long cap, long long* len) {
  int rc = check_member(c, member);
  if (rc) return rc;
  std::string js;
  const int state_rc = phase_summary_text(c, member, step, step_start_seconds, phase, js);
  if (state_rc != GWM_B200_OK && state_rc != GWM_B200_ERR_STATE) return state_rc;
  rc = put_text(c, js, buf, cap, len);
  return rc ? rc : state_rc;
}

int gwm_b200_prepared_steps(gwm_b200_ctx* c, int nsteps, float* sim_time, const char* phase_summary_dir,
                            int only_step, int step_min, int step_max) {
  if (!c || nsteps < 0 || c->m.empty()) return GWM_B200_ERR_ARG;
  float t = sim_time ? *sim_time : 0.0f;
  const float dt = c->m[0].md.step.dt;
  const bool phases = phase_summary_dir && *phase_summary_dir;
  auto selected = [&](int step) {  // phase_summary_step_selected (:71-88)
    if (only_step >= 0) return step == only_step;
    return !(step_min >= 0 && step < step_min) && !(step_max >= 0 && step > step_max);
  };
  auto write = [&](int step, const char* phase) {
    for (int m = 0; m < (int)c->m.size(); ++m) {
      std::string js;
      const int rc = phase_summary_text(c, m, step, t, phase, js);
      if (rc != GWM_B200_OK && rc != GWM_B200_ERR_STATE) return rc;
      std::string path = std::string(phase_summary_dir) + "/step_" + std::to_string(step) + "_" + phase;
      if (m > 0) path += "_member" + std::to_string(m);
      path += ".json";
      std::FILE* f = std::fopen(path.c_str(), "wb");
      if (!f) return fail(c, GWM_B200_ERR_ARG, "Failed to open phase summary path: " + path);
      const bool ok = std::fwrite(js.data(), 1, js.size(), f) == js.size();
      std::fclose(f);
      if (!ok) return fail(c, GWM_B200_ERR_ARG, "Failed to write phase summary: " + path);
    }
    return GWM_B200_OK;
  };
  for (int step = 0; step < nsteps; ++step) {
    int rc;
    if (!phases || !selected(step)) {
      rc = run_steps(c, 1, enqueue_full_step);
    } else {
      bool tracers = false, rain = false;
      for (const auto& M : c->m) {
        tracers |= M.md.enable_tracer_transport && !M.reg.empty();
        rain |= M.md.moist && M.md.enable_warm_rain;
      }
      rc = run_steps(c, 1, enqueue_dry);
      if (!rc) rc = write(step, "dry");
      if (!rc && tracers) rc = run_steps(c, 1, enqueue_phase_tracers);
      if (!rc && tracers) rc = write(step, "tracers");
      if (!rc && rain) rc = run_steps(c, 1, enqueue_phase_rain);
      if (!rc && rain) rc = write(step, "warm_rain");
    }
    if (rc) return rc;
    t += dt;
  }
  if (sim_time) *sim_time = t;
  CK(cudaStreamSynchronize(c->stream));
  return check_device_errors(c);
}

int gwm_b200_prepared_summary_json(gwm_b200_ctx* c, int member, const gwm_b200_prepared_meta* meta, int steps,
                                   const char* initial_json, char* buf, long long cap, long long* len) {
  int rc = check_member(c, member);
  if (rc) return rc;
  if (!meta || !initial_json || steps < 0) return fail(c, GWM_B200_ERR_ARG, "prepared summary: missing input");
  const Member& M = c->m[member];
  std::string final_js;
  const int state_rc = runtime_summary_text(c, member, "    ", final_js);
  if (state_rc != GWM_B200_OK && state_rc != GWM_B200_ERR_STATE) return state_rc;
  // prepared_summary_json (gwm_prepared_case_driver.cpp:252-350)
  const float dt = M.md.step.dt;
  const gwm_b200_warm_rain_config& w = M.md.rain;
  auto b = [](int v) { return v ? "true" : "false"; };
  const double elapsed = (double)steps * (double)dt;
  std::ostringstream o;
  o << std::setprecision(17);
  o << "{\n";
  o << "  \"case\": \"prepared_case\",\n";
  o << "  \"source\": \"" << (meta->source ? meta->source : "") << "\",\n";
  o << "  \"cycle_time_utc\": \"" << (meta->cycle_time_utc ? meta->cycle_time_utc : "") << "\",\n";
  o << "  \"analysis_valid_time_utc\": \""
    << (meta->analysis_valid_time_utc ? meta->analysis_valid_time_utc : "") << "\",\n";
  o << "  \"steps\": " << steps << ",\n";
  o << "  \"dt\": " << dt << ",\n";
  o << "  \"fast_substeps\": " << M.md.step.fast_substeps << ",\n";
  o << "  \"enable_boundaries\": " << b(meta->enable_boundaries) << ",\n";
  o << "  \"enable_fast_modes\": " << b(M.md.step.enable_fast_modes) << ",\n";
  o << "  \"enable_tracer_transport\": " << b(M.md.enable_tracer_transport) << ",\n";
  o << "  \"enable_warm_rain\": " << b(M.md.enable_warm_rain) << ",\n";
  o << "  \"fast_update_horizontal_momentum\": " << b(M.md.step.fast_update_horizontal_momentum) << ",\n";
  o << "  \"fast_update_density\": " << b(M.md.step.fast_update_density) << ",\n";
  o << "  \"warm_rain\": {\n";
  o << "    \"condensation_relaxation\": " << w.condensation_relaxation << ",\n";
  o << "    \"cloud_autoconversion_threshold\": " << w.cloud_autoconversion_threshold << ",\n";
  o << "    \"cloud_autoconversion_rate\": " << w.cloud_autoconversion_rate << ",\n";
  o << "    \"rain_evaporation_rate\": " << w.rain_evaporation_rate << ",\n";
  o << "    \"rain_terminal_velocity\": " << w.rain_terminal_velocity << ",\n";
  o << "    \"sedimentation_layer_depth_m\": " << w.sedimentation_layer_depth_m << ",\n";
  o << "    \"enable_latent_heating\": " << b(w.enable_latent_heating) << "\n";
  o << "  },\n";
  o << "  \"elapsed_seconds\": " << elapsed << ",\n";
  o << "  \"elapsed_hours\": " << elapsed / 3600.0 << ",\n";
  o << "  \"grid\": {\n";
  o << "    \"nx\": " << M.gd.nx << ",\n    \"ny\": " << M.gd.ny << ",\n    \"nz\": " << M.gd.nz << ",\n";
  o << "    \"dx\": " << M.gd.dx << ",\n    \"dy\": " << M.gd.dy << ",\n    \"z_top\": " << M.gd.z_top << "\n";
  o << "  },\n";
  o << "  \"surface_runtime\": {\n";
  o << "    \"ntile\": " << meta->surface_ntile << ",\n    \"nsoil\": " << meta->surface_nsoil << "\n";
  o << "  },\n";
  o << "  \"startup_balance\": {\n";
  o << "    \"max_rel_eos\": " << meta->max_rel_eos << ",\n";
  o << "    \"max_rel_hydrostatic\": " << meta->max_rel_hydrostatic << ",\n";
  o << "    \"max_rel_fast_vertical\": " << meta->max_rel_fast_vertical << ",\n";
  o << "    \"max_abs_mass_divergence\": " << meta->max_abs_mass_divergence << ",\n";
  o << "    \"max_rel_mass_divergence\": " << meta->max_rel_mass_divergence << ",\n";
  o << "    \"max_abs_mom_w_bottom\": " << meta->max_abs_mom_w_bottom << ",\n";
  o << "    \"max_abs_mom_w_top\": " << meta->max_abs_mom_w_top << ",\n";
  o << "    \"max_abs_tracer_closure\": " << meta->max_abs_tracer_closure;
  if (meta->has_max_abs_z_src_minus_metric)
    o << ",\n    \"max_abs_z_src_minus_metric\": " << meta->max_abs_z_src_minus_metric << "\n";
  else
    o << "\n";
  o << "  },\n";
  o << "  \"initial\": " << initial_json << ",\n";
  o << "  \"final\": " << final_js << "\n";
  o << "}";
  rc = put_text(c, o.str(), buf, cap, len);
  return rc ? rc : state_rc;
}

// ---------------------------------------------------------------------------
// Runtime plan view (extract_runtime_plan_view, src/io/plan_view_output.cpp:715-834).
namespace {
struct PlanViewName {
  const char* name;
  const char* units;
};
const PlanViewName kPlanViewNames[kPvAll] = {
    {"terrain_height", "m"}, {"z_center", "m"}, {"rho_d", "kg m^-3"}, {"theta_m", "K"},
    {"air_pressure", "Pa"}, {"air_temperature", "K"}, {"u_velocity", "m s^-1"}, {"v_velocity", "m s^-1"},
    {"wind_speed", "m s^-1"}, {"w_velocity", "m s^-1"}, {"specific_humidity", "kg kg^-1"},
    {"relative_humidity", "%"}, {"dewpoint", "K"}, {"cloud_water_mixing_ratio", "kg kg^-1"},
    {"rain_water_mixing_ratio", "kg kg^-1"}, {"total_condensate", "kg kg^-1"}, {"column_cloud_water", "kg m^-2"},
    {"column_rain_water", "kg m^-2"}, {"column_total_condensate", "kg m^-2"}, {"column_rain_fraction", "1"},
    {"synthetic_reflectivity", "dBZ"}, {"accumulated_surface_precipitation", "mm"},
    {"mean_surface_precipitation_rate", "mm h^-1"}};

const Member::Tracer* find_tracer(const Member& M, const char* name) {
  for (const auto& t : M.reg)
    if (t.name == name) return &t;
  return nullptr;
}

// The bundle's fields for the member's state at level k into a host vector; the
// field count follows the member's tracers as extract_runtime_plan_view's branches do.
int plan_view_fields(gwm_b200_ctx* c, Member& M, int k, int steps, double dt, std::vector<double>& host,
                     int* nfields) {
  const Geom& g = M.g;
  PlanViewArgs a{};
  a.g = g;
  a.k = k;
  a.rho = M.Q[0]; a.rt = M.Q[1]; a.u = M.Q[2]; a.v = M.Q[3]; a.w = M.Q[4];
  a.zc = M.zc; a.idc = M.idc; a.metric_3d = M.terrain_active ? 1 : 0;
  a.nfields = kPvDry;
  if (!M.reg.empty()) {  // a runtime tracer state: specific humidity is required
    const auto* qv = find_tracer(M, "specific_humidity");
    if (!qv) return fail(c, GWM_B200_ERR_ARG, "specific_humidity tracer missing from runtime tracer state");
    a.qv = qv->f[0];
    a.nfields = kPvVapour;
    const auto *qc = find_tracer(M, "cloud_water_mixing_ratio"), *qr = find_tracer(M, "rain_water_mixing_ratio");
    if (qc && qr) {
      a.qc = qc->f[0];
      a.qr = qr->f[0];
      a.nfields = kPvWarmRain;
      if (M.md.moist) {  // the warm-rain surface accumulation
        a.precip = M.precip;
        a.precip_comp = M.pcomp;
        a.inv_hours = 1.0 / std::max((double)steps * (double)(float)dt / 3600.0, 1.0e-9);
        a.nfields = kPvAll;
      }
    }
  }
  const size_t plane = (size_t)g.nx * g.ny;
  double* dev = nullptr;
  CK(cudaMalloc(&dev, (size_t)a.nfields * plane * sizeof(double)));
  a.out = dev;
  host.assign((size_t)a.nfields * plane, 0.0);
  cudaError_t e = launch_plan_view(a, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host.data() + plane, dev + plane, (size_t)(a.nfields - 1) * plane * sizeof(double),
                        cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(dev);
  CK(e);
  if (!M.terrain.empty())  // terrain height (the metric's input; zero on flat grids)
    for (size_t q = 0; q < plane; ++q) host[q] = (double)M.terrain[q];
  *nfields = a.nfields;
  return GWM_B200_OK;
}
}  // namespace

int gwm_b200_plan_view_field(int field, const char** name, const char** units) {
  if (field < 0 || field >= kPvAll) return GWM_B200_ERR_ARG;
  if (name) *name = kPlanViewNames[field].name;
  if (units) *units = kPlanViewNames[field].units;
  return GWM_B200_OK;
}

int gwm_b200_plan_view(gwm_b200_ctx* c, int member, int level, int steps, double dt, double* out, long long cap,
                       int* nfields) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  const int k = std::clamp(level, 0, M.g.nz - 1);
  std::vector<double> host;
  int nf = 0;
  rc = plan_view_fields(c, M, k, steps, dt, host, &nf);
  if (rc) return rc;
  if (nfields) *nfields = nf;
  if (out) {
    if (cap < (long long)host.size()) return fail(c, GWM_B200_ERR_ARG, "plan-view buffer too small");
    std::copy(host.begin(), host.end(), out);
  }
  return GWM_B200_OK;
}

int gwm_b200_plan_view_json(gwm_b200_ctx* c, int member, int level, const char* case_kind, int steps, double dt,
                            char* buf, long long cap, long long* len) {
  int rc = check_member(c, member);
  if (rc) return rc;
  Member& M = c->m[member];
  const Geom& g = M.g;
  const int k = std::clamp(level, 0, g.nz - 1);
  std::vector<double> f;
  int nf = 0;
  rc = plan_view_fields(c, M, k, steps, dt, f, &nf);
  if (rc) return rc;
  // plan_view_bundle_to_json (plan_view_output.cpp:950-1003); dt is the bundle's FP32 real,
  // the mean height the FP64 mean of the level's z_center in row order
  const size_t plane = (size_t)g.nx * g.ny;
  const HostMetrics H = build_metrics(M);
  double zsum = 0.0;
  for (size_t q = 0; q < plane; ++q) zsum += (double)H.zc[(size_t)k * plane + q];
  auto jstr = [](const std::string& v) {
    std::string o = "\"";
    for (char ch : v) {
      if (ch == '"' || ch == '\\') o += '\\';
      o += ch;
    }
    return o + "\"";
  };
  std::ostringstream o;
  o << std::setprecision(10);
  o << "{\n  \"schema_version\": " << jstr("gwm-next-plan-view/v1") << ",\n";
  o << "  \"case\": " << jstr(case_kind ? case_kind : "") << ",\n";
  o << "  \"steps\": " << steps << ",\n  \"dt\": " << (float)dt << ",\n  \"slice_k\": " << k << ",\n";
  o << "  \"grid\": {\n    \"nx\": " << g.nx << ",\n    \"ny\": " << g.ny << ",\n    \"dx\": " << M.gd.dx
    << ",\n    \"dy\": " << M.gd.dy << ",\n    \"slice_mean_height_m\": " << zsum / (double)(g.nx * g.ny)
    << "\n  },\n";
  o << "  \"fields\": [\n";
  for (int n = 0; n < nf; ++n) {
    o << "    {\n      \"name\": " << jstr(kPlanViewNames[n].name) << ",\n      \"units\": "
      << jstr(kPlanViewNames[n].units) << ",\n      \"location\": \"cell_center\",\n      \"nx\": " << g.nx
      << ",\n      \"ny\": " << g.ny << ",\n      \"storage\": \"row_major_yx\",\n      \"values\": [";
    const double* v = f.data() + (size_t)n * plane;
    for (size_t q = 0; q < plane; ++q) {
      if (q) o << ", ";
      o << v[q];
    }
    o << "]\n    }" << (n + 1 < nf ? "," : "") << "\n";
  }
  o << "  ]\n}";
  const std::string js = o.str();
  if (len) *len = (long long)js.size() + 1;
  if (buf && cap > 0) {
    const size_t n = std::min<size_t>(js.size(), (size_t)cap - 1);
    std::memcpy(buf, js.data(), n);
    buf[n] = 0;
    if ((long long)js.size() + 1 > cap) return fail(c, GWM_B200_ERR_ARG, "plan-view buffer too small");
  }
  return GWM_B200_OK;
}

// ---------------------------------------------------------------------------
static int layout_rows(const gwm_b200_layout_desc* d, std::vector<int>& rows) {
  if (!d || d->global_nx <= 0 || d->global_ny <= 0 || d->nz <= 0 || d->ranks_x <= 0 ||
      d->ranks_y <= 0 || d->halo < 0)
    return GWM_B200_ERR_ARG;
  const int rx = d->ranks_x, ry = d->ranks_y;
  const int bnx = d->global_nx / rx, rnx = d->global_nx % rx;
  const int bny = d->global_ny / ry, rny = d->global_ny % ry;
  rows.assign((size_t)12 * rx * ry, 0);
  int jb = 0, r = 0;
  for (int y = 0; y < ry; ++y) {  // virtual_rank_layout.cpp:7-47
    const int nyl = bny + (y < rny ? 1 : 0);
    int ib = 0;
    for (int x = 0; x < rx; ++x, ++r) {
      const int nxl = bnx + (x < rnx ? 1 : 0);
      int* o = &rows[(size_t)12 * r];
      o[0] = r; o[1] = x; o[2] = y; o[3] = ib; o[4] = ib + nxl; o[5] = jb; o[6] = jb + nyl; o[11] = d->nz;
      ib += nxl;
    }
    jb += nyl;
  }
  auto rank_at = [&](int cx, int cy) {  // cartesian_topology.cpp:29-53
    if (d->periodic_x) cx = ((cx % rx) + rx) % rx; else if (cx < 0 || cx >= rx) return -1;
    if (d->periodic_y) cy = ((cy % ry) + ry) % ry; else if (cy < 0 || cy >= ry) return -1;
    return cy * rx + cx;
  };
  for (int q = 0; q < rx * ry; ++q) {
    int* o = &rows[(size_t)12 * q];
    o[7] = rank_at(o[1] - 1, o[2]); o[8] = rank_at(o[1] + 1, o[2]);
    o[9] = rank_at(o[1], o[2] - 1); o[10] = rank_at(o[1], o[2] + 1);
  }
  return GWM_B200_OK;
}

int gwm_b200_grid_z_center(const gwm_b200_grid_desc* d, float* out) {
  if (!d || !out || d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || !(d->z_top > 0)) return GWM_B200_ERR_ARG;
  Member M;  // host fields only: the metric builder reads the grid, terrain and levels
  M.gd = *d;
  if (d->terrain) M.terrain.assign(d->terrain, d->terrain + (size_t)d->nx * d->ny);
  if (d->eta_interfaces) M.eta.assign(d->eta_interfaces, d->eta_interfaces + d->nz + 1);
  const HostMetrics H = build_metrics(M);
  std::copy(H.zc.begin(), H.zc.end(), out);
  return GWM_B200_OK;
}

int gwm_b200_layout(const gwm_b200_layout_desc* d, int* out, int capacity) {
  std::vector<int> rows;
  int rc = layout_rows(d, rows);
  if (rc) return rc;
  const int n = (int)(rows.size() / 12);
  if (out) {
    if (capacity < n) return GWM_B200_ERR_ARG;
    std::memcpy(out, rows.data(), rows.size() * sizeof(int));
  }
  return n;
}

int gwm_b200_halo_exchange(const gwm_b200_layout_desc* d, int orientation, int op,
                           float* const* rank_fields, void* stream) {
  std::vector<int> rows;
  int rc = layout_rows(d, rows);
  if (rc) return rc;
  const int n = (int)(rows.size() / 12);
  if (n > kMaxRanks || orientation < 0 || orientation > 3 || op < 0 || op > 1 || !rank_fields)
    return GWM_B200_ERR_ARG;
  if (op == 1 && orientation == 0) return GWM_B200_ERR_ARG;
  RankTable t{};
  t.n = n; t.nz = d->nz; t.halo = d->halo; t.orient = orientation;
  for (int r = 0; r < n; ++r) {
    const int* o = &rows[(size_t)12 * r];
    t.r[r].nxl = o[4] - o[3]; t.r[r].nyl = o[6] - o[5];
    t.r[r].west = o[7]; t.r[r].east = o[8]; t.r[r].south = o[9]; t.r[r].north = o[10];
    t.r[r].data = rank_fields[r];
    if (!t.r[r].data) return GWM_B200_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (launch_rank_halo(t, op, s) != cudaSuccess) return GWM_B200_ERR_CUDA;
  if (!stream && cudaStreamSynchronize(s) != cudaSuccess) return GWM_B200_ERR_CUDA;
  return GWM_B200_OK;
}

int gwm_b200_dry_pressure(const float* rho, const float* rt, float* p, long long n, void* stream) {
  if (!rho || !rt || !p || n < 0) return GWM_B200_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (launch_pressure(rho, rt, p, n, s) != cudaSuccess) return GWM_B200_ERR_CUDA;
  if (!stream && cudaStreamSynchronize(s) != cudaSuccess) return GWM_B200_ERR_CUDA;
  return GWM_B200_OK;
}

static void rank_shape(const int* row, int nz, int halo, int o, int& ox, int& oy, int& oz, int& px,
                       int& py) {
  ox = row[4] - row[3] + (o == 1);
  oy = row[6] - row[5] + (o == 2);
  oz = nz + (o == 3);
  px = ox + 2 * halo;
  py = oy + 2 * halo;
}

int gwm_b200_ranks_to_global(const gwm_b200_layout_desc* d, int o, const float* const* rf, float* glob) {
  std::vector<int> rows;
  int rc = layout_rows(d, rows);
  if (rc) return rc;
  if (o < 0 || o > 3 || !rf || !glob) return GWM_B200_ERR_ARG;
  const int gx = d->global_nx + (o == 1), gy = d->global_ny + (o == 2), gz = d->nz + (o == 3);
  const size_t n = (size_t)gx * gy * gz;
  std::vector<float> sum(n, 0.0f);
  std::vector<unsigned char> cnt(n, 0);
  std::vector<float> first(n, 0.0f);
  for (size_t r = 0; r < rows.size() / 12; ++r) {
    const int* row = &rows[12 * r];
    int ox, oy, oz, px, py;
    rank_shape(row, d->nz, d->halo, o, ox, oy, oz, px, py);
    for (int k = 0; k < oz; ++k)
      for (int j = 0; j < oy; ++j)
        for (int i = 0; i < ox; ++i) {
          const float v = rf[r][((size_t)k * py + (j + d->halo)) * px + (i + d->halo)];
          const size_t q = ((size_t)k * gy + (row[5] + j)) * gx + (row[3] + i);
          if (cnt[q] == 0) first[q] = v; else sum[q] = v;
          cnt[q]++;
        }
  }
  for (size_t q = 0; q < n; ++q) glob[q] = cnt[q] >= 2 ? 0.5f * (first[q] + sum[q]) : first[q];
  return GWM_B200_OK;
}

int gwm_b200_global_to_ranks(const gwm_b200_layout_desc* d, int o, const float* glob, float* const* rf) {
  std::vector<int> rows;
  int rc = layout_rows(d, rows);
  if (rc) return rc;
  if (o < 0 || o > 3 || !rf || !glob) return GWM_B200_ERR_ARG;
  const int gx = d->global_nx + (o == 1), gy = d->global_ny + (o == 2);
  for (size_t r = 0; r < rows.size() / 12; ++r) {
    const int* row = &rows[12 * r];
    int ox, oy, oz, px, py;
    rank_shape(row, d->nz, d->halo, o, ox, oy, oz, px, py);
    for (int k = 0; k < oz; ++k)
      for (int j = 0; j < oy; ++j)
        for (int i = 0; i < ox; ++i)
          rf[r][((size_t)k * py + (j + d->halo)) * px + (i + d->halo)] =
              glob[((size_t)k * gy + (row[5] + j)) * gx + (row[3] + i)];
  }
  return GWM_B200_OK;
}

}  // extern "C"
