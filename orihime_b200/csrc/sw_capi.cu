// C ABI of the soft Smith-Waterman kernels (declared in include/orihime_b200.h).
// This is the library's single translation unit: it includes the kernels so
// that every launch sees the kernel definitions.
//
// Every entry point is asynchronous on the caller's stream, allocates nothing
// and calls no synchronising CUDA API, so a sequence of calls can be captured
// in a CUDA graph.  Device scratch comes from the caller as one workspace
// buffer whose size the *_workspace_bytes functions report.
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>

#include "sw_kernels.cu"
#include "sw_lin.cu"
#include "sw_tan.cu"
#include "sw_xband.cu"
#include "sw_prelude.cuh"
#include "sw_probe.cuh"
#include "../../include/orihime_b200.h"

// Workspace of swb_sw_affine_forward_static: a fixed device array (one copy
// per device, created when the module loads on that device), so that entry
// point needs no caller-provided or allocated scratch.
static __device__ __align__(256) unsigned char g_static_scratch[SWB_STATIC_SCRATCH_BYTES];

namespace {

using swb::Args;

constexpr int kDefaultR = 4;          // columns per lane unless the caller picks another
constexpr int kChainLag = 31;         // wavefront steps band b+1 trails band b
constexpr int kWarpsFwd = 4;          // forward CTA: 4 independent warps
constexpr int kWarpsBwd = 1;          // adjoint CTA: 1 warp (shared memory bound)
constexpr size_t kAlign = 256;

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

template <int NS, int G = 0> constexpr int np() { return swb::push_fields<NS, G>(); }
template <int NS, int R> constexpr int ckrs() { return swb::ck_record_floats<NS, R>(); }
template <int NS, int R> constexpr int ne() { return swb::Dims<NS, R>::NE; }

bool valid_r(int r) { return r == 2 || r == 4; }
// 8 columns per lane: the linear-domain kernels of the local families only
bool valid_r_local(int r) { return r == 2 || r == 4 || r == 8; }
constexpr int ridx(int r) { return r == 2 ? 0 : (r == 4 ? 1 : 2); }
// Whether a launch with these parameters runs the linear-domain kernels
// (the local families, gaps <= 0, not forced to the log domain).
template <int NS, int G>
bool lin_eligible(float go, float ge, float T, const swb_options* opt) {
  if (G != 0 || !(T > 0.f) || !(T < INFINITY)) return false;
  if (opt && opt->domain == SWB_DOMAIN_LOG) return false;
  const float k = 1.4426950408889634f / T;
  const double xo = (double)go * (double)k, xe = NS == 3 ? (double)ge * (double)k : 0.0;
  return xo <= 0.0 && xe <= 0.0;
}
// Default columns per lane of the padded entry points, for the linear-domain
// kernels: 8 on batches at least 256 columns wide (half the bands, each
// step's fixed work spread over twice the cells: measured faster from
// 64 x 1024^2 to 4 x 4096^2); 2 on batches at most 64 columns wide (one band
// with every lane live: forward + adjoint of 1 x 64^2 in 84 us against 105 at
// 4, 128 x 64^2 in 87 against 106); else 4.  The log domain always takes 4.
int default_r(long long L2m, bool lin) {
  if (!lin) return kDefaultR;
  return L2m >= 256 ? 8 : (L2m <= 64 ? 2 : kDefaultR);
}
int pick_r(const swb_options* opt, long long L2m, bool lin) {
  return (opt && opt->cols_per_lane) ? opt->cols_per_lane : default_r(L2m, lin);
}

struct Layout {
  int nb, nchunks;
  size_t off_hdr, off_pair_done, off_part, off_gpart, off_sent, off_edge, off_bpush, off_ckpt;
  size_t sent_bytes;   // sentinel-initialised span (never_written + edge + bpush)
  size_t total;
  size_t ck_band = 0;  // checkpoint floats per band slot when not nchunks records
};

// Workspace layout for `slots` band slots and the given buffer sizes (floats).
Layout layout_sizes(long long B, size_t slots, size_t edge_floats, size_t bp_floats,
                    size_t ck_floats) {
  Layout l{};
  size_t o = 0;
  l.off_hdr = o;        o = align_up(o + 64);
  l.off_pair_done = o;  o = align_up(o + sizeof(unsigned) * (size_t)B);
  l.off_part = o;       o = align_up(o + sizeof(float) * 2 * slots);
  l.off_gpart = o;      o = align_up(o + sizeof(float) * 4 * slots);
  l.off_sent = o;       o = o + kAlign;   // never_written word lives here
  l.off_edge = o;       o = align_up(o + sizeof(float) * edge_floats);
  l.off_bpush = o;      o = align_up(o + sizeof(float) * bp_floats);
  l.sent_bytes = o - l.off_sent;
  l.off_ckpt = o;       o = align_up(o + sizeof(float) * ck_floats);
  l.total = o;
  return l;
}

int chunks_for(long long L1) { return (int)((L1 + 31 + swb::C_STEPS - 1) / swb::C_STEPS); }

// Padded batch: every pair gets the slices of a Lmax1 x Lmax2 pair.
template <int NS, int R, int G = 0>
Layout layout_for(long long B, long long L1m, long long L2m) {
  int nb = (int)((L2m + 32 * R - 1) / (32 * R));
  if (nb < 1) nb = 1;
  const int nch = chunks_for(L1m);
  const size_t slots = (size_t)B * nb;
  Layout l = layout_sizes(B, slots, slots * ne<NS, R>() * (size_t)L1m,
                          slots * np<NS, G>() * (size_t)(L1m + 1),
                          slots * (size_t)nch * ckrs<NS, R>());
  l.nb = nb;
  l.nchunks = nch;
  return l;
}

// Ragged plan header (int64 words), followed by B * PLAN_PAIR_WORDS pair
// words and ntasks (pair, band) int32 pairs.
enum HeaderWord : int {
  HW_MAGIC = 0, HW_B = 1, HW_NTASKS = 2, HW_SLOTS = 3, HW_CK = 4, HW_EDGE = 5, HW_BP = 6,
  HW_FAMILY = 7, HW_MAP_ELEMS = 8, HW_WORDS = 10
};
constexpr long long kPlanMagic = 0x53574232504c414eLL;  // "SWB2PLAN"

size_t plan_bytes_for(long long B, long long ntasks) {
  return sizeof(long long) * (HW_WORDS + (size_t)B * swb::PLAN_PAIR_WORDS) +
         sizeof(int) * 2 * (size_t)ntasks;
}

// Occupancy of each kernel instantiation on one device, computed once.
struct DevInfo {
  int sms = 0;
  int occ[2][5][2] = {};   // [kernel fwd/bwd][model_index][R == 4?]
  int locc[2][2][3] = {};  // linear-domain kernels: [fwd/bwd][NS == 3?][R: 2, 4, 8]
  int locc_sparse[2][3] = {};  // linear-domain adjoint, sparse checkpoints: [NS == 3?][R: 2, 4, 8]
  bool ready = false;
};
DevInfo g_dev[64];
std::mutex g_mu;

template <int NS, int R>
size_t bwd_smem() { return (size_t)kWarpsBwd * swb::bwd_smem_floats<NS, R>() * sizeof(float); }

// occupancy slots: linear, affine, global linear, global affine, Saigo-Vert
template <int NS, int G> constexpr int model_index() {
  return NS == 3 ? (G == 1 ? 3 : (G == 2 ? 4 : 1)) : (G == 1 ? 2 : 0);
}

template <int NS, int R>
size_t lbwd_smem() { return (size_t)kWarpsBwd * swb::lbwd_smem_floats<NS, R>() * sizeof(float); }

template <int NS, int R>
cudaError_t setup_lin(DevInfo& d) {
  cudaError_t e = cudaFuncSetAttribute(swb::lbwd_kernel<NS, R, kWarpsBwd>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)lbwd_smem<NS, R>());
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.locc[0][NS == 3][ridx(R)],
                                                    swb::lfwd_kernel<NS, R>, 32 * kWarpsFwd, 0);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &d.locc[1][NS == 3][ridx(R)], swb::lbwd_kernel<NS, R, kWarpsBwd>, 32 * kWarpsBwd,
      lbwd_smem<NS, R>());
  if (e != cudaSuccess || R == 2) return e;   // the checkpointed op runs 4 or 8 columns per lane
  e = cudaFuncSetAttribute(swb::lbwd_kernel<NS, R, kWarpsBwd, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lbwd_smem<NS, R>());
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &d.locc_sparse[NS == 3][ridx(R)], swb::lbwd_kernel<NS, R, kWarpsBwd, true>, 32 * kWarpsBwd,
      lbwd_smem<NS, R>());
}

template <int NS, int R, int G = 0>
cudaError_t setup_pair(DevInfo& d) {
  constexpr int m = model_index<NS, G>();
  cudaError_t e = cudaFuncSetAttribute(swb::bwd_kernel<NS, R, kWarpsBwd, G>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bwd_smem<NS, R>());
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ[0][m][R == 4],
                                                    swb::fwd_kernel<NS, R, G>, 32 * kWarpsFwd, 0);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &d.occ[1][m][R == 4], swb::bwd_kernel<NS, R, kWarpsBwd, G>, 32 * kWarpsBwd,
      bwd_smem<NS, R>());
}

int dev_info(DevInfo** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SWB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  DevInfo& d = g_dev[dev];
  if (!d.ready) {
    if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return SWB_ERR_CUDA;
    if (setup_pair<1, 2>(d) || setup_pair<1, 4>(d) || setup_pair<3, 2>(d) || setup_pair<3, 4>(d) ||
        setup_pair<1, 2, 1>(d) || setup_pair<1, 4, 1>(d) || setup_pair<3, 2, 1>(d) ||
        setup_pair<3, 4, 1>(d) || setup_pair<3, 2, 2>(d) || setup_pair<3, 4, 2>(d) ||
        setup_lin<1, 2>(d) || setup_lin<1, 4>(d) || setup_lin<3, 2>(d) || setup_lin<3, 4>(d) ||
        setup_lin<1, 8>(d) || setup_lin<3, 8>(d))
      return SWB_ERR_CUDA;
    d.ready = true;
  }
  *out = &d;
  return SWB_OK;
}

// Device address of g_static_scratch on the current device, looked up once
// per device context (the first lookup may load the module on that device).
// The cache is keyed on the current CUDA context as well as the device: a
// device reset or a re-created primary context makes the old address
// invalid, and the next call looks it up again.  The context comes from the
// driver's cuCtxGetCurrent, reached through cudaGetDriverEntryPoint, so the
// library needs no link against the driver library.
void* g_static_ptr[64];
void* g_static_ctx[64];

using CtxGetCurrentFn = int (*)(void**);

void* current_context() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

int static_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SWB_ERR_CUDA;
  void* ctx = current_context();   // null before the runtime first touches the device
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_static_ptr[dev] || !ctx || ctx != g_static_ctx[dev]) {
    void* p = nullptr;   // the lookup initialises the device's primary context if needed
    if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) return SWB_ERR_CUDA;
    g_static_ptr[dev] = p;
    g_static_ctx[dev] = current_context();
  }
  *out = g_static_ptr[dev];
  return SWB_OK;
}

// Common launch: per-call resets, then the forward and adjoint kernels.
template <int NS, int R, int G = 0>
int launch(Args a, const Layout& l, long long ntasks, size_t map_elems, bool clear_map, void* ws,
           size_t ws_bytes, void* stream_v, const swb_options* opt, bool value_only = false) {
  if (!ws || ws_bytes < l.total) return SWB_ERR_WORKSPACE;
  DevInfo* d = nullptr;
  int rc = dev_info(&d);
  if (rc != SWB_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream_v);
  char* w = static_cast<char*>(ws);
  a.k = 1.4426950408889634f / a.T;
  a.counters = reinterpret_cast<unsigned*>(w + l.off_hdr);
  a.status = a.counters + 4;
  a.pair_done = reinterpret_cast<unsigned*>(w + l.off_pair_done);
  a.part = reinterpret_cast<float*>(w + l.off_part);
  a.gpart = reinterpret_cast<float*>(w + l.off_gpart);
  a.never_written = reinterpret_cast<float*>(w + l.off_sent);
  a.edge = reinterpret_cast<float*>(w + l.off_edge);
  a.bpush = reinterpret_cast<float*>(w + l.off_bpush);
  a.ckpt = value_only ? nullptr : reinterpret_cast<float*>(w + l.off_ckpt);
  a.spin_limit_ns = (opt && opt->spin_limit_ns) ? opt->spin_limit_ns : 20ull * 1000000000ull;
  a.fault_inject = opt ? opt->fault_inject : 0;
  // the local models run in the scaled linear domain (sw_lin.cu) when every
  // transition factor 2^(gap k) is at most 1, else in the log domain
  const double xo = (double)a.go * (double)a.k, xe = NS == 3 ? (double)a.ge * (double)a.k : 0.0;
  const int domain = opt ? opt->domain : SWB_DOMAIN_AUTO;
  const bool lin = G == 0 && domain != SWB_DOMAIN_LOG && xo <= 0.0 && xe <= 0.0;
  if (G == 0 && domain == SWB_DOMAIN_LINEAR && !lin) return SWB_ERR_ARG;
  a.xgo = (float)exp2(xo);
  a.xge = (float)exp2(xe);
  if (a.ck_every < 1) a.ck_every = 1;
  a.dparams = opt ? opt->params_device : nullptr;
  if (a.dparams && !lin) return SWB_ERR_ARG;   // device parameters: linear-domain kernels only

  // per-call resets: counters, status and completion counts to 0, cross-band
  // buffers to the NaN sentinel, the map to 0 (cells outside lengths stay 0)
  if (cudaMemsetAsync(w, 0, l.off_part, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (cudaMemsetAsync(w + l.off_sent, 0xff, l.sent_bytes, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (clear_map && map_elems > 0 &&
      cudaMemsetAsync(a.map, 0, map_elems * sizeof(float), st) != cudaSuccess)
    return SWB_ERR_CUDA;

  if (R == 8 && !lin) return SWB_ERR_ARG;   // 8 columns per lane: linear domain only
  constexpr int m = model_index<NS, G>();
  const int of = lin ? d->locc[0][NS == 3][ridx(R)] : d->occ[0][m][R == 4];
  const int ob = lin ? d->locc[1][NS == 3][ridx(R)] : d->occ[1][m][R == 4];
  const int cta_cap_f = d->sms * (of > 0 ? of : 1);
  const int cta_cap_b = d->sms * (ob > 0 ? ob : 1);
  const long long need_f = (ntasks + kWarpsFwd - 1) / kWarpsFwd;
  const long long need_b = (ntasks + kWarpsBwd - 1) / kWarpsBwd;
  int grid_f = (int)(need_f < cta_cap_f ? need_f : cta_cap_f);
  int grid_b = (int)(need_b < cta_cap_b ? need_b : cta_cap_b);
  if (opt && opt->max_ctas > 0) {
    if (grid_f > opt->max_ctas) grid_f = opt->max_ctas;
    if (grid_b > opt->max_ctas) grid_b = opt->max_ctas;
  }
  if (grid_f < 1) grid_f = 1;
  if (grid_b < 1) grid_b = 1;
  if (lin) {
    if constexpr (G == 0) {
      swb::lfwd_kernel<NS, R><<<grid_f, 32 * kWarpsFwd, 0, st>>>(a);
      if (cudaPeekAtLastError() != cudaSuccess) return SWB_ERR_CUDA;
      if (opt && opt->split_event &&
          cudaEventRecord(reinterpret_cast<cudaEvent_t>(opt->split_event), st) != cudaSuccess)
        return SWB_ERR_CUDA;
      if (value_only) {
        swb::lvalue_kernel<NS, R><<<(a.B + 3) / 4, 128, 0, st>>>(a);
        return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
      }
      swb::lbwd_kernel<NS, R, kWarpsBwd><<<grid_b, 32 * kWarpsBwd, lbwd_smem<NS, R>(), st>>>(a);
      return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
    }
  }
  if constexpr (R != 8) {   // the log-domain kernels have 2 or 4 columns per lane
    swb::fwd_kernel<NS, R, G><<<grid_f, 32 * kWarpsFwd, 0, st>>>(a);
    if (cudaPeekAtLastError() != cudaSuccess) return SWB_ERR_CUDA;
    if (opt && opt->split_event &&
        cudaEventRecord(reinterpret_cast<cudaEvent_t>(opt->split_event), st) != cudaSuccess)
      return SWB_ERR_CUDA;
    if (value_only) {
      swb::value_kernel<NS, R, G><<<(a.B + 3) / 4, 128, 0, st>>>(a);
      return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
    }
    swb::bwd_kernel<NS, R, kWarpsBwd, G><<<grid_b, 32 * kWarpsBwd, bwd_smem<NS, R>(), st>>>(a);
    if (cudaPeekAtLastError() != cudaSuccess) return SWB_ERR_CUDA;
  }
  return SWB_OK;
}

template <int NS, int R, int G = 0>
int launch_padded_r(const float* scores, const int* lengths, int B, int L1m, int L2m, float go,
                    float ge, float T, float* value, float* map, float* g_open, float* g_ext,
                    float* g_T, void* ws, size_t ws_bytes, void* stream, const swb_options* opt) {
  if (B < 0 || L1m < 0 || L2m < 0) return SWB_ERR_ARG;
  if (!(T > 0.f) || !(T < INFINITY)) return SWB_ERR_ARG;
  if (B == 0) return SWB_OK;
  const size_t map_elems = (size_t)B * L1m * L2m;
  if (!value || !g_open || !g_T || (NS == 3 && !g_ext)) return SWB_ERR_ARG;
  if (map_elems > 0 && (!scores || !map)) return SWB_ERR_ARG;
  const Layout l = layout_for<NS, R, G>(B, L1m, L2m);
  Args a{};
  a.scores = scores; a.map = map; a.lengths = lengths;
  a.B = B; a.Lmax1 = L1m; a.Lmax2 = L2m; a.layout = 0;
  a.go = go; a.ge = ge; a.T = T;
  a.nb = l.nb; a.nchunks = l.nchunks;
  a.value = value; a.g_open = g_open; a.g_ext = g_ext; a.g_T = g_T;
  return launch<NS, R, G>(a, l, (long long)B * l.nb, map_elems, true, ws, ws_bytes, stream, opt);
}

template <int NS, int G = 0>
int launch_padded(const float* scores, const int* lengths, int B, int L1m, int L2m, float go,
                  float ge, float T, float* value, float* map, float* g_open, float* g_ext,
                  float* g_T, void* ws, size_t ws_bytes, void* stream, const swb_options* opt) {
  const int r = pick_r(opt, L2m, lin_eligible<NS, G>(go, ge, T, opt));
  if (r == 2)
    return launch_padded_r<NS, 2, G>(scores, lengths, B, L1m, L2m, go, ge, T, value, map, g_open,
                                     g_ext, g_T, ws, ws_bytes, stream, opt);
  if (r == 4)
    return launch_padded_r<NS, 4, G>(scores, lengths, B, L1m, L2m, go, ge, T, value, map, g_open,
                                     g_ext, g_T, ws, ws_bytes, stream, opt);
  if constexpr (G == 0) {   // 8 columns per lane: the local families' linear-domain kernels
    if (r == 8)
      return launch_padded_r<NS, 8, G>(scores, lengths, B, L1m, L2m, go, ge, T, value, map, g_open,
                                       g_ext, g_T, ws, ws_bytes, stream, opt);
  }
  return SWB_ERR_ARG;
}

// Padded value-only batch: the forward wavefront, no checkpoints, no adjoint.
// Columns per lane as the full call's default (the values are equal bit for
// bit only for equal band decompositions).
template <int NS, int G = 0, int R = kDefaultR>
Layout value_layout(long long B, long long L1m, long long L2m) {
  int nb = (int)((L2m + 32 * R - 1) / (32 * R));
  if (nb < 1) nb = 1;
  const size_t slots = (size_t)B * nb;
  Layout l = layout_sizes(B, slots, slots * ne<NS, R>() * (size_t)L1m,
                          slots * np<NS, G>() * (size_t)(L1m + 1), 0);
  l.nb = nb;
  l.nchunks = chunks_for(L1m);
  return l;
}

template <int NS, int G = 0>
int launch_value(const float* scores, const int* lengths, int B, int L1m, int L2m, float go,
                 float ge, float T, float* value, void* ws, size_t ws_bytes, void* stream) {
  if (B < 0 || L1m < 0 || L2m < 0) return SWB_ERR_ARG;
  if (!(T > 0.f) || !(T < INFINITY)) return SWB_ERR_ARG;
  if (B == 0) return SWB_OK;
  if (!value || ((size_t)B * L1m * L2m > 0 && !scores)) return SWB_ERR_ARG;
  auto run = [&](auto rt) {
    constexpr int R = decltype(rt)::value;
    const Layout l = value_layout<NS, G, R>(B, L1m, L2m);
    Args a{};
    a.scores = scores; a.map = nullptr; a.lengths = lengths;
    a.B = B; a.Lmax1 = L1m; a.Lmax2 = L2m; a.layout = 0;
    a.go = go; a.ge = ge; a.T = T;
    a.nb = l.nb; a.nchunks = l.nchunks;
    a.value = value;
    return launch<NS, R, G>(a, l, (long long)B * l.nb, 0, false, ws, ws_bytes, stream, nullptr, true);
  };
  if constexpr (G == 0) {
    const int r = default_r(L2m, lin_eligible<NS, G>(go, ge, T, nullptr));
    if (r == 8) return run(std::integral_constant<int, 8>{});
    if (r == 2) return run(std::integral_constant<int, 2>{});
  }
  return run(std::integral_constant<int, kDefaultR>{});
}

template <int NS, int G = 0>
size_t value_workspace(long long B, long long L1m, long long L2m) {
  size_t n = value_layout<NS, G, kDefaultR>(B, L1m, L2m).total;
  if constexpr (G == 0)
    n = std::max({n, value_layout<NS, G, 8>(B, L1m, L2m).total, value_layout<NS, G, 2>(B, L1m, L2m).total});
  return n;
}

template <int NS, int G = 0>
int launch_ragged(const float* scores, const void* host_plan, const void* dev_plan, float go,
                  float ge, float T, float* value, float* map, float* g_open, float* g_ext,
                  float* g_T, void* ws, size_t ws_bytes, void* stream, const swb_options* opt,
                  bool value_only = false) {
  if (!host_plan || !dev_plan) return SWB_ERR_ARG;
  const long long* h = static_cast<const long long*>(host_plan);
  // plan families: 1 linear, 3 affine, 2 global linear, 4 global affine, 5 Saigo-Vert
  constexpr int fam = G == 2 ? 5 : (G == 1 ? (NS == 3 ? 4 : 2) : NS);
  if (h[HW_MAGIC] != kPlanMagic || (h[HW_FAMILY] & 0xff) != fam) return SWB_ERR_ARG;
  const int r = (int)(h[HW_FAMILY] >> 8);
  if (!(T > 0.f) || !(T < INFINITY)) return SWB_ERR_ARG;
  const long long B = h[HW_B], ntasks = h[HW_NTASKS];
  if (B == 0) return SWB_OK;
  if (!value) return SWB_ERR_ARG;
  if (!value_only && (!g_open || !g_T || (NS == 3 && !g_ext))) return SWB_ERR_ARG;
  if (h[HW_MAP_ELEMS] > 0 && (!scores || (!value_only && !map))) return SWB_ERR_ARG;
  const Layout l = layout_sizes(B, (size_t)h[HW_SLOTS], (size_t)h[HW_EDGE], (size_t)h[HW_BP],
                                (size_t)h[HW_CK]);
  const long long* dp = static_cast<const long long*>(dev_plan);
  Args a{};
  a.scores = scores; a.map = map;
  a.plan_pairs = dp + HW_WORDS;
  a.plan_tasks = reinterpret_cast<const int*>(dp + HW_WORDS + B * swb::PLAN_PAIR_WORDS);
  a.ntasks = (int)ntasks;
  a.B = (int)B; a.layout = 1;
  a.go = go; a.ge = ge; a.T = T;
  a.value = value; a.g_open = g_open; a.g_ext = g_ext; a.g_T = g_T;
  if (r == 2)
    return launch<NS, 2, G>(a, l, ntasks, (size_t)h[HW_MAP_ELEMS], false, ws, ws_bytes, stream,
                            opt, value_only);
  if (r == 4)
    return launch<NS, 4, G>(a, l, ntasks, (size_t)h[HW_MAP_ELEMS], false, ws, ws_bytes, stream,
                            opt, value_only);
  if constexpr (G == 0) {
    if (r == 8)
      return launch<NS, 8, G>(a, l, ntasks, (size_t)h[HW_MAP_ELEMS], false, ws, ws_bytes, stream,
                              opt, value_only);
  }
  return SWB_ERR_ARG;
}

// ---- second-order ops as band wavefronts ----

// Columns per lane of the second-order kernels: 4 once the batch has at least
// kXTasksR4 bands of 128 columns (measured at 256 x 512^2: HVP 3.2 ms at 4
// against 4.5 ms at 2), else 2, which doubles the warps for small batches.
constexpr long long kXTasksR4 = 256;
#ifndef SWB_XR
#define SWB_XR 0
#endif

int xpick_r(long long B, long long L2m) {
  if (SWB_XR == 2 || SWB_XR == 4) return SWB_XR;
  const long long nb4 = std::max(1LL, (L2m + 127) / 128);
  return B * nb4 >= kXTasksR4 ? 4 : 2;
}

struct XLayout {
  int R, nb, nsteps;
  size_t off_pair_done, off_part, off_gpart, off_cmax, off_sent, off_edge, off_bpush, off_fld;
  size_t sent_bytes, total;
};

template <int NS, int G = 0>
XLayout xlayout(long long B, long long L1m, long long L2m) {
  XLayout l{};
  l.R = xpick_r(B, L2m);
  l.nb = (int)std::max(1LL, (L2m + 32 * l.R - 1) / (32 * l.R));
  l.nsteps = (int)((L1m + 31 + swb::XC - 1) / swb::XC * swb::XC);
  const size_t slots = (size_t)B * l.nb;
  using XS = swb::XShape<NS, G>;
  const size_t step = (size_t)l.R * XS::G * 128;
  size_t o = align_up(64);   // counters [0, 1], status [4]
  l.off_pair_done = o; o = align_up(o + sizeof(unsigned) * (size_t)B);
  l.off_part = o;      o = align_up(o + sizeof(float) * swb::XPART * slots);
  l.off_gpart = o;     o = align_up(o + sizeof(float) * 4 * slots);
  l.off_cmax = o;      o = align_up(o + sizeof(float) * slots * (size_t)(l.nsteps / swb::XC));
  l.off_sent = o;
  l.off_edge = o;      o = align_up(o + sizeof(float) * slots * XS::NE * (size_t)L1m);
  l.off_bpush = o;
  o = align_up(o + sizeof(float) * slots * 2 * XS::NP * (size_t)(L1m + 1));
  l.sent_bytes = o - l.off_sent;
  l.off_fld = o;       o = align_up(o + sizeof(float) * slots * (size_t)l.nsteps * step);
  l.total = o;
  return l;
}

// Occupancy of each second-order instantiation on one device, computed once.
struct XOcc {
  int f = 0, b = 0;
  bool ready = false;
};
XOcc g_xocc[64][5][2][4];   // [device][model_index][R == 4?][mode]

template <int NS, int R, int MODE, int G = 0>
int launch_xband_r(swb::XArgs a, cudaStream_t st) {
  DevInfo* d = nullptr;
  int rc = dev_info(&d);
  if (rc != SWB_OK) return rc;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SWB_ERR_CUDA;
  const size_t smem = sizeof(float) * swb::XSTAGES * swb::xstep_floats<NS, R, G>();
  XOcc& o = g_xocc[dev][model_index<NS, G>()][R == 4][MODE];
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!o.ready) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.f, swb::xfwd_kernel<NS, R, MODE, G>, 128,
                                                        0) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.b, swb::xbwd_kernel<NS, R, MODE, G>, 32,
                                                        smem) != cudaSuccess)
        return SWB_ERR_CUDA;
      o.ready = true;
    }
  }
  const long long ntasks = (long long)a.B * a.nb;
  const long long cap_f = (long long)d->sms * (o.f > 0 ? o.f : 1);
  const long long cap_b = (long long)d->sms * (o.b > 0 ? o.b : 1);
  const int grid_f = (int)std::min((ntasks + 3) / 4, cap_f);
  const int grid_b = (int)std::min(ntasks, cap_b);
  swb::xfwd_kernel<NS, R, MODE, G><<<grid_f, 128, 0, st>>>(a);
  swb::xbwd_kernel<NS, R, MODE, G><<<grid_b, 32, smem, st>>>(a);
  return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
}

// ---- second-order ops of the local models in the linear domain ----

constexpr int kTanR = 4;   // columns per lane of the tangent kernels
static_assert((int)swb::TM_SCORE == (int)swb::AUX_HVP && (int)swb::TM_G0 == (int)swb::AUX_P0 &&
                  (int)swb::TM_G1 == (int)swb::AUX_P1 && (int)swb::TM_T == (int)swb::AUX_PT,
              "tangent directions follow the second-order op modes");

// Workspace of the tangent kernels: counters and status, per-pair completion
// counts, per-band (frame, Z) and (frame, Z') partials and parameter-tangent
// partials, then (sentinel-filled) edge and push records, then checkpoints.
struct TLayout {
  size_t off_pair_done, off_part, off_zdot, off_gpart, off_edge, off_bpush, off_ckpt, total;
  int nb, nchunks;
};

template <int NS>
TLayout tlayout(long long B, long long L1m, long long L2m) {
  using D = swb::TDims<NS, kTanR>;
  TLayout l{};
  l.nb = (int)std::max(1LL, (L2m + 32 * kTanR - 1) / (32 * kTanR));
  l.nchunks = chunks_for(L1m);
  const size_t slots = (size_t)B * l.nb;
  size_t o = align_up(64);   // counters [0, 1], status [4]
  l.off_pair_done = o; o = align_up(o + sizeof(unsigned) * (size_t)B);
  l.off_part = o;      o = align_up(o + sizeof(float) * 2 * slots);
  l.off_zdot = o;      o = align_up(o + sizeof(float) * 2 * slots);
  l.off_gpart = o;     o = align_up(o + sizeof(float) * 8 * slots);
  l.off_edge = o;      o = align_up(o + sizeof(float) * slots * D::NEF * (size_t)L1m);
  l.off_bpush = o;     o = align_up(o + sizeof(float) * slots * D::NPF * (size_t)(L1m + 1));
  l.off_ckpt = o;      o = align_up(o + sizeof(float) * slots * (size_t)l.nchunks * D::LREC);
  l.total = o;
  return l;
}

// The linear-domain tangent kernels serve the local models when every gap is
// <= 0 and T is finite and positive (the first-order linear domain's range).
bool tan_eligible(float go, float ge, float T) {
  if (!SWB_TAN || !(T > 0.f) || !(T < INFINITY)) return false;
  const float k = 1.4426950408889634f / T;
  return (double)go * k <= 0.0 && (double)ge * k <= 0.0;
}

struct TOcc {
  int f = 0, b = 0;
  bool ready = false;
};
TOcc g_tocc[64][2][4];   // [device][affine?][mode]

template <int NS, int MODE>
int launch_tan(const float* scores, const float* v, const int* lengths, int B, int L1m, int L2m,
               float go, float ge, float T, float* out, float* gt, void* ws, size_t ws_bytes,
               cudaStream_t st) {
  constexpr int R = kTanR;
  const TLayout l = tlayout<NS>(B, L1m, L2m);
  if (!ws || ws_bytes < l.total) return SWB_ERR_WORKSPACE;
  DevInfo* d = nullptr;
  int rc = dev_info(&d);
  if (rc != SWB_OK) return rc;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SWB_ERR_CUDA;
  const size_t smem = sizeof(float) * swb::ltbwd_smem_floats<NS, R>();
  TOcc& o = g_tocc[dev][NS == 3][MODE];
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!o.ready) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.f, swb::ltfwd_kernel<NS, R, MODE>, 128, 0) !=
              cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.b, swb::ltbwd_kernel<NS, R, MODE>, 32, smem) !=
              cudaSuccess)
        return SWB_ERR_CUDA;
      o.ready = true;
    }
  }
  char* w = static_cast<char*>(ws);
  // per-call resets: header, completion counts and partials to 0; the edge and
  // push records to the NaN sentinel; the output to 0 (cells outside lengths)
  if (cudaMemsetAsync(w, 0, l.off_edge, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (cudaMemsetAsync(w + l.off_edge, 0xff, l.off_ckpt - l.off_edge, st) != cudaSuccess) return SWB_ERR_CUDA;
  const size_t map_elems = (size_t)B * L1m * L2m;
  if (map_elems > 0 && cudaMemsetAsync(out, 0, map_elems * sizeof(float), st) != cudaSuccess)
    return SWB_ERR_CUDA;
  swb::Args a{};
  a.scores = scores; a.map = out; a.lengths = lengths;
  a.B = B; a.Lmax1 = L1m; a.Lmax2 = L2m; a.layout = 0;
  a.go = go; a.ge = ge; a.T = T; a.k = 1.4426950408889634f / T;
  a.xgo = (float)exp2((double)go * (double)a.k);
  a.xge = (float)exp2((double)ge * (double)a.k);
  a.nb = l.nb; a.nchunks = l.nchunks;
  a.counters = reinterpret_cast<unsigned*>(w);
  a.status = a.counters + 4;
  a.pair_done = reinterpret_cast<unsigned*>(w + l.off_pair_done);
  a.part = reinterpret_cast<float*>(w + l.off_part);
  a.zdot = reinterpret_cast<float*>(w + l.off_zdot);
  a.gpart = reinterpret_cast<float*>(w + l.off_gpart);
  a.edge = reinterpret_cast<float*>(w + l.off_edge);
  a.bpush = reinterpret_cast<float*>(w + l.off_bpush);
  a.ckpt = reinterpret_cast<float*>(w + l.off_ckpt);
  a.tdir = v; a.tgt = gt; a.tmode = MODE;
  a.spin_limit_ns = 20ull * 1000000000ull;
  const long long ntasks = (long long)B * l.nb;
  const long long cap_f = (long long)d->sms * (o.f > 0 ? o.f : 1);
  const long long cap_b = (long long)d->sms * (o.b > 0 ? o.b : 1);
  const int grid_f = (int)std::min((ntasks + 3) / 4, cap_f);
  const int grid_b = (int)std::min(ntasks, cap_b);
  swb::ltfwd_kernel<NS, R, MODE><<<grid_f, 128, 0, st>>>(a);
  swb::ltbwd_kernel<NS, R, MODE><<<grid_b, 32, smem, st>>>(a);
  return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
}

template <int NS, int MODE, int G = 0>
int launch_xband(const float* scores, const float* v, const int* lengths, int B, int L1m, int L2m,
                 float go, float ge, float T, float* out, float* gt, void* ws, size_t ws_bytes,
                 void* stream_v) {
  if (B < 0 || L1m < 0 || L2m < 0) return SWB_ERR_ARG;
  if (!(T > 0.f) || !(T < INFINITY)) return SWB_ERR_ARG;
  if (B == 0) return SWB_OK;
  if constexpr (G == 0) {
    if (tan_eligible(go, NS == 3 ? ge : 0.f, T)) {
      const size_t map_elems = (size_t)B * L1m * L2m;
      if (map_elems > 0 && (!scores || !out || (MODE == swb::AUX_HVP && !v))) return SWB_ERR_ARG;
      return launch_tan<NS, MODE>(scores, v, lengths, B, L1m, L2m, go, ge, T, out, gt, ws, ws_bytes,
                                  reinterpret_cast<cudaStream_t>(stream_v));
    }
  }
  const size_t map_elems = (size_t)B * L1m * L2m;
  if (map_elems > 0 && (!scores || !out || (MODE == swb::AUX_HVP && !v))) return SWB_ERR_ARG;
  const XLayout l = xlayout<NS, G>(B, L1m, L2m);
  if (!ws || ws_bytes < l.total) return SWB_ERR_WORKSPACE;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream_v);
  char* w = static_cast<char*>(ws);
  // per-call resets: counters, status, completion counts to 0; cross-band
  // buffers to the NaN sentinel; the output to 0 (cells outside lengths stay 0)
  if (cudaMemsetAsync(w, 0, l.off_part, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (cudaMemsetAsync(w + l.off_sent, 0xff, l.sent_bytes, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (map_elems > 0 && cudaMemsetAsync(out, 0, map_elems * sizeof(float), st) != cudaSuccess)
    return SWB_ERR_CUDA;
  swb::XArgs a{};
  a.scores = scores; a.v = v; a.lengths = lengths;
  a.B = B; a.L1m = L1m; a.L2m = L2m; a.nb = l.nb; a.nsteps = l.nsteps;
  a.go = go; a.ge = ge; a.T = T; a.k = 1.4426950408889634f / T;
  a.out = out; a.gt = gt;
  a.counters = reinterpret_cast<unsigned*>(w);
  a.status = a.counters + 4;
  a.pair_done = reinterpret_cast<unsigned*>(w + l.off_pair_done);
  a.part = reinterpret_cast<float*>(w + l.off_part);
  a.gpart = reinterpret_cast<float*>(w + l.off_gpart);
  a.cmax = reinterpret_cast<float*>(w + l.off_cmax);
  a.edge = reinterpret_cast<float*>(w + l.off_edge);
  a.bpush = reinterpret_cast<float*>(w + l.off_bpush);
  a.fld = reinterpret_cast<float*>(w + l.off_fld);
  a.spin_limit_ns = 20ull * 1000000000ull;
  return l.R == 4 ? launch_xband_r<NS, 4, MODE, G>(a, st) : launch_xband_r<NS, 2, MODE, G>(a, st);
}

// ---- checkpointed value: forward now (checkpoints kept), adjoint later ----

constexpr int kMaxCkEvery = 16;

template <int NS, int R>
Layout ck_layout(long long B, long long L1m, long long L2m, int kc) {
  using LD = swb::LDims<NS, R>;
  int nb = (int)((L2m + 32 * R - 1) / (32 * R));
  if (nb < 1) nb = 1;
  const int nch = chunks_for(L1m);
  const size_t band = ((size_t)((nch + kc - 1) / kc) * LD::LREC + (size_t)nch + 3) / 4 * 4;
  const size_t slots = (size_t)B * nb;
  Layout l = layout_sizes(B, slots, slots * ne<NS, R>() * (size_t)L1m,
                          slots * np<NS, 0>() * (size_t)(L1m + 1), slots * band);
  l.nb = nb;
  l.nchunks = nch;
  l.ck_band = band;
  return l;
}

// Shared set-up of the two halves: argument checks, parameters (linear
// domain only), workspace pointers.  Returns SWB_OK or an error code.
template <int NS, int R>
int ck_setup(Args& a, Layout& l, const float* scores, const int* lengths, int B, int L1m, int L2m,
             float go, float ge, float T, int kc, void* ws, size_t ws_bytes) {
  if (B < 0 || L1m < 0 || L2m < 0 || kc < 1 || kc > kMaxCkEvery) return SWB_ERR_ARG;
  if (!(T > 0.f) || !(T < INFINITY)) return SWB_ERR_ARG;
  if ((size_t)B * L1m * L2m > 0 && !scores) return SWB_ERR_ARG;
  a = Args{};
  a.k = 1.4426950408889634f / T;
  const double xo = (double)go * (double)a.k, xe = NS == 3 ? (double)ge * (double)a.k : 0.0;
  if (!(xo <= 0.0 && xe <= 0.0)) return SWB_ERR_ARG;   // the linear domain needs gaps <= 0
  l = ck_layout<NS, R>(B, L1m, L2m, kc);
  if (!ws || ws_bytes < l.total) return SWB_ERR_WORKSPACE;
  char* w = static_cast<char*>(ws);
  a.scores = scores; a.lengths = lengths;
  a.B = B; a.Lmax1 = L1m; a.Lmax2 = L2m; a.layout = 0;
  a.go = go; a.ge = NS == 3 ? ge : 0.f; a.T = T;
  a.xgo = (float)exp2(xo);
  a.xge = (float)exp2(xe);
  a.nb = l.nb; a.nchunks = l.nchunks;
  a.ck_every = kc;
  a.ck_band_floats = l.ck_band;
  a.counters = reinterpret_cast<unsigned*>(w + l.off_hdr);
  a.status = a.counters + 4;
  a.pair_done = reinterpret_cast<unsigned*>(w + l.off_pair_done);
  a.part = reinterpret_cast<float*>(w + l.off_part);
  a.gpart = reinterpret_cast<float*>(w + l.off_gpart);
  a.never_written = reinterpret_cast<float*>(w + l.off_sent);
  a.edge = reinterpret_cast<float*>(w + l.off_edge);
  a.bpush = reinterpret_cast<float*>(w + l.off_bpush);
  a.ckpt = reinterpret_cast<float*>(w + l.off_ckpt);
  a.spin_limit_ns = 20ull * 1000000000ull;
  return SWB_OK;
}

template <int NS, int R>
int ck_forward_r(const float* scores, const int* lengths, int B, int L1m, int L2m, float go, float ge,
                 float T, int kc, float* value, void* ws, size_t ws_bytes, void* stream_v) {
  Args a;
  Layout l;
  int rc = ck_setup<NS, R>(a, l, scores, lengths, B, L1m, L2m, go, ge, T, kc, ws, ws_bytes);
  if (rc != SWB_OK) return rc;
  if (B == 0) return SWB_OK;
  if (!value) return SWB_ERR_ARG;
  a.value = value;
  DevInfo* d = nullptr;
  if ((rc = dev_info(&d)) != SWB_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream_v);
  char* w = static_cast<char*>(ws);
  if (cudaMemsetAsync(w, 0, l.off_part, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (cudaMemsetAsync(w + l.off_sent, 0xff, l.sent_bytes, st) != cudaSuccess) return SWB_ERR_CUDA;
  const long long ntasks = (long long)B * l.nb;
  const int of = d->locc[0][NS == 3][ridx(R)];
  const long long cap = (long long)d->sms * (of > 0 ? of : 1);
  const int grid = (int)std::max(1LL, std::min((ntasks + kWarpsFwd - 1) / kWarpsFwd, cap));
  swb::lfwd_kernel<NS, R><<<grid, 32 * kWarpsFwd, 0, st>>>(a);
  swb::lvalue_kernel<NS, R><<<(B + 3) / 4, 128, 0, st>>>(a);
  return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
}

template <int NS, int R>
int ck_adjoint_r(const float* scores, const int* lengths, int B, int L1m, int L2m, float go, float ge,
                 float T, int kc, float* value, float* map, float* g_open, float* g_ext, float* g_T,
                 void* ws, size_t ws_bytes, void* stream_v) {
  Args a;
  Layout l;
  int rc = ck_setup<NS, R>(a, l, scores, lengths, B, L1m, L2m, go, ge, T, kc, ws, ws_bytes);
  if (rc != SWB_OK) return rc;
  if (B == 0) return SWB_OK;
  const size_t map_elems = (size_t)B * L1m * L2m;
  if (!value || !g_open || !g_T || (NS == 3 && !g_ext) || (map_elems > 0 && !map)) return SWB_ERR_ARG;
  a.value = value; a.map = map; a.g_open = g_open; a.g_ext = g_ext; a.g_T = g_T;
  DevInfo* d = nullptr;
  if ((rc = dev_info(&d)) != SWB_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream_v);
  char* w = static_cast<char*>(ws);
  // the forward's edge records, partials and checkpoints stay; the adjoint's
  // counter, the completion counts (not the failure flags) and the push
  // records are reset, so the adjoint can run more than once
  swb::adjoint_reset_kernel<<<(B + 255) / 256, 256, 0, st>>>(a.counters, a.pair_done, B);
  if (cudaMemsetAsync(w + l.off_bpush, 0xff, l.off_ckpt - l.off_bpush, st) != cudaSuccess)
    return SWB_ERR_CUDA;
  if (map_elems > 0 && cudaMemsetAsync(map, 0, map_elems * sizeof(float), st) != cudaSuccess)
    return SWB_ERR_CUDA;
  const long long ntasks = (long long)B * l.nb;
  const int ob = kc > 1 ? d->locc_sparse[NS == 3][ridx(R)] : d->locc[1][NS == 3][ridx(R)];
  const long long cap = (long long)d->sms * (ob > 0 ? ob : 1);
  const int grid = (int)std::max(1LL, std::min((ntasks + kWarpsBwd - 1) / kWarpsBwd, cap));
  if (kc > 1)
    swb::lbwd_kernel<NS, R, kWarpsBwd, true><<<grid, 32 * kWarpsBwd, lbwd_smem<NS, R>(), st>>>(a);
  else
    swb::lbwd_kernel<NS, R, kWarpsBwd><<<grid, 32 * kWarpsBwd, lbwd_smem<NS, R>(), st>>>(a);
  return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
}

// The checkpointed op's columns per lane: the padded default for the linear
// domain (its results then equal the one-call entry points' bit for bit).
template <int NS>
int ck_forward(const float* scores, const int* lengths, int B, int L1m, int L2m, float go, float ge,
               float T, int kc, float* value, void* ws, size_t ws_bytes, void* stream_v) {
  const int r = default_r(L2m, true);
  if (r == 8)
    return ck_forward_r<NS, 8>(scores, lengths, B, L1m, L2m, go, ge, T, kc, value, ws, ws_bytes, stream_v);
  if (r == 2)
    return ck_forward_r<NS, 2>(scores, lengths, B, L1m, L2m, go, ge, T, kc, value, ws, ws_bytes, stream_v);
  return ck_forward_r<NS, 4>(scores, lengths, B, L1m, L2m, go, ge, T, kc, value, ws, ws_bytes, stream_v);
}

template <int NS>
int ck_adjoint(const float* scores, const int* lengths, int B, int L1m, int L2m, float go, float ge,
               float T, int kc, float* value, float* map, float* g_open, float* g_ext, float* g_T,
               void* ws, size_t ws_bytes, void* stream_v) {
  const int r = default_r(L2m, true);
  if (r == 8)
    return ck_adjoint_r<NS, 8>(scores, lengths, B, L1m, L2m, go, ge, T, kc, value, map, g_open, g_ext,
                               g_T, ws, ws_bytes, stream_v);
  if (r == 2)
    return ck_adjoint_r<NS, 2>(scores, lengths, B, L1m, L2m, go, ge, T, kc, value, map, g_open, g_ext,
                               g_T, ws, ws_bytes, stream_v);
  return ck_adjoint_r<NS, 4>(scores, lengths, B, L1m, L2m, go, ge, T, kc, value, map, g_open, g_ext,
                             g_T, ws, ws_bytes, stream_v);
}

template <int NS>
size_t ck_workspace(long long B, long long L1m, long long L2m, int kc) {
  const int r = default_r(L2m, true);
  return r == 8 ? ck_layout<NS, 8>(B, L1m, L2m, kc).total
                : (r == 2 ? ck_layout<NS, 2>(B, L1m, L2m, kc).total : ck_layout<NS, 4>(B, L1m, L2m, kc).total);
}

}  // namespace

extern "C" {

int swb_cols_per_lane(int family, int L2max, float gap_open, float gap_ext, float temp) {
  // family: 1 linear, 3 affine (local); 2, 4, 5 global and Saigo-Vert
  if (family == 1) return default_r(L2max, lin_eligible<1, 0>(gap_open, 0.f, temp, nullptr));
  if (family == 3) return default_r(L2max, lin_eligible<3, 0>(gap_open, gap_ext, temp, nullptr));
  return (family >= 1 && family <= 5) ? kDefaultR : SWB_ERR_ARG;
}

size_t swb_sw_affine_checkpoint_workspace_bytes(int B, int L1max, int L2max, int ck_every) {
  if (B <= 0 || ck_every < 1 || ck_every > kMaxCkEvery) return 0;
  return ck_workspace<3>(B, L1max, L2max, ck_every);
}

size_t swb_sw_checkpoint_workspace_bytes(int B, int L1max, int L2max, int ck_every) {
  if (B <= 0 || ck_every < 1 || ck_every > kMaxCkEvery) return 0;
  return ck_workspace<1>(B, L1max, L2max, ck_every);
}

int swb_sw_affine_checkpoint(const float* scores, const int* lengths, int B, int L1max, int L2max,
                             float gap_open, float gap_ext, float temp, int ck_every, float* value,
                             void* workspace, size_t workspace_bytes, void* stream) {
  return ck_forward<3>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, ck_every, value,
                       workspace, workspace_bytes, stream);
}

int swb_sw_affine_adjoint(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, int ck_every, float* value,
                          float* map, float* grad_open, float* grad_ext, float* grad_temp,
                          void* workspace, size_t workspace_bytes, void* stream) {
  return ck_adjoint<3>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, ck_every, value,
                       map, grad_open, grad_ext, grad_temp, workspace, workspace_bytes, stream);
}

int swb_sw_checkpoint(const float* scores, const int* lengths, int B, int L1max, int L2max,
                      float gap, float temp, int ck_every, float* value, void* workspace,
                      size_t workspace_bytes, void* stream) {
  return ck_forward<1>(scores, lengths, B, L1max, L2max, gap, 0.f, temp, ck_every, value, workspace,
                       workspace_bytes, stream);
}

int swb_sw_adjoint(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                   float temp, int ck_every, float* value, float* map, float* grad_gap,
                   float* grad_temp, void* workspace, size_t workspace_bytes, void* stream) {
  return ck_adjoint<1>(scores, lengths, B, L1max, L2max, gap, 0.f, temp, ck_every, value, map,
                       grad_gap, nullptr, grad_temp, workspace, workspace_bytes, stream);
}

size_t swb_sw_affine_aux_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? std::max(xlayout<3>(B, L1max, L2max).total, tlayout<3>(B, L1max, L2max).total) : 0;
}

size_t swb_sw_aux_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? std::max(xlayout<1>(B, L1max, L2max).total, tlayout<1>(B, L1max, L2max).total) : 0;
}

// What the second-order call with these parameters launches: the tangent
// kernels' layout when tan_eligible holds (launch_xband's own test), else the
// log-domain kernels'.
size_t swb_sw_affine_aux_workspace_bytes_for(int B, int L1max, int L2max, float gap_open,
                                             float gap_ext, float temp) {
  if (B <= 0) return 0;
  return tan_eligible(gap_open, gap_ext, temp) ? tlayout<3>(B, L1max, L2max).total
                                               : xlayout<3>(B, L1max, L2max).total;
}

size_t swb_sw_aux_workspace_bytes_for(int B, int L1max, int L2max, float gap, float temp) {
  if (B <= 0) return 0;
  return tan_eligible(gap, 0.f, temp) ? tlayout<1>(B, L1max, L2max).total
                                      : xlayout<1>(B, L1max, L2max).total;
}

int swb_sw_affine_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
                      int L2max, float gap_open, float gap_ext, float temp, float* out,
                      float* grad_tangents, void* workspace, size_t workspace_bytes, void* stream) {
  return launch_xband<3, swb::AUX_HVP>(scores, v, lengths, B, L1max, L2max, gap_open, gap_ext, temp,
                                     out, grad_tangents, workspace, workspace_bytes, stream);
}

int swb_sw_affine_param_jacobian(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp, int param,
                                 float* out, void* workspace, size_t workspace_bytes, void* stream) {
  switch (param) {
    case 0: return launch_xband<3, swb::AUX_P0>(scores, nullptr, lengths, B, L1max, L2max, gap_open,
                                              gap_ext, temp, out, nullptr, workspace, workspace_bytes, stream);
    case 1: return launch_xband<3, swb::AUX_P1>(scores, nullptr, lengths, B, L1max, L2max, gap_open,
                                              gap_ext, temp, out, nullptr, workspace, workspace_bytes, stream);
    case 2: return launch_xband<3, swb::AUX_PT>(scores, nullptr, lengths, B, L1max, L2max, gap_open,
                                              gap_ext, temp, out, nullptr, workspace, workspace_bytes, stream);
    default: return SWB_ERR_ARG;
  }
}

int swb_sw_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max, int L2max,
               float gap, float temp, float* out, float* grad_tangents, void* workspace,
               size_t workspace_bytes, void* stream) {
  return launch_xband<1, swb::AUX_HVP>(scores, v, lengths, B, L1max, L2max, gap, 0.f, temp, out,
                                     grad_tangents, workspace, workspace_bytes, stream);
}

int swb_sw_param_jacobian(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap, float temp, int param, float* out, void* workspace,
                          size_t workspace_bytes, void* stream) {
  switch (param) {
    case 0: return launch_xband<1, swb::AUX_P0>(scores, nullptr, lengths, B, L1max, L2max, gap, 0.f,
                                              temp, out, nullptr, workspace, workspace_bytes, stream);
    case 1: return launch_xband<1, swb::AUX_PT>(scores, nullptr, lengths, B, L1max, L2max, gap, 0.f,
                                              temp, out, nullptr, workspace, workspace_bytes, stream);
    default: return SWB_ERR_ARG;
  }
}


size_t swb_nw_affine_aux_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? xlayout<3, 1>(B, L1max, L2max).total : 0;
}

int swb_nw_affine_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
                      int L2max, float gap_open, float gap_ext, float temp, float* out,
                      float* grad_tangents, void* workspace, size_t workspace_bytes, void* stream) {
  return launch_xband<3, swb::AUX_HVP, 1>(scores, v, lengths, B, L1max, L2max, gap_open, gap_ext,
                                             temp, out, grad_tangents, workspace, workspace_bytes,
                                             stream);
}

int swb_nw_affine_param_jacobian(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp, int param,
                                 float* out, void* workspace, size_t workspace_bytes, void* stream) {
  switch (param) {
    case 0: return launch_xband<3, swb::AUX_P0, 1>(scores, nullptr, lengths, B, L1max, L2max,
                                                      gap_open, gap_ext, temp, out, nullptr,
                                                      workspace, workspace_bytes, stream);
    case 1: return launch_xband<3, swb::AUX_P1, 1>(scores, nullptr, lengths, B, L1max, L2max,
                                                      gap_open, gap_ext, temp, out, nullptr,
                                                      workspace, workspace_bytes, stream);
    case 2: return launch_xband<3, swb::AUX_PT, 1>(scores, nullptr, lengths, B, L1max, L2max,
                                                      gap_open, gap_ext, temp, out, nullptr,
                                                      workspace, workspace_bytes, stream);
    default: return SWB_ERR_ARG;
  }
}

size_t swb_sv_affine_aux_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? xlayout<3, 2>(B, L1max, L2max).total : 0;
}

int swb_sv_affine_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
                      int L2max, float gap_open, float gap_ext, float temp, float* out,
                      float* grad_tangents, void* workspace, size_t workspace_bytes, void* stream) {
  return launch_xband<3, swb::AUX_HVP, 2>(scores, v, lengths, B, L1max, L2max, gap_open, gap_ext,
                                          temp, out, grad_tangents, workspace, workspace_bytes,
                                          stream);
}

int swb_sv_affine_param_jacobian(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp, int param,
                                 float* out, void* workspace, size_t workspace_bytes, void* stream) {
  switch (param) {
    case 0: return launch_xband<3, swb::AUX_P0, 2>(scores, nullptr, lengths, B, L1max, L2max,
                                                   gap_open, gap_ext, temp, out, nullptr, workspace,
                                                   workspace_bytes, stream);
    case 1: return launch_xband<3, swb::AUX_P1, 2>(scores, nullptr, lengths, B, L1max, L2max,
                                                   gap_open, gap_ext, temp, out, nullptr, workspace,
                                                   workspace_bytes, stream);
    case 2: return launch_xband<3, swb::AUX_PT, 2>(scores, nullptr, lengths, B, L1max, L2max,
                                                   gap_open, gap_ext, temp, out, nullptr, workspace,
                                                   workspace_bytes, stream);
    default: return SWB_ERR_ARG;
  }
}

size_t swb_nw_aux_workspace_bytes(int B, int L1max, int L2max) {
  return swb_sw_aux_workspace_bytes(B, L1max, L2max);
}

int swb_nw_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max, int L2max,
               float gap, float temp, float* out, float* grad_tangents, void* workspace,
               size_t workspace_bytes, void* stream) {
  return launch_xband<1, swb::AUX_HVP, 1>(scores, v, lengths, B, L1max, L2max, gap, 0.f, temp,
                                             out, grad_tangents, workspace, workspace_bytes, stream);
}

int swb_nw_param_jacobian(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap, float temp, int param, float* out, void* workspace,
                          size_t workspace_bytes, void* stream) {
  switch (param) {
    case 0: return launch_xband<1, swb::AUX_P0, 1>(scores, nullptr, lengths, B, L1max, L2max, gap,
                                                      0.f, temp, out, nullptr, workspace,
                                                      workspace_bytes, stream);
    case 1: return launch_xband<1, swb::AUX_PT, 1>(scores, nullptr, lengths, B, L1max, L2max, gap,
                                                      0.f, temp, out, nullptr, workspace,
                                                      workspace_bytes, stream);
    default: return SWB_ERR_ARG;
  }
}

size_t swb_sw_affine_workspace_bytes(int B, int L1max, int L2max) {
  if (B <= 0) return 0;
  return std::max({layout_for<3, 2>(B, L1max, L2max).total, layout_for<3, 4>(B, L1max, L2max).total,
                   layout_for<3, 8>(B, L1max, L2max).total});
}

int swb_scan_scores(const float* x, int B, long long per_item, float limit, float sentinel,
                    unsigned* words, float* amax, void* stream) {
  if (B < 0 || per_item < 0 || !words || !amax) return SWB_ERR_ARG;
  if (B == 0) return SWB_OK;
  if (per_item > 0 && !x) return SWB_ERR_ARG;
  DevInfo* d = nullptr;
  int rc = dev_info(&d);
  if (rc != SWB_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  swb::scan_init_kernel<<<(B + 1 + 255) / 256, 256, 0, st>>>(words, B);
  if (per_item > 0) {
    // about 8 blocks of 256 threads per SM in all, at least one per item
    const long long want = (long long)d->sms * 8;
    long long bpi = (want + B - 1) / B;
    const long long most = (per_item + 1023) / 1024;
    if (bpi > most) bpi = most;
    if (bpi < 1) bpi = 1;
    if ((long long)B * bpi > 0x7fffffffLL) return SWB_ERR_ARG;
    swb::scan_kernel<<<(unsigned)(B * bpi), 256, 0, st>>>(x, per_item, (int)bpi, limit, sentinel,
                                                          words);
  }
  swb::scan_finish_kernel<<<(B + 255) / 256, 256, 0, st>>>(words, amax, B);
  return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
}

size_t swb_sw_affine_value_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? value_workspace<3>(B, L1max, L2max) : 0;
}

size_t swb_sw_value_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? value_workspace<1>(B, L1max, L2max) : 0;
}

int swb_sw_affine_value(const float* scores, const int* lengths, int B, int L1max, int L2max,
                        float gap_open, float gap_ext, float temp, float* value, void* workspace,
                        size_t workspace_bytes, void* stream) {
  return launch_value<3>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, value, workspace,
                         workspace_bytes, stream);
}

int swb_sw_value(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                 float temp, float* value, void* workspace, size_t workspace_bytes, void* stream) {
  return launch_value<1>(scores, lengths, B, L1max, L2max, gap, 0.f, temp, value, workspace,
                         workspace_bytes, stream);
}

size_t swb_sw_workspace_bytes(int B, int L1max, int L2max) {
  if (B <= 0) return 0;
  return std::max({layout_for<1, 2>(B, L1max, L2max).total, layout_for<1, 4>(B, L1max, L2max).total,
                   layout_for<1, 8>(B, L1max, L2max).total});
}

int swb_sw_affine_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, float* value, float* map,
                          float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                          size_t workspace_bytes, void* stream, const swb_options* opt) {
  return launch_padded<3>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, value, map,
                          grad_open, grad_ext, grad_temp, workspace, workspace_bytes, stream, opt);
}

int swb_sw_affine_forward_static(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp,
                                 float* value, float* map, float* grad_open, float* grad_ext,
                                 float* grad_temp, void* stream, const swb_options* opt) {
  // size check first: an oversize batch is rejected before any CUDA call
  const int r = pick_r(opt, L2max, lin_eligible<3, 0>(gap_open, gap_ext, temp, opt));
  if (B > 0 && L1max >= 0 && L2max >= 0 && valid_r_local(r)) {
    const size_t need = r == 2 ? layout_for<3, 2>(B, L1max, L2max).total
                               : (r == 4 ? layout_for<3, 4>(B, L1max, L2max).total
                                         : layout_for<3, 8>(B, L1max, L2max).total);
    if (need > (size_t)SWB_STATIC_SCRATCH_BYTES) return SWB_ERR_WORKSPACE;
  }
  void* ws = nullptr;
  if (B > 0) {
    const int rc = static_scratch(&ws);
    if (rc != SWB_OK) return rc;
  }
  // the shared launch path resets the counters, status word and completion
  // counts to 0 and the cross-band buffers to the sentinel on every call
  return launch_padded<3>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, value, map,
                          grad_open, grad_ext, grad_temp, ws, (size_t)SWB_STATIC_SCRATCH_BYTES,
                          stream, opt);
}

int swb_sw_forward(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                   float temp, float* value, float* map, float* grad_gap, float* grad_temp,
                   void* workspace, size_t workspace_bytes, void* stream,
                   const swb_options* opt) {
  return launch_padded<1>(scores, lengths, B, L1max, L2max, gap, 0.f, temp, value, map, grad_gap,
                          nullptr, grad_temp, workspace, workspace_bytes, stream, opt);
}

size_t swb_nw_workspace_bytes(int B, int L1max, int L2max) { return swb_sw_workspace_bytes(B, L1max, L2max); }

int swb_nw_forward(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                   float temp, float* value, float* map, float* grad_gap, float* grad_temp,
                   void* workspace, size_t workspace_bytes, void* stream,
                   const swb_options* opt) {
  return launch_padded<1, 1>(scores, lengths, B, L1max, L2max, gap, 0.f, temp, value, map,
                                grad_gap, nullptr, grad_temp, workspace, workspace_bytes, stream,
                                opt);
}

size_t swb_nw_affine_workspace_bytes(int B, int L1max, int L2max) {
  if (B <= 0) return 0;
  return std::max(layout_for<3, 2, 1>(B, L1max, L2max).total,
                  layout_for<3, 4, 1>(B, L1max, L2max).total);
}

int swb_nw_affine_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, float* value, float* map,
                          float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                          size_t workspace_bytes, void* stream, const swb_options* opt) {
  return launch_padded<3, 1>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, value,
                                map, grad_open, grad_ext, grad_temp, workspace, workspace_bytes,
                                stream, opt);
}

size_t swb_nw_affine_value_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? value_workspace<3, 1>(B, L1max, L2max) : 0;
}

int swb_nw_affine_value(const float* scores, const int* lengths, int B, int L1max, int L2max,
                        float gap_open, float gap_ext, float temp, float* value, void* workspace,
                        size_t workspace_bytes, void* stream) {
  return launch_value<3, 1>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, value,
                               workspace, workspace_bytes, stream);
}

int swb_nw_affine_ragged(const float* scores, const void* host_plan, const void* dev_plan,
                         float gap_open, float gap_ext, float temp, float* value, float* map,
                         float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                         size_t workspace_bytes, void* stream, const swb_options* opt) {
  return launch_ragged<3, 1>(scores, host_plan, dev_plan, gap_open, gap_ext, temp, value, map,
                                grad_open, grad_ext, grad_temp, workspace, workspace_bytes, stream,
                                opt);
}

int swb_nw_affine_ragged_value(const float* scores, const void* host_plan, const void* dev_plan,
                               float gap_open, float gap_ext, float temp, float* value,
                               void* workspace, size_t workspace_bytes, void* stream) {
  return launch_ragged<3, 1>(scores, host_plan, dev_plan, gap_open, gap_ext, temp, value,
                                nullptr, nullptr, nullptr, nullptr, workspace, workspace_bytes,
                                stream, nullptr, true);
}

size_t swb_sv_affine_workspace_bytes(int B, int L1max, int L2max) {
  if (B <= 0) return 0;
  return std::max(layout_for<3, 2, 2>(B, L1max, L2max).total,
                  layout_for<3, 4, 2>(B, L1max, L2max).total);
}

int swb_sv_affine_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, float* value, float* map,
                          float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                          size_t workspace_bytes, void* stream, const swb_options* opt) {
  return launch_padded<3, 2>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, value, map,
                             grad_open, grad_ext, grad_temp, workspace, workspace_bytes, stream,
                             opt);
}

size_t swb_sv_affine_value_workspace_bytes(int B, int L1max, int L2max) {
  return B > 0 ? value_workspace<3, 2>(B, L1max, L2max) : 0;
}

int swb_sv_affine_value(const float* scores, const int* lengths, int B, int L1max, int L2max,
                        float gap_open, float gap_ext, float temp, float* value, void* workspace,
                        size_t workspace_bytes, void* stream) {
  return launch_value<3, 2>(scores, lengths, B, L1max, L2max, gap_open, gap_ext, temp, value,
                            workspace, workspace_bytes, stream);
}

int swb_sv_affine_ragged(const float* scores, const void* host_plan, const void* dev_plan,
                         float gap_open, float gap_ext, float temp, float* value, float* map,
                         float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                         size_t workspace_bytes, void* stream, const swb_options* opt) {
  return launch_ragged<3, 2>(scores, host_plan, dev_plan, gap_open, gap_ext, temp, value, map,
                             grad_open, grad_ext, grad_temp, workspace, workspace_bytes, stream, opt);
}

int swb_sv_affine_ragged_value(const float* scores, const void* host_plan, const void* dev_plan,
                               float gap_open, float gap_ext, float temp, float* value,
                               void* workspace, size_t workspace_bytes, void* stream) {
  return launch_ragged<3, 2>(scores, host_plan, dev_plan, gap_open, gap_ext, temp, value, nullptr,
                             nullptr, nullptr, nullptr, workspace, workspace_bytes, stream, nullptr,
                             true);
}

size_t swb_nw_value_workspace_bytes(int B, int L1max, int L2max) {
  return swb_sw_value_workspace_bytes(B, L1max, L2max);
}

int swb_nw_value(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                 float temp, float* value, void* workspace, size_t workspace_bytes, void* stream) {
  return launch_value<1, 1>(scores, lengths, B, L1max, L2max, gap, 0.f, temp, value, workspace,
                               workspace_bytes, stream);
}

int swb_ragged_plan(int family, int cols_per_lane, const int* lengths, const long long* offsets,
                    int B, void* plan, size_t plan_capacity, size_t* plan_bytes,
                    size_t* workspace_bytes) {
  const int R = cols_per_lane ? cols_per_lane : kDefaultR;
  // family: 1 linear, 3 affine, 2 global linear, 4 global affine, 5 Saigo-Vert
  const bool local = family == 1 || family == 3;
  if ((family < 1 || family > 5) || !(local ? valid_r_local(R) : valid_r(R)) || B < 0 ||
      (B > 0 && (!lengths || !offsets)))
    return SWB_ERR_ARG;
  const int ns = (family >= 3) ? 3 : 1;
  const int NE = 2 * ns;
  const int NP = family >= 4 ? swb::push_fields<3, 1>()
                             : (ns == 3 ? swb::push_fields<3, 0>() : swb::push_fields<1, 0>());
  const int CKRS = ns == 3 ? (R == 2 ? swb::ck_record_floats<3, 2>()
                                     : (R == 4 ? swb::ck_record_floats<3, 4>() : swb::ck_record_floats<3, 8>()))
                           : (R == 2 ? swb::ck_record_floats<1, 2>()
                                     : (R == 4 ? swb::ck_record_floats<1, 4>() : swb::ck_record_floats<1, 8>()));
  // validate the packing: row pitch round4(L2), offsets multiples of 4 floats
  long long ntasks = 0;
  for (int b = 0; b < B; ++b) {
    const long long L1 = lengths[2 * b], L2 = lengths[2 * b + 1];
    if (L1 < 0 || L2 < 0 || L1 > (1 << 24) || L2 > (1 << 24)) return SWB_ERR_ARG;
    const long long pitch = (L2 + 3) & ~3LL;
    if (offsets[b] < 0 || (offsets[b] & 3) || offsets[b + 1] - offsets[b] < L1 * pitch)
      return SWB_ERR_ARG;
    long long nb = (L2 + 32 * R - 1) / (32 * R);
    ntasks += nb < 1 ? 1 : nb;
  }
  const size_t need = plan_bytes_for(B, ntasks);
  if (plan_bytes) *plan_bytes = need;
  if (!plan) {  // size query
    if (workspace_bytes) *workspace_bytes = 0;
    if (!plan_bytes) return SWB_ERR_ARG;
    // fall through to compute the workspace size without writing a plan
  } else if (plan_capacity < need) {
    return SWB_ERR_ARG;
  }
  // longest-chain-first order.  A band task lasts L1 + 31 wavefront steps
  // whatever its width, and band b+1 of a pair trails band b by about 31
  // steps, so a pair's critical path is L1 + 31 * nb steps: queue pairs by
  // that (then by cells, then by index), their bands in order.
  std::vector<int> order(B);
  for (int b = 0; b < B; ++b) order[b] = b;
  auto chain = [&](int b) {
    const long long L1 = lengths[2 * b], L2 = lengths[2 * b + 1];
    if (L1 <= 0 || L2 <= 0) return 0LL;
    return L1 + (long long)kChainLag * ((L2 + 32 * R - 1) / (32 * R));
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const long long cx = chain(x), cy = chain(y);
    if (cx != cy) return cx > cy;
    return (long long)lengths[2 * x] * lengths[2 * x + 1] >
           (long long)lengths[2 * y] * lengths[2 * y + 1];
  });
  long long* h = static_cast<long long*>(plan);
  long long* pw = plan ? h + HW_WORDS : nullptr;
  int* tk = plan ? reinterpret_cast<int*>(h + HW_WORDS + (size_t)B * swb::PLAN_PAIR_WORDS)
                 : nullptr;
  size_t slots = 0, ck = 0, ed = 0, bp = 0;
  long long t = 0;
  for (int b : order) {
    const long long L1 = lengths[2 * b], L2 = lengths[2 * b + 1];
    long long nb = (L2 + 32 * R - 1) / (32 * R);
    if (nb < 1) nb = 1;
    if (pw) {
      long long* q = pw + (size_t)b * swb::PLAN_PAIR_WORDS;
      q[swb::PW_SCORE_OFF] = offsets[b];
      q[swb::PW_L1] = L1;
      q[swb::PW_L2] = L2;
      q[swb::PW_SLOT0] = (long long)slots;
      q[swb::PW_NB] = nb;
      q[swb::PW_CK0] = (long long)ck;
      q[swb::PW_EDGE0] = (long long)ed;
      q[swb::PW_BP0] = (long long)bp;
      for (long long j = 0; j < nb; ++j) { tk[2 * t] = b; tk[2 * t + 1] = (int)j; ++t; }
    }
    slots += nb;
    ck += (size_t)nb * chunks_for(L1) * CKRS;
    ed += (size_t)nb * NE * L1;
    bp += (size_t)nb * NP * (L1 + 1);
  }
  const Layout l = layout_sizes(B, slots, ed, bp, ck);
  if (workspace_bytes) *workspace_bytes = B > 0 ? l.total : 0;
  if (pw) {
    h[HW_MAGIC] = kPlanMagic; h[HW_B] = B; h[HW_NTASKS] = ntasks; h[HW_SLOTS] = (long long)slots;
    h[HW_CK] = (long long)ck; h[HW_EDGE] = (long long)ed; h[HW_BP] = (long long)bp;
    h[HW_FAMILY] = family | (R << 8); h[HW_MAP_ELEMS] = B > 0 ? offsets[B] : 0; h[9] = 0;
  }
  return SWB_OK;
}

int swb_sw_affine_ragged(const float* scores, const void* host_plan, const void* dev_plan,
                         float gap_open, float gap_ext, float temp, float* value, float* map,
                         float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                         size_t workspace_bytes, void* stream, const swb_options* opt) {
  return launch_ragged<3>(scores, host_plan, dev_plan, gap_open, gap_ext, temp, value, map,
                          grad_open, grad_ext, grad_temp, workspace, workspace_bytes, stream, opt);
}

int swb_sw_affine_ragged_value(const float* scores, const void* host_plan, const void* dev_plan,
                               float gap_open, float gap_ext, float temp, float* value,
                               void* workspace, size_t workspace_bytes, void* stream) {
  return launch_ragged<3>(scores, host_plan, dev_plan, gap_open, gap_ext, temp, value, nullptr,
                          nullptr, nullptr, nullptr, workspace, workspace_bytes, stream, nullptr, true);
}

int swb_sw_ragged_value(const float* scores, const void* host_plan, const void* dev_plan, float gap,
                        float temp, float* value, void* workspace, size_t workspace_bytes,
                        void* stream) {
  return launch_ragged<1>(scores, host_plan, dev_plan, gap, 0.f, temp, value, nullptr, nullptr,
                          nullptr, nullptr, workspace, workspace_bytes, stream, nullptr, true);
}

int swb_sw_ragged(const float* scores, const void* host_plan, const void* dev_plan, float gap,
                  float temp, float* value, float* map, float* grad_gap, float* grad_temp,
                  void* workspace, size_t workspace_bytes, void* stream,
                  const swb_options* opt) {
  return launch_ragged<1>(scores, host_plan, dev_plan, gap, 0.f, temp, value, map, grad_gap,
                          nullptr, grad_temp, workspace, workspace_bytes, stream, opt);
}

int swb_nw_ragged(const float* scores, const void* host_plan, const void* dev_plan, float gap,
                  float temp, float* value, float* map, float* grad_gap, float* grad_temp,
                  void* workspace, size_t workspace_bytes, void* stream,
                  const swb_options* opt) {
  return launch_ragged<1, 1>(scores, host_plan, dev_plan, gap, 0.f, temp, value, map, grad_gap,
                                nullptr, grad_temp, workspace, workspace_bytes, stream, opt);
}

int swb_nw_ragged_value(const float* scores, const void* host_plan, const void* dev_plan, float gap,
                        float temp, float* value, void* workspace, size_t workspace_bytes,
                        void* stream) {
  return launch_ragged<1, 1>(scores, host_plan, dev_plan, gap, 0.f, temp, value, nullptr,
                                nullptr, nullptr, nullptr, workspace, workspace_bytes, stream,
                                nullptr, true);
}

int swb_static_read_status(void* stream, unsigned* status) {
  if (!status) return SWB_ERR_ARG;
  void* ws = nullptr;
  const int rc = static_scratch(&ws);
  if (rc != SWB_OK) return rc;
  return swb_read_status(ws, stream, status);
}

int swb_read_status(const void* workspace, void* stream, unsigned* status) {
  if (!workspace || !status) return SWB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const unsigned* p = reinterpret_cast<const unsigned*>(workspace) + 4;
  if (cudaMemcpyAsync(status, p, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return SWB_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return SWB_ERR_CUDA;
  return SWB_OK;
}

const char* swb_error_string(int code) {
  switch (code) {
    case SWB_OK: return "ok";
    case SWB_ERR_ARG: return "invalid argument";
    case SWB_ERR_WORKSPACE: return "workspace missing or too small";
    case SWB_ERR_CUDA: return "CUDA error";
    default: return "unknown error";
  }
}

int swb_abi_version(void) { return SWB_ABI_VERSION; }

int swb_mufu_probe(float* scratch, int blocks, int iters, void* stream) {
  if (!scratch || blocks <= 0 || iters <= 0) return SWB_ERR_ARG;
  swb::mufu_probe_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(scratch, iters);
  return cudaPeekAtLastError() == cudaSuccess ? SWB_OK : SWB_ERR_CUDA;
}

}  // extern "C"
