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
#include <mutex>
#include <cuda_runtime.h>

#include "sw_kernels.cu"
#include "sw_probe.cuh"
#include "../../include/orihime_b200.h"

namespace {

using swb::Args;

constexpr int kR = 4;                 // columns per lane
constexpr int kWarpsFwd = 4;          // forward CTA: 4 independent warps
constexpr int kWarpsBwd = 1;          // adjoint CTA: 1 warp (shared memory bound)
constexpr size_t kAlign = 256;

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

template <int NS> constexpr int np() { return swb::Dims<NS, kR>::NP; }
template <int NS> constexpr int ckf() { return swb::Dims<NS, kR>::CKF; }
template <int NS> constexpr int ne() { return swb::Dims<NS, kR>::NE; }

struct Layout {
  int nb, nchunks;
  size_t off_hdr, off_pair_done, off_part, off_gpart, off_sent, off_edge, off_bpush, off_ckpt;
  size_t sent_bytes;   // sentinel-initialised span (never_written + edge + bpush)
  size_t total;
};

template <int NS>
Layout layout_for(long long B, long long L1m, long long L2m) {
  Layout l{};
  l.nb = (int)((L2m + 32 * kR - 1) / (32 * kR));
  if (l.nb < 1) l.nb = 1;
  l.nchunks = (int)((L1m + 31 + swb::C_STEPS - 1) / swb::C_STEPS);  // = band_chunks(L1m)
  const size_t slots = (size_t)B * l.nb;
  size_t o = 0;
  l.off_hdr = o;        o = align_up(o + 64);
  l.off_pair_done = o;  o = align_up(o + sizeof(unsigned) * (size_t)B);
  l.off_part = o;       o = align_up(o + sizeof(float) * 2 * slots);
  l.off_gpart = o;      o = align_up(o + sizeof(float) * 4 * slots);
  l.off_sent = o;       o = o + kAlign;   // never_written word lives here
  l.off_edge = o;       o = align_up(o + sizeof(float) * slots * ne<NS>() * (size_t)L1m);
  l.off_bpush = o;      o = align_up(o + sizeof(float) * slots * np<NS>() * (size_t)(L1m + 1));
  l.sent_bytes = o - l.off_sent;
  l.off_ckpt = o;       o = align_up(o + sizeof(float) * slots * l.nchunks * ckf<NS>() * 32);
  l.total = o;
  return l;
}

struct DevInfo {
  int sms = 0;
  int occ_fwd[2] = {0, 0};   // [linear, affine]
  int occ_bwd[2] = {0, 0};
  bool ready = false;
};
DevInfo g_dev[64];
std::mutex g_mu;

template <int NS>
size_t bwd_smem() { return (size_t)kWarpsBwd * swb::bwd_smem_floats<NS, kR>() * sizeof(float); }

int dev_info(DevInfo** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SWB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  DevInfo& d = g_dev[dev];
  if (!d.ready) {
    if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return SWB_ERR_CUDA;
    if (cudaFuncSetAttribute(swb::bwd_kernel<3, kR, kWarpsBwd>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bwd_smem<3>()) != cudaSuccess)
      return SWB_ERR_CUDA;
    if (cudaFuncSetAttribute(swb::bwd_kernel<1, kR, kWarpsBwd>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bwd_smem<1>()) != cudaSuccess)
      return SWB_ERR_CUDA;
    const int tf = 32 * kWarpsFwd, tb = 32 * kWarpsBwd;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_fwd[0], swb::fwd_kernel<1, kR>, tf, 0) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_fwd[1], swb::fwd_kernel<3, kR>, tf, 0) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_bwd[0], swb::bwd_kernel<1, kR, kWarpsBwd>, tb,
                                                      bwd_smem<1>()) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_bwd[1], swb::bwd_kernel<3, kR, kWarpsBwd>, tb,
                                                      bwd_smem<3>()))
      return SWB_ERR_CUDA;
    d.ready = true;
  }
  *out = &d;
  return SWB_OK;
}

template <int NS>
int launch(const float* scores, const int* lengths, const long long* offsets, const int* order,
           int layout, int B, int L1m, int L2m, float go, float ge, float T, float* value,
           float* map, size_t map_elems, float* g_open, float* g_ext, float* g_T, void* ws,
           size_t ws_bytes, void* stream_v, const swb_options* opt) {
  if (B < 0 || L1m < 0 || L2m < 0) return SWB_ERR_ARG;
  if (!(T > 0.f) || !(T < INFINITY)) return SWB_ERR_ARG;
  if (B == 0) return SWB_OK;
  if (!value || !g_open || !g_T || (NS == 3 && !g_ext)) return SWB_ERR_ARG;
  if (map_elems > 0 && (!scores || !map)) return SWB_ERR_ARG;
  if (layout == 1 && (!offsets || !lengths)) return SWB_ERR_ARG;
  const Layout l = layout_for<NS>(B, L1m, L2m);
  if (!ws || ws_bytes < l.total) return SWB_ERR_WORKSPACE;
  DevInfo* d = nullptr;
  int rc = dev_info(&d);
  if (rc != SWB_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream_v);
  char* w = static_cast<char*>(ws);

  Args a{};
  a.scores = scores; a.map = map; a.lengths = lengths; a.offsets = offsets; a.order = order;
  a.B = B; a.Lmax1 = L1m; a.Lmax2 = L2m; a.layout = layout;
  a.go = go; a.ge = ge; a.T = T; a.k = 1.4426950408889634f / T;
  a.nb = l.nb; a.nchunks = l.nchunks;
  a.value = value; a.g_open = g_open; a.g_ext = g_ext; a.g_T = g_T;
  a.counters = reinterpret_cast<unsigned*>(w + l.off_hdr);
  a.status = a.counters + 4;
  a.pair_done = reinterpret_cast<unsigned*>(w + l.off_pair_done);
  a.part = reinterpret_cast<float*>(w + l.off_part);
  a.gpart = reinterpret_cast<float*>(w + l.off_gpart);
  a.never_written = reinterpret_cast<float*>(w + l.off_sent);
  a.edge = reinterpret_cast<float*>(w + l.off_edge);
  a.bpush = reinterpret_cast<float*>(w + l.off_bpush);
  a.ckpt = reinterpret_cast<float*>(w + l.off_ckpt);
  a.spin_limit_ns = (opt && opt->spin_limit_ns) ? opt->spin_limit_ns : 20ull * 1000000000ull;
  a.fault_inject = opt ? opt->fault_inject : 0;

  // per-call resets: counters, status and completion counts to 0, cross-band
  // buffers to the NaN sentinel, the map to 0 (cells outside lengths stay 0)
  if (cudaMemsetAsync(w, 0, l.off_part, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (cudaMemsetAsync(w + l.off_sent, 0xff, l.sent_bytes, st) != cudaSuccess) return SWB_ERR_CUDA;
  if (map_elems > 0 && cudaMemsetAsync(map, 0, map_elems * sizeof(float), st) != cudaSuccess)
    return SWB_ERR_CUDA;

  const long long ntasks = (long long)B * l.nb;
  const int cta_cap_f = d->sms * (d->occ_fwd[NS == 3] > 0 ? d->occ_fwd[NS == 3] : 1);
  const int cta_cap_b = d->sms * (d->occ_bwd[NS == 3] > 0 ? d->occ_bwd[NS == 3] : 1);
  const long long need_f = (ntasks + kWarpsFwd - 1) / kWarpsFwd;
  const long long need_b = (ntasks + kWarpsBwd - 1) / kWarpsBwd;
  int grid_f = (int)(need_f < cta_cap_f ? need_f : cta_cap_f);
  int grid_b = (int)(need_b < cta_cap_b ? need_b : cta_cap_b);
  if (opt && opt->max_ctas > 0) {
    if (grid_f > opt->max_ctas) grid_f = opt->max_ctas;
    if (grid_b > opt->max_ctas) grid_b = opt->max_ctas;
  }
  swb::fwd_kernel<NS, kR><<<grid_f, 32 * kWarpsFwd, 0, st>>>(a);
  if (cudaPeekAtLastError() != cudaSuccess) return SWB_ERR_CUDA;
  swb::bwd_kernel<NS, kR, kWarpsBwd><<<grid_b, 32 * kWarpsBwd, bwd_smem<NS>(), st>>>(a);
  if (cudaPeekAtLastError() != cudaSuccess) return SWB_ERR_CUDA;
  return SWB_OK;
}

}  // namespace

extern "C" {

size_t swb_sw_affine_workspace_bytes(int B, int L1max, int L2max) {
  if (B <= 0) return 0;
  return layout_for<3>(B, L1max, L2max).total;
}

size_t swb_sw_workspace_bytes(int B, int L1max, int L2max) {
  if (B <= 0) return 0;
  return layout_for<1>(B, L1max, L2max).total;
}

int swb_sw_affine_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, float* value, float* map,
                          float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                          size_t workspace_bytes, void* stream, const swb_options* opt) {
  return launch<3>(scores, lengths, nullptr, nullptr, 0, B, L1max, L2max, gap_open, gap_ext, temp,
                   value, map, (size_t)B * L1max * L2max, grad_open, grad_ext, grad_temp,
                   workspace, workspace_bytes, stream, opt);
}

int swb_sw_forward(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                   float temp, float* value, float* map, float* grad_gap, float* grad_temp,
                   void* workspace, size_t workspace_bytes, void* stream,
                   const swb_options* opt) {
  return launch<1>(scores, lengths, nullptr, nullptr, 0, B, L1max, L2max, gap, 0.f, temp, value,
                   map, (size_t)B * L1max * L2max, grad_gap, nullptr, grad_temp, workspace,
                   workspace_bytes, stream, opt);
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
