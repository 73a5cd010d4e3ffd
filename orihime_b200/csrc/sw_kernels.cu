// Soft Smith-Waterman forward / adjoint kernels (sm_100a).  Layout and
// protocol are described in sw_kernels.cuh.  Compiled as part of sw_capi.cu.
//
// Reference semantics restated here (megure-labs/orihime):
//   affine  src/sw_affine/kernels_gpu.cu:274-347 (forward cell),
//           :350-410 (partition incl. M[0,0] = 0), :413-573 (adjoint),
//           :576-616 (dS/dT);
//   linear  src/sw/kernels_gpu.cu:175-239, :242-299, :325-460, :463-497.
// In the scaled domain x' = x*log2(e)/T the reference's
//   LSE_T(v) = m + T*log(sum exp((v-m)/T))
// becomes m' + lg2(sum ex2(v'-m')), and the softmax weight of a predecessor
// is its term ex2(v'-m') divided by the sum, which is what the adjoint uses.
#include "sw_kernels.cuh"

namespace swb {

// ---------------------------------------------------------------------------
// scalar helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ float ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float lg2(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// 1/x for x in [1, 4]: MUFU approximation refined by one Newton-Raphson step
// (y' = y + y (1 - x y)), which leaves an error of about half an ulp with no
// systematic sign; the adjoint's per-cell weight normalisation relies on that.
__device__ __forceinline__ float recip(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return fmaf(y, fmaf(-x, y, 1.f), y);
}

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Strong (L1-bypassing) load used for cross-warp polling.
__device__ __forceinline__ float ld_poll(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool is_sentinel(float v) {
  return __float_as_uint(v) == SENTINEL_BITS;
}

// Kahan-compensated accumulator.
struct KSum {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

#ifndef SWB_POLL_SLEEP
#define SWB_POLL_SLEEP 128
#endif
// A bounded wait that expires marks its pair: bit 31 of the pair's
// completion word (zeroed with the workspace header at every call).  The
// pair's finisher then writes NaN into its value and gradients (second-order
// ops: into its output map), so a timeout shows in the results without any
// host synchronisation; the status word records it as well.
constexpr unsigned PAIR_TIMEOUT = 0x80000000u;

__device__ __forceinline__ void mark_timeout(unsigned* status, unsigned* flag) {
  atomicOr(status, ERR_WAIT_TIMEOUT);
  if (flag) atomicOr(flag, PAIR_TIMEOUT);
}

// Bounded wait until none of x.v[0..N) is the sentinel, x.v[f] read from
// base[f * stride].  Every round re-reads all missing fields together, so their
// load latencies overlap.  The fields travel by value (the caller's values
// need no memory address).  On timeout it records the error (status word and
// the pair's flag) and substitutes NEG for the missing fields f < NSV, 0 for
// the others.
template <int N> struct FieldVec { float v[N]; };
template <int N, int NSV>
__device__ __noinline__ FieldVec<N> poll_fields_v(FieldVec<N> x, const float* base, size_t stride,
                                                  uint64_t deadline, unsigned* status,
                                                  unsigned* flag) {
  while (true) {
    bool miss = false;
#pragma unroll
    for (int f = 0; f < N; ++f)
      if (is_sentinel(x.v[f])) x.v[f] = ld_poll(base + f * stride);
#pragma unroll
    for (int f = 0; f < N; ++f) miss |= is_sentinel(x.v[f]);
    if (!miss) return x;
    if (gtimer() > deadline) {
      mark_timeout(status, flag);
#pragma unroll
      for (int f = 0; f < N; ++f)
        if (is_sentinel(x.v[f])) x.v[f] = f < NSV ? NEG : 0.f;
      return x;
    }
    __nanosleep(SWB_POLL_SLEEP);
  }
}

// Bounded wait until *p is not the sentinel.  On timeout records the error
// (status word and the pair's flag) and returns `fallback`.
__device__ __noinline__ float poll_value(const float* p, float v, uint64_t deadline,
                                         unsigned* status, unsigned* flag, float fallback) {
  while (is_sentinel(v)) {
    if (gtimer() > deadline) {
      mark_timeout(status, flag);
      return fallback;
    }
    __nanosleep(SWB_POLL_SLEEP);
    v = ld_poll(p);
  }
  return v;
}

// ---------------------------------------------------------------------------
// pair descriptors
// ---------------------------------------------------------------------------

struct Pair {
  const float* s;   // score row 0
  float* m;         // map row 0
  int L1, L2, ld;
  bool vec;         // row starts are 16-byte aligned and ld % 4 == 0
};

// Where a band task lives: its pair, band, and the pair's workspace slices.
struct Place {
  int p, band, nb;          // pair, band, bands of the pair
  size_t slot0;             // slot of band 0 (partials, completion count)
  size_t ck0, ckb;          // checkpoint floats: band 0 offset, per-band stride
  size_t ed0, edb;          // edge floats
  size_t bp0, bpb;          // push floats
  int Lm;                   // row stride of the edge / push buffers (>= L1)
  Pair pr;
};

// Push channels crossing a lane or band edge backward: local affine 5 (left
// M, D; diagonal M, I, D), global affine 6 (left M, I, D; diagonal M, I, D),
// linear 2 (left, diagonal); the first push_left of them are left pushes.
// Model variants of the band kernels (template argument GM): 0 the local
// alignments (soft Smith-Waterman), 1 the global ones (soft Needleman-
// Wunsch), 2 Saigo-Vert (local, affine states with D <- I, only M ends).
// Global and Saigo-Vert affine take six push channels (D pushes to M, I, D).
template <int NS, int GM> __host__ __device__ constexpr int push_channels() {
  return NS == 3 ? (GM ? 6 : 5) : 2;
}
template <int NS, int GM> __host__ __device__ constexpr int push_left() {
  return NS == 3 ? (GM ? 3 : 2) : 1;
}
// Floats per row of a band's push buffer in the workspace: the push channels
// of the log-domain adjoint, or the 3 fields (beta_D or beta, t, frame) the
// linear-domain adjoint of the local models passes, whichever is more.
template <int NS, int GM> __host__ __device__ constexpr int push_fields() {
  return push_channels<NS, GM>() > 3 ? push_channels<NS, GM>() : 3;
}
// Floats of one checkpoint chunk record: the larger of the log-domain record
// (double-float values) and the linear-domain one (sw_lin.cu), so one
// workspace layout serves both kernel families.
template <int NS, int R> __host__ __device__ constexpr int ck_record_floats() {
  constexpr int lg = (2 * NS * R + 2 * NS) * 32 + 4;
  constexpr int lv = ((NS * R + NS + 3 + 3) / 4 * 4) * 32 + 4;
  return lg > lv ? lg : lv;
}

template <int NS, int R, int GM = 0>
__device__ __forceinline__ Place place_of(const Args& a, int task, bool reverse_band) {
  constexpr int NE = 2 * NS, NP = push_fields<NS, GM>(), CKRS = ck_record_floats<NS, R>();
  Place w;
  Pair& r = w.pr;
  if (a.layout == 0) {
    int p = task / a.nb;
    const int j = task - p * a.nb;
    if (a.order) p = a.order[p];
    w.p = p;
    w.nb = a.nb;
    w.band = reverse_band ? a.nb - 1 - j : j;
    w.slot0 = (size_t)p * a.nb;
    w.Lm = a.Lmax1;
    w.ckb = a.ck_band_floats ? a.ck_band_floats : (size_t)a.nchunks * CKRS;
    w.edb = (size_t)NE * a.Lmax1;
    w.bpb = (size_t)NP * (a.Lmax1 + 1);
    w.ck0 = w.slot0 * w.ckb;
    w.ed0 = w.slot0 * w.edb;
    w.bp0 = w.slot0 * w.bpb;
    const size_t base = (size_t)p * a.Lmax1 * a.Lmax2;
    r.s = a.scores + base;
    r.m = a.map + base;
    r.ld = a.Lmax2;
    if (a.lengths) {  // never index outside the padded slab
      r.L1 = min(max(a.lengths[2 * p], 0), a.Lmax1);
      r.L2 = min(max(a.lengths[2 * p + 1], 0), a.Lmax2);
    } else {
      r.L1 = a.Lmax1;
      r.L2 = a.Lmax2;
    }
  } else {
    const int p = a.plan_tasks[2 * task];
    const int j = a.plan_tasks[2 * task + 1];
    const long long* q = a.plan_pairs + (size_t)p * PLAN_PAIR_WORDS;
    w.p = p;
    w.nb = (int)q[PW_NB];
    w.band = reverse_band ? w.nb - 1 - j : j;
    w.slot0 = (size_t)q[PW_SLOT0];
    r.L1 = (int)q[PW_L1];
    r.L2 = (int)q[PW_L2];
    r.ld = (r.L2 + 3) & ~3;
    w.Lm = r.L1;
    const int nch = (r.L1 + 31 + C_STEPS - 1) / C_STEPS;
    w.ckb = (size_t)nch * CKRS;
    w.edb = (size_t)NE * r.L1;
    w.bpb = (size_t)NP * (r.L1 + 1);
    w.ck0 = (size_t)q[PW_CK0];
    w.ed0 = (size_t)q[PW_EDGE0];
    w.bp0 = (size_t)q[PW_BP0];
    r.s = a.scores + q[PW_SCORE_OFF];
    r.m = a.map + q[PW_SCORE_OFF];
  }
  r.vec = ((r.ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(r.s) & 15) == 0) &&
          ((reinterpret_cast<uintptr_t>(r.m) & 15) == 0);
  return w;
}

// Lengths of pair p in a padded batch outside [0, padded size]: the kernels
// clamp them (so nothing is read or written out of bounds); the first band
// task of the pair marks it so its outputs come back NaN, and sets the
// status bit.  (The host range-checks lengths with the reference's messages
// before launching, except while a stream is being captured.)
__device__ __forceinline__ void check_lengths(const Args& a, const Place& w, int lane) {
  if (a.layout != 0 || !a.lengths || w.band != 0 || lane != 0) return;
  const int l1 = a.lengths[2 * w.p], l2 = a.lengths[2 * w.p + 1];
  if (l1 < 0 || l1 > a.Lmax1 || l2 < 0 || l2 > a.Lmax2) {
    atomicOr(a.status, ERR_BAD_LENGTHS);
    atomicOr(a.pair_done + w.p, PAIR_TIMEOUT);
  }
}

template <int R>
__device__ __forceinline__ void load_row(const Pair& pr, int i, int jl, bool ok, float (&o)[R]) {
  // i: 1-based row; jl: 0-based first column of the lane
  if (!ok) {
#pragma unroll
    for (int c = 0; c < R; ++c) o[c] = 0.f;
    return;
  }
  const float* src = pr.s + (size_t)(i - 1) * pr.ld + jl;
  if (R == 8 && pr.vec && jl + 8 <= pr.L2) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(src));
    const float4 u = __ldg(reinterpret_cast<const float4*>(src) + 1);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    o[R > 4 ? 4 : 0] = u.x; o[R > 5 ? 5 : 0] = u.y; o[R > 6 ? 6 : 0] = u.z; o[R > 7 ? 7 : 0] = u.w;
  } else if (R == 4 && pr.vec && jl + 4 <= pr.L2) {
    float4 v = __ldg(reinterpret_cast<const float4*>(src));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  } else if (R == 2 && pr.vec && jl + 2 <= pr.L2) {
    float2 v = __ldg(reinterpret_cast<const float2*>(src));
    o[0] = v.x; o[1] = v.y;
  } else {
#pragma unroll
    for (int c = 0; c < R; ++c) o[c] = (jl + c < pr.L2) ? __ldg(src + c) : 0.f;
  }
}

// Writes row i of the map for the lane's columns; columns in [L2, ld) (row
// pitch padding) receive 0, so a packed map needs no separate clearing.
template <int R>
__device__ __forceinline__ void store_row(const Pair& pr, int i, int jl, const float (&v)[R]) {
  float* dst = pr.m + (size_t)(i - 1) * pr.ld + jl;
  if (R == 8 && pr.vec && jl + 8 <= pr.ld) {
    float z[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) z[c] = (c < R && jl + c < pr.L2) ? v[c < R ? c : 0] : 0.f;
    reinterpret_cast<float4*>(dst)[0] = make_float4(z[0], z[1], z[2], z[3]);
    reinterpret_cast<float4*>(dst)[1] = make_float4(z[4], z[5], z[6], z[7]);
  } else if (R == 4 && pr.vec && jl + 4 <= pr.ld) {
    *reinterpret_cast<float4*>(dst) = make_float4(jl + 0 < pr.L2 ? v[0] : 0.f, jl + 1 < pr.L2 ? v[1] : 0.f,
                                                  jl + 2 < pr.L2 ? v[2] : 0.f, jl + 3 < pr.L2 ? v[3] : 0.f);
  } else if (R == 2 && pr.vec && jl + 2 <= pr.ld) {
    *reinterpret_cast<float2*>(dst) = make_float2(jl + 0 < pr.L2 ? v[0] : 0.f, jl + 1 < pr.L2 ? v[1] : 0.f);
  } else {
#pragma unroll
    for (int c = 0; c < R; ++c)
      if (jl + c < pr.ld) dst[c] = (jl + c < pr.L2) ? v[c] : 0.f;
  }
}

// Values crossing a band edge forward (2*NS: hi and lo of each state), pushes
// crossing it backward (NP), checkpoint floats per lane (CKF), and
// shared-memory floats per lane per recomputed step (EW: WF adjoint fields per
// cell).
// WF: adjoint fields per cell.  affine: the weights of M's diagonal
// predecessors M, I, D, of I's upper predecessors M, I and of D's left
// predecessors M, D, the beta-init terms of M, I, D and the scaled score.
// linear: the map factor (diagonal + start weights), the diagonal, upper and
// left weights, the beta-init term and the scaled score.
template <int NS> struct Shape;
template <> struct Shape<3> { static constexpr int NP = 5, WF = 11; };
template <> struct Shape<1> { static constexpr int NP = 2, WF = 6; };

template <int NS, int R> struct Dims {
  static constexpr int NE = 2 * NS;
  static constexpr int NP = Shape<NS>::NP;
  static constexpr int CKF = 2 * NS * R + 2 * NS;   // checkpoint floats per lane (even)
  static constexpr int CKRS = CKF * 32 + 4;         // chunk record floats: checkpoint, chunk max, pad
  static constexpr int CK4 = CKF / 4;               // ... stored as CK4 float4
  static constexpr int CK2 = (CKF % 4) / 2;         // ... and CK2 (0 or 1) float2
  static constexpr int WF = Shape<NS>::WF;         // adjoint fields per cell
  static constexpr int EW = WF * R;                 // shared floats per lane per step
};

// Checkpoint of one lane: hi of its R columns per state, lo of the same, then
// hi and lo of its left neighbour per state.
template <int NS, int R>
__device__ __forceinline__ void ck_pack(const float (&ph)[NS][R], const float (&pl)[NS][R],
                                        const float (&lh)[NS], const float (&ll)[NS],
                                        float (&v)[Dims<NS, R>::CKF]) {
#pragma unroll
  for (int q = 0; q < NS; ++q) {
#pragma unroll
    for (int c = 0; c < R; ++c) { v[q * R + c] = ph[q][c]; v[NS * R + q * R + c] = pl[q][c]; }
    v[2 * NS * R + q] = lh[q];
    v[2 * NS * R + NS + q] = ll[q];
  }
}

// Checkpoint record of a chunk: CK4 groups of [lane][4] floats, then [lane][2]
// (ck_store / ck_load), then one float: the largest hi alpha of the band's
// live cells in the chunk (written by the forward at the chunk's end), and
// 3 floats of padding that keep records 16-byte aligned.
template <int NS, int R>
__device__ __forceinline__ void ck_store(float* chunk, int lane, const float (&v)[Dims<NS, R>::CKF]) {
  using D = Dims<NS, R>;
#pragma unroll
  for (int g = 0; g < D::CK4; ++g)
    reinterpret_cast<float4*>(chunk + g * 128)[lane] =
        make_float4(v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3]);
  if constexpr (D::CK2 == 1)
    reinterpret_cast<float2*>(chunk + D::CK4 * 128)[lane] =
        make_float2(v[4 * D::CK4], v[4 * D::CK4 + 1]);
}

template <int NS, int R>
__device__ __forceinline__ void ck_load(const float* chunk, int lane, float (&v)[Dims<NS, R>::CKF]) {
  using D = Dims<NS, R>;
#pragma unroll
  for (int g = 0; g < D::CK4; ++g) {
    const float4 x = reinterpret_cast<const float4*>(chunk + g * 128)[lane];
    v[4 * g] = x.x; v[4 * g + 1] = x.y; v[4 * g + 2] = x.z; v[4 * g + 3] = x.w;
  }
  if constexpr (D::CK2 == 1) {
    const float2 x = reinterpret_cast<const float2*>(chunk + D::CK4 * 128)[lane];
    v[4 * D::CK4] = x.x; v[4 * D::CK4 + 1] = x.y;
  }
}

template <int NS, int R>
__device__ __forceinline__ void ck_unpack(const float (&v)[Dims<NS, R>::CKF], float (&ph)[NS][R],
                                          float (&pl)[NS][R], float (&lh)[NS], float (&ll)[NS]) {
#pragma unroll
  for (int q = 0; q < NS; ++q) {
#pragma unroll
    for (int c = 0; c < R; ++c) { ph[q][c] = v[q * R + c]; pl[q][c] = v[NS * R + q * R + c]; }
    lh[q] = v[2 * NS * R + q];
    ll[q] = v[2 * NS * R + NS + q];
  }
}

// ---------------------------------------------------------------------------
// forward cell
// ---------------------------------------------------------------------------

// r + t as a pair when r is the large part: hi = r + t, lo = exact error
// (Fast2Sum; exact whenever |r| >= |t|, and only ever inexact at the scale of
// small values).
__device__ __forceinline__ void fast2(float r, float t, float& h, float& l) {
  h = r + t;
  l = (r - h) + t;
}

// a + b as an exact pair (TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float& h, float& l) {
  h = a + b;
  const float bb = h - a;
  l = (a - (h - bb)) + (b - bb);
}

// n * g as an exact pair (the global-alignment boundaries A[i,0] = i * gap,
// A[0,j] = j * gap in the scaled domain; n < 2^24 is exact in float).
__device__ __forceinline__ void nmul(int n, float g, float& h, float& l) {
  h = (float)n * g;
  l = fmaf((float)n, g, -h);
}

// go + n * ge as a pair (the affine global boundaries I(i,0), D(0,j) with
// n = i - 1, j - 1; scaled gaps).
__device__ __forceinline__ void gpair(int n, float go, float ge, float& h, float& l) {
  float ph, pl, th, tl;
  nmul(n, ge, ph, pl);
  two_sum(go, ph, th, tl);
  h = th;
  l = tl + pl;
}

// Row-0 values of a global alignment at column j (1-based; j = 0 is the
// origin): linear A = j * gap; affine M = [j == 0] * 0, I = NEG,
// D = go + (j - 1) ge.  (h, l) per state.
template <int NS>
__device__ __forceinline__ void row0(int j, float g0, float g1, float (&h)[NS], float (&l)[NS]) {
  if constexpr (NS == 1) {
    nmul(j, g0, h[0], l[0]);
  } else {
    h[0] = j == 0 ? 0.f : NEG; l[0] = 0.f;
    h[1] = NEG; l[1] = 0.f;
    if (j >= 1) gpair(j - 1, g0, g1, h[2], l[2]);
    else { h[2] = NEG; l[2] = 0.f; }
  }
}

// Column-0 values at row i >= 1 as an edge record (hi of each state, then lo):
// linear A = i * gap; affine M = NEG, I = go + (i - 1) ge, D = NEG.
template <int NS>
__device__ __forceinline__ void col0_edge(int i, float g0, float g1, float (&e)[2 * NS]) {
  if constexpr (NS == 1) {
    nmul(i, g0, e[0], e[1]);
  } else {
    e[0] = NEG; e[3] = 0.f;
    gpair(i - 1, g0, g1, e[1], e[4]);
    e[2] = NEG; e[5] = 0.f;
  }
}

// Adjoint fields of column c in one step's shared-memory entry `ent`, stored
// column block by column block; inside a block each field group is one
// vector per lane (lane-contiguous, so every warp access is conflict-free).
// affine (11 floats): A = (wMM, wMI, wMD, wIM), B = (wII, wDM, wDD, s), then
// the beta-init terms C = (bM0, bI0) and D = bD0; linear (6 floats):
// A = (map factor, wA, wU, wL), then s, then the beta-init term b0.  s is the
// cell's scaled score.  The init terms are written only for steps where some
// lane's init can be nonzero (fwd_cells returns that flag).
template <int NS, int R>
__device__ __forceinline__ void put_weights(float* ent, int lane, int c, float4 A, float4 B,
                                            float sc) {
  float* col = ent + c * Shape<NS>::WF * 32;
  reinterpret_cast<float4*>(col)[lane] = A;
  if constexpr (NS == 3) {
    reinterpret_cast<float4*>(col + 128)[lane] = make_float4(B.x, B.y, B.z, sc);
  } else {
    col[128 + lane] = sc;
  }
}
template <int NS, int R>
__device__ __forceinline__ void put_inits(float* ent, int lane, int c, float b0, float b1,
                                          float b2) {
  float* col = ent + c * Shape<NS>::WF * 32;
  if constexpr (NS == 3) {
    reinterpret_cast<float2*>(col + 256)[lane] = make_float2(b0, b1);
    col[320 + lane] = b2;
  } else {
    col[160 + lane] = b0;
  }
}
// Saigo-Vert: the D <- I weight lives in the slot the local affine model
// uses for D's beta-init (its only beta-init is M's, in the first of the
// init pair).
template <int R>
__device__ __forceinline__ void put_wdi(float* ent, int lane, int c, float w) {
  ent[c * Shape<3>::WF * 32 + 320 + lane] = w;
}
template <int R>
__device__ __forceinline__ float get_wdi(const float* ent, int lane, int c) {
  return ent[c * Shape<3>::WF * 32 + 320 + lane];
}
template <int R>
__device__ __forceinline__ void put_init_m(float* ent, int lane, int c, float b0) {
  reinterpret_cast<float2*>(ent + c * Shape<3>::WF * 32 + 256)[lane] = make_float2(b0, 0.f);
}

template <int NS, int R>
__device__ __forceinline__ void get_weights(const float* ent, int lane, int c, float4& A, float4& B,
                                            float& sc) {
  const float* col = ent + c * Shape<NS>::WF * 32;
  A = reinterpret_cast<const float4*>(col)[lane];
  if constexpr (NS == 3) {
    B = reinterpret_cast<const float4*>(col + 128)[lane];
    sc = B.w;
  } else {
    sc = col[128 + lane];
  }
}
template <int NS, int R>
__device__ __forceinline__ void get_inits(const float* ent, int lane, int c, float& b0, float& b1,
                                          float& b2) {
  const float* col = ent + c * Shape<NS>::WF * 32;
  if constexpr (NS == 3) {
    const float2 x = reinterpret_cast<const float2*>(col + 256)[lane];
    b0 = x.x; b1 = x.y;
    b2 = col[320 + lane];
  } else {
    b0 = col[160 + lane];
  }
}

// One step of the forward wavefront for one lane.  Inputs: previous-row pairs
// (ph, pl), left pairs of this row (lfh, lfl, already received), diag pairs of
// column 0 (dgh0, dgl0: left lane, previous row) and the scaled scores s.
// Overwrites (ph, pl) with the new row.  A lane whose row has not started yet
// gets s = NEG from its caller, which keeps every state at NEG (the row-0
// boundary); rows past the pair's end compute values nothing reads.
//
// WT (adjoint recompute): also writes each cell's adjoint fields to the
// shared-memory entry `went` (put_weights, put_inits).  The predecessor
// weights are the recurrence's own softmax terms divided by their sum, so
// they add up to 1 per cell up to rounding and the adjoint conserves
// probability flow exactly; beta-init = exp2(min(x - S, 0)) for the first
// `nlive` columns, 0 beyond.  Returns (warp-uniform) whether the inits were
// written; when not, every one of them is 0.
//
// G (global alignment, NS == 1 only): A = LSE(diag + s, up + g, left + g),
// no local start, no beta-inits.  `hold` (a row before the lane's first)
// keeps (ph, pl) at the row-0 boundary values and writes zero weights, so the
// boundary cells neither change nor push.
template <int NS, int R, bool WT = false, int GM = 0>
__device__ __forceinline__ bool fwd_cells(float (&ph)[NS][R], float (&pl)[NS][R],
                                          const float (&lfh)[NS], const float (&lfl)[NS],
                                          const float (&dgh0)[NS], const float (&dgl0)[NS],
                                          const float (&s)[R], float g0, float g1,
                                          float Sh = 0.f, float Sl = 0.f, int nlive = 0,
                                          float* went = nullptr, int lane = 0, bool hold = false) {
  constexpr bool G = GM == 1;
  [[maybe_unused]] constexpr bool SV = GM == 2;
  // G, NS == 3 (global affine): M = s + LSE(M, I, D at diag);
  // I = LSE(M + go, I + ge, D + go) from above; D = LSE(M + go, I + go, D + ge)
  // from the left.  Fields: A = (wMM, wMI, wMD, wIM), B = (wII, wDM, wDD, s),
  // and the init slots carry (wID, wDI).
  float dgh[NS], dgl[NS], lh[NS], ll[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) { dgh[q] = dgh0[q]; dgl[q] = dgl0[q]; lh[q] = lfh[q]; ll[q] = lfl[q]; }
#pragma unroll
  for (int c = 0; c < R; ++c) {
    if constexpr (NS == 3 && G) {
      const float uMh = ph[0][c], uMl = pl[0][c], uIh = ph[1][c], uIl = pl[1][c];
      const float uDh = ph[2][c], uDl = pl[2][c];
      const float r = fmaxf(fmaxf(dgh[0], dgh[1]), dgh[2]);
      const float tM = ex2((dgh[0] - r) + dgl[0]), tI = ex2((dgh[1] - r) + dgl[1]);
      const float tD = ex2((dgh[2] - r) + dgl[2]);
      const float sm = (tM + tI) + tD;
      float Mh, Ml;
      two_sum(r, s[c], Mh, Ml);
      Ml += lg2(sm);
      const float ru = fmaxf(fmaxf(uMh + g0, uIh + g1), uDh + g0);
      const float ta = ex2(((uMh - ru) + g0) + uMl), tb = ex2(((uIh - ru) + g1) + uIl);
      const float tc = ex2(((uDh - ru) + g0) + uDl);
      const float si = (ta + tb) + tc;
      float Ih, Il;
      fast2(ru, lg2(si), Ih, Il);
      const float rl = fmaxf(fmaxf(lh[0] + g0, lh[1] + g0), lh[2] + g1);
      const float td = ex2(((lh[0] - rl) + g0) + ll[0]), te = ex2(((lh[1] - rl) + g0) + ll[1]);
      const float tf = ex2(((lh[2] - rl) + g1) + ll[2]);
      const float sd = (td + te) + tf;
      float Dh, Dl;
      fast2(rl, lg2(sd), Dh, Dl);
      if (hold) { Mh = uMh; Ml = uMl; Ih = uIh; Il = uIl; Dh = uDh; Dl = uDl; }
      if constexpr (WT) {
        const float vm = hold ? 0.f : recip(sm), vi = hold ? 0.f : recip(si);
        const float vd = hold ? 0.f : recip(sd);
        put_weights<NS, R>(went, lane, c, make_float4(tM * vm, tI * vm, tD * vm, ta * vi),
                           make_float4(tb * vi, td * vd, tf * vd, 0.f), s[c]);
        put_inits<NS, R>(went, lane, c, tc * vi, te * vd, 0.f);
      }
      dgh[0] = uMh; dgl[0] = uMl; dgh[1] = uIh; dgl[1] = uIl; dgh[2] = uDh; dgl[2] = uDl;
      lh[0] = Mh; ll[0] = Ml; lh[1] = Ih; ll[1] = Il; lh[2] = Dh; ll[2] = Dl;
      ph[0][c] = Mh; pl[0][c] = Ml; ph[1][c] = Ih; pl[1][c] = Il; ph[2][c] = Dh; pl[2][c] = Dl;
    } else if constexpr (NS == 3) {
      const float uMh = ph[0][c], uMl = pl[0][c], uIh = ph[1][c], uIl = pl[1][c];
      const float uDh = ph[2][c], uDl = pl[2][c];
      // M = s + LSE(M, I, D at diag, 0).  The reference point of each LSE
      // comes from the hi parts only: any r close to the maximum keeps every
      // term <= ~1, and the lo parts enter the exponents exactly.
      const float r = fmaxf(fmaxf(dgh[0], dgh[1]), fmaxf(dgh[2], 0.f));
      const float tM = ex2((dgh[0] - r) + dgl[0]), tI = ex2((dgh[1] - r) + dgl[1]);
      const float tD = ex2((dgh[2] - r) + dgl[2]);
      const float sm = (tM + tI) + (tD + ex2(-r));
      float Mh, Ml;
      two_sum(r, s[c], Mh, Ml);
      Ml += lg2(sm);
      // I = LSE(M up + go, I up + ge)
      const float ru = fmaxf(uMh + g0, uIh + g1);
      const float ta = ex2(((uMh - ru) + g0) + uMl), tb = ex2(((uIh - ru) + g1) + uIl);
      const float si = ta + tb;
      float Ih, Il;
      fast2(ru, lg2(si), Ih, Il);
      // D = LSE(M left + go, D left + ge); Saigo-Vert adds I left + go
      const float rl = SV ? fmaxf(fmaxf(lh[0] + g0, lh[1] + g0), lh[2] + g1)
                          : fmaxf(lh[0] + g0, lh[2] + g1);
      const float tc = ex2(((lh[0] - rl) + g0) + ll[0]), td = ex2(((lh[2] - rl) + g1) + ll[2]);
      const float te = SV ? ex2(((lh[1] - rl) + g0) + ll[1]) : 0.f;
      const float sd = SV ? (tc + te) + td : tc + td;
      float Dh, Dl;
      fast2(rl, lg2(sd), Dh, Dl);
      if constexpr (WT) {
        const float vm = recip(sm), vi = recip(si), vd = recip(sd);
        put_weights<NS, R>(went, lane, c, make_float4(tM * vm, tI * vm, tD * vm, ta * vi),
                           make_float4(tb * vi, tc * vd, td * vd, 0.f), s[c]);
        if constexpr (SV) put_wdi<R>(went, lane, c, te * vd);
      }
      dgh[0] = uMh; dgl[0] = uMl; dgh[1] = uIh; dgl[1] = uIl; dgh[2] = uDh; dgl[2] = uDl;
      lh[0] = Mh; ll[0] = Ml; lh[1] = Ih; ll[1] = Il; lh[2] = Dh; ll[2] = Dl;
      ph[0][c] = Mh; pl[0][c] = Ml; ph[1][c] = Ih; pl[1][c] = Il; ph[2][c] = Dh; pl[2][c] = Dl;
    } else if constexpr (G) {
      const float uh = ph[0][c], ul = pl[0][c];
      // A = LSE(diag + s, up + g, left + g), reference point from hi parts
      const float r = fmaxf(dgh[0] + s[c], fmaxf(uh + g0, lh[0] + g0));
      const float va = ((dgh[0] - r) + s[c]) + dgl[0];
      const float vu = ((uh - r) + g0) + ul;
      const float vl = ((lh[0] - r) + g0) + ll[0];
      const float ta = ex2(va), tu = ex2(vu), tl = ex2(vl);
      const float sm = (ta + tu) + tl;
      float Ah, Al;
      fast2(r, lg2(sm), Ah, Al);
      if (hold) { Ah = uh; Al = ul; }
      if constexpr (WT) {
        const float v = hold ? 0.f : recip(sm);
        put_weights<NS, R>(went, lane, c, make_float4(ta * v, ta * v, tu * v, tl * v),
                           make_float4(0.f, 0.f, 0.f, 0.f), s[c]);
      }
      dgh[0] = uh; dgl[0] = ul;
      lh[0] = Ah; ll[0] = Al;
      ph[0][c] = Ah; pl[0][c] = Al;
    } else {
      const float uh = ph[0][c], ul = pl[0][c];
      // A = LSE(diag + s, up + g, left + g, s), reference point from hi parts
      const float r = fmaxf(fmaxf(dgh[0] + s[c], uh + g0), fmaxf(lh[0] + g0, s[c]));
      const float va = ((dgh[0] - r) + s[c]) + dgl[0];
      const float vu = ((uh - r) + g0) + ul;
      const float vl = ((lh[0] - r) + g0) + ll[0];
      const float vs = s[c] - r;
      const float ta = ex2(va), tu = ex2(vu), tl = ex2(vl), ts = ex2(vs);
      const float sm = (ta + tu) + (tl + ts);
      float Ah, Al;
      fast2(r, lg2(sm), Ah, Al);
      if constexpr (WT) {
        const float v = recip(sm);
        put_weights<NS, R>(went, lane, c, make_float4((ta + ts) * v, ta * v, tu * v, tl * v),
                           make_float4(0.f, 0.f, 0.f, 0.f), s[c]);
      }
      dgh[0] = uh; dgl[0] = ul;
      lh[0] = Ah; ll[0] = Al;
      ph[0][c] = Ah; pl[0][c] = Al;
    }
  }
  if constexpr (WT && !G) {
    // beta-init exp2(min(x - S, 0)) of the first `nlive` columns.  The lo
    // parts stay below ~2.1 (lo of M carries lg2 of a sum of at most four
    // terms <= 1), so a hi part below S - 135 gives an exponent below -130
    // and an init of exactly 0 (ex2.approx.ftz flushes it): when that holds
    // for every lane the step's inits are not computed or stored.
    constexpr int NI = SV ? 1 : NS;   // states that end an alignment (Saigo-Vert: M only)
    bool near = false;
#pragma unroll
    for (int c = 0; c < R; ++c)
#pragma unroll
      for (int q = 0; q < NI; ++q) near |= (c < nlive) && (ph[q][c] - Sh > -135.f);
    if (!__any_sync(FULL, near)) return false;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const bool lv = c < nlive;
      float b[NI];
#pragma unroll
      for (int q = 0; q < NI; ++q) b[q] = lv ? ex2(fminf((ph[q][c] - Sh) + (pl[q][c] - Sl), 0.f)) : 0.f;
      if constexpr (SV) put_init_m<R>(went, lane, c, b[0]);
      else if constexpr (NS == 3) put_inits<NS, R>(went, lane, c, b[0], b[1], b[2]);
      else put_inits<NS, R>(went, lane, c, b[0], 0.f, 0.f);
    }
    return true;
  }
  return false;
}

// Value of a global alignment at a terminal cell (column c): linear A;
// affine LSE(M, I, D) as a pair.
template <int NS, int R>
__device__ __forceinline__ void term_value(const float (&ph)[NS][R], const float (&pl)[NS][R], int c,
                                           float& h, float& l) {
  if constexpr (NS == 1) {
    h = ph[0][c];
    l = pl[0][c];
  } else {
    const float r = fmaxf(fmaxf(ph[0][c], ph[1][c]), ph[2][c]);
    const float sm = (ex2((ph[0][c] - r) + pl[0][c]) + ex2((ph[1][c] - r) + pl[1][c])) +
                     ex2((ph[2][c] - r) + pl[2][c]);
    fast2(r, lg2(sm), h, l);
  }
}

// Steps of a band, padded to whole checkpoint chunks (the padding steps find
// every lane past the last row and do nothing).
__device__ __forceinline__ int band_chunks(int L1) { return (L1 + 31 + C_STEPS - 1) / C_STEPS; }

// ---------------------------------------------------------------------------
// forward band task
// ---------------------------------------------------------------------------

// G: global alignment (see fwd_cells).  Lanes start from the row-0 boundary,
// band 0's lane 0 takes A[i,0] = i * gap as its left input, and instead of
// partition partials the band holding the pair's last column writes the
// terminal value A[L1,L2] (hi, lo) to its partial slot.  The chunk maximum
// becomes a marker: +1e30 for the chunk holding the terminal, NEG elsewhere,
// so the adjoint's quiet-chunk test sees the one beta-init there is.
template <int NS, int R, int GM = 0>
__device__ void fwd_band(const Args& a, const Place& w, int lane, uint64_t deadline) {
  constexpr bool G = GM == 1;
  [[maybe_unused]] constexpr bool SV = GM == 2;
  using D = Dims<NS, R>;
  constexpr int NE = D::NE;
  check_lengths(a, w, lane);
  const Pair& pr = w.pr;
  const int L1 = pr.L1, L2 = pr.L2;
  const int band = w.band;
  const size_t slot = w.slot0 + band;
  const int col0 = band * 32 * R;
  float* part = a.part + 2 * (size_t)slot;
  if (!(L1 > 0 && col0 < L2)) {
    if (!G && lane == 0) { part[0] = 0.f; part[1] = (band == 0) ? 1.f : 0.f; }
    return;
  }
  const int jl = col0 + lane * R;
  const float k = a.k, g0 = a.go * k, g1 = a.ge * k;
  const size_t Lm = (size_t)w.Lm;
  const bool term_lane = G && jl < L2 && L2 <= jl + R;   // holds the pair's last column
  float* eout = a.edge + w.ed0 + (size_t)band * w.edb;
  const float* ein = (band > 0) ? eout - w.edb : nullptr;
  const bool fault = a.fault_inject && band > 0;
  if (fault) ein = nullptr;
  // value-only calls (no adjoint to follow) pass no checkpoint buffer
  const bool keep_ck = a.ckpt != nullptr;
  float* ck = keep_ck ? a.ckpt + w.ck0 + (size_t)band * w.ckb : nullptr;
  const int nch = band_chunks(L1);

  float ph[NS][R], pl[NS][R], lh[NS], ll[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    lh[q] = NEG; ll[q] = 0.f;
#pragma unroll
    for (int c = 0; c < R; ++c) { ph[q][c] = NEG; pl[q][c] = 0.f; }
  }
  if constexpr (G) {   // row 0 (A[0,j] = j * gap, affine D(0,j) = go + (j-1) ge); lh = column jl
    row0<NS>(jl, g0, g1, lh, ll);
#pragma unroll
    for (int c = 0; c < R; ++c) {
      float h[NS], l[NS];
      row0<NS>(jl + c + 1, g0, g1, h, l);
#pragma unroll
      for (int q = 0; q < NS; ++q) { ph[q][c] = h[q]; pl[q][c] = l[q]; }
    }
  }
  float ref = 0.f;
  KSum acc;
  if (!G && band == 0 && lane == 0) acc.s = 1.f;  // the M[0,0] = 0 origin term

  // Lane u < C holds the left band's edge values that lane 0 needs at step u
  // of a chunk, loaded one chunk ahead; lane 0 takes them by shuffle.  Band 0
  // of a global alignment takes the column-0 boundary i * gap instead.
  const bool left_bnd = G && band == 0 && !fault;
  float eb[NE], ebn[NE];
  auto load_edge = [&](int kc, float (&dst)[NE]) {
    const int i = kc * C_STEPS + lane + 1;  // lane 0's row at step kc*C + lane
    const bool ok = ein && lane < C_STEPS && i <= L1;
#pragma unroll
    for (int f = 0; f < NE; ++f) dst[f] = ok ? ld_poll(ein + f * Lm + (i - 1)) : 0.f;
    if (left_bnd) col0_edge<NS>(i, g0, g1, dst);
  };
  load_edge(0, eb);
  float sb[PF][R];  // per-lane score ring, PF steps ahead
#pragma unroll
  for (int u = 0; u < PF; ++u) {
    const int i = u - lane + 1;
    load_row<R>(pr, i, jl, i >= 1 && i <= L1, sb[u]);
  }

  for (int kc = 0; kc < nch; ++kc) {
    if (keep_ck) {  // checkpoint: state before step kc*C
      float v[D::CKF];
      ck_pack<NS, R>(ph, pl, lh, ll, v);
      ck_store<NS, R>(ck + (size_t)kc * D::CKRS, lane, v);
    }
    float cmx = NEG;   // largest hi alpha of the lane's live cells in this chunk
    if (kc + 1 < nch) load_edge(kc + 1, ebn);
#pragma unroll 1
    for (int u0 = 0; u0 < C_STEPS; u0 += PF)
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int cu = u0 + u;
      const int t = kc * C_STEPS + cu;
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      float xh[NS], xl[NS], ev[NE];
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        xh[q] = __shfl_up_sync(FULL, ph[q][R - 1], 1);
        xl[q] = __shfl_up_sync(FULL, pl[q][R - 1], 1);
      }
#pragma unroll
      for (int f = 0; f < NE; ++f) ev[f] = __shfl_sync(FULL, eb[f], cu);
      // lane 0 takes the left band's values; a value still at the sentinel
      // (producer not there yet) is polled on a warp-uniform slow path
      bool miss = false;
#pragma unroll
      for (int f = 0; f < NE; ++f) miss |= is_sentinel(ev[f]);
      miss = (lane == 0) && ein && act && miss;
      if (__any_sync(FULL, miss) || fault) {
        if (lane == 0 && fault && act) {
          float v = poll_value(a.never_written, ld_poll(a.never_written), deadline, a.status,
                               a.pair_done + w.p, NEG);
#pragma unroll
          for (int f = 0; f < NE; ++f) ev[f] = (f < NS) ? v : 0.f;
        } else if (miss) {
          FieldVec<NE> x;
#pragma unroll
          for (int f = 0; f < NE; ++f) x.v[f] = ev[f];
          x = poll_fields_v<NE, NS>(x, ein + (i - 1), Lm, deadline, a.status, a.pair_done + w.p);
#pragma unroll
          for (int f = 0; f < NE; ++f) ev[f] = x.v[f];
        }
      }
      if (lane == 0) {
        const bool take = act && (ein || fault || left_bnd);
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          xh[q] = take ? ev[q] : NEG;
          xl[q] = take ? ev[NS + q] : 0.f;
        }
      }
      float dgh[NS], dgl[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        dgh[q] = lh[q]; dgl[q] = ll[q];
        lh[q] = xh[q]; ll[q] = xl[q];
      }
      float s[R];
#pragma unroll
      for (int c = 0; c < R; ++c) s[c] = i >= 1 ? __fmul_rn(sb[u][c], k) : NEG;
      {
        const int ip = i + PF;
        load_row<R>(pr, ip, jl, ip >= 1 && ip <= L1, sb[u]);
      }
      if constexpr (G) {
        fwd_cells<NS, R, false, GM>(ph, pl, lh, ll, dgh, dgl, s, g0, g1, 0.f, 0.f, 0, nullptr,
                                    lane, i < 1);
        if (act) {
          if (term_lane && i == L1) {   // the terminal: A[L1, L2], affine LSE of M, I, D there
            float th = 0.f, tl = 0.f;
#pragma unroll
            for (int c = 0; c < R; ++c)
              if (jl + c == L2 - 1) term_value<NS>(ph, pl, c, th, tl);
            part[0] = th;
            part[1] = tl;
            cmx = 1e30f;
          }
          if (lane == 31) {
#pragma unroll
            for (int q = 0; q < NS; ++q) {
              eout[q * Lm + (i - 1)] = ph[q][R - 1];
              eout[(NS + q) * Lm + (i - 1)] = pl[q][R - 1];
            }
          }
        }
        continue;
      }
      fwd_cells<NS, R, false, GM>(ph, pl, lh, ll, dgh, dgl, s, g0, g1);
      if (act) {
        // partition: lazily rescaled Kahan sum of ex2(x - ref); exponents stay
        // <= 8 so (hi - ref) + lo rounds at <= 2^-21 absolute
        // the partition's terms: every state of the local models, M alone
        // for Saigo-Vert (S = LSE(0, M cells))
        constexpr int NT = SV ? 1 : NS;
        float mx = NEG;
#pragma unroll
        for (int c = 0; c < R; ++c)
          if (jl + c < L2)
#pragma unroll
            for (int q = 0; q < NT; ++q) mx = fmaxf(mx, ph[q][c]);
        cmx = fmaxf(cmx, mx);
        if (mx > ref + 8.f) {
          float f = ex2(ref - mx);
          acc.s *= f;
          acc.c *= f;
          ref = mx;
        }
        float tsum = 0.f;
#pragma unroll
        for (int c = 0; c < R; ++c)
          if (jl + c < L2)
#pragma unroll
            for (int q = 0; q < NT; ++q) tsum += ex2((ph[q][c] - ref) + pl[q][c]);
        acc.add(tsum);
        if (lane == 31) {
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            eout[q * Lm + (i - 1)] = ph[q][R - 1];
            eout[(NS + q) * Lm + (i - 1)] = pl[q][R - 1];
          }
        }
      }
    }
#pragma unroll
    for (int f = 0; f < NE; ++f) eb[f] = ebn[f];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cmx = fmaxf(cmx, __shfl_xor_sync(FULL, cmx, o));
    if (keep_ck && lane == 0) ck[(size_t)kc * D::CKRS + D::CKF * 32] = cmx;
  }
  if constexpr (G) return;
  // warp-combine (ref, sum) pairs
  float s_ = acc.s;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float r2 = __shfl_xor_sync(FULL, ref, o);
    float s2 = __shfl_xor_sync(FULL, s_, o);
    float m = fmaxf(ref, r2);
    s_ = s_ * ex2(ref - m) + s2 * ex2(r2 - m);
    ref = m;
  }
  if (lane == 0) { part[0] = ref; part[1] = s_; }
}

template <int NS, int R, int GM = 0>
__global__ void __launch_bounds__(128) fwd_kernel(Args a) {
  const int lane = threadIdx.x & 31;
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = (a.layout == 0) ? a.B * a.nb : a.ntasks;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 0, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    fwd_band<NS, R, GM>(a, place_of<NS, R, GM>(a, task, false), lane, deadline);
  }
}

// ---------------------------------------------------------------------------
// adjoint band task
// ---------------------------------------------------------------------------

// Combine the forward partials of pair p into the scaled log-partition
// S' = Sh + Sl.
__device__ __forceinline__ void pair_logz(const Args& a, const Place& w, int lane, float& Sh,
                                          float& Sl) {
  float ref = NEG, s = 0.f;
  for (int b = lane; b < w.nb; b += 32) {
    const float* q = a.part + 2 * (w.slot0 + b);
    float r2 = q[0], s2 = q[1];
    if (s2 > 0.f) {
      float m = fmaxf(ref, r2);
      s = s * ex2(ref - m) + s2 * ex2(r2 - m);
      ref = m;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float r2 = __shfl_xor_sync(FULL, ref, o);
    float s2 = __shfl_xor_sync(FULL, s, o);
    float m = fmaxf(ref, r2);
    s = s * ex2(ref - m) + s2 * ex2(r2 - m);
    ref = m;
  }
  // S = ref + log2(s) as a double-float with a small lo part: with s = m * 2^e,
  // m in [1, 2), lg2 sees only the mantissa and the integer e joins ref by
  // TwoSum.  (lg2 of a large s would round at ~1e-6 absolute, which shows up
  // in every exp2(x - S) of the adjoint.)
  const unsigned bits = __float_as_uint(s);
  const int e = (int)((bits >> 23) & 0xffu) - 127;
  if (s > 0.f && e > -127 && e < 128) {
    float h, l;
    two_sum(ref, (float)e, h, l);
    Sh = h;
    Sl = l + lg2(__uint_as_float((bits & 0x7fffffu) | 0x3f800000u));
  } else {
    Sh = ref;
    Sl = lg2(s);
  }
}

// Global alignment: S' = the terminal value the band holding column L2 wrote,
// or, when a side is empty, the boundary cell's: linear (L1 + L2) * gap;
// affine go + (n - 1) ge for n = L1 + L2 > 0, 0 at the origin.
template <int NS, int R>
__device__ __forceinline__ void pair_term(const Args& a, const Place& w, float& Sh, float& Sl) {
  const int L1 = w.pr.L1, L2 = w.pr.L2;
  if (L1 == 0 || L2 == 0) {
    const int n = L1 + L2;
    if (NS == 1) {
      nmul(n, a.go * a.k, Sh, Sl);
    } else if (n > 0) {
      gpair(n - 1, a.go * a.k, a.ge * a.k, Sh, Sl);
    } else {
      Sh = 0.f;
      Sl = 0.f;
    }
    return;
  }
  const float* q = a.part + 2 * (w.slot0 + (L2 - 1) / (32 * R));
  Sh = q[0];
  Sl = q[1];
}

// Natural-unit value and dS/d(go, ge) of a global alignment with an empty
// side (the reference's float expressions: n * gap; go + (n - 1) * ge).
template <int NS>
__device__ __forceinline__ float empty_global_value(const Args& a, int n, float& dgo, float& dge) {
  if (NS == 1) {
    dgo = (float)n;
    dge = 0.f;
    return (float)n * a.go;
  }
  dgo = n > 0 ? 1.f : 0.f;
  dge = n > 0 ? (float)(n - 1) : 0.f;
  return n > 0 ? a.go + (float)(n - 1) * a.ge : 0.f;
}

// Value-only calls: one warp per pair folds the forward's band partials into
// S, as finish_pair does after a full adjoint (4 warps per CTA).  Only the
// pair's band count and first partial slot (and, for a global alignment, its
// lengths) are needed.
template <int NS, int R, int GM = 0>
__global__ void __launch_bounds__(128) value_kernel(Args a) {
  constexpr bool G = GM == 1;
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (q >= a.B) return;
  Place w;
  if (a.layout == 0) {
    w = place_of<NS, R, GM>(a, q * a.nb, false);
  } else {
    const long long* pw = a.plan_pairs + (size_t)q * PLAN_PAIR_WORDS;
    w.p = q;
    w.nb = (int)pw[PW_NB];
    w.slot0 = (size_t)pw[PW_SLOT0];
    w.pr.L1 = (int)pw[PW_L1];
    w.pr.L2 = (int)pw[PW_L2];
  }
  float Sh, Sl;
  if (a.pair_done[w.p] & PAIR_TIMEOUT) {   // a bounded wait of this pair expired
    if (lane == 0) a.value[w.p] = __int_as_float(0x7fc00000);
    return;
  }
  if constexpr (G) {
    if (lane == 0) {
      if (w.pr.L1 == 0 || w.pr.L2 == 0) {   // exactly the boundary cell's value
        float dgo, dge;
        a.value[w.p] = empty_global_value<NS>(a, w.pr.L1 + w.pr.L2, dgo, dge);
      } else {
        pair_term<NS, R>(a, w, Sh, Sl);
        a.value[w.p] = (Sh + Sl) * (1.f / a.k);
      }
    }
    return;
  }
  pair_logz(a, w, lane, Sh, Sl);
  if (lane == 0) a.value[w.p] = (Sh + Sl) * (1.f / a.k);
}

// Parameters a pair's finish needs (natural units, and k = log2(e) / T).
struct PParams { float go, ge, T, k; };

// Last band task of a pair to finish folds the per-band gradient partials (in
// band order, so the result is deterministic) into the outputs.
template <int NS, int GM = 0>
__device__ void finish_pair_p(const Args& a, const Place& w, int lane, float Sh, float Sl,
                              float g0sum, float g1sum, float pssum, PParams pp);

template <int NS, int GM = 0>
__device__ void finish_pair(const Args& a, const Place& w, int lane, float Sh, float Sl,
                            float g0sum, float g1sum, float pssum) {
  finish_pair_p<NS, GM>(a, w, lane, Sh, Sl, g0sum, g1sum, pssum, PParams{a.go, a.ge, a.T, a.k});
}

template <int NS, int GM>
__device__ void finish_pair_p(const Args& a, const Place& w, int lane, float Sh, float Sl,
                              float g0sum, float g1sum, float pssum, PParams pp) {
  constexpr bool G = GM == 1;
  const int p = w.p;
  if (lane == 0) {
    float* gp = a.gpart + 4 * (w.slot0 + w.band);
    gp[0] = g0sum; gp[1] = g1sum; gp[2] = pssum; gp[3] = 0.f;
    __threadfence();
    unsigned done = atomicAdd(a.pair_done + p, 1u);
    if ((done & ~PAIR_TIMEOUT) == (unsigned)w.nb - 1) {
      __threadfence();
      if (done & PAIR_TIMEOUT) {   // a bounded wait of this pair expired
        const float nan = __int_as_float(0x7fc00000);
        a.value[p] = nan; a.g_open[p] = nan; a.g_T[p] = nan;
        if (a.g_ext) a.g_ext[p] = nan;
        return;
      }
      float o = 0.f, e = 0.f, ps = 0.f;
      for (int b = 0; b < w.nb; ++b) {
        const float* q = a.gpart + 4 * (w.slot0 + b);
        o += ld_poll(q + 0);
        e += ld_poll(q + 1);
        ps += ld_poll(q + 2);
      }
      const float inv_k = 1.f / pp.k;         // = T * ln 2
      const float S = (Sh + Sl) * inv_k;
      const float match = ps * inv_k;
      if (G && (w.pr.L1 == 0 || w.pr.L2 == 0)) {
        // the terminal is a boundary cell: its value, its gap derivatives, dS/dT = 0
        float dgo, dge;
        a.value[p] = empty_global_value<NS>(a, w.pr.L1 + w.pr.L2, dgo, dge);
        a.g_open[p] = dgo;
        if (a.g_ext) a.g_ext[p] = dge;
        a.g_T[p] = 0.f;
        return;
      }
      a.value[p] = S;
      if (NS == 3) {
        a.g_open[p] = o;
        a.g_ext[p] = e;
        a.g_T[p] = (S - (match + (o * pp.go + e * pp.ge))) / pp.T;
      } else {
        a.g_open[p] = o;
        if (a.g_ext) a.g_ext[p] = 0.f;
        a.g_T[p] = (S - (match + o * pp.go)) / pp.T;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// adjoint band task
// ---------------------------------------------------------------------------

// Per band, checkpoint chunks in reverse.  Each chunk restores its checkpoint
// and recomputes C steps of alpha, writing every cell's adjoint fields
// (normalised predecessor weights, beta-init, scaled score) to shared memory;
// then the adjoint runs the same C steps backwards in push form, where a
// cell's beta = beta-init + pushes received, and it pushes beta * weight to
// each predecessor: within the lane through registers, to the left lane
// through __shfl_down_sync, to the left band through the push buffer.
//
// G (global alignment): the only beta-init is beta = 1 at the terminal cell
// A[L1, L2]; pushes that leave the grid into the row-0 and column-0 boundary
// cells (values j * gap and i * gap) add index * push to dS/dgap there.
template <int NS, int R, int GM = 0>
__device__ void bwd_band(const Args& a, const Place& w, int lane, float* sm, uint64_t deadline) {
  constexpr bool G = GM == 1;
  [[maybe_unused]] constexpr bool SV = GM == 2;
  using D = Dims<NS, R>;
  constexpr int NP = push_channels<NS, GM>(), NL = push_left<NS, GM>();
  constexpr int EW = D::EW, CKF = D::CKF, CKRS = D::CKRS, NE = D::NE;
  const Pair& pr = w.pr;
  const int L1 = pr.L1, L2 = pr.L2;
  const int band = w.band;
  const int col0 = band * 32 * R;
  float Sh, Sl;
  if constexpr (G) pair_term<NS, R>(a, w, Sh, Sl);
  else pair_logz(a, w, lane, Sh, Sl);
  if (!(L1 > 0 && col0 < L2)) {
    finish_pair<NS, GM>(a, w, lane, Sh, Sl, 0.f, 0.f, 0.f);
    return;
  }
  const int jl = col0 + lane * R;
  const bool term_lane = G && jl < L2 && L2 <= jl + R;   // holds the pair's last column
  const int ncols = min(max(L2 - jl, 0), R);  // columns of this lane inside the pair
  const float k = a.k, g0 = a.go * k, g1 = a.ge * k;
  const size_t Lm = (size_t)w.Lm;
  const float* ein = (band > 0) ? a.edge + w.ed0 + (size_t)(band - 1) * w.edb : nullptr;
  float* pout = (band > 0) ? a.bpush + w.bp0 + (size_t)band * w.bpb : nullptr;
  const bool right_live = (col0 + 32 * R) < L2 && (band + 1) < w.nb;
  const float* pin = right_live ? a.bpush + w.bp0 + (size_t)(band + 1) * w.bpb : nullptr;
  const float* ck = a.ckpt + w.ck0 + (size_t)band * w.ckb;
  const int nch = band_chunks(L1);

  // ---- chunk-ahead prefetch state ----
  float ckr[CKF];           // checkpoint of the next chunk to recompute
  float ckm;                // ... and the largest hi alpha of the band's live cells in it
  float ebr[NE];            // lane u < C: left-band edge pair of lane 0's row at recompute step u
  float pbc[NP], pbn[NP];   // lane u < C: right-band pushes lane 31 needs at adjoint step u
  float sb[PF][R];          // per-lane scores of the first PF recompute steps
  auto load_ck = [&](int kc) {
    const float* rec = ck + (size_t)kc * CKRS;
    ck_load<NS, R>(rec, lane, ckr);
    ckm = rec[CKF * 32];
  };
  auto load_eb = [&](int kc) {
    const int i = kc * C_STEPS + lane + 1;
    const bool ok = ein && lane < C_STEPS && i <= L1;
#pragma unroll
    for (int f = 0; f < NE; ++f) ebr[f] = ok ? ein[f * Lm + (i - 1)] : (f < NS ? NEG : 0.f);
    if (G && band == 0) col0_edge<NS>(i, g0, g1, ebr);   // column-0 boundary
  };
  auto load_pb = [&](int kc, float (&dst)[NP]) {
    const int i = kc * C_STEPS + C_STEPS - 1 - lane - 30;  // lane 31's row at step end-1-lane
    const bool ok = pin && lane < C_STEPS && i >= 1 && i <= L1;
#pragma unroll
    for (int f = 0; f < NP; ++f) {
      const bool left = f < NL;
      dst[f] = (ok && (left || i < L1)) ? ld_poll(pin + f * (Lm + 1) + i) : 0.f;
    }
  };
  auto load_sb = [&](int kc) {
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int i = kc * C_STEPS + u - lane + 1;
      load_row<R>(pr, i, jl, i >= 1 && i <= L1, sb[u]);
    }
  };
  load_ck(nch - 1);
  load_eb(nch - 1);
  load_sb(nch - 1);
  load_pb(nch - 1, pbc);

  // ---- adjoint state ----
  float ac[NS][R], nx[NS][R];   // pushes received by this row / the row above
#pragma unroll
  for (int q = 0; q < NS; ++q)
#pragma unroll
    for (int c = 0; c < R; ++c) { ac[q][c] = 0.f; nx[q][c] = 0.f; }
  float hold[NS], outp[NP];
#pragma unroll
  for (int q = 0; q < NS; ++q) hold[q] = 0.f;
#pragma unroll
  for (int q = 0; q < NP; ++q) outp[q] = 0.f;
  KSum gA, gB, gS;   // chunk sums folded in with compensation

  for (int kc = nch - 1; kc >= 0; --kc) {
    const int t0 = kc * C_STEPS;
    // ---- quiet chunk.  Flows only split or leave (a cell pushes beta * w
    // with the weights summing to at most 1), so every value inside a chunk
    // is at most the sum of the flows entering it plus its beta-inits.  When
    // every entering push is below kFlowTiny and every init is too (all hi
    // alphas of the chunk kInitQuiet below S), nothing in the chunk exceeds
    // ~2e-15: it writes zeros (map rows, pushes to the left band) instead of
    // restoring and recomputing. ----
    {
      // the right band's pushes for this chunk, resolved now so that the
      // decision does not depend on timing (results are deterministic)
      {
        bool miss = false;
#pragma unroll
        for (int q = 0; q < NP; ++q) miss |= is_sentinel(pbc[q]);
        if (__any_sync(FULL, miss) && miss) {
          const int ir = kc * C_STEPS + C_STEPS - 1 - lane - 30;   // as in load_pb
#pragma unroll
          for (int q = 0; q < NP; ++q)
            if (is_sentinel(pbc[q]))
              pbc[q] = poll_value(pin + q * (Lm + 1) + ir, ld_poll(pin + q * (Lm + 1) + ir), deadline,
                                  a.status, a.pair_done + w.p, 0.f);
        }
      }
      float inmax = 0.f;
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        inmax = fmaxf(inmax, hold[q]);
#pragma unroll
        for (int c = 0; c < R; ++c) inmax = fmaxf(inmax, ac[q][c]);
      }
#pragma unroll
      for (int q = 0; q < NP; ++q) inmax = fmaxf(fmaxf(inmax, outp[q]), pbc[q]);
      const bool ok = inmax < kFlowTiny && ckm - Sh < kInitQuiet;
      if (__all_sync(FULL, ok)) {
        // zero map rows and pushes to the left band for the rows of chunk kq
        auto zero_chunk = [&](int kq) {
          float z[R];
#pragma unroll
          for (int c = 0; c < R; ++c) z[c] = 0.f;
          for (int cu = 0; cu < C_STEPS; ++cu) {
            const int i = kq * C_STEPS + (C_STEPS - 1 - cu) - lane + 1;
            if (i >= 1 && i <= L1) {
              store_row<R>(pr, i, jl, z);
              if (lane == 0 && pout) {
#pragma unroll
                for (int f = 0; f < NP; ++f) {
                  const bool left = f < NL;
                  pout[f * (Lm + 1) + (left ? i : i - 1)] = 0.f;
                }
              }
            }
          }
        };
        zero_chunk(kc);
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          hold[q] = 0.f;
#pragma unroll
          for (int c = 0; c < R; ++c) ac[q][c] = 0.f;
        }
#pragma unroll
        for (int q = 0; q < NP; ++q) outp[q] = 0.f;
        // ---- quiet run.  After a quiet chunk nothing enters the next one
        // from below or from the right lane, so the following chunks are
        // quiet when the right band's pushes for their rows are written and
        // below kFlowTiny and their alpha maxima are low.  One round of loads
        // checks 32 / C chunks (lane l: chunk kn - l / C, lane 31's row at
        // its step C - 1 - l % C); a push not written yet ends the run, and
        // that chunk is then decided above from the same values, so results
        // do not depend on timing. ----
        constexpr int RUN = 32 / C_STEPS;
        int kn = kc - 1;   // first chunk not known to be quiet
        while (kn >= 0) {
          const int j = lane / C_STEPS, u = lane - j * C_STEPS;
          const int kq = kn - j;
          bool q = kq >= 0;
          if (q) {
            const int ir = kq * C_STEPS + C_STEPS - 1 - u - 30;
            if (pin && ir >= 1 && ir <= L1) {
#pragma unroll
              for (int f = 0; f < NP; ++f) {
                const bool left = f < NL;
                if (left || ir < L1) {
                  const float v = ld_poll(pin + f * (Lm + 1) + ir);
                  q = q && !is_sentinel(v) && v < kFlowTiny;
                }
              }
            }
            q = q && (ck[(size_t)kq * CKRS + CKF * 32] - Sh < kInitQuiet);
          }
          const unsigned ball = __ballot_sync(FULL, q);
          constexpr unsigned grp = (1u << C_STEPS) - 1u;
          int n = 0;
          while (n < RUN && kn - n >= 0 && ((ball >> (n * C_STEPS)) & grp) == grp) ++n;
          for (int m = 0; m < n; ++m) zero_chunk(kn - m);
          kn -= n;
          if (n < RUN) break;
        }
        if (kn >= 0) {   // inputs of the next chunk to run
          load_ck(kn);
          load_eb(kn);
          load_sb(kn);
          load_pb(kn, pbc);
        }
        kc = kn + 1;     // the loop continues with chunk kn
        continue;
      }
    }
    float cA = 0.f, cB = 0.f, cS = 0.f;   // this chunk's plain sums
    // ---- restore the checkpoint and recompute the chunk's adjoint fields ----
    float ph[NS][R], pl[NS][R], lh[NS], ll[NS];
    ck_unpack<NS, R>(ckr, ph, pl, lh, ll);
    unsigned initbits = 0;   // bit u: step u of the chunk wrote its beta-inits
    float tw[NS];            // G: the terminal's beta-inits (softmax of its states; linear 1)
#pragma unroll
    for (int q = 0; q < NS; ++q) tw[q] = 0.f;
#pragma unroll 1
    for (int u0 = 0; u0 < C_STEPS; u0 += PF)
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int cu = u0 + u;
      const int t = t0 + cu;
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      float xh[NS], xl[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        xh[q] = __shfl_up_sync(FULL, ph[q][R - 1], 1);
        xl[q] = __shfl_up_sync(FULL, pl[q][R - 1], 1);
        const float evh = __shfl_sync(FULL, ebr[q], cu);
        const float evl = __shfl_sync(FULL, ebr[NS + q], cu);
        if (lane == 0) {
          xh[q] = act ? evh : NEG;
          xl[q] = act ? evl : 0.f;
        }
      }
      float dgh[NS], dgl[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        dgh[q] = lh[q]; dgl[q] = ll[q];
        lh[q] = xh[q]; ll[q] = xl[q];
      }
      float s[R];
#pragma unroll
      for (int c = 0; c < R; ++c) s[c] = i >= 1 ? __fmul_rn(sb[u][c], k) : NEG;
      if (cu + PF < C_STEPS) {
        const int ip = i + PF;
        load_row<R>(pr, ip, jl, ip >= 1 && ip <= L1, sb[u]);
      }
      if (fwd_cells<NS, R, true, GM>(ph, pl, lh, ll, dgh, dgl, s, g0, g1, Sh, Sl, act ? ncols : 0,
                                    sm + (size_t)cu * EW * 32, lane, G && i < 1))
        initbits |= 1u << cu;
      if (G && term_lane && i == L1) {
#pragma unroll
        for (int c = 0; c < R; ++c)
          if (jl + c == L2 - 1)
#pragma unroll
            for (int q = 0; q < NS; ++q)
              tw[q] = NS == 1 ? 1.f : ex2((ph[q][c] - Sh) + (pl[q][c] - Sl));
      }
    }
    if (kc > 0) {  // prefetch the next chunk's inputs while the adjoint runs
      load_ck(kc - 1);
      load_eb(kc - 1);
      load_sb(kc - 1);
      load_pb(kc - 1, pbn);
    }
    __syncwarp();
    // ---- adjoint over the chunk, last step first ----
#pragma unroll 1
    for (int cu = 0; cu < C_STEPS; ++cu) {
      const int ent = C_STEPS - 1 - cu;        // entry of this step's row
      const bool hasinit = (initbits >> ent) & 1u;   // else every beta-init is 0
      const int t = t0 + ent;
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      const float* E = sm + (size_t)ent * EW * 32;
      float r[NP], pw[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        r[q] = __shfl_down_sync(FULL, outp[q], 1);
        pw[q] = __shfl_sync(FULL, pbc[q], cu);
      }
      // pushes arriving at column R-1 of row i: left pushes (local affine: M, D;
      // global affine: M, I, D; linear: A) and diag pushes (M, I, D; linear: A)
      float inL[3], inD[NS];
      {
        bool miss = false;
#pragma unroll
        for (int q = 0; q < NP; ++q) miss |= is_sentinel(pw[q]);
        miss = miss && (lane == 31);
        if (__any_sync(FULL, miss) && miss) {
#pragma unroll
          for (int q = 0; q < NP; ++q)
            if (is_sentinel(pw[q]))
              pw[q] = poll_value(pin + q * (Lm + 1) + i, ld_poll(pin + q * (Lm + 1) + i), deadline,
                                 a.status, a.pair_done + w.p, 0.f);
        }
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) inL[q] = 0.f;
      if (lane == 31) {
#pragma unroll
        for (int q = 0; q < NL; ++q) inL[q] = pw[q];
#pragma unroll
        for (int q = 0; q < NS; ++q) inD[q] = pw[NL + q];
      } else {
#pragma unroll
        for (int q = 0; q < NL; ++q) inL[q] = r[q];
#pragma unroll
        for (int q = 0; q < NS; ++q) { inD[q] = hold[q]; hold[q] = r[NL + q]; }
      }
      if constexpr (NS == 3 && (G || SV)) {
        ac[0][R - 1] += inL[0] + inD[0];
        ac[1][R - 1] += inL[1] + inD[1];
        ac[2][R - 1] += inL[2] + inD[2];
      } else if constexpr (NS == 3) {
        ac[0][R - 1] += inL[0] + inD[0];
        ac[1][R - 1] += inD[1];
        ac[2][R - 1] += inL[1] + inD[2];
      } else {
        ac[0][R - 1] += inL[0] + inD[0];
      }
      if constexpr (G) {
        if (term_lane && i == L1) {   // the terminal's beta-inits
#pragma unroll
          for (int c = 0; c < R; ++c)
            if (jl + c == L2 - 1)
#pragma unroll
              for (int q = 0; q < NS; ++q) ac[q][c] += tw[q];
        }
      }
#pragma unroll
      for (int q = 0; q < NP; ++q) outp[q] = 0.f;
      float pm[R];
#pragma unroll
      for (int c = R - 1; c >= 0; --c) {
        // cells outside the pair carry beta-init 0 and receive only zero
        // pushes (their successors are outside too, or their weight toward
        // a NEG predecessor is 0), so beta needs no mask
        if constexpr (NS == 3 && G) {
          float4 f0, f1;
          float sc, wID, wDI, unused;
          get_weights<NS, R>(E, lane, c, f0, f1, sc);
          get_inits<NS, R>(E, lane, c, wID, wDI, unused);
          // f0 = (wMM, wMI, wMD, wIM), f1 = (wII, wDM, wDD, s), (wID, wDI)
          const float bM = ac[0][c], bI = ac[1][c], bD = ac[2][c];
          pm[c] = bM;
          const float pIM = bI * f0.w, pII = bI * f1.x, pID = bI * wID;
          const float pDM = bD * f1.y, pDI = bD * wDI, pDD = bD * f1.z;
          const float qM = bM * f0.x, qI = bM * f0.y, qD = bM * f0.z;
          cA += (pIM + pID) + (pDM + pDI);
          cB += pII + pDD;
          cS += bM * sc;
          // pushes into the boundary states D(0, j) (row 0) and I(i, 0)
          // (column 0): gap_open once, gap_ext (n - 1) times; pushes toward
          // the NEG boundary states are 0
          if (i == 1) {
            cA += pID + qD;
            cB += (float)(jl + c) * pID + (float)(jl + c - 1) * qD;
          }
          if (band == 0 && lane == 0 && c == 0) {
            cA += pDI + qI;
            cB += (float)(i - 1) * pDI + (float)(i - 2) * qI;
          }
          nx[0][c] += pIM; nx[1][c] += pII; nx[2][c] += pID;
          if (c > 0) {
            nx[0][c - 1] += qM; nx[1][c - 1] += qI; nx[2][c - 1] += qD;
            ac[0][c - 1] += pDM; ac[1][c - 1] += pDI; ac[2][c - 1] += pDD;
          } else {
            outp[0] = pDM; outp[1] = pDI; outp[2] = pDD; outp[3] = qM; outp[4] = qI; outp[5] = qD;
          }
        } else if constexpr (NS == 3 && SV) {
          float4 f0, f1;
          float sc;
          get_weights<NS, R>(E, lane, c, f0, f1, sc);
          const float wDI = get_wdi<R>(E, lane, c);
          // f0 = (wMM, wMI, wMD, wIM), f1 = (wII, wDM, wDD, s), wDI; M's beta-init
          float i0 = 0.f, i1 = 0.f, unused = 0.f;
          if (hasinit) get_inits<NS, R>(E, lane, c, i0, i1, unused);
          const float bM = i0 + ac[0][c];
          const float bI = ac[1][c];
          const float bD = ac[2][c];
          pm[c] = bM;
          const float pIM = bI * f0.w, pII = bI * f1.x;
          const float pDM = bD * f1.y, pDI = bD * wDI, pDD = bD * f1.z;
          cA += (pIM + pDM) + pDI;
          cB += pII + pDD;
          cS += bM * sc;
          nx[0][c] += pIM;
          nx[1][c] += pII;
          const float qM = bM * f0.x, qI = bM * f0.y, qD = bM * f0.z;
          if (c > 0) {
            nx[0][c - 1] += qM; nx[1][c - 1] += qI; nx[2][c - 1] += qD;
            ac[0][c - 1] += pDM; ac[1][c - 1] += pDI; ac[2][c - 1] += pDD;
          } else {
            outp[0] = pDM; outp[1] = pDI; outp[2] = pDD; outp[3] = qM; outp[4] = qI; outp[5] = qD;
          }
        } else if constexpr (NS == 3) {
          float4 f0, f1;
          float sc;
          get_weights<NS, R>(E, lane, c, f0, f1, sc);
          // f0 = (wMM, wMI, wMD, wIM), f1 = (wII, wDM, wDD, s)
          float i0 = 0.f, i1 = 0.f, i2 = 0.f;
          if (hasinit) get_inits<NS, R>(E, lane, c, i0, i1, i2);
          const float bM = i0 + ac[0][c];
          const float bI = i1 + ac[1][c];
          const float bD = i2 + ac[2][c];
          pm[c] = bM;
          const float pIM = bI * f0.w, pII = bI * f1.x;
          const float pDM = bD * f1.y, pDD = bD * f1.z;
          cA += pIM + pDM;
          cB += pII + pDD;
          cS += bM * sc;
          nx[0][c] += pIM;
          nx[1][c] += pII;
          const float qM = bM * f0.x, qI = bM * f0.y, qD = bM * f0.z;
          if (c > 0) {
            nx[0][c - 1] += qM; nx[1][c - 1] += qI; nx[2][c - 1] += qD;
            ac[0][c - 1] += pDM; ac[2][c - 1] += pDD;
          } else {
            outp[0] = pDM; outp[1] = pDD; outp[2] = qM; outp[3] = qI; outp[4] = qD;
          }
        } else {
          float4 f0, f1;
          float sc;
          get_weights<NS, R>(E, lane, c, f0, f1, sc);
          // f0 = (map factor, wA, wU, wL)
          float i0 = 0.f, i1 = 0.f, i2 = 0.f;
          if (hasinit) get_inits<NS, R>(E, lane, c, i0, i1, i2);
          const float b = i0 + ac[0][c];
          const float pv_ = b * f0.x;
          pm[c] = pv_;
          const float pU = b * f0.z, pL = b * f0.w, pD = b * f0.y;
          cA += pU + pL;
          cS += pv_ * sc;
          if constexpr (G) {
            // pushes into the boundary: row 0 (up to column j, diag to j - 1)
            // and column 0 (left to row i, diag to row i - 1)
            if (i == 1) cA += (float)(jl + c + 1) * pU + (float)(jl + c) * pD;
            if (band == 0 && lane == 0 && c == 0) cA += (float)i * pL + (float)(i - 1) * pD;
          }
          nx[0][c] += pU;
          if (c > 0) {
            nx[0][c - 1] += pD;
            ac[0][c - 1] += pL;
          } else {
            outp[0] = pL; outp[1] = pD;
          }
        }
      }
      if (act) {
        store_row<R>(pr, i, jl, pm);
        if (lane == 0 && pout) {
#pragma unroll
          for (int f = 0; f < NP; ++f) pout[f * (Lm + 1) + (f < NL ? i : i - 1)] = outp[f];
        }
      }
#pragma unroll
      for (int q = 0; q < NS; ++q)
#pragma unroll
        for (int c = 0; c < R; ++c) { ac[q][c] = nx[q][c]; nx[q][c] = 0.f; }
    }
#pragma unroll
    for (int q = 0; q < NP; ++q) pbc[q] = pbn[q];
    gA.add(cA);
    gB.add(cB);
    gS.add(cS);
    __syncwarp();
  }
  // warp-reduce the gradient partials (fixed shuffle tree: deterministic)
  float v0 = gA.s, v1 = gB.s, v2 = gS.s;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_xor_sync(FULL, v0, o);
    v1 += __shfl_xor_sync(FULL, v1, o);
    v2 += __shfl_xor_sync(FULL, v2, o);
  }
  finish_pair<NS, GM>(a, w, lane, Sh, Sl, v0, v1, v2);
}

// Shared memory per adjoint warp (floats): one chunk of adjoint fields.
template <int NS, int R>
__host__ __device__ constexpr int bwd_smem_floats() {
  return C_STEPS * Dims<NS, R>::EW * 32;
}

template <int NS, int R, int WARPS, int GM = 0>
__global__ void __launch_bounds__(32 * WARPS) bwd_kernel(Args a) {
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  float* sm = smem + (size_t)w * bwd_smem_floats<NS, R>();
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = (a.layout == 0) ? a.B * a.nb : a.ntasks;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 1, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    bwd_band<NS, R, GM>(a, place_of<NS, R, GM>(a, task, true), lane, sm, deadline);
  }
}

}  // namespace swb

