// Soft Smith-Waterman forward / adjoint in the scaled linear domain (sm_100a),
// local alignment with linear or affine gaps.  Compiled as part of sw_capi.cu
// after sw_kernels.cu, whose band decomposition, task queue, cross-band
// buffers, polling and pair finish this file reuses.
//
// Why a linear domain
// -------------------
// Every term of the reference recurrence is positive, so instead of
// log-sum-exp over scaled log values (one ex2 per term, one lg2 per state:
// 14 MUFU ops per affine cell forward, 15 more in the adjoint) the DP can run
// on the exponentials themselves.  With E = 2^(s k) (k = log2(e) / T),
// G_o = 2^(go k), G_e = 2^(ge k) the local affine recurrence of
// src/sw_affine/kernels_cpu.cpp:94-196 becomes
//     M[i,j] = E[i,j] * (M + I + D)[i-1,j-1] + E[i,j]      (the "+ E": a fresh start)
//     I[i,j] = G_o * M[i-1,j] + G_e * I[i-1,j]
//     D[i,j] = G_o * M[i,j-1] + G_e * D[i,j-1]
//     Z      = 1 + sum over all cells and states,  S = T ln Z,
// and the linear one (src/sw/kernels_cpu.cpp:70-160)
//     A[i,j] = E[i,j] * (A[i-1,j-1] + 1) + G (A[i-1,j] + A[i,j-1]).
// The adjoint is the outside recursion beta = dZ/d(cell) over the successors,
//     beta_M = 1 + t(i+1,j+1) + G_o (beta_I(i+1,j) + beta_D(i,j+1)),  t = E * beta_M,
//     beta_I = 1 + t(i+1,j+1) + G_e beta_I(i+1,j),   beta_D = 1 + t + G_e beta_D(i,j+1),
// with the map P = M beta_M / Z (linear: E (A_diag + 1) beta / Z) and the
// parameter gradients as expected transition counts.  One ex2 per cell
// (the emission E), the rest multiply-adds.
//
// Range
// -----
// Values span far more than fp32's exponent range, so each lane keeps its R
// columns of a row as float mantissas under one power-of-two frame:
// value = m * 2^e.  A step computes its row in the frame et = max of its
// inputs' normalised frames (the lane's previous row, the left lane's row and
// the left lane's previous row), which makes every converted input <= 1;
// then the row's sum gives the normalised frame n = et + exponent(sum) in
// which the row is <= 1.  Rows are never rescaled: the raw values keep the
// compute frame et and every use scales them by 2^(frame - target) (a
// power-of-two factor built from the exponent bits, folded into the gap
// factors).  Frames are floored at 0: the empty alignment's weight 1 is
// always representable and Z >= 1, so values below 2^-149 of it are dropped,
// as the reference drops exponentials below e^-88 of their LSE's maximum.
// Scores are within |s|/T <= 80 (the host's domain check), so E <= 2^115.4
// and a step's raw values stay below 2^122.
//
// The kernels run when every transition factor is at most 1 (gaps <= 0);
// otherwise the host uses the log-domain kernels of sw_kernels.cu.
#include "sw_kernels.cuh"

namespace swb {

// 2^d for an integer d <= 127 (0 for d < -126): frame conversion factors.
// Conversions go to a frame at least as large as the source's normalised
// frame, so d <= 126 always (a raw value's frame exceeds its normalised frame
// by at most 126, when the values are below 1).
__device__ __forceinline__ float p2i(int d) {
  d = max(d, -127);
  return __int_as_float((d + 127) << 23);
}
// 2^d for any integer d, saturated to [0, 2^127].
__device__ __forceinline__ float p2any(int d) {
  d = min(max(d, -127), 127);
  return __int_as_float((d + 127) << 23);
}
// Upper bound k of log2 of a non-negative float: m <= 2^k, tight within a
// factor 2 for normal m (0 and subnormals give -126).
__device__ __forceinline__ int fexp(float m) {
  return (int)((__float_as_uint(m) >> 23) & 0xffu) - 126;
}

constexpr float XMAX = 118.f;   // scaled scores above this are clamped (|s|/T <= 80 gives 115.4)

// Quiet chunks of the adjoint: every posterior in the chunk and every flow
// out of it below 2^-SWB_LQUIET (relative to Z).  At 45 the posterior mass a
// pair can lose over all its chunks stays below ~1e-9.
#ifndef SWB_LQUIET
#define SWB_LQUIET 45
#endif

// Asynchronous global -> shared copy (cp.async): the adjoint stages the next
// chunk's checkpoint while it runs the current chunk, so it occupies no
// registers in between.
__device__ __forceinline__ void lcp16(float* dst, const float* src, int src_size) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_size)
               : "memory");
}
__device__ __forceinline__ void lcp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void lcp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---------------------------------------------------------------------------
// whole-chunk row pieces
// ---------------------------------------------------------------------------
// In the skewed wavefront lane l works on row t - l + 1 at step t, so one
// store of every lane touches 32 rows: 32 cache lines per warp instruction.
// Over a checkpoint chunk (C steps), though, row i is worked on by C
// adjacent lanes, whose columns are one contiguous piece of 4 C R bytes.  The
// adjoint writes the map rows of a quiet chunk (zeros) in whole row pieces:
// round `it`, item k = 32 it + lane is float4 h of lane l at step cu with
// q = k % NI, rho = k / NI, cu = q / HR, h = q % HR, l = rho - (C - 1) + cu;
// its row is kc C + cu - l + 1.  Every (cu, l, h) is one item; NI
// consecutive items are one row piece.
template <int R> struct Pieces {
  static constexpr int HR = R / 4;                    // float4 per lane and row
  static constexpr int NI = C_STEPS * HR;             // items per row piece
  static constexpr int ROWS = 32 + C_STEPS - 1;       // rows a chunk touches
  static constexpr int ROUNDS = (ROWS * NI + 31) / 32;
};

// Zero chunk kc's map rows of a band (a quiet chunk) in whole row pieces.
// Rows outside [1, L1] are not written; every column up to the row pitch is.
// The rounds run as a loop: unrolled, their per-lane item indices would stay
// live in registers across the adjoint.
template <int R>
__device__ __forceinline__ void zero_chunk_rows(const Pair& pr, int kc, int col0, int lane) {
  using P = Pieces<R>;
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 1
  for (int it = 0; it < P::ROUNDS; ++it) {
    const int k = it * 32 + lane;
    const int rho = k / P::NI, q = k - rho * P::NI;
    const int cu = q / P::HR, h = q - cu * P::HR;
    const int l = rho - (C_STEPS - 1) + cu;
    if (rho < P::ROWS && l >= 0 && l < 32) {
      const int i = kc * C_STEPS + cu - l + 1;
      const int col = col0 + R * l + 4 * h;
      if (i >= 1 && i <= pr.L1 && col < pr.ld) {
        float* dst = pr.m + (size_t)(i - 1) * pr.ld + col;
        if (pr.vec) {
          *reinterpret_cast<float4*>(dst) = z;
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (col + e < pr.ld) dst[e] = 0.f;
        }
      }
    }
  }
}

// Checkpoint floats per lane (CKF, padded to float4), one checkpoint record
// (LREC: CK4 groups of [lane][4]) and adjoint shared-memory floats per lane
// per step (FW).  A band's checkpoint region holds ceil(nchunks / ck_every)
// records, then one float per chunk: the chunk's largest normalised alpha
// frame (the adjoint's quiet-chunk test).  An affine record keeps M and I of
// the lane's row but not D: D is rebuilt from M, the left lane's values and
// the frames with the forward's own operations (lck_unpack), bit for bit, so
// a record is 24 floats per lane instead of 32 at 8 columns per lane.
template <int NS, int R> struct LDims {
  static constexpr int NSTORE = NS == 3 ? 2 : 1;         // states stored per column
  static constexpr int CKV = NSTORE * R + NS + 3;        // raw row, left values, e, n, nl
  static constexpr int CKF = (CKV + 3) / 4 * 4;
  static constexpr int CK4 = CKF / 4;
  static constexpr int LREC = CKF * 32;
  // affine: M, I, D (raw) and the scaled score per column; linear: A, the
  // emission part E (A_diag + 1), and the scaled score; then e and n
  static constexpr int NF = NS == 3 ? 4 : 3;
  static constexpr int FW = NF * R + 2;
};

// Lane state of the forward wavefront.
template <int NS, int R> struct LState {
  float v[NS][R];   // raw values of the lane's latest row (frame e)
  float cs[NS == 3 ? R : 1];   // affine: their column sums (M + I) + D (frame e)
  float lv[NS];     // the left lane's latest row, last column (normalised frame nl)
  float vs[NS];     // the lane's last column in its normalised frame n
  int e, n, nl;
};

// Affine: the column sums of the lane's row, the diagonal inputs of the next
// row's M (formed once per row, not once per cell).
template <int NS, int R>
__device__ __forceinline__ void lstate_sums(LState<NS, R>& s) {
  if constexpr (NS == 3) {
#pragma unroll
    for (int c = 0; c < R; ++c) s.cs[c] = (s.v[0][c] + s.v[1][c]) + s.v[2][c];
  }
}

template <int NS, int R>
__device__ __forceinline__ void lstate_zero(LState<NS, R>& s) {
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    s.lv[q] = 0.f; s.vs[q] = 0.f;
#pragma unroll
    for (int c = 0; c < R; ++c) s.v[q][c] = 0.f;
  }
  lstate_sums(s);
  s.e = 0; s.n = 0; s.nl = 0;
}

template <int NS, int R>
__device__ __forceinline__ void lck_store(float* rec, int lane, const LState<NS, R>& s) {
  using L = LDims<NS, R>;
  constexpr int V = L::NSTORE * R;   // where the left values start
  float x[L::CKF];
#pragma unroll
  for (int q = 0; q < L::NSTORE; ++q)
#pragma unroll
    for (int c = 0; c < R; ++c) x[q * R + c] = s.v[q][c];
#pragma unroll
  for (int q = 0; q < NS; ++q) x[V + q] = s.lv[q];
  x[V + NS] = __int_as_float(s.e);
  x[V + NS + 1] = __int_as_float(s.n);
  x[V + NS + 2] = __int_as_float(s.nl);
#pragma unroll
  for (int f = L::CKV; f < L::CKF; ++f) x[f] = 0.f;
#pragma unroll
  for (int g = 0; g < L::CK4; ++g)
    reinterpret_cast<float4*>(rec + g * 128)[lane] = make_float4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]);
}

template <int NS, int R>
__device__ __forceinline__ void lck_load(const float* rec, int lane, float (&x)[LDims<NS, R>::CKF]) {
  using L = LDims<NS, R>;
#pragma unroll
  for (int g = 0; g < L::CK4; ++g) {
    const float4 y = reinterpret_cast<const float4*>(rec + g * 128)[lane];
    x[4 * g] = y.x; x[4 * g + 1] = y.y; x[4 * g + 2] = y.z; x[4 * g + 3] = y.w;
  }
}

// Restores the lane state of a record.  Affine: D is rebuilt as lcells
// computed it for that row -- column 0 from the left lane's values (in its
// frame nl, converted to the row's frame e), column c > 0 from column c - 1
// of M and D, then zero past the pair -- with the same operations in the
// same order, so the restored state equals the forward's bit for bit.
template <int NS, int R>
__device__ __forceinline__ void lck_unpack(const float (&x)[LDims<NS, R>::CKF], LState<NS, R>& s,
                                           float gO, float gE, int nlive, bool has_dead) {
  using L = LDims<NS, R>;
  constexpr int V = L::NSTORE * R;
#pragma unroll
  for (int q = 0; q < L::NSTORE; ++q)
#pragma unroll
    for (int c = 0; c < R; ++c) s.v[q][c] = x[q * R + c];
#pragma unroll
  for (int q = 0; q < NS; ++q) s.lv[q] = x[V + q];
  s.e = __float_as_int(x[V + NS]);
  s.n = __float_as_int(x[V + NS + 1]);
  s.nl = __float_as_int(x[V + NS + 2]);
  if constexpr (NS == 3) {
    const float fL = p2i(s.nl - s.e);
    const float gOl = gO * fL, gEl = gE * fL;
#pragma unroll
    for (int c = 0; c < R; ++c)
      s.v[2][c] = c == 0 ? fmaf(gEl, s.lv[2], gOl * s.lv[0]) : fmaf(gE, s.v[2][c - 1], gO * s.v[0][c - 1]);
    if (has_dead) {
#pragma unroll
      for (int c = 0; c < R; ++c)
        if (c >= nlive) s.v[2][c] = 0.f;
    }
  }
  lstate_sums(s);
  const float f = p2i(s.e - s.n);
#pragma unroll
  for (int q = 0; q < NS; ++q) s.vs[q] = s.v[q][R - 1] * f;
}

// One step of the forward wavefront for one lane: (xl, xn) is the left
// lane's last column of this row (normalised frame xn), xs the scaled scores
// (NEG where the cell does not exist).  Updates the state to this row;
// returns the step's compute frame in `et` (the raw values' frame) and the
// row's sum over its columns and states in `rs` (frame et).
// Affine: M, I, D; linear: A (and, for the adjoint, the emission part em).
template <int NS, int R>
__device__ __forceinline__ void lcells(LState<NS, R>& s, const float (&xl)[NS], int xn,
                                       const float (&xs)[R], bool live, float gO, float gE, int nlive,
                                       bool has_dead, int& et, float (&em)[R], float& rs) {
  // diagonal inputs of column 0: the left lane's previous row
  const int nd = s.nl;
  float dg[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) { dg[q] = s.lv[q]; s.lv[q] = xl[q]; }
  s.nl = xn;
  et = max(max(s.n, xn), nd);
  // st: the fresh-start term 1 in frame et.  Before the lane's first row every
  // input of the step is 0, so st = 0 keeps the whole row at 0 (E is finite:
  // the scores of such rows are 0)
  const float fU = p2i(s.e - et), fL = p2i(xn - et), fD = p2i(nd - et), st = live ? p2i(-et) : 0.f;
  float E[R];
#pragma unroll
  for (int c = 0; c < R; ++c) E[c] = ex2(xs[c]);
  if constexpr (NS == 3) {
    const float gOu = gO * fU, gEu = gE * fU, gOl = gO * fL, gEl = gE * fL;
    float pS = (dg[0] + dg[1]) + dg[2], fP = fD;   // diagonal (M + I) + D of column 0
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const float oM = s.v[0][c], oI = s.v[1][c];
      const float m = E[c] * fmaf(fP, pS, st);
      const float iv = fmaf(gOu, oM, gEu * oI);
      // D runs along the lane's columns: one fma per column on that chain
      const float dv = c == 0 ? fmaf(gEl, s.lv[2], gOl * s.lv[0])
                              : fmaf(gE, s.v[2][c - 1], gO * s.v[0][c - 1]);
      s.v[0][c] = m; s.v[1][c] = iv; s.v[2][c] = dv;
      pS = s.cs[c]; fP = fU;   // the previous row's column sum: column c + 1's diagonal
      em[c] = 0.f;
    }
    if (has_dead) {   // columns past the pair: D would run on from the last live column
#pragma unroll
      for (int c = 0; c < R; ++c)
        if (c >= nlive) s.v[2][c] = 0.f;
    }
  } else {
    const float gU = gO * fU, gL = gO * fL;
    float pA = dg[0], fP = fD;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const float oA = s.v[0][c];
      const float m = E[c] * fmaf(fP, pA, st);
      const float left = c == 0 ? gL * s.lv[0] : gO * s.v[0][c - 1];
      const float a = fmaf(gU, oA, m + left);
      em[c] = m;
      s.v[0][c] = a;
      pA = oA; fP = fU;
    }
    if (has_dead) {
#pragma unroll
      for (int c = 0; c < R; ++c)
        if (c >= nlive) { s.v[0][c] = 0.f; em[c] = 0.f; }
    }
  }
  // the row sum over columns and states bounds every value of the row (all
  // are >= 0; it exceeds the largest by at most a factor 3R) and is the row's
  // partition term
  lstate_sums(s);
  float cs[R];
#pragma unroll
  for (int c = 0; c < R; ++c) {
    if constexpr (NS == 3) cs[c] = s.cs[c];
    else cs[c] = s.v[0][c];
  }
#pragma unroll
  for (int h = 1; h < R; h *= 2)   // pairwise: a short dependency chain
#pragma unroll
    for (int c = 0; c + h < R; c += 2 * h) cs[c] += cs[c + h];
  rs = cs[0];
  s.e = et;
  s.n = max(et + fexp(rs), 0);
  const float f = p2i(et - s.n);
#pragma unroll
  for (int q = 0; q < NS; ++q) s.vs[q] = s.v[q][R - 1] * f;
}

// Scaled scores of one step, clamped at XMAX; NEG in columns past the pair
// (E = 0 there).  Rows outside the pair hold scores 0 (load_row).
template <int R>
__device__ __forceinline__ void lscores(const float (&sb)[R], float k, int nlive, bool has_dead,
                                        float (&xs)[R]) {
#pragma unroll
  for (int c = 0; c < R; ++c) xs[c] = fminf(__fmul_rn(sb[c], k), XMAX);
  if (has_dead) {
#pragma unroll
    for (int c = 0; c < R; ++c)
      if (c >= nlive) xs[c] = NEG;
  }
}

// Parameters of a linear-domain launch: the launch's floats, or read from the
// device parameter array when there is one (a stream capture with tensor
// parameters: each replay reads their current values).  k and the transition
// factors are formed exactly as the host forms them.  ok is false for a
// temperature that is not finite and positive or a positive gap: the linear
// domain needs every transition factor <= 1.
struct LParams {
  float go, ge, T, k, xgo, xge;
  bool ok;
};
template <int NS>
__device__ __forceinline__ LParams lparams(const Args& a) {
  LParams p{a.go, a.ge, a.T, a.k, a.xgo, a.xge, true};
  if (a.dparams) {
    p.go = a.dparams[0];
    p.ge = NS == 3 ? a.dparams[1] : 0.f;
    p.T = a.dparams[NS == 3 ? 2 : 1];
    p.k = 1.4426950408889634f / p.T;
    p.xgo = (float)exp2((double)p.go * (double)p.k);
    p.xge = (float)exp2((double)p.ge * (double)p.k);
    p.ok = p.T > 0.f && p.T < INFINITY && p.go * p.k <= 0.f && p.ge * p.k <= 0.f;
  }
  return p;
}

// ---------------------------------------------------------------------------
// forward band task
// ---------------------------------------------------------------------------

// Score prefetch distance of the forward (steps; C_STEPS % SWB_FPF == 0).  A
// whole chunk: each row is requested a chunk before its step (measured on the
// 4096-pair bench batch at 8 columns per lane: forward 2.27 ms at 4 steps,
// 2.59 at 2, 3.05 at 1).
#ifndef SWB_FPF
#define SWB_FPF SWB_C_STEPS
#endif
constexpr int FPF = SWB_FPF;
static_assert(C_STEPS % FPF == 0, "the forward's prefetch distance must divide the chunk");

// Forward wavefront of one band: per-lane partition sums (Kahan, in the
// lane's largest normalised frame), the left-to-right edge records
// (last column normalised, then its frame) and, every C steps, a checkpoint
// of the lane state plus the chunk's largest normalised frame.  The band's
// partition partial is (frame, mantissa sum): Z_band = sum * 2^frame.
template <int NS, int R>
__device__ void lfwd_band(const Args& a, const LParams& lp, const Place& w, int lane,
                          uint64_t deadline, float4* sedge) {
  using LD = LDims<NS, R>;
  check_lengths(a, w, lane);
  if (!lp.ok && w.band == 0 && lane == 0) {
    atomicOr(a.status, ERR_BAD_PARAMS);
    atomicOr(a.pair_done + w.p, PAIR_TIMEOUT);
  }
  const Pair& pr = w.pr;
  const int L1 = pr.L1, L2 = pr.L2;
  const int band = w.band;
  const size_t slot = w.slot0 + band;
  const int col0 = band * 32 * R;
  float* part = a.part + 2 * (size_t)slot;
  if (!(L1 > 0 && col0 < L2)) {
    if (lane == 0) { part[0] = 0.f; part[1] = (band == 0) ? 1.f : 0.f; }
    return;
  }
  const int jl = col0 + lane * R;
  const int nlive = min(max(L2 - jl, 0), R);
  const bool has_dead = __any_sync(FULL, nlive < R);
  const float k = lp.k, gO = lp.xgo, gE = lp.xge;
  const size_t Lm = (size_t)w.Lm;
  float* eout = a.edge + w.ed0 + (size_t)band * w.edb;
  const float* ein = (band > 0) ? eout - w.edb : nullptr;
  const bool fault = a.fault_inject && band > 0;
  if (fault) ein = nullptr;
  const bool keep_ck = a.ckpt != nullptr;
  float* ck = keep_ck ? a.ckpt + w.ck0 + (size_t)band * w.ckb : nullptr;
  const int nch = band_chunks(L1);
  const int KC = a.ck_every;
  float* ckmax = keep_ck ? ck + (size_t)((nch + KC - 1) / KC) * LD::LREC : nullptr;

  LState<NS, R> s;
  lstate_zero(s);
  float zm = (band == 0 && lane == 0) ? 1.f : 0.f, zc = 0.f;   // M[0,0]: the empty alignment
  int ze = 0;

  // lane u < C holds the left band's edge record lane 0 needs at step u of a
  // chunk (NS values, then the frame), loaded one chunk ahead
  constexpr int NEF = NS + 1;
  float eb[NEF], ebn[NEF];
  auto load_edge = [&](int kc, float (&dst)[NEF]) {
    const int i = kc * C_STEPS + lane + 1;
    const bool ok = ein && lane < C_STEPS && i <= L1;
#pragma unroll
    for (int f = 0; f < NEF; ++f) dst[f] = ok ? ld_poll(ein + f * Lm + (i - 1)) : 0.f;
  };
  load_edge(0, eb);
#pragma unroll
  for (int f = 0; f < NEF; ++f) ebn[f] = 0.f;
  float sb[FPF][R];   // per-lane score ring, FPF steps ahead
#pragma unroll
  for (int u = 0; u < FPF; ++u) {
    const int i = u - lane + 1;
    load_row<R>(pr, i, jl, i >= 1 && i <= L1, sb[u]);
  }

  for (int kc = 0; kc < nch; ++kc) {
    // resolve this chunk's edge records before its first step: lane u < C
    // polls its own record until the left band has written it (one bounded
    // wait per chunk, not per row); fault injection waits on a word nobody
    // writes and substitutes zeros
    {
      const int ie = kc * C_STEPS + lane + 1;
      const bool mine = lane < C_STEPS && ie <= L1;
      bool miss = false;
#pragma unroll
      for (int f = 0; f < NEF; ++f) miss |= is_sentinel(eb[f]);
      miss = miss && ein && mine;
      if (__any_sync(FULL, miss || (fault && mine))) {
        if (fault && mine) {
          poll_value(a.never_written, ld_poll(a.never_written), deadline, a.status, a.pair_done + w.p,
                     0.f);
#pragma unroll
          for (int f = 0; f < NEF; ++f) eb[f] = 0.f;
        } else if (miss) {
          FieldVec<NEF> x;
#pragma unroll
          for (int f = 0; f < NEF; ++f) x.v[f] = eb[f];
          x = poll_fields_v<NEF, 0>(x, ein + (ie - 1), Lm, deadline, a.status, a.pair_done + w.p);
#pragma unroll
          for (int f = 0; f < NEF; ++f) eb[f] = x.v[f];
        }
      }
    }
    // the resolved records go to shared memory, where lane 0 reads the one of
    // each step (one load instead of NS + 1 shuffles per step)
    __syncwarp();
    if (lane < C_STEPS) sedge[lane] = make_float4(eb[0], eb[1], eb[NEF > 2 ? 2 : 0], eb[NEF > 3 ? 3 : 0]);
    __syncwarp();
    if (keep_ck && kc % KC == 0) lck_store<NS, R>(ck + (size_t)(kc / KC) * LD::LREC, lane, s);
    int cmx = -(1 << 30);   // largest normalised frame of the lane's live rows in this chunk
    if (kc + 1 < nch) load_edge(kc + 1, ebn);
#pragma unroll 1
    for (int u0 = 0; u0 < C_STEPS; u0 += FPF)
#pragma unroll
    for (int u = 0; u < FPF; ++u) {
      const int cu = u0 + u;
      const int t = kc * C_STEPS + cu;
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      float xl[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) xl[q] = __shfl_up_sync(FULL, s.vs[q], 1);
      int xn = __shfl_up_sync(FULL, s.n, 1);
      if (lane == 0) {   // the chunk's records are resolved (0 where there is no left band)
        const float4 e4 = sedge[cu];
        const float ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
        for (int q = 0; q < NS; ++q) xl[q] = act ? ev[q] : 0.f;
        xn = act ? __float_as_int(ev[NS]) : 0;
      }
      float xs[R];
      lscores<R>(sb[u], k, nlive, has_dead, xs);
      {
        const int ip = i + FPF;
        load_row<R>(pr, ip, jl, ip >= 1 && ip <= L1, sb[u]);
      }
      int et;
      float em[R], rs;
      lcells<NS, R>(s, xl, xn, xs, i >= 1, gO, gE, nlive, has_dead, et, em, rs);
      if (act) {
        // partition: the row's live values (dead columns are 0) in the frame
        // ze (the largest normalised frame so far), Kahan-compensated
        if (s.n > ze) {
          const float f = p2i(ze - s.n);
          zm *= f; zc *= f; ze = s.n;
        }
        const float y = rs * p2i(et - ze) - zc;
        const float tt = zm + y;
        zc = (tt - zm) - y;
        zm = tt;
        cmx = max(cmx, s.n);
        if (lane == 31) {
#pragma unroll
          for (int q = 0; q < NS; ++q) eout[q * Lm + (i - 1)] = s.vs[q];
          eout[NS * Lm + (i - 1)] = __int_as_float(s.n);
        }
      }
    }
#pragma unroll
    for (int f = 0; f < NEF; ++f) eb[f] = ebn[f];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cmx = max(cmx, __shfl_xor_sync(FULL, cmx, o));
    if (keep_ck && lane == 0) ckmax[kc] = __int_as_float(cmx);
  }
  // warp-combine (frame, sum) pairs, fixed shuffle tree
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int z2 = __shfl_xor_sync(FULL, ze, o);
    const float m2 = __shfl_xor_sync(FULL, zm, o);
    const int m = max(ze, z2);
    zm = zm * p2i(ze - m) + m2 * p2i(z2 - m);
    ze = m;
  }
  if (lane == 0) { part[0] = (float)ze; part[1] = zm; }
}

#ifndef SWB_LFWD_MINB
#define SWB_LFWD_MINB 5
#endif
template <int NS, int R>
__global__ void __launch_bounds__(128, (R >= 8 ? 4 : SWB_LFWD_MINB)) lfwd_kernel(Args a) {
  __shared__ float4 s_edge[4][C_STEPS];   // per warp: the left band's records of a chunk
  const int lane = threadIdx.x & 31;
  const LParams lp = lparams<NS>(a);
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = (a.layout == 0) ? a.B * a.nb : a.ntasks;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 0, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    lfwd_band<NS, R>(a, lp, place_of<NS, R>(a, task, false), lane, deadline, s_edge[threadIdx.x >> 5]);
  }
}

// ---------------------------------------------------------------------------
// partition of a pair
// ---------------------------------------------------------------------------

// Z of pair w as (integer frame ze, mantissa zm): Z = zm * 2^ze, combined
// from the band partials in a fixed order (deterministic).
__device__ __forceinline__ void lpair_z(const Args& a, const Place& w, int lane, int& ze, float& zm) {
  int ref = 0;
  float s = 0.f;
  for (int b = lane; b < w.nb; b += 32) {
    const float* q = a.part + 2 * (w.slot0 + b);
    const int r2 = (int)q[0];
    const float s2 = q[1];
    if (s2 > 0.f) {
      const int m = max(ref, r2);
      s = s * p2i(ref - m) + s2 * p2i(r2 - m);
      ref = m;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int r2 = __shfl_xor_sync(FULL, ref, o);
    const float s2 = __shfl_xor_sync(FULL, s, o);
    const int m = max(ref, r2);
    s = s * p2i(ref - m) + s2 * p2i(r2 - m);
    ref = m;
  }
  ze = ref;
  zm = s;
}

// S' = log2 Z as a double-float (Sh, Sl): the integer part joins the frame
// exactly and lg2 sees only the mantissa.
__device__ __forceinline__ void lz_log2(int ze, float zm, float& Sh, float& Sl) {
  const unsigned bits = __float_as_uint(zm);
  const int e = (int)((bits >> 23) & 0xffu) - 127;
  if (zm > 0.f && e > -127 && e < 128) {
    float h, l;
    two_sum((float)ze, (float)e, h, l);
    Sh = h;
    Sl = l + lg2(__uint_as_float((bits & 0x7fffffu) | 0x3f800000u));
  } else {
    Sh = (float)ze;
    Sl = lg2(zm);
  }
}

// Value-only calls: one warp per pair folds the band partials into S.
template <int NS, int R>
__global__ void __launch_bounds__(128) lvalue_kernel(Args a) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (q >= a.B) return;
  Place w;
  if (a.layout == 0) {
    w = place_of<NS, R>(a, q * a.nb, false);
  } else {
    const long long* pw = a.plan_pairs + (size_t)q * PLAN_PAIR_WORDS;
    w.p = q;
    w.nb = (int)pw[PW_NB];
    w.slot0 = (size_t)pw[PW_SLOT0];
  }
  if (a.pair_done[w.p] & PAIR_TIMEOUT) {   // a bounded wait of this pair expired
    if (lane == 0) a.value[w.p] = __int_as_float(0x7fc00000);
    return;
  }
  int ze;
  float zm, Sh, Sl;
  lpair_z(a, w, lane, ze, zm);
  lz_log2(ze, zm, Sh, Sl);
  if (lane == 0) a.value[w.p] = (Sh + Sl) * (1.f / lparams<NS>(a).k);
}

// ---------------------------------------------------------------------------
// adjoint band task
// ---------------------------------------------------------------------------

// Shared memory per adjoint warp (floats): one chunk of recomputed fields,
// the staged checkpoint of the next chunk, then the chunk's cross-band
// records as float4 per step: the left band's edge records (lane 0,
// recompute) and the right band's push records (lane 31, outside recursion).
// The next chunk's score rows wait in registers.
template <int NS, int R>
__host__ __device__ constexpr int lbwd_smem_floats() {
  return (C_STEPS * LDims<NS, R>::FW + LDims<NS, R>::CKF) * 32 + 2 * C_STEPS * 4;
}

// Per band, checkpoint chunks in reverse.  Each chunk restores its checkpoint
// and recomputes C steps of the forward, keeping every cell's raw values and
// scaled score (and each step's frames) in shared memory; then the outside
// recursion runs the same C steps backwards.  Lane l + 1 is one step ahead of
// lane l (it processes row i one step earlier); a lane receives from its right
// neighbour that row's beta_D (beta, linear) of column 0 in the neighbour's
// normalised frame, its t = E beta_M of column 0 and the frame, and holds
// the t for one more step (it is the diagonal successor of the next row).
// Lane 0 passes the same three values to the left band through the push
// buffer; lane 31 reads the right band's.  No atomics; the map is written row
// by row (a quiet chunk writes its zero rows in whole row pieces); the
// gradient sums are folded per pair in band order.
template <int NS, int R, bool SPARSE = false>
__device__ void lbwd_band(const Args& a, const LParams& lp, const Place& w, int lane, float* sm,
                          uint64_t deadline) {
  using LD = LDims<NS, R>;
  constexpr int CKF = LD::CKF, LREC = LD::LREC, FW = LD::FW, NEF = NS + 1, NPF = 3;
  const Pair& pr = w.pr;
  const int L1 = pr.L1, L2 = pr.L2;
  const int band = w.band;
  const int col0 = band * 32 * R;
  int ze;
  float zm, Sh, Sl;
  lpair_z(a, w, lane, ze, zm);
  lz_log2(ze, zm, Sh, Sl);
  const PParams pp{lp.go, lp.ge, lp.T, lp.k};
  if (!(L1 > 0 && col0 < L2)) {
    finish_pair_p<NS>(a, w, lane, Sh, Sl, 0.f, 0.f, 0.f, pp);
    return;
  }
  const float invZ = 1.f / zm;
  const int jl = col0 + lane * R;
  const int nlive = min(max(L2 - jl, 0), R);
  const bool has_dead = __any_sync(FULL, nlive < R);
  const float k = lp.k, gO = lp.xgo, gE = lp.xge, gX = fmaxf(gO, gE);
  const size_t Lm = (size_t)w.Lm;
  const float* ein = (band > 0) ? a.edge + w.ed0 + (size_t)(band - 1) * w.edb : nullptr;
  float* pout = (band > 0) ? a.bpush + w.bp0 + (size_t)band * w.bpb : nullptr;
  const bool right_live = (col0 + 32 * R) < L2 && (band + 1) < w.nb;
  const float* pin = right_live ? a.bpush + w.bp0 + (size_t)(band + 1) * w.bpb : nullptr;
  const float* ck = a.ckpt + w.ck0 + (size_t)band * w.ckb;
  const int nch = band_chunks(L1);
  const int KC = SPARSE ? a.ck_every : 1;   // checkpoint records every KC chunks
  const float* ckmax = ck + (size_t)((nch + KC - 1) / KC) * LREC;

  // ---- chunk-ahead prefetch state: the next chunk's checkpoint is staged in
  // shared memory (cp.async), its score rows and records wait in registers ----
  float* stg_ck = sm + C_STEPS * FW * 32;   // [CK4][lane][4]
  float4* s_eb = reinterpret_cast<float4*>(stg_ck + CKF * 32);   // [C] edge records
  float4* s_pb = s_eb + C_STEPS;                                 // [C] push records
  float nsb[C_STEPS][R];   // the next chunk's score rows, requested a chunk ahead
  int ckm;                 // the next chunk's largest normalised alpha frame
  float ebr[NEF];          // lane u < C: left-band edge record of lane 0's row at recompute step u
  float pbc[NPF], pbn[NPF];// lane u < C: right-band record lane 31 needs at backward step u
  auto load_ck = [&](int kc) {   // the record at or before chunk kc, and kc's alpha frame
    const float* rec = ck + (size_t)(kc / KC) * LREC;
#pragma unroll
    for (int g = 0; g < LD::CK4; ++g) lcp16(stg_ck + g * 128 + lane * 4, rec + g * 128 + lane * 4, 16);
    lcp_commit();
    ckm = __float_as_int(ckmax[kc]);
  };
  auto load_eb = [&](int kc) {
    const int i = kc * C_STEPS + lane + 1;
    const bool ok = ein && lane < C_STEPS && i <= L1;
#pragma unroll
    for (int f = 0; f < NEF; ++f) ebr[f] = ok ? ein[f * Lm + (i - 1)] : 0.f;
  };
  auto load_pb = [&](int kc, float (&dst)[NPF]) {
    const int i = kc * C_STEPS + C_STEPS - 1 - lane - 30;   // lane 31's row at backward step lane
    const bool ok = pin && lane < C_STEPS && i >= 1 && i <= L1;
#pragma unroll
    for (int f = 0; f < NPF; ++f) dst[f] = ok ? ld_poll(pin + f * (Lm + 1) + i) : 0.f;
  };
  auto load_sb = [&](int kc) {
#pragma unroll
    for (int u = 0; u < C_STEPS; ++u) {
      const int i = kc * C_STEPS + u - lane + 1;
      load_row<R>(pr, i, jl, i >= 1 && i <= L1, nsb[u]);
    }
  };
  load_ck(nch - 1);
  load_eb(nch - 1);
  load_sb(nch - 1);
  load_pb(nch - 1, pbc);
#pragma unroll
  for (int f = 0; f < NPF; ++f) pbn[f] = 0.f;

  // ---- outside-recursion state: the row below (raw beta_I / beta in frame
  // fb, t = E beta_M in frame nb), the right neighbour's held t and frame,
  // and this lane's outputs of its latest row (for the left neighbour) ----
  float bdn[R], tdn[R];
#pragma unroll
  for (int c = 0; c < R; ++c) { bdn[c] = 0.f; tdn[c] = 0.f; }
  int fb = 0, nb = 0;
  float ht = 0.f;
  int hn = 0;
  float o_b = 0.f, o_t = 0.f;
  int o_n = 0;
  KSum gA, gB, gS;

  // log2 of Z is at least zlog; a chunk is quiet (below) when every cell's
  // posterior and every flow out of it is below 2^-SWB_LQUIET
  const int zlog = ze + fexp(zm) - 1 - SWB_LQUIET;
  for (int kc = nch - 1; kc >= 0; --kc) {
    const int t0 = kc * C_STEPS;
    lcp_wait_all();   // this chunk's staged checkpoint
    __syncwarp();
    // ---- quiet chunk.  For a cell u of the chunk, alpha_u beta_u / Z sums,
    // over the chunk cells x where u's continuations stay inside, terms
    // alpha_x (1 + w beta_out) / Z (alpha_u W(u -> x) <= alpha_x: all weights
    // are positive), where beta_out are the successors outside the chunk: the
    // row below, the right neighbour's held t and, for lane 31, the right
    // band's records.  With at most 2^9 cells, alpha_x <= 2^ckm and
    // 1 + w beta_out <= 4 max(1, inflow), every posterior in the chunk and
    // every flow across its top and left edges is below 2^-SWB_LQUIET when
    // ckm + 11 + max(log2 inflow, 0) < log2 Z - SWB_LQUIET.  Such a chunk writes zero
    // map rows and zero records to the left band, and passes zero beta up:
    // the flows it drops are among those bounded.  The right band's records
    // are resolved first, so the decision does not depend on timing. ----
    {
      {
        bool miss = false;
#pragma unroll
        for (int f = 0; f < NPF; ++f) miss |= is_sentinel(pbc[f]);
        if (__any_sync(FULL, miss) && miss) {
          const int ir = kc * C_STEPS + C_STEPS - 1 - lane - 30;   // as in load_pb
          FieldVec<NPF> x;
#pragma unroll
          for (int f = 0; f < NPF; ++f) x.v[f] = pbc[f];
          x = poll_fields_v<NPF, 0>(x, pin + ir, Lm + 1, deadline, a.status, a.pair_done + w.p);
#pragma unroll
          for (int f = 0; f < NPF; ++f) pbc[f] = x.v[f];
        }
      }
      int inl = hn + fexp(ht);
#pragma unroll
      for (int c = 0; c < R; ++c) inl = max(inl, max(fb + fexp(bdn[c]), nb + fexp(tdn[c])));
      if (lane < C_STEPS) {
        const int pn = __float_as_int(pbc[2]);
        inl = max(inl, pn + fexp(fmaxf(pbc[0], pbc[1])));
      }
      const bool ok = ckm + 11 + max(inl, 0) < zlog;
#ifdef SWB_COUNT_QUIET   // measurement builds: quiet and computed chunks in header words 8, 9
      {
        const bool all_ok = __all_sync(FULL, ok);   // the vote runs on every lane
        if (lane == 0) atomicAdd(a.counters + (all_ok ? 8 : 9), 1u);
      }
#endif
      if (__all_sync(FULL, ok)) {
        // zero map rows and left-band records for the rows of chunk kq
        auto zero_chunk = [&](int kq) {
          if constexpr (R % 4 == 0) zero_chunk_rows<R>(pr, kq, col0, lane);
          for (int cu = 0; cu < C_STEPS; ++cu) {
            const int i = kq * C_STEPS + cu - lane + 1;
            if (i >= 1 && i <= L1) {
              if constexpr (R % 4 != 0) {
                float z[R];
#pragma unroll
                for (int c = 0; c < R; ++c) z[c] = 0.f;
                store_row<R>(pr, i, jl, z);
              }
              if (lane == 0 && pout) {
                pout[0 * (Lm + 1) + i] = 0.f;
                pout[1 * (Lm + 1) + i] = 0.f;
                pout[2 * (Lm + 1) + i] = 0.f;
              }
            }
          }
        };
        zero_chunk(kc);
        // the row above the chunk sees zero beta; lane 31 keeps the right
        // band's t of its top chunk row as the held diagonal successor
        float pt = __shfl_sync(FULL, pbc[1], C_STEPS - 1);
        int pn = __shfl_sync(FULL, __float_as_int(pbc[2]), C_STEPS - 1);
        // ---- quiet run.  After a quiet chunk only lane 31's held t and the
        // right band's records enter the chunks above, so one round of loads
        // decides the next 32 / C chunks: lane l takes chunk kn - l / C at
        // backward step l % C (lane 31's row there), checking that record
        // and the one of the row below (lane l - 1's; lane 0: the held t).
        // A record not written yet ends the run; that chunk is then decided
        // as above from the same values, so results do not depend on timing. ----
        constexpr int RUN = 32 / C_STEPS;
        int kn = kc - 1;
        while (kn >= 0) {
          const int j = lane / C_STEPS, u = lane - j * C_STEPS;
          const int kq = kn - j;
          float r0 = 0.f, r1 = 0.f;
          int rn2 = 0, cm = -(1 << 30);
          bool written = true;
          if (kq >= 0) {
            const int ir = kq * C_STEPS + C_STEPS - 1 - u - 30;
            if (pin && ir >= 1 && ir <= L1) {
              r0 = ld_poll(pin + 0 * (Lm + 1) + ir);
              r1 = ld_poll(pin + 1 * (Lm + 1) + ir);
              const float r2 = ld_poll(pin + 2 * (Lm + 1) + ir);
              written = !is_sentinel(r0) && !is_sentinel(r1) && !is_sentinel(r2);
              rn2 = __float_as_int(r2);
            }
            cm = __float_as_int(ckmax[kq]);
          }
          const int lg = written ? rn2 + fexp(fmaxf(r0, r1)) : 0;
          const int lgu = __shfl_up_sync(FULL, lg, 1);
          const bool wu = __shfl_up_sync(FULL, (int)written, 1) != 0;
          const int lgb = lane == 0 ? pn + fexp(pt) : lgu;
          const bool wb = lane == 0 || wu;
          const bool q = kq >= 0 && written && wb && cm + 11 + max(max(lg, lgb), 0) < zlog;
          const unsigned ball = __ballot_sync(FULL, q);
          constexpr unsigned grp = (1u << C_STEPS) - 1u;
          int n = 0;
          while (n < RUN && kn - n >= 0 && ((ball >> (n * C_STEPS)) & grp) == grp) ++n;
          for (int m = 0; m < n; ++m) zero_chunk(kn - m);
          if (n > 0) {   // lane 31's held t: the record of its top row of the last zeroed chunk
            const int src = (n - 1) * C_STEPS + C_STEPS - 1;
            pt = __shfl_sync(FULL, r1, src);
            pn = __shfl_sync(FULL, rn2, src);
          }
          kn -= n;
          if (n < RUN) break;
        }
#pragma unroll
        for (int c = 0; c < R; ++c) { bdn[c] = 0.f; tdn[c] = 0.f; }
        fb = 0; nb = 0;
        o_b = 0.f; o_t = 0.f; o_n = 0;
        ht = lane == 31 ? pt : 0.f;
        hn = lane == 31 ? pn : 0;
        if (kn >= 0) {   // inputs of the next chunk to run
          load_ck(kn);
          load_eb(kn);
          load_sb(kn);
          load_pb(kn, pbc);
        }
        kc = kn + 1;   // the loop continues with chunk kn
        continue;
      }
    }
    // ---- restore the checkpoint and recompute the chunk ----
    LState<NS, R> st;
    {
      float ckr[CKF];
      lck_load<NS, R>(stg_ck, lane, ckr);
      lck_unpack<NS, R>(ckr, st, gO, gE, nlive, has_dead);
    }
    if (lane < C_STEPS) s_eb[lane] = make_float4(ebr[0], ebr[1], ebr[NEF > 2 ? 2 : 0], ebr[NEF > 3 ? 3 : 0]);
    __syncwarp();   // the staged checkpoint is read before the next chunk's copy is issued
    if (SPARSE && kc % KC != 0) {
      // sparse checkpoints: the restored state is that of chunk kc - kc % KC;
      // run the forward over the chunks in between (the same steps as the
      // forward kernel, so the state reached is bit for bit the same)
      const int k0 = kc - kc % KC;
      float ab[PF][R];
#pragma unroll
      for (int u = 0; u < PF; ++u) {
        const int i = k0 * C_STEPS + u - lane + 1;
        load_row<R>(pr, i, jl, i >= 1 && i <= L1, ab[u]);
      }
      for (int ka = k0; ka < kc; ++ka) {
        float er[NEF];
        {
          const int ie = ka * C_STEPS + lane + 1;
          const bool ok = ein && lane < C_STEPS && ie <= L1;
#pragma unroll
          for (int f = 0; f < NEF; ++f) er[f] = ok ? ein[f * Lm + (ie - 1)] : 0.f;
        }
#pragma unroll 1
        for (int u0 = 0; u0 < C_STEPS; u0 += PF)
#pragma unroll
        for (int u = 0; u < PF; ++u) {
          const int cu = u0 + u;
          const int i = ka * C_STEPS + cu - lane + 1;
          const bool act = (i >= 1) && (i <= L1);
          float xl[NS];
#pragma unroll
          for (int q = 0; q < NS; ++q) xl[q] = __shfl_up_sync(FULL, st.vs[q], 1);
          int xn = __shfl_up_sync(FULL, st.n, 1);
          float ev[NEF];
#pragma unroll
          for (int f = 0; f < NEF; ++f) ev[f] = __shfl_sync(FULL, er[f], cu);
          if (lane == 0) {
#pragma unroll
            for (int q = 0; q < NS; ++q) xl[q] = act ? ev[q] : 0.f;
            xn = act ? __float_as_int(ev[NS]) : 0;
          }
          float xs[R];
          lscores<R>(ab[u], k, nlive, has_dead, xs);
          {
            const int ip = i + PF;
            load_row<R>(pr, ip, jl, ip >= 1 && ip <= L1, ab[u]);
          }
          int et;
          float em[R], rs;
          lcells<NS, R>(st, xl, xn, xs, i >= 1, gO, gE, nlive, has_dead, et, em, rs);
        }
      }
    }
#pragma unroll
    for (int cu = 0; cu < C_STEPS; ++cu) {
      const int t = t0 + cu;
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      float xl[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) xl[q] = __shfl_up_sync(FULL, st.vs[q], 1);
      int xn = __shfl_up_sync(FULL, st.n, 1);
      if (lane == 0) {
        const float4 e4 = s_eb[cu];
        const float ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
        for (int q = 0; q < NS; ++q) xl[q] = act ? ev[q] : 0.f;
        xn = act ? __float_as_int(ev[NS]) : 0;
      }
      float xs[R];
      lscores<R>(nsb[cu], k, nlive, has_dead, xs);
      int et;
      float em[R], rs;
      lcells<NS, R>(st, xl, xn, xs, i >= 1, gO, gE, nlive, has_dead, et, em, rs);
      float* ent = sm + (size_t)cu * FW * 32;
      if constexpr (R % 4 == 0) {
        // field g's R columns as R / 4 float4 per lane: [g][quad][lane][4]
        auto put = [&](int g, const float (&x)[R]) {
#pragma unroll
          for (int h = 0; h < R / 4; ++h)
            reinterpret_cast<float4*>(ent + g * R * 32 + h * 128)[lane] =
                make_float4(x[4 * h], x[4 * h + 1], x[4 * h + 2], x[4 * h + 3]);
        };
        put(0, st.v[0]);
        if constexpr (NS == 3) {
          put(1, st.v[1]);
          put(2, st.v[2]);
        } else {
          put(1, em);
        }
        put(LD::NF - 1, xs);
      } else {
#pragma unroll
        for (int c = 0; c < R; ++c) {
          ent[(0 * R + c) * 32 + lane] = st.v[0][c];
          if constexpr (NS == 3) {
            ent[(1 * R + c) * 32 + lane] = st.v[1][c];
            ent[(2 * R + c) * 32 + lane] = st.v[2][c];
          } else {
            ent[(1 * R + c) * 32 + lane] = em[c];
          }
          ent[((LD::NF - 1) * R + c) * 32 + lane] = xs[c];
        }
      }
      ent[LD::NF * R * 32 + lane] = __int_as_float(et);
      ent[LD::NF * R * 32 + 32 + lane] = __int_as_float(st.n);
    }
    if (kc > 0) {   // prefetch the next chunk's inputs while the outside recursion runs
      load_ck(kc - 1);
      load_eb(kc - 1);
      load_sb(kc - 1);
      load_pb(kc - 1, pbn);
    }
    if (lane < C_STEPS) s_pb[lane] = make_float4(pbc[0], pbc[1], pbc[2], 0.f);
    __syncwarp();
    float cA = 0.f, cB = 0.f, cS = 0.f;   // this chunk's plain sums
    // ---- outside recursion over the chunk, last step first ----
#pragma unroll 1
    for (int cu = 0; cu < C_STEPS; ++cu) {
      const int ent_i = C_STEPS - 1 - cu;
      const int t = t0 + ent_i;
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      const float* ent = sm + (size_t)ent_i * FW * 32;
      // the right neighbour's latest row (row i): beta_D / beta of its column
      // 0, its t and frame; lane 31 takes the right band's record of row i
      float rb = __shfl_down_sync(FULL, o_b, 1);
      float rt = __shfl_down_sync(FULL, o_t, 1);
      int rn = __shfl_down_sync(FULL, o_n, 1);
      if (lane == 31) {   // resolved at the chunk's start (the quiet-chunk test polls them)
        const float4 p4 = s_pb[cu];
        rb = p4.x; rt = p4.y; rn = __float_as_int(p4.z);
      }
      // frames: the row is computed in ft >= every input's normalised frame
      const int ft = max(max(nb, rn), hn);
      const float fBd = p2i(fb - ft), fTd = p2i(nb - ft), fR = p2i(rn - ft), fH = p2i(hn - ft);
      const float st1 = p2i(-ft);
      const int ea = __float_as_int(ent[LD::NF * R * 32 + lane]);
      const int na = __float_as_int(ent[LD::NF * R * 32 + 32 + lane]);
      const float as = p2i(ea - na);                       // raw alpha -> normalised
      const float sc = p2any(na + ft - ze) * invZ; // real alpha * beta / Z factor
      float fa[LD::NF][R];
      if constexpr (R % 4 == 0) {
#pragma unroll
        for (int g = 0; g < LD::NF; ++g)
#pragma unroll
          for (int h = 0; h < R / 4; ++h) {
            const float4 y = reinterpret_cast<const float4*>(ent + g * R * 32 + h * 128)[lane];
            fa[g][4 * h] = y.x; fa[g][4 * h + 1] = y.y; fa[g][4 * h + 2] = y.z; fa[g][4 * h + 3] = y.w;
          }
      } else {
#pragma unroll
        for (int g = 0; g < LD::NF; ++g)
#pragma unroll
          for (int c = 0; c < R; ++c) fa[g][c] = ent[(g * R + c) * 32 + lane];
      }
      const float one = act ? st1 : 0.f;
      // per-row factors folded out of the cells: the frame of the row below
      // (fBd), alpha's normalisation (as) and the posterior scale (sc)
      const float asc = as * sc, gEb = gE * fBd, gOb = gO * fBd;
      float br = fR * rb;   // right successor's beta_D (beta)
      float nbv[R], nmv[R], pm[R], mxv[R];
      float so = 0.f, sxi = 0.f, sxd = 0.f, sp = 0.f;   // sums of raw alpha x beta
#pragma unroll
      for (int c = R - 1; c >= 0; --c) {
        const float oc = c < nlive ? one : 0.f;
        // plus the diagonal successor's t
        const float base = c == R - 1 ? fmaf(fH, ht, oc) : fmaf(fTd, tdn[c + 1], oc);
        const float sr = fmaf(fBd, bdn[c], br);   // beta_I (beta) below + beta_D right
        if constexpr (NS == 3) {
          const float vm = fmaf(gO, sr, base);
          const float vi = fmaf(gEb, bdn[c], base);
          const float vd = fmaf(gE, br, base);
          const float P = fminf((fa[0][c] * asc) * vm, 1.f);   // a posterior: rounding may pass 1
          pm[c] = P;
          so = fmaf(fa[0][c], sr, so);
          sxi = fmaf(fa[1][c], bdn[c], sxi);
          sxd = fmaf(fa[2][c], br, sxd);
          sp = fmaf(P, fa[3][c], sp);
          nbv[c] = vi;
          nmv[c] = vm;
          mxv[c] = fmaf(gX, sr, base);   // >= vm, vi, vd
          br = vd;
        } else {
          const float vb = fmaf(gO, br, fmaf(gOb, bdn[c], base));   // one fma on the column chain
          const float P = fminf((fa[1][c] * asc) * vb, 1.f);
          pm[c] = P;
          so = fmaf(fa[0][c], sr, so);
          sp = fmaf(P, fa[2][c], sp);
          nbv[c] = vb;
          nmv[c] = vb;
          mxv[c] = vb;
          br = vb;
        }
      }
      // normalise: t = E beta_M in the row's normalised frame
#pragma unroll
      for (int h = 1; h < R; h *= 2)   // pairwise maximum: a short dependency chain
#pragma unroll
        for (int c = 0; c + h < R; c += 2 * h) mxv[c] = fmaxf(mxv[c], mxv[c + h]);
      const int nn = max(ft + fexp(mxv[0]), 0);
      const float bs = p2i(ft - nn);
#pragma unroll
      for (int c = 0; c < R; ++c) {
        tdn[c] = (nmv[c] * bs) * ex2(fa[LD::NF - 1][c]);
        bdn[c] = nbv[c];
      }
      fb = ft;
      nb = nn;
      o_b = br * bs;   // column 0's beta_D (beta), normalised
      o_t = tdn[0];
      o_n = nn;
      ht = rt;
      hn = rn;
      if constexpr (NS == 3) {
        cA = fmaf(so * asc, gO, cA);
        cB = fmaf(fmaf(sxi, fBd, sxd) * asc, gE, cB);
      } else {
        cA = fmaf(so * asc, gO, cA);
      }
      cS += sp;
      if (act) {
        store_row<R>(pr, i, jl, pm);
        if (lane == 0 && pout) {
          pout[0 * (Lm + 1) + i] = o_b;
          pout[1 * (Lm + 1) + i] = o_t;
          pout[2 * (Lm + 1) + i] = __int_as_float(o_n);
        }
      }
    }
#pragma unroll
    for (int f = 0; f < NPF; ++f) pbc[f] = pbn[f];
    gA.add(cA);
    gB.add(cB);
    gS.add(cS);
    __syncwarp();
  }
  float v0 = gA.s, v1 = gB.s, v2 = gS.s;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_xor_sync(FULL, v0, o);
    v1 += __shfl_xor_sync(FULL, v1, o);
    v2 += __shfl_xor_sync(FULL, v2, o);
  }
  finish_pair_p<NS>(a, w, lane, Sh, Sl, v0, v1, v2, pp);
}

// Before a separate adjoint launch on a workspace the forward filled: the
// adjoint task counter to 0 and the pairs' completion counts to 0, keeping
// the failure flags the forward set.
__global__ void adjoint_reset_kernel(unsigned* counters, unsigned* pair_done, int B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) counters[1] = 0u;
  if (i < B) pair_done[i] &= PAIR_TIMEOUT;
}

// SPARSE: checkpoints every a.ck_every chunks (the chunks between are
// recomputed); otherwise every chunk (a.ck_every must be 1).
template <int NS, int R, int WARPS, bool SPARSE = false>
__global__ void __launch_bounds__(32 * WARPS) lbwd_kernel(Args a) {
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31;
  const int wi = threadIdx.x >> 5;
  float* sm = smem + (size_t)wi * lbwd_smem_floats<NS, R>();
  const LParams lp = lparams<NS>(a);
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = (a.layout == 0) ? a.B * a.nb : a.ntasks;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 1, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    lbwd_band<NS, R, SPARSE>(a, lp, place_of<NS, R>(a, task, true), lane, sm, deadline);
  }
}

}  // namespace swb
