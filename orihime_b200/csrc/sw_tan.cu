// Second-order ops of the local soft Smith-Waterman models (linear and affine
// gaps) in the scaled linear domain (sm_100a): directional derivatives of the
// marginal map.  Compiled as part of sw_capi.cu after sw_lin.cu, whose frames,
// cell layout, band decomposition and polling this file reuses.
//
// The linear-domain recurrences (sw_lin.cu) are linear in the DP values and
// in the outside values beta, with coefficients E = 2^(s k), G_o, G_e.  Along
// a direction (a score tangent v, or one of gap_open, gap_ext, T) every value
// x therefore has a tangent x' that follows the same recurrence plus source
// terms from the coefficients' own tangents:
//     E' = E e   with e = v / T (score direction) or -s / T^2 (temperature),
//     G' = G g   with g = 1 / T along its own gap, -gap / T^2 along T.
// Forward (per cell, affine; the diagonal sum S = (M + I + D) of (i-1, j-1)):
//     M = E (S + 1),                  M' = E (e (S + 1) + S')
//     I = G_o M^ + G_e I^,            I' = G_o (M^' + g_o M^) + G_e (I^' + g_e I^)
//     D = G_o M< + G_e D<,            D' likewise from the left
//     Z = 1 + sum (M + I + D),        Z' = sum (M' + I' + D')
// Adjoint (beta_M = 1 + t + G_o (b_I below + b_D right), t = E beta_M of the
// diagonal successor):
//     beta_M' = t' + G_o (b' + g_o b),   t' = E (beta_M' + e beta_M), ...
//     P = M beta_M / Z,               P' = (M' beta_M + M beta_M') / Z - P Z' / Z.
// Tangents live in the same power-of-two frame as their values (the
// recurrences are linear), so the frames of sw_lin.cu carry over; a tangent
// is bounded by its value times the largest accumulated |e| or |g| along a
// path, far inside the fp32 range.
//
// The forward kernel writes per band (frame, Z, Z') partials, the tangent
// edge records and per-chunk checkpoints of (values, tangents).  The adjoint
// kernel recomputes each chunk (values and tangents) into shared memory and
// runs the outside recursion and its tangent backwards, writing P' row by row
// (every chunk is computed: no quiet-chunk skip).  Along the score direction
// it also sums the tangents of the parameter gradients (expected transition
// counts) for marginals_backward; dS/dT's tangent then follows from the
// homogeneity of S in (s, gaps, T).
#include "sw_kernels.cuh"

namespace swb {

enum : int { TM_SCORE = 0, TM_G0 = 1, TM_G1 = 2, TM_T = 3 };

#ifndef SWB_TAN
#define SWB_TAN 1   // 0: second-order ops of the local models use the log-domain kernels
#endif

// Relative tangents of the coefficients along the launch's direction:
// d ln G_o = gOd, d ln G_e = gEd, and the emission's d ln E = eT * x with x
// the direction's score tangent (score direction) or the score (temperature).
struct TConst {
  float gOd, gEd, eT;
};
template <int NS, int MODE>
__device__ __forceinline__ TConst tconst(float go, float ge, float T) {
  const float iT = 1.f / T;
  TConst c{0.f, 0.f, 0.f};
  if (MODE == TM_G0) c.gOd = iT;
  if (MODE == TM_G1) c.gEd = iT;
  if (MODE == TM_T) {
    c.gOd = -go * iT * iT;
    c.gEd = NS == 3 ? -ge * iT * iT : 0.f;
    c.eT = -iT * iT;
  }
  if (MODE == TM_SCORE) c.eT = iT;
  return c;
}

// Checkpoint floats per lane (values, tangents, left column of both, three
// frames), edge and push record fields, adjoint shared-memory floats per lane
// and step (affine: M, I, D, their tangents, the scaled score and e; linear:
// A, A', the emission part E (A_diag + 1) and its tangent, the scaled score
// and e; then the two frames).
// An affine record keeps M, I and their tangents but not D and D': restoring
// it rebuilds them from M, M', the left lane's values and tangents and the
// frames with tcells' own operations, bit for bit (28 floats per lane at 4
// columns per lane instead of 36).
template <int NS, int R> struct TDims {
  static constexpr int NSTORE = NS == 3 ? 2 : 1;   // states stored per column
  static constexpr int CKV = 2 * NSTORE * R + 2 * NS + 3;
  static constexpr int CKF = (CKV + 3) / 4 * 4;
  static constexpr int CK4 = CKF / 4;
  static constexpr int LREC = CKF * 32;
  static constexpr int NEF = 2 * NS + 1;
  static constexpr int NPF = 5;   // beta_D (beta), t, frame, and the two tangents
  static constexpr int NF = NS == 3 ? 8 : 6;
  static constexpr int FW = NF * R + 2;
};

template <int NS, int R> struct TState {
  float v[NS][R], w[NS][R];     // raw values and tangents of the lane's latest row (frame e)
  float cs[R], cw[R];           // affine: their column sums (M + I) + D
  float lv[NS], lw[NS];         // the left lane's latest row, last column (frame nl)
  float vs[NS], ws[NS];         // the lane's last column in its normalised frame n
  int e, n, nl;
};

template <int NS, int R>
__device__ __forceinline__ void tstate_sums(TState<NS, R>& s) {
  if constexpr (NS == 3) {
#pragma unroll
    for (int c = 0; c < R; ++c) {
      s.cs[c] = (s.v[0][c] + s.v[1][c]) + s.v[2][c];
      s.cw[c] = (s.w[0][c] + s.w[1][c]) + s.w[2][c];
    }
  }
}

template <int NS, int R>
__device__ __forceinline__ void tstate_zero(TState<NS, R>& s) {
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    s.lv[q] = 0.f; s.lw[q] = 0.f; s.vs[q] = 0.f; s.ws[q] = 0.f;
#pragma unroll
    for (int c = 0; c < R; ++c) { s.v[q][c] = 0.f; s.w[q][c] = 0.f; }
  }
  tstate_sums(s);
  s.e = 0; s.n = 0; s.nl = 0;
}

template <int NS, int R>
__device__ __forceinline__ void tck_store(float* rec, int lane, const TState<NS, R>& s) {
  using D = TDims<NS, R>;
  constexpr int K = D::NSTORE, V = 2 * K * R;   // V: where the left column starts
  float x[D::CKF];
#pragma unroll
  for (int q = 0; q < K; ++q)
#pragma unroll
    for (int c = 0; c < R; ++c) { x[q * R + c] = s.v[q][c]; x[(K + q) * R + c] = s.w[q][c]; }
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    x[V + q] = s.lv[q];
    x[V + NS + q] = s.lw[q];
  }
  x[V + 2 * NS] = __int_as_float(s.e);
  x[V + 2 * NS + 1] = __int_as_float(s.n);
  x[V + 2 * NS + 2] = __int_as_float(s.nl);
#pragma unroll
  for (int f = D::CKV; f < D::CKF; ++f) x[f] = 0.f;
#pragma unroll
  for (int g = 0; g < D::CK4; ++g)
    reinterpret_cast<float4*>(rec + g * 128)[lane] = make_float4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]);
}

// Restores a record.  Affine: D and D' are rebuilt as tcells computed them
// for that row (column 0 from the left lane's values and tangents converted
// to the row's frame, column c > 0 from column c - 1 of M, D and their
// tangents, zero past the pair), with the same operations in the same order.
template <int NS, int R>
__device__ __forceinline__ void tck_restore(const float* rec, int lane, TState<NS, R>& s, float gO,
                                            float gE, const TConst& tc, int nlive, bool has_dead) {
  using D = TDims<NS, R>;
  constexpr int K = D::NSTORE, V = 2 * K * R;
  float x[D::CKF];
#pragma unroll
  for (int g = 0; g < D::CK4; ++g) {
    const float4 y = reinterpret_cast<const float4*>(rec + g * 128)[lane];
    x[4 * g] = y.x; x[4 * g + 1] = y.y; x[4 * g + 2] = y.z; x[4 * g + 3] = y.w;
  }
#pragma unroll
  for (int q = 0; q < K; ++q)
#pragma unroll
    for (int c = 0; c < R; ++c) { s.v[q][c] = x[q * R + c]; s.w[q][c] = x[(K + q) * R + c]; }
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    s.lv[q] = x[V + q];
    s.lw[q] = x[V + NS + q];
  }
  s.e = __float_as_int(x[V + 2 * NS]);
  s.n = __float_as_int(x[V + 2 * NS + 1]);
  s.nl = __float_as_int(x[V + 2 * NS + 2]);
  if constexpr (NS == 3) {
    const float fL = p2i(s.nl - s.e);
    const float gOl = gO * fL, gEl = gE * fL;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      if (c == 0) {
        s.v[2][c] = fmaf(gEl, s.lv[2], gOl * s.lv[0]);
        s.w[2][c] = fmaf(gEl, fmaf(tc.gEd, s.lv[2], s.lw[2]), gOl * fmaf(tc.gOd, s.lv[0], s.lw[0]));
      } else {
        s.v[2][c] = fmaf(gE, s.v[2][c - 1], gO * s.v[0][c - 1]);
        s.w[2][c] = fmaf(gE, fmaf(tc.gEd, s.v[2][c - 1], s.w[2][c - 1]),
                         gO * fmaf(tc.gOd, s.v[0][c - 1], s.w[0][c - 1]));
      }
    }
    if (has_dead) {
#pragma unroll
      for (int c = 0; c < R; ++c)
        if (c >= nlive) { s.v[2][c] = 0.f; s.w[2][c] = 0.f; }
    }
  }
  tstate_sums(s);
  const float f = p2i(s.e - s.n);
#pragma unroll
  for (int q = 0; q < NS; ++q) { s.vs[q] = s.v[q][R - 1] * f; s.ws[q] = s.w[q][R - 1] * f; }
}

// One step of the tangent forward for one lane: (xl, xw, xn) the left lane's
// last column of this row (values, tangents, normalised frame), xs the scaled
// scores (NEG in columns past the pair), xe the emission's relative tangent
// e per column, live false before the lane's first row.  Returns the step's
// frame et and the row's sums of values (rs) and tangents (rw) in frame et;
// linear: em / ed the emission part E (A_diag + 1) and its tangent.
template <int NS, int R>
__device__ __forceinline__ void tcells(TState<NS, R>& s, const float (&xl)[NS], const float (&xw)[NS], int xn,
                                       const float (&xs)[R], const float (&xe)[R], bool live, float gO,
                                       float gE, const TConst& tc, int nlive, bool has_dead, int& et,
                                       float (&em)[R], float (&ed)[R], float& rs, float& rw) {
  const int nd = s.nl;
  float dg[NS], dgw[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    dg[q] = s.lv[q]; dgw[q] = s.lw[q];
    s.lv[q] = xl[q]; s.lw[q] = xw[q];
  }
  s.nl = xn;
  et = max(max(s.n, xn), nd);
  const float fU = p2i(s.e - et), fL = p2i(xn - et), fD = p2i(nd - et), st = live ? p2i(-et) : 0.f;
  float E[R];
#pragma unroll
  for (int c = 0; c < R; ++c) E[c] = ex2(xs[c]);
  if constexpr (NS == 3) {
    const float gOu = gO * fU, gEu = gE * fU, gOl = gO * fL, gEl = gE * fL;
    float pS = (dg[0] + dg[1]) + dg[2], pW = (dgw[0] + dgw[1]) + dgw[2], fP = fD;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const float oM = s.v[0][c], oI = s.v[1][c], oMw = s.w[0][c], oIw = s.w[1][c];
      const float dS = fmaf(fP, pS, st);
      const float m = E[c] * dS;
      const float mw = E[c] * fmaf(xe[c], dS, fP * pW);
      const float iv = fmaf(gOu, oM, gEu * oI);
      const float iw = fmaf(gOu, fmaf(tc.gOd, oM, oMw), gEu * fmaf(tc.gEd, oI, oIw));
      float dv, dw;
      if (c == 0) {
        dv = fmaf(gEl, s.lv[2], gOl * s.lv[0]);
        dw = fmaf(gEl, fmaf(tc.gEd, s.lv[2], s.lw[2]), gOl * fmaf(tc.gOd, s.lv[0], s.lw[0]));
      } else {
        dv = fmaf(gE, s.v[2][c - 1], gO * s.v[0][c - 1]);
        dw = fmaf(gE, fmaf(tc.gEd, s.v[2][c - 1], s.w[2][c - 1]),
                  gO * fmaf(tc.gOd, s.v[0][c - 1], s.w[0][c - 1]));
      }
      s.v[0][c] = m; s.v[1][c] = iv; s.v[2][c] = dv;
      s.w[0][c] = mw; s.w[1][c] = iw; s.w[2][c] = dw;
      pS = s.cs[c]; pW = s.cw[c]; fP = fU;   // the previous row's sums: column c + 1's diagonal
      em[c] = 0.f; ed[c] = 0.f;
    }
    if (has_dead) {
#pragma unroll
      for (int c = 0; c < R; ++c)
        if (c >= nlive) { s.v[2][c] = 0.f; s.w[2][c] = 0.f; }
    }
  } else {
    const float gU = gO * fU, gL = gO * fL;
    float pA = dg[0], pAw = dgw[0], fP = fD;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const float oA = s.v[0][c], oAw = s.w[0][c];
      const float dS = fmaf(fP, pA, st);
      const float m = E[c] * dS;
      const float mw = E[c] * fmaf(xe[c], dS, fP * pAw);
      const float left = c == 0 ? gL * s.lv[0] : gO * s.v[0][c - 1];
      const float leftw = c == 0 ? gL * fmaf(tc.gOd, s.lv[0], s.lw[0])
                                 : gO * fmaf(tc.gOd, s.v[0][c - 1], s.w[0][c - 1]);
      s.v[0][c] = fmaf(gU, oA, m + left);
      s.w[0][c] = fmaf(gU, fmaf(tc.gOd, oA, oAw), mw + leftw);
      em[c] = m; ed[c] = mw;
      pA = oA; pAw = oAw; fP = fU;
    }
    if (has_dead) {
#pragma unroll
      for (int c = 0; c < R; ++c)
        if (c >= nlive) { s.v[0][c] = 0.f; s.w[0][c] = 0.f; em[c] = 0.f; ed[c] = 0.f; }
    }
  }
  tstate_sums(s);
  float cs[R], cw[R];
#pragma unroll
  for (int c = 0; c < R; ++c) {
    cs[c] = NS == 3 ? s.cs[c] : s.v[0][c];
    cw[c] = NS == 3 ? s.cw[c] : s.w[0][c];
  }
#pragma unroll
  for (int h = 1; h < R; h *= 2)
#pragma unroll
    for (int c = 0; c + h < R; c += 2 * h) { cs[c] += cs[c + h]; cw[c] += cw[c + h]; }
  rs = cs[0];
  rw = cw[0];
  s.e = et;
  s.n = max(et + fexp(rs), 0);
  const float f = p2i(et - s.n);
#pragma unroll
  for (int q = 0; q < NS; ++q) { s.vs[q] = s.v[q][R - 1] * f; s.ws[q] = s.w[q][R - 1] * f; }
}

// The emission's relative tangent per column: the direction's score tangent
// (score direction) or the score itself (temperature), times eT; 0 along a gap.
template <int R, int MODE>
__device__ __forceinline__ void temission(const float (&sb)[R], const float (&vb)[R], const TConst& tc,
                                          float (&xe)[R]) {
#pragma unroll
  for (int c = 0; c < R; ++c)
    xe[c] = MODE == TM_SCORE ? vb[c] * tc.eT : (MODE == TM_T ? sb[c] * tc.eT : 0.f);
}

// Where a band task of the tangent kernels lives (padded batches only).
template <int NS, int R>
__device__ __forceinline__ Place tplace(const Args& a, int task, bool reverse_band) {
  using D = TDims<NS, R>;
  Place w;
  Pair& r = w.pr;
  const int p = task / a.nb;
  const int j = task - p * a.nb;
  w.p = p;
  w.nb = a.nb;
  w.band = reverse_band ? a.nb - 1 - j : j;
  w.slot0 = (size_t)p * a.nb;
  w.Lm = a.Lmax1;
  w.ckb = (size_t)a.nchunks * D::LREC;
  w.edb = (size_t)D::NEF * a.Lmax1;
  w.bpb = (size_t)D::NPF * (a.Lmax1 + 1);
  w.ck0 = w.slot0 * w.ckb;
  w.ed0 = w.slot0 * w.edb;
  w.bp0 = w.slot0 * w.bpb;
  const size_t base = (size_t)p * a.Lmax1 * a.Lmax2;
  r.s = a.scores + base;
  r.m = a.map + base;
  r.ld = a.Lmax2;
  if (a.lengths) {
    r.L1 = min(max(a.lengths[2 * p], 0), a.Lmax1);
    r.L2 = min(max(a.lengths[2 * p + 1], 0), a.Lmax2);
  } else {
    r.L1 = a.Lmax1;
    r.L2 = a.Lmax2;
  }
  r.vec = ((r.ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(r.s) & 15) == 0) &&
          ((reinterpret_cast<uintptr_t>(r.m) & 15) == 0);
  return w;
}

// The direction rows of a pair (score direction): the same offsets in a.tdir.
__device__ __forceinline__ Pair tdir_pair(const Args& a, const Pair& pr) {
  Pair q = pr;
  q.s = a.tdir + (pr.s - a.scores);
  q.vec = pr.vec && ((reinterpret_cast<uintptr_t>(q.s) & 15) == 0);
  return q;
}

// ---------------------------------------------------------------------------
// tangent forward band task
// ---------------------------------------------------------------------------
template <int NS, int R, int MODE>
__device__ void ltfwd_band(const Args& a, const LParams& lp, const TConst& tc, const Place& w, int lane,
                           uint64_t deadline) {
  using D = TDims<NS, R>;
  constexpr int NEF = D::NEF;
  check_lengths(a, w, lane);
  const Pair& pr = w.pr;
  const int L1 = pr.L1, L2 = pr.L2;
  const int band = w.band;
  const size_t slot = w.slot0 + band;
  const int col0 = band * 32 * R;
  float* part = a.part + 2 * slot;
  float* zd = a.zdot + 2 * slot;
  if (!(L1 > 0 && col0 < L2)) {
    if (lane == 0) {
      part[0] = 0.f; part[1] = (band == 0) ? 1.f : 0.f;
      zd[0] = 0.f; zd[1] = 0.f;
    }
    return;
  }
  const int jl = col0 + lane * R;
  const int nlive = min(max(L2 - jl, 0), R);
  const bool has_dead = __any_sync(FULL, nlive < R);
  const float k = lp.k, gO = lp.xgo, gE = lp.xge;
  const size_t Lm = (size_t)w.Lm;
  float* eout = a.edge + w.ed0 + (size_t)band * w.edb;
  const float* ein = (band > 0) ? eout - w.edb : nullptr;
  float* ck = a.ckpt + w.ck0 + (size_t)band * w.ckb;
  const int nch = band_chunks(L1);
  const Pair pv = MODE == TM_SCORE ? tdir_pair(a, pr) : pr;

  TState<NS, R> s;
  tstate_zero(s);
  float zm = (band == 0 && lane == 0) ? 1.f : 0.f, zc = 0.f, zw = 0.f, zwc = 0.f;
  int ze = 0;

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
  constexpr int VR = MODE == TM_SCORE ? FPF : 1;
  float sb[FPF][R], vb[VR][R];
#pragma unroll
  for (int u = 0; u < FPF; ++u) {
    const int i = u - lane + 1;
    load_row<R>(pr, i, jl, i >= 1 && i <= L1, sb[u]);
    if constexpr (MODE == TM_SCORE) load_row<R>(pv, i, jl, i >= 1 && i <= L1, vb[u]);
  }

  for (int kc = 0; kc < nch; ++kc) {
    {   // this chunk's edge records (bounded waits, as the first-order forward)
      const int ie = kc * C_STEPS + lane + 1;
      const bool mine = lane < C_STEPS && ie <= L1;
      bool miss = false;
#pragma unroll
      for (int f = 0; f < NEF; ++f) miss |= is_sentinel(eb[f]);
      miss = miss && ein && mine;
      if (__any_sync(FULL, miss) && miss) {
        FieldVec<NEF> x;
#pragma unroll
        for (int f = 0; f < NEF; ++f) x.v[f] = eb[f];
        x = poll_fields_v<NEF, 0>(x, ein + (ie - 1), Lm, deadline, a.status, a.pair_done + w.p);
#pragma unroll
        for (int f = 0; f < NEF; ++f) eb[f] = x.v[f];
      }
    }
    tck_store<NS, R>(ck + (size_t)kc * D::LREC, lane, s);
    if (kc + 1 < nch) load_edge(kc + 1, ebn);
#pragma unroll 1
    for (int u0 = 0; u0 < C_STEPS; u0 += FPF)
#pragma unroll
    for (int u = 0; u < FPF; ++u) {
      const int cu = u0 + u;
      const int t = kc * C_STEPS + cu;
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      float xl[NS], xw[NS], ev[NEF];
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        xl[q] = __shfl_up_sync(FULL, s.vs[q], 1);
        xw[q] = __shfl_up_sync(FULL, s.ws[q], 1);
      }
      int xn = __shfl_up_sync(FULL, s.n, 1);
#pragma unroll
      for (int f = 0; f < NEF; ++f) ev[f] = __shfl_sync(FULL, eb[f], cu);
      if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          xl[q] = act ? ev[q] : 0.f;
          xw[q] = act ? ev[NS + q] : 0.f;
        }
        xn = act ? __float_as_int(ev[2 * NS]) : 0;
      }
      float xs[R], xe[R];
      lscores<R>(sb[u], k, nlive, has_dead, xs);
      temission<R, MODE>(sb[u], vb[MODE == TM_SCORE ? u : 0], tc, xe);
      {
        const int ip = i + FPF;
        load_row<R>(pr, ip, jl, ip >= 1 && ip <= L1, sb[u]);
        if constexpr (MODE == TM_SCORE) load_row<R>(pv, ip, jl, ip >= 1 && ip <= L1, vb[u]);
      }
      int et;
      float em[R], ed[R], rs, rw;
      tcells<NS, R>(s, xl, xw, xn, xs, xe, i >= 1, gO, gE, tc, nlive, has_dead, et, em, ed, rs, rw);
      if (act) {
        if (s.n > ze) {
          const float f = p2i(ze - s.n);
          zm *= f; zc *= f; zw *= f; zwc *= f; ze = s.n;
        }
        const float g = p2i(et - ze);
        {
          const float y = rs * g - zc;
          const float tt = zm + y;
          zc = (tt - zm) - y;
          zm = tt;
        }
        {
          const float y = rw * g - zwc;
          const float tt = zw + y;
          zwc = (tt - zw) - y;
          zw = tt;
        }
        if (lane == 31) {
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            eout[q * Lm + (i - 1)] = s.vs[q];
            eout[(NS + q) * Lm + (i - 1)] = s.ws[q];
          }
          eout[2 * NS * Lm + (i - 1)] = __int_as_float(s.n);
        }
      }
    }
#pragma unroll
    for (int f = 0; f < NEF; ++f) eb[f] = ebn[f];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int z2 = __shfl_xor_sync(FULL, ze, o);
    const float m2 = __shfl_xor_sync(FULL, zm, o);
    const float w2 = __shfl_xor_sync(FULL, zw, o);
    const int m = max(ze, z2);
    const float fa = p2i(ze - m), fb = p2i(z2 - m);
    zm = zm * fa + m2 * fb;
    zw = zw * fa + w2 * fb;
    ze = m;
  }
  if (lane == 0) {
    part[0] = (float)ze; part[1] = zm;
    zd[0] = (float)ze; zd[1] = zw;
  }
}

template <int NS, int R, int MODE>
__global__ void __launch_bounds__(128) ltfwd_kernel(Args a) {
  const int lane = threadIdx.x & 31;
  const LParams lp = lparams<NS>(a);
  const TConst tc = tconst<NS, MODE>(lp.go, lp.ge, lp.T);
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = a.B * a.nb;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 0, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    ltfwd_band<NS, R, MODE>(a, lp, tc, tplace<NS, R>(a, task, false), lane, deadline);
  }
}

// ---------------------------------------------------------------------------
// tangent adjoint band task
// ---------------------------------------------------------------------------

template <int NS, int R>
__host__ __device__ constexpr int ltbwd_smem_floats() {
  return (C_STEPS * TDims<NS, R>::FW) * 32;
}

// Z' / Z of pair w from the band partials (frame, Z') and Z's frame ze.
__device__ __forceinline__ float tpair_zrel(const Args& a, const Place& w, int lane, int ze, float zm) {
  float s = 0.f;
  for (int b = lane; b < w.nb; b += 32) {
    const float* q = a.zdot + 2 * (w.slot0 + b);
    s += q[1] * p2i((int)q[0] - ze);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
  return s / zm;
}

// The last band of a pair to finish folds the bands' partial sums (in band
// order) into the pair's parameter tangents (score direction with tgt), or
// fills the pair's map with NaN when one of its bounded waits expired.
template <int NS>
__device__ void tfinish(const Args& a, const Place& w, int lane, const float (&sums)[5], float zz,
                        bool empty, const LParams& lp) {
  const int p = w.p;
  const bool tangents = a.tmode == TM_SCORE && a.tgt;
  unsigned done = 0;
  if (lane == 0) {
    if (tangents) {
      float* gp = a.gpart + 8 * (w.slot0 + w.band);
#pragma unroll
      for (int f = 0; f < 5; ++f) gp[f] = sums[f];
      __threadfence();
    }
    done = atomicAdd(a.pair_done + p, 1u);
  }
  done = __shfl_sync(FULL, done, 0);
  if ((done & ~PAIR_TIMEOUT) != (unsigned)w.nb - 1) return;
  if (done & PAIR_TIMEOUT) {
    const float nan = __int_as_float(0x7fc00000);
    const Pair& pr = w.pr;
    for (int i = 0; i < pr.L1; ++i)
      for (int j = lane; j < pr.L2; j += 32) pr.m[(size_t)i * pr.ld + j] = nan;
    if (tangents && lane < 4) a.tgt[4 * p + lane] = nan;
    return;
  }
  if (!tangents || lane != 0) return;
  __threadfence();
  float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int b = 0; b < w.nb; ++b) {
    const float* q = a.gpart + 8 * (w.slot0 + b);
#pragma unroll
    for (int f = 0; f < 5; ++f) s[f] += ld_poll(q + f);
  }
  float* g = a.tgt + 4 * p;
  if (empty) {
    g[0] = 0.f; g[1] = 0.f; g[2] = 0.f; g[3] = 0.f;
    return;
  }
  // s: g_o, its tangent, g_e, its tangent, sum (P' s + P v); the tangent of
  // g_theta is its summed tangent minus g_theta Z'/Z
  const float dS = lp.T * zz;
  const float go_t = s[1] - s[0] * zz;
  const float ge_t = s[3] - s[2] * zz;
  const float gT_t = (dS - s[4] - (NS == 3 ? lp.go * go_t + lp.ge * ge_t : lp.go * go_t)) / lp.T;
  g[0] = go_t;
  g[1] = NS == 3 ? ge_t : gT_t;
  g[2] = NS == 3 ? gT_t : 0.f;
  g[3] = dS;
}

template <int NS, int R, int MODE>
__device__ void ltbwd_band(const Args& a, const LParams& lp, const TConst& tc, const Place& w, int lane,
                           float* sm, uint64_t deadline) {
  using D = TDims<NS, R>;
  constexpr int NEF = D::NEF, NPF = D::NPF, NF = D::NF, FW = D::FW;
  constexpr int FX = NF - 2, FE = NF - 1;   // fields of the scaled score and of e
  const Pair& pr = w.pr;
  const int L1 = pr.L1, L2 = pr.L2;
  const int band = w.band;
  const int col0 = band * 32 * R;
  int ze;
  float zm;
  lpair_z(a, w, lane, ze, zm);
  const float zz = tpair_zrel(a, w, lane, ze, zm);
  float sums[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  if (!(L1 > 0 && col0 < L2)) {
    tfinish<NS>(a, w, lane, sums, zz, L1 == 0 || L2 == 0, lp);
    return;
  }
  const float invZ = 1.f / zm;
  const int jl = col0 + lane * R;
  const int nlive = min(max(L2 - jl, 0), R);
  const bool has_dead = __any_sync(FULL, nlive < R);
  const float k = lp.k, gO = lp.xgo, gE = lp.xge, gX = fmaxf(gO, gE);
  const float inv_k = 1.f / k;
  const size_t Lm = (size_t)w.Lm;
  const float* ein = (band > 0) ? a.edge + w.ed0 + (size_t)(band - 1) * w.edb : nullptr;
  float* pout = (band > 0) ? a.bpush + w.bp0 + (size_t)band * w.bpb : nullptr;
  const bool right_live = (col0 + 32 * R) < L2 && (band + 1) < w.nb;
  const float* pin = right_live ? a.bpush + w.bp0 + (size_t)(band + 1) * w.bpb : nullptr;
  const float* ck = a.ckpt + w.ck0 + (size_t)band * w.ckb;
  const int nch = band_chunks(L1);
  const Pair pv = MODE == TM_SCORE ? tdir_pair(a, pr) : pr;

  // outside-recursion state: the row below (beta_I / beta and tangent in frame
  // fb; t and tangent in frame nb), the right neighbour's held t (frame hn)
  // and this lane's outputs of its latest row
  float bdn[R], bdw[R], tdn[R], tdw[R];
#pragma unroll
  for (int c = 0; c < R; ++c) { bdn[c] = 0.f; bdw[c] = 0.f; tdn[c] = 0.f; tdw[c] = 0.f; }
  int fb = 0, nb = 0, hn = 0, o_n = 0;
  float ht = 0.f, htw = 0.f, o_b = 0.f, o_bw = 0.f, o_t = 0.f, o_tw = 0.f;
  float cA = 0.f, cAd = 0.f, cB = 0.f, cBd = 0.f, cC = 0.f;

  for (int kc = nch - 1; kc >= 0; --kc) {
    const int t0 = kc * C_STEPS;
    // the right band's push records lane 31 needs at backward step u (lane u)
    float pbc[NPF];
    {
      const int ir = t0 + C_STEPS - 1 - lane - 30;
      const bool ok = pin && lane < C_STEPS && ir >= 1 && ir <= L1;
#pragma unroll
      for (int f = 0; f < NPF; ++f) pbc[f] = ok ? ld_poll(pin + f * (Lm + 1) + ir) : 0.f;
      bool miss = false;
#pragma unroll
      for (int f = 0; f < NPF; ++f) miss |= is_sentinel(pbc[f]);
      if (__any_sync(FULL, miss) && miss) {
        FieldVec<NPF> x;
#pragma unroll
        for (int f = 0; f < NPF; ++f) x.v[f] = pbc[f];
        x = poll_fields_v<NPF, 0>(x, pin + ir, Lm + 1, deadline, a.status, a.pair_done + w.p);
#pragma unroll
        for (int f = 0; f < NPF; ++f) pbc[f] = x.v[f];
      }
    }
    // this chunk's left-band edge records for lane 0 (written by the forward)
    float ebr[NEF];
    {
      const int ie = t0 + lane + 1;
      const bool ok = ein && lane < C_STEPS && ie <= L1;
#pragma unroll
      for (int f = 0; f < NEF; ++f) ebr[f] = ok ? ein[f * Lm + (ie - 1)] : 0.f;
    }
    // ---- restore and recompute the chunk (values and tangents) ----
    {
      TState<NS, R> st;
      tck_restore<NS, R>(ck + (size_t)kc * D::LREC, lane, st, gO, gE, tc, nlive, has_dead);
#pragma unroll
      for (int cu = 0; cu < C_STEPS; ++cu) {
        const int i = t0 + cu - lane + 1;
        const bool act = (i >= 1) && (i <= L1);
        float xl[NS], xw[NS], ev[NEF];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          xl[q] = __shfl_up_sync(FULL, st.vs[q], 1);
          xw[q] = __shfl_up_sync(FULL, st.ws[q], 1);
        }
        int xn = __shfl_up_sync(FULL, st.n, 1);
#pragma unroll
        for (int f = 0; f < NEF; ++f) ev[f] = __shfl_sync(FULL, ebr[f], cu);
        if (lane == 0) {
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            xl[q] = act ? ev[q] : 0.f;
            xw[q] = act ? ev[NS + q] : 0.f;
          }
          xn = act ? __float_as_int(ev[2 * NS]) : 0;
        }
        float sbr[R], vbr[R], xs[R], xe[R];
        load_row<R>(pr, i, jl, act, sbr);
        if constexpr (MODE == TM_SCORE) load_row<R>(pv, i, jl, act, vbr);
        else {
#pragma unroll
          for (int c = 0; c < R; ++c) vbr[c] = 0.f;
        }
        lscores<R>(sbr, k, nlive, has_dead, xs);
        temission<R, MODE>(sbr, vbr, tc, xe);
        int et;
        float em[R], ed[R], rs, rw;
        tcells<NS, R>(st, xl, xw, xn, xs, xe, i >= 1, gO, gE, tc, nlive, has_dead, et, em, ed, rs, rw);
        float* ent = sm + (size_t)cu * FW * 32;
#pragma unroll
        for (int c = 0; c < R; ++c) {
          if constexpr (NS == 3) {
            ent[(0 * R + c) * 32 + lane] = st.v[0][c];
            ent[(1 * R + c) * 32 + lane] = st.v[1][c];
            ent[(2 * R + c) * 32 + lane] = st.v[2][c];
            ent[(3 * R + c) * 32 + lane] = st.w[0][c];
            ent[(4 * R + c) * 32 + lane] = st.w[1][c];
            ent[(5 * R + c) * 32 + lane] = st.w[2][c];
          } else {
            ent[(0 * R + c) * 32 + lane] = st.v[0][c];
            ent[(1 * R + c) * 32 + lane] = st.w[0][c];
            ent[(2 * R + c) * 32 + lane] = em[c];
            ent[(3 * R + c) * 32 + lane] = ed[c];
          }
          ent[(FX * R + c) * 32 + lane] = xs[c];
          ent[(FE * R + c) * 32 + lane] = xe[c];
        }
        ent[NF * R * 32 + lane] = __int_as_float(et);
        ent[NF * R * 32 + 32 + lane] = __int_as_float(st.n);
      }
    }
    __syncwarp();
    // ---- outside recursion and its tangent over the chunk, last step first ----
#pragma unroll 1
    for (int cu = 0; cu < C_STEPS; ++cu) {
      const int ent_i = C_STEPS - 1 - cu;
      const int i = t0 + ent_i - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      const float* ent = sm + (size_t)ent_i * FW * 32;
      float rb = __shfl_down_sync(FULL, o_b, 1);
      float rbw = __shfl_down_sync(FULL, o_bw, 1);
      float rt = __shfl_down_sync(FULL, o_t, 1);
      float rtw = __shfl_down_sync(FULL, o_tw, 1);
      int rn = __shfl_down_sync(FULL, o_n, 1);
      {
        float pw[NPF];
#pragma unroll
        for (int f = 0; f < NPF; ++f) pw[f] = __shfl_sync(FULL, pbc[f], cu);
        if (lane == 31) { rb = pw[0]; rt = pw[1]; rn = __float_as_int(pw[2]); rbw = pw[3]; rtw = pw[4]; }
      }
      const int ft = max(max(nb, rn), hn);
      const float fBd = p2i(fb - ft), fTd = p2i(nb - ft), fR = p2i(rn - ft), fH = p2i(hn - ft);
      const float st1 = p2i(-ft);
      const int ea = __float_as_int(ent[NF * R * 32 + lane]);
      const int na = __float_as_int(ent[NF * R * 32 + 32 + lane]);
      const float as = p2i(ea - na);
      const float sc = p2any(na + ft - ze) * invZ;
      float fa[NF][R];
#pragma unroll
      for (int g = 0; g < NF; ++g)
#pragma unroll
        for (int c = 0; c < R; ++c) fa[g][c] = ent[(g * R + c) * 32 + lane];
      const float one = act ? st1 : 0.f;
      float br = fR * rb, brw = fR * rbw;
      float nbv[R], nbw[R], nmv[R], nmw[R], pd[R], mxv[R];
      float so = 0.f, sow = 0.f, sx = 0.f, sxw = 0.f, cc = 0.f;
#pragma unroll
      for (int c = R - 1; c >= 0; --c) {
        const float oc = c < nlive ? one : 0.f;
        const float td = c == R - 1 ? fH * ht : fTd * tdn[c + 1 < R ? c + 1 : 0];
        const float tw = c == R - 1 ? fH * htw : fTd * tdw[c + 1 < R ? c + 1 : 0];
        const float base = oc + td;
        const float bd = fBd * bdn[c], bdt = fBd * bdw[c];
        const float sr = bd + br, srw = bdt + brw;
        if constexpr (NS == 3) {
          const float vm = fmaf(gO, sr, base);
          const float vmw = fmaf(gO, fmaf(tc.gOd, sr, srw), tw);
          const float vi = fmaf(gE, bd, base);
          const float viw = fmaf(gE, fmaf(tc.gEd, bd, bdt), tw);
          const float vd = fmaf(gE, br, base);
          const float vdw = fmaf(gE, fmaf(tc.gEd, br, brw), tw);
          const float am = fa[0][c] * as, ai = fa[1][c] * as, ad = fa[2][c] * as;
          const float amw = fa[3][c] * as, aiw = fa[4][c] * as, adw = fa[5][c] * as;
          const float P = (am * sc) * vm;
          const float Pd = fmaf(sc, fmaf(amw, vm, am * vmw), -P * zz);
          pd[c] = Pd;
          so = fmaf(am, sr, so);
          sow = fmaf(amw, sr, fmaf(am, srw, sow));
          sx = fmaf(ai, bd, fmaf(ad, br, sx));
          sxw = fmaf(aiw, bd, fmaf(ai, bdt, fmaf(adw, br, fmaf(ad, brw, sxw))));
          cc = fmaf(Pd, fa[FX][c] * inv_k, fmaf(P * lp.T, fa[FE][c], cc));
          nbv[c] = vi; nbw[c] = viw;
          nmv[c] = vm; nmw[c] = vmw;
          mxv[c] = fmaf(gX, sr, base);
          br = vd; brw = vdw;
        } else {
          const float vb = fmaf(gO, sr, base);
          const float vbw = fmaf(gO, fmaf(tc.gOd, sr, srw), tw);
          const float A = fa[0][c] * as, Aw = fa[1][c] * as;
          const float em = fa[2][c] * as, emw = fa[3][c] * as;
          const float P = (em * sc) * vb;
          const float Pd = fmaf(sc, fmaf(emw, vb, em * vbw), -P * zz);
          pd[c] = Pd;
          so = fmaf(A, sr, so);
          sow = fmaf(Aw, sr, fmaf(A, srw, sow));
          cc = fmaf(Pd, fa[FX][c] * inv_k, fmaf(P * lp.T, fa[FE][c], cc));
          nbv[c] = vb; nbw[c] = vbw;
          nmv[c] = vb; nmw[c] = vbw;
          mxv[c] = vb;
          br = vb; brw = vbw;
        }
      }
#pragma unroll
      for (int h = 1; h < R; h *= 2)
#pragma unroll
        for (int c = 0; c + h < R; c += 2 * h) mxv[c] = fmaxf(mxv[c], mxv[c + h]);
      const int nn = max(ft + fexp(mxv[0]), 0);
      const float bs = p2i(ft - nn);
#pragma unroll
      for (int c = 0; c < R; ++c) {
        const float E = ex2(fa[FX][c]);
        tdn[c] = (nmv[c] * bs) * E;
        tdw[c] = (fmaf(fa[FE][c], nmv[c], nmw[c]) * bs) * E;   // t' = E (beta_M' + e beta_M)
        bdn[c] = nbv[c];
        bdw[c] = nbw[c];
      }
      fb = ft;
      nb = nn;
      o_b = br * bs; o_bw = brw * bs;
      o_t = tdn[0]; o_tw = tdw[0];
      o_n = nn;
      ht = rt; htw = rtw; hn = rn;
      if (MODE == TM_SCORE && a.tgt) {
        cA = fmaf(so * sc, gO, cA);
        cAd = fmaf(fmaf(tc.gOd, so, sow) * sc, gO, cAd);
        if constexpr (NS == 3) {
          cB = fmaf(sx * sc, gE, cB);
          cBd = fmaf(fmaf(tc.gEd, sx, sxw) * sc, gE, cBd);
        }
        cC += cc;
      }
      if (act) {
        store_row<R>(pr, i, jl, pd);
        if (lane == 0 && pout) {
          pout[0 * (Lm + 1) + i] = o_b;
          pout[1 * (Lm + 1) + i] = o_t;
          pout[2 * (Lm + 1) + i] = __int_as_float(o_n);
          pout[3 * (Lm + 1) + i] = o_bw;
          pout[4 * (Lm + 1) + i] = o_tw;
        }
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cA += __shfl_xor_sync(FULL, cA, o);
    cAd += __shfl_xor_sync(FULL, cAd, o);
    cB += __shfl_xor_sync(FULL, cB, o);
    cBd += __shfl_xor_sync(FULL, cBd, o);
    cC += __shfl_xor_sync(FULL, cC, o);
  }
  sums[0] = cA; sums[1] = cAd; sums[2] = cB; sums[3] = cBd; sums[4] = cC;
  tfinish<NS>(a, w, lane, sums, zz, false, lp);
}

template <int NS, int R, int MODE>
__global__ void __launch_bounds__(32) ltbwd_kernel(Args a) {
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31;
  const LParams lp = lparams<NS>(a);
  const TConst tc = tconst<NS, MODE>(lp.go, lp.ge, lp.T);
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = a.B * a.nb;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 1, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    ltbwd_band<NS, R, MODE>(a, lp, tc, tplace<NS, R>(a, task, true), lane, smem, deadline);
  }
}

}  // namespace swb
