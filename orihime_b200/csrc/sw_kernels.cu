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
// becomes m' + lg2(sum ex2(v'-m')), and its softmax weight of a predecessor
// is ex2(pred' + edge' - cell'), which is what the adjoint uses.
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

// Bounded wait until *p is not the sentinel.  On timeout records the error and
// returns `fallback`.
__device__ __noinline__ float poll_value(const float* p, float v, uint64_t deadline,
                                         unsigned* status, float fallback) {
  while (is_sentinel(v)) {
    if (gtimer() > deadline) {
      atomicOr(status, ERR_WAIT_TIMEOUT);
      return fallback;
    }
    __nanosleep(128);
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

__device__ __forceinline__ Pair pair_of(const Args& a, int p) {
  Pair r;
  if (a.layout == 0) {
    size_t base = (size_t)p * a.Lmax1 * a.Lmax2;
    r.s = a.scores + base;
    r.m = a.map + base;
    r.ld = a.Lmax2;
  } else {
    long long off = a.offsets[p];
    r.s = a.scores + off;
    r.m = a.map + off;
  }
  if (a.lengths) {
    r.L1 = a.lengths[2 * p];
    r.L2 = a.lengths[2 * p + 1];
    if (a.layout == 0) {  // never index outside the padded slab
      r.L1 = min(max(r.L1, 0), a.Lmax1);
      r.L2 = min(max(r.L2, 0), a.Lmax2);
    }
  } else {
    r.L1 = a.Lmax1;
    r.L2 = a.Lmax2;
  }
  if (a.layout == 1) r.ld = (r.L2 + 3) & ~3;
  r.vec = ((r.ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(r.s) & 15) == 0) &&
          ((reinterpret_cast<uintptr_t>(r.m) & 15) == 0);
  return r;
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
  if (R == 4 && pr.vec && jl + 4 <= pr.L2) {
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

template <int R>
__device__ __forceinline__ void store_row(const Pair& pr, int i, int jl, const float (&v)[R]) {
  float* dst = pr.m + (size_t)(i - 1) * pr.ld + jl;
  if (R == 4 && pr.vec && jl + 4 <= pr.L2) {
    *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
  } else if (R == 2 && pr.vec && jl + 2 <= pr.L2) {
    *reinterpret_cast<float2*>(dst) = make_float2(v[0], v[1]);
  } else {
#pragma unroll
    for (int c = 0; c < R; ++c)
      if (jl + c < pr.L2) dst[c] = v[c];
  }
}

// Number of values crossing a band edge forward (NS) and pushes crossing it
// backward (NP), checkpoint fields per lane (CKF) and shared-memory fields per
// lane per recomputed step (EF).
template <int NS> struct Shape;
template <> struct Shape<3> { static constexpr int NP = 5; };
template <> struct Shape<1> { static constexpr int NP = 2; };

template <int NS, int R> struct Dims {
  static constexpr int NP = Shape<NS>::NP;
  static constexpr int CKF = NS * R + NS;
  static constexpr int EF = NS * R + NS + R;
};

// ---------------------------------------------------------------------------
// forward cell
// ---------------------------------------------------------------------------

// One step of the forward wavefront for one lane: consumes the previous-row
// values pv, the left values of this row lf (already received), the diag
// values dg of column 0 (left lane, previous row) and the scaled scores s.
// Writes the new row into pv when act.  Returns per-column new values in nv.
template <int NS, int R>
__device__ __forceinline__ void fwd_cells(float (&pv)[NS][R], const float (&lf)[NS],
                                          const float (&dg0)[NS], const float (&s)[R],
                                          float g0, float g1, bool act, float (&nv)[NS][R]) {
  float dg[NS], left[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) { dg[q] = dg0[q]; left[q] = lf[q]; }
#pragma unroll
  for (int c = 0; c < R; ++c) {
    if constexpr (NS == 3) {
      const float upM = pv[0][c], upI = pv[1][c], upD = pv[2][c];
      // M = s + LSE(M, I, D at diag, 0)
      float mx = fmaxf(fmaxf(dg[0], dg[1]), fmaxf(dg[2], 0.f));
      float sm = ex2(dg[0] - mx) + ex2(dg[1] - mx) + ex2(dg[2] - mx) + ex2(-mx);
      float M = s[c] + (mx + lg2(sm));
      // I = LSE(M up + go, I up + ge)
      float ia = upM + g0, ib = upI + g1;
      float im = fmaxf(ia, ib);
      float I = im + lg2(1.f + ex2(fminf(ia, ib) - im));
      // D = LSE(M left + go, D left + ge)
      float da = left[0] + g0, db = left[2] + g1;
      float dm = fmaxf(da, db);
      float D = dm + lg2(1.f + ex2(fminf(da, db) - dm));
      nv[0][c] = M; nv[1][c] = I; nv[2][c] = D;
      dg[0] = upM; dg[1] = upI; dg[2] = upD;
      left[0] = M; left[1] = I; left[2] = D;
    } else {
      const float up = pv[0][c];
      // A = LSE(diag + s, up + g, left + g, s)
      float va = dg[0] + s[c], vu = up + g0, vl = left[0] + g0, vs = s[c];
      float mx = fmaxf(fmaxf(va, vu), fmaxf(vl, vs));
      float sm = ex2(va - mx) + ex2(vu - mx) + ex2(vl - mx) + ex2(vs - mx);
      float A = mx + lg2(sm);
      nv[0][c] = A;
      dg[0] = up;
      left[0] = A;
    }
  }
  if (act) {
#pragma unroll
    for (int q = 0; q < NS; ++q)
#pragma unroll
      for (int c = 0; c < R; ++c) pv[q][c] = nv[q][c];
  }
}

// ---------------------------------------------------------------------------
// forward band task
// ---------------------------------------------------------------------------

template <int NS, int R>
__device__ void fwd_band(const Args& a, int p, int band, int lane, uint64_t deadline) {
  using D = Dims<NS, R>;
  const Pair pr = pair_of(a, p);
  const int L1 = pr.L1, L2 = pr.L2;
  const int slot = p * a.nb + band;
  const int col0 = band * 32 * R;
  float* part = a.part + 2 * (size_t)slot;
  if (!(L1 > 0 && col0 < L2)) {
    if (lane == 0) { part[0] = 0.f; part[1] = (band == 0) ? 1.f : 0.f; }
    return;
  }
  const int jl = col0 + lane * R;
  const float k = a.k, g0 = a.go * k, g1 = a.ge * k;
  const size_t Lm = (size_t)a.Lmax1;
  float* eout = a.edge + (size_t)slot * NS * Lm;
  const float* ein = (band > 0) ? a.edge + (size_t)(slot - 1) * NS * Lm : nullptr;
  if (a.fault_inject && band > 0) ein = nullptr;
  float* ck = a.ckpt + (size_t)slot * a.nchunks * D::CKF * 32;
  const int nsteps = L1 + 31;

  float pv[NS][R], lv[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    lv[q] = NEG;
#pragma unroll
    for (int c = 0; c < R; ++c) pv[q][c] = NEG;
  }
  float ref = 0.f;
  KSum acc;
  if (band == 0 && lane == 0) acc.s = 1.f;  // the M[0,0] = 0 origin term

  float sb[PF][R], eb[PF][NS];
#pragma unroll
  for (int u = 0; u < PF; ++u) {
    const int i = u - lane + 1;
    load_row<R>(pr, i, jl, i >= 1 && i <= L1, sb[u]);
#pragma unroll
    for (int q = 0; q < NS; ++q)
      eb[u][q] = (lane == 0 && ein && i >= 1 && i <= L1) ? ld_poll(ein + q * Lm + (i - 1)) : NEG;
  }

  for (int tb = 0; tb < nsteps; tb += PF) {
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int t = tb + u;
      if (t < nsteps) {
        if (u == 0 && (tb % C_STEPS) == 0) {
          float* dst = ck + (size_t)(tb / C_STEPS) * D::CKF * 32 + lane;
#pragma unroll
          for (int q = 0; q < NS; ++q) {
#pragma unroll
            for (int c = 0; c < R; ++c) dst[(q * R + c) * 32] = pv[q][c];
            dst[(NS * R + q) * 32] = lv[q];
          }
        }
        const int i = t - lane + 1;
        const bool act = (i >= 1) && (i <= L1);
        float x[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) x[q] = __shfl_up_sync(FULL, pv[q][R - 1], 1);
        if (lane == 0) {
          if (a.fault_inject && band > 0 && act) {
            float v = poll_value(a.never_written, ld_poll(a.never_written), deadline, a.status,
                                 NEG);
#pragma unroll
            for (int q = 0; q < NS; ++q) x[q] = v;
          } else if (ein && act) {
#pragma unroll
            for (int q = 0; q < NS; ++q)
              x[q] = poll_value(ein + q * Lm + (i - 1), eb[u][q], deadline, a.status, NEG);
          } else {
#pragma unroll
            for (int q = 0; q < NS; ++q) x[q] = NEG;
          }
        }
        float dg[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) { dg[q] = lv[q]; lv[q] = x[q]; }
        float s[R];
#pragma unroll
        for (int c = 0; c < R; ++c) s[c] = sb[u][c] * k;
        {  // prefetch step t + PF
          const int ip = i + PF;
          load_row<R>(pr, ip, jl, ip >= 1 && ip <= L1, sb[u]);
#pragma unroll
          for (int q = 0; q < NS; ++q)
            eb[u][q] = (lane == 0 && ein && ip >= 1 && ip <= L1) ? ld_poll(ein + q * Lm + (ip - 1))
                                                                  : NEG;
        }
        float nv[NS][R];
        fwd_cells<NS, R>(pv, lv, dg, s, g0, g1, act, nv);
        if (act) {
          // partition: lazily rescaled Kahan sum of ex2(x - ref)
          float mx = NEG;
#pragma unroll
          for (int c = 0; c < R; ++c)
            if (jl + c < L2)
#pragma unroll
              for (int q = 0; q < NS; ++q) mx = fmaxf(mx, nv[q][c]);
          if (mx > ref + 64.f) {
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
              for (int q = 0; q < NS; ++q) tsum += ex2(nv[q][c] - ref);
          acc.add(tsum);
          if (lane == 31) {
#pragma unroll
            for (int q = 0; q < NS; ++q) eout[q * Lm + (i - 1)] = pv[q][R - 1];
          }
        }
      }
    }
  }
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

template <int NS, int R>
__global__ void __launch_bounds__(128) fwd_kernel(Args a) {
  const int lane = threadIdx.x & 31;
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = a.B * a.nb;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 0, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    int p = task / a.nb, band = task - p * a.nb;
    if (a.order) p = a.order[p];
    fwd_band<NS, R>(a, p, band, lane, deadline);
  }
}

// ---------------------------------------------------------------------------
// adjoint band task
// ---------------------------------------------------------------------------

// Combine the forward partials of pair p into the scaled log-partition S'.
__device__ __forceinline__ float pair_logz(const Args& a, int p, int lane) {
  float ref = NEG, s = 0.f;
  for (int b = lane; b < a.nb; b += 32) {
    const float* q = a.part + 2 * ((size_t)p * a.nb + b);
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
  return ref + lg2(s);
}

// Last band task of a pair to finish folds the per-band gradient partials (in
// band order, so the result is deterministic) into the outputs.
template <int NS>
__device__ void finish_pair(const Args& a, int p, int slot, int lane, float S2, float g0sum,
                            float g1sum, float pssum) {
  if (lane == 0) {
    float* gp = a.gpart + 4 * (size_t)slot;
    gp[0] = g0sum; gp[1] = g1sum; gp[2] = pssum; gp[3] = 0.f;
    __threadfence();
    unsigned done = atomicAdd(a.pair_done + p, 1u);
    if (done == (unsigned)a.nb - 1) {
      __threadfence();
      float o = 0.f, e = 0.f, ps = 0.f;
      for (int b = 0; b < a.nb; ++b) {
        const float* q = a.gpart + 4 * ((size_t)p * a.nb + b);
        o += ld_poll(q + 0);
        e += ld_poll(q + 1);
        ps += ld_poll(q + 2);
      }
      const float inv_k = 1.f / a.k;          // = T * ln 2
      const float S = S2 * inv_k;
      const float match = ps * inv_k;
      a.value[p] = S;
      if (NS == 3) {
        a.g_open[p] = o;
        a.g_ext[p] = e;
        a.g_T[p] = (S - (match + (o * a.go + e * a.ge))) / a.T;
      } else {
        a.g_open[p] = o;
        if (a.g_ext) a.g_ext[p] = 0.f;
        a.g_T[p] = (S - (match + o * a.go)) / a.T;
      }
    }
  }
}

template <int NS, int R>
__device__ void bwd_band(const Args& a, int p, int band, int lane, float* sm, uint64_t deadline) {
  using D = Dims<NS, R>;
  constexpr int NP = D::NP, EF = D::EF, CKF = D::CKF;
  const Pair pr = pair_of(a, p);
  const int L1 = pr.L1, L2 = pr.L2;
  const int slot = p * a.nb + band;
  const int col0 = band * 32 * R;
  const float S2 = pair_logz(a, p, lane);
  if (!(L1 > 0 && col0 < L2)) {
    finish_pair<NS>(a, p, slot, lane, S2, 0.f, 0.f, 0.f);
    return;
  }
  const int jl = col0 + lane * R;
  const float k = a.k, g0 = a.go * k, g1 = a.ge * k;
  const size_t Lm = (size_t)a.Lmax1;
  const float* ein = (band > 0) ? a.edge + (size_t)(slot - 1) * NS * Lm : nullptr;
  float* pout = (band > 0) ? a.bpush + (size_t)slot * NP * (Lm + 1) : nullptr;
  const bool right_live = (col0 + 32 * R) < L2 && (band + 1) < a.nb;
  const float* pin = right_live ? a.bpush + (size_t)(slot + 1) * NP * (Lm + 1) : nullptr;
  const float* ck = a.ckpt + (size_t)slot * a.nchunks * CKF * 32;
  const int nsteps = L1 + 31;
  const int nch = (nsteps + C_STEPS - 1) / C_STEPS;

  // adjoint state
  float ac[NS][R], nx[NS][R];
#pragma unroll
  for (int q = 0; q < NS; ++q)
#pragma unroll
    for (int c = 0; c < R; ++c) { ac[q][c] = 0.f; nx[q][c] = 0.f; }
  float hold[NS], outp[NP];
#pragma unroll
  for (int q = 0; q < NS; ++q) hold[q] = 0.f;
#pragma unroll
  for (int q = 0; q < NP; ++q) outp[q] = 0.f;
  KSum gA, gB, gS;

  for (int kc = nch - 1; kc >= 0; --kc) {
    const int t0 = kc * C_STEPS;
    const int t1 = min(t0 + C_STEPS, nsteps);
    // ---- restore checkpoint and recompute the chunk into shared memory ----
    float pv[NS][R], lv[NS];
    {
      const float* src = ck + (size_t)kc * CKF * 32 + lane;
#pragma unroll
      for (int q = 0; q < NS; ++q) {
#pragma unroll
        for (int c = 0; c < R; ++c) pv[q][c] = src[(q * R + c) * 32];
        lv[q] = src[(NS * R + q) * 32];
      }
      float* e0 = sm + lane;
#pragma unroll
      for (int q = 0; q < NS; ++q) {
#pragma unroll
        for (int c = 0; c < R; ++c) e0[(q * R + c) * 32] = pv[q][c];
        e0[(NS * R + q) * 32] = lv[q];
      }
    }
    float sb[PF][R];
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int i = t0 + u - lane + 1;
      load_row<R>(pr, i, jl, (t0 + u < t1) && i >= 1 && i <= L1, sb[u]);
    }
#pragma unroll
    for (int u0 = 0; u0 < C_STEPS; u0 += PF) {
#pragma unroll
      for (int u = 0; u < PF; ++u) {
        const int t = t0 + u0 + u;
        if (t < t1) {
          const int i = t - lane + 1;
          const bool act = (i >= 1) && (i <= L1);
          float x[NS];
#pragma unroll
          for (int q = 0; q < NS; ++q) x[q] = __shfl_up_sync(FULL, pv[q][R - 1], 1);
          if (lane == 0) {
#pragma unroll
            for (int q = 0; q < NS; ++q) x[q] = (ein && act) ? ein[q * Lm + (i - 1)] : NEG;
          }
          float dg[NS];
#pragma unroll
          for (int q = 0; q < NS; ++q) { dg[q] = lv[q]; lv[q] = x[q]; }
          float s[R];
#pragma unroll
          for (int c = 0; c < R; ++c) s[c] = sb[u][c] * k;
          {
            const int tp = t + PF;
            const int ip = tp - lane + 1;
            if (u0 + u + PF < C_STEPS) load_row<R>(pr, ip, jl, tp < t1 && ip >= 1 && ip <= L1, sb[u]);
          }
          float nv[NS][R];
          fwd_cells<NS, R>(pv, lv, dg, s, g0, g1, act, nv);
          float* e = sm + (size_t)(t - t0 + 1) * EF * 32 + lane;
#pragma unroll
          for (int q = 0; q < NS; ++q) {
#pragma unroll
            for (int c = 0; c < R; ++c) e[(q * R + c) * 32] = pv[q][c];
            e[(NS * R + q) * 32] = lv[q];
          }
#pragma unroll
          for (int c = 0; c < R; ++c) e[(NS * R + NS + c) * 32] = s[c];
        }
      }
    }
    __syncwarp();
    // ---- adjoint over the chunk, last step first ----
    for (int t = t1 - 1; t >= t0; --t) {
      const int i = t - lane + 1;
      const bool act = (i >= 1) && (i <= L1);
      const float* E = sm + (size_t)(t - t0 + 1) * EF * 32 + lane;   // row i
      const float* P = sm + (size_t)(t - t0) * EF * 32 + lane;       // row i-1
      float r[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q) r[q] = __shfl_down_sync(FULL, outp[q], 1);
      // pushes arriving at column R-1 of row i: left pushes (NS==3: M,D; NS==1: A)
      // and diag pushes (NS==3: M,I,D; NS==1: A)
      float inL[2], inD[NS];
      if (lane == 31) {
        if (pin && act) {
          if constexpr (NS == 3) {
            // left pushes for row i come from the right band's row i; diag
            // pushes into row i from its row i+1, which exists only below L1
            inL[0] = poll_value(pin + 0 * (Lm + 1) + i, ld_poll(pin + 0 * (Lm + 1) + i), deadline, a.status, 0.f);
            inL[1] = poll_value(pin + 1 * (Lm + 1) + i, ld_poll(pin + 1 * (Lm + 1) + i), deadline, a.status, 0.f);
#pragma unroll
            for (int q = 0; q < 3; ++q)
              inD[q] = (i < L1) ? poll_value(pin + (2 + q) * (Lm + 1) + i,
                                             ld_poll(pin + (2 + q) * (Lm + 1) + i), deadline,
                                             a.status, 0.f)
                                : 0.f;
          } else {
            inL[0] = poll_value(pin + i, ld_poll(pin + i), deadline, a.status, 0.f);
            inL[1] = 0.f;
            inD[0] = (i < L1) ? poll_value(pin + (Lm + 1) + i, ld_poll(pin + (Lm + 1) + i), deadline,
                                           a.status, 0.f)
                              : 0.f;
          }
        } else {
          inL[0] = inL[1] = 0.f;
#pragma unroll
          for (int q = 0; q < NS; ++q) inD[q] = 0.f;
        }
      } else {
        if constexpr (NS == 3) {
          inL[0] = r[0]; inL[1] = r[1];
#pragma unroll
          for (int q = 0; q < 3; ++q) { inD[q] = hold[q]; hold[q] = r[2 + q]; }
        } else {
          inL[0] = r[0]; inL[1] = 0.f;
          inD[0] = hold[0]; hold[0] = r[1];
        }
      }
      if constexpr (NS == 3) {
        ac[0][R - 1] += inL[0] + inD[0];
        ac[1][R - 1] += inD[1];
        ac[2][R - 1] += inL[1] + inD[2];
      } else {
        ac[0][R - 1] += inL[0] + inD[0];
      }
#pragma unroll
      for (int q = 0; q < NP; ++q) outp[q] = 0.f;
      float pm[R];
#pragma unroll
      for (int c = R - 1; c >= 0; --c) {
        const bool live = act && (jl + c < L2);
        const bool has_up = i > 1;
        const bool has_left = (jl + c) > 0;
        const float sp = E[(NS * R + NS + c) * 32];
        if constexpr (NS == 3) {
          const float M = E[(0 * R + c) * 32], I = E[(1 * R + c) * 32], Dv = E[(2 * R + c) * 32];
          const float uM = P[(0 * R + c) * 32], uI = P[(1 * R + c) * 32];
          float dM, dI, dD, lM, lD;
          if (c > 0) {
            dM = P[(0 * R + c - 1) * 32]; dI = P[(1 * R + c - 1) * 32]; dD = P[(2 * R + c - 1) * 32];
            lM = E[(0 * R + c - 1) * 32]; lD = E[(2 * R + c - 1) * 32];
          } else {
            dM = P[(3 * R + 0) * 32]; dI = P[(3 * R + 1) * 32]; dD = P[(3 * R + 2) * 32];
            lM = E[(3 * R + 0) * 32]; lD = E[(3 * R + 2) * 32];
          }
          const float bM = live ? ex2(fminf(M - S2, 0.f)) + ac[0][c] : 0.f;
          const float bI = live ? ex2(fminf(I - S2, 0.f)) + ac[1][c] : 0.f;
          const float bD = live ? ex2(fminf(Dv - S2, 0.f)) + ac[2][c] : 0.f;
          const float lse = M - sp;
          const float wMM = ex2(fminf(dM - lse, 0.f));
          const float wMI = ex2(fminf(dI - lse, 0.f));
          const float wMD = ex2(fminf(dD - lse, 0.f));
          const float wIM = has_up ? ex2(fminf(uM + g0 - I, 0.f)) : 0.f;
          const float wII = has_up ? ex2(fminf(uI + g1 - I, 0.f)) : 0.f;
          const float wDM = has_left ? ex2(fminf(lM + g0 - Dv, 0.f)) : 0.f;
          const float wDD = has_left ? ex2(fminf(lD + g1 - Dv, 0.f)) : 0.f;
          pm[c] = bM;
          const float pIM = bI * wIM, pII = bI * wII, pDM = bD * wDM, pDD = bD * wDD;
          gA.add(pIM + pDM);
          gB.add(pII + pDD);
          gS.add(bM * sp);
          nx[0][c] += pIM;
          nx[1][c] += pII;
          const float qM = bM * wMM, qI = bM * wMI, qD = bM * wMD;
          if (c > 0) {
            nx[0][c - 1] += qM; nx[1][c - 1] += qI; nx[2][c - 1] += qD;
            ac[0][c - 1] += pDM; ac[2][c - 1] += pDD;
          } else {
            outp[0] = pDM; outp[1] = pDD; outp[2] = qM; outp[3] = qI; outp[4] = qD;
          }
        } else {
          const float A = E[c * 32];
          const float uA = P[c * 32];
          const float dA = (c > 0) ? P[(c - 1) * 32] : P[R * 32];
          const float lA = (c > 0) ? E[(c - 1) * 32] : E[R * 32];
          const float b = live ? ex2(fminf(A - S2, 0.f)) + ac[0][c] : 0.f;
          const float wA = ex2(fminf(dA + sp - A, 0.f));
          const float wS = ex2(fminf(sp - A, 0.f));
          const float wU = has_up ? ex2(fminf(uA + g0 - A, 0.f)) : 0.f;
          const float wL = has_left ? ex2(fminf(lA + g0 - A, 0.f)) : 0.f;
          const float pv_ = b * (wA + wS);
          pm[c] = pv_;
          const float pU = b * wU, pL = b * wL, pD = b * wA;
          gA.add(pU + pL);
          gS.add(pv_ * sp);
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
          if constexpr (NS == 3) {
            pout[0 * (Lm + 1) + i] = outp[0];
            pout[1 * (Lm + 1) + i] = outp[1];
            pout[2 * (Lm + 1) + (i - 1)] = outp[2];
            pout[3 * (Lm + 1) + (i - 1)] = outp[3];
            pout[4 * (Lm + 1) + (i - 1)] = outp[4];
          } else {
            pout[i] = outp[0];
            pout[(Lm + 1) + (i - 1)] = outp[1];
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NS; ++q)
#pragma unroll
        for (int c = 0; c < R; ++c) { ac[q][c] = nx[q][c]; nx[q][c] = 0.f; }
    }
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
  finish_pair<NS>(a, p, slot, lane, S2, v0, v1, v2);
}

template <int NS, int R>
__global__ void __launch_bounds__(128) bwd_kernel(Args a) {
  extern __shared__ float smem[];
  using D = Dims<NS, R>;
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  float* sm = smem + (size_t)w * (C_STEPS + 1) * D::EF * 32;
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = a.B * a.nb;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 1, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    int p = task / a.nb;
    const int band = a.nb - 1 - (task - p * a.nb);
    if (a.order) p = a.order[p];
    bwd_band<NS, R>(a, p, band, lane, sm, deadline);
  }
}

}  // namespace swb
