// Second-order soft Smith-Waterman ops (sm_100a): Hessian-vector product of
// the marginal map, parameter Jacobians of the map, and the tangent of the
// parameter gradients that the map's full VJP needs.  Compiled as part of
// sw_capi.cu.
//
// Reference semantics (megure-labs/orihime):
//   affine  HVP          src/sw_affine/kernels_gpu.cu:623-785 (launcher :1566)
//           dP/dtheta    src/sw_affine/kernels_gpu.cu:1011-1473 (launcher :1638)
//           full VJP     src/sw_affine/torch_cuda.cpp:681-811
//   linear  HVP          src/sw/kernels_cpu.cpp:279-485 (CUDA twin src/sw/kernels_gpu.cu)
//           dP/dtheta    src/sw/kernels_cpu.cpp:491-710
//
// Work decomposition: one CTA per pair sweeps the anti-diagonals; the threads
// split each diagonal.  Forward: alpha (double-float, scaled log2 domain) and
// the tangent U of alpha (dalpha along the score direction V, or dalpha /
// dtheta) are stored for every cell in a compact diagonal-major table.  Then
// the CTA reduces S, the tangent of S, and sweeps back: a cell's beta and its
// tangent are its init terms plus what its successors pushed, read from a
// rolling buffer that holds the pushes of the last three diagonals.  Each cell
// recomputes its own predecessor weights from the stored alpha, normalised by
// their sum as in the first-order adjoint, so flow is conserved per cell.
//
// Tangents are in natural units.  A weight's tangent along a direction with
// candidate tangents t_k is w_k (t_k - sum_l w_l t_l) / T; the temperature
// direction adds w_k (-ln w_k - H) / T, H the entropy of the cell's softmax.
namespace swb {

enum : int { AUX_HVP = 0, AUX_P0 = 1, AUX_P1 = 2, AUX_PT = 3 };
#ifndef SWB_AUX_THREADS
#define SWB_AUX_THREADS 256
#endif
constexpr int AUX_THREADS = SWB_AUX_THREADS;
constexpr float LN2 = 0.69314718055994531f;

struct AuxArgs {
  const float* scores;   // [B, L1m, L2m]
  const float* v;        // AUX_HVP: direction [B, L1m, L2m]
  const int* lengths;    // [B, 2] or null
  int B, L1m, L2m;
  float go, ge, T, k;    // natural parameters (linear: go = gap), k = log2(e) / T
  float* out;            // [B, L1m, L2m], zero outside lengths (cleared by the host)
  float* gt;             // AUX_HVP: [B][4] tangents of (g0, g1, g_T, S), or null
  float* tab;            // per pair: 3 * NS planes of cells(L1m, L2m) floats
  float* roll;           // per pair: 3 diagonals x (L1m + 1) x 2 * NPUSH floats
  size_t tab_pair, roll_pair;
};

template <int NS> struct AuxShape;
template <> struct AuxShape<3> { static constexpr int NPUSH = 7; };
template <> struct AuxShape<1> { static constexpr int NPUSH = 3; };

__host__ __device__ __forceinline__ long long aux_tri(long long n) { return n > 0 ? n * (n + 1) / 2 : 0; }

// Compact diagonal-major index of the (L1+1) x (L2+1) cell grid: cells with
// i + j = d are contiguous, i ascending.
struct DiagIx {
  int L1, L2;
  __device__ __forceinline__ long long base(int d) const {
    return aux_tri(d) - aux_tri(d - L1 - 1) - aux_tri(d - L2 - 1) + aux_tri(d - L1 - L2 - 2);
  }
  __device__ __forceinline__ long long at(int i, int j) const {
    const int d = i + j;
    return base(d) + (i - max(0, d - L2));
  }
};

__host__ __device__ __forceinline__ size_t aux_cells(int L1, int L2) {
  return (size_t)(L1 + 1) * (size_t)(L2 + 1);
}

// Weights below the smallest normal float count as 0 in the log terms: the
// MUFU lg2 flushes a subnormal input to 0 and would return -inf.
constexpr float W_TINY = 1.17549435e-38f;

// x * log2(x) with 0 * log2(0) = 0.
__device__ __forceinline__ float xlg2(float x) { return x > W_TINY ? x * lg2(x) : 0.f; }

// Block-wide reductions (AUX_THREADS threads), results broadcast to all.
__device__ __forceinline__ void aux_reduce_logsum(float& ref, float& s, float* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float r2 = __shfl_xor_sync(FULL, ref, o), s2 = __shfl_xor_sync(FULL, s, o);
    const float m = fmaxf(ref, r2);
    s = s * ex2(ref - m) + s2 * ex2(r2 - m);
    ref = m;
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) { red[2 * w] = ref; red[2 * w + 1] = s; }
  __syncthreads();
  ref = NEG; s = 0.f;
  for (int q = 0; q < AUX_THREADS / 32; ++q) {  // same order in every thread
    const float r2 = red[2 * q], s2 = red[2 * q + 1];
    if (s2 > 0.f) {
      const float m = fmaxf(ref, r2);
      s = s * ex2(ref - m) + s2 * ex2(r2 - m);
      ref = m;
    }
  }
  __syncthreads();
}

template <int N>
__device__ __forceinline__ void aux_reduce_sum(float (&v)[N], float* red) {
#pragma unroll
  for (int q = 0; q < N; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(FULL, v[q], o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < N; ++q) red[N * w + q] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < N; ++q) {
    float t = 0.f;
    for (int u = 0; u < AUX_THREADS / 32; ++u) t += red[N * u + q];
    v[q] = t;
  }
  __syncthreads();
}

// Softmax terms and weights of one affine cell from its predecessors' alpha
// pairs (scaled domain).  M: diag M, I, D and the start term; I: up M, I;
// D: left M, D.  Returns the cell's own alpha pairs too.
struct AffCell {
  float wm[4], wi[2], wd[2];    // normalised weights (wm[3]: start term)
  float Mh, Ml, Ih, Il, Dh, Dl; // alpha of the cell
};

__device__ __forceinline__ void aff_cell(const float (&dh)[3], const float (&dl)[3],
                                         float uMh, float uMl, float uIh, float uIl,
                                         float lMh, float lMl, float lDh, float lDl, float s,
                                         float g0, float g1, AffCell& c) {
  const float r = fmaxf(fmaxf(dh[0] + dl[0], dh[1] + dl[1]), fmaxf(dh[2] + dl[2], 0.f));
  const float tM = ex2((dh[0] - r) + dl[0]), tI = ex2((dh[1] - r) + dl[1]);
  const float tD = ex2((dh[2] - r) + dl[2]), tZ = ex2(-r);
  const float sm = (tM + tI) + (tD + tZ);
  two_sum(r, s, c.Mh, c.Ml);
  c.Ml += lg2(sm);
  const float vm = recip(sm);
  c.wm[0] = tM * vm; c.wm[1] = tI * vm; c.wm[2] = tD * vm; c.wm[3] = tZ * vm;
  const float ru = fmaxf((uMh + uMl) + g0, (uIh + uIl) + g1);
  const float ia = ((uMh - ru) + g0) + uMl, ib = ((uIh - ru) + g1) + uIl;
  const float ta = ex2(ia), tb = ex2(ib), si = ta + tb;
  fast2(ru, lg2(si), c.Ih, c.Il);
  const float vi = recip(si);
  c.wi[0] = ta * vi; c.wi[1] = tb * vi;
  const float rl = fmaxf((lMh + lMl) + g0, (lDh + lDl) + g1);
  const float da = ((lMh - rl) + g0) + lMl, db = ((lDh - rl) + g1) + lDl;
  const float tc = ex2(da), td = ex2(db), sd = tc + td;
  fast2(rl, lg2(sd), c.Dh, c.Dl);
  const float vd = recip(sd);
  c.wd[0] = tc * vd; c.wd[1] = td * vd;
}

struct LinCell {
  float w[4];   // diag, up, left, start
  float Ah, Al;
};

__device__ __forceinline__ void lin_cell(float dh, float dl, float uh, float ul, float lh, float ll,
                                         float s, float g, LinCell& c) {
  const float r = fmaxf(fmaxf((dh + dl) + s, (uh + ul) + g), fmaxf((lh + ll) + g, s));
  const float ta = ex2(((dh - r) + s) + dl), tu = ex2(((uh - r) + g) + ul);
  const float tl = ex2(((lh - r) + g) + ll), ts = ex2(s - r);
  const float sm = (ta + tu) + (tl + ts);
  fast2(r, lg2(sm), c.Ah, c.Al);
  const float v = recip(sm);
  c.w[0] = ta * v; c.w[1] = tu * v; c.w[2] = tl * v; c.w[3] = ts * v;
}

// Entropy (nats) of a softmax from its weights.
template <int N>
__device__ __forceinline__ float ent(const float* w) {
  float h = 0.f;
#pragma unroll
  for (int q = 0; q < N; ++q) h -= xlg2(w[q]);
  return h * LN2;
}

// Weight tangents: dw_k = w_k (t_k - tbar) / T (+ temperature term).
template <int N, bool TM>
__device__ __forceinline__ void wtan(const float* w, const float* t, float iT, float* dw) {
  float tb = 0.f;
#pragma unroll
  for (int q = 0; q < N; ++q) tb += w[q] * t[q];
  float h = 0.f;
  if (TM) h = ent<N>(w);
#pragma unroll
  for (int q = 0; q < N; ++q) {
    float x = t[q] - tb;
    if (TM) x += (w[q] > W_TINY ? -lg2(w[q]) * LN2 : 0.f) - h;
    dw[q] = w[q] * x * iT;
  }
}

// Shared-memory variant (SM): the forward sweep reads its predecessors from a
// ring of the last three diagonals' alpha / tangent values in shared memory,
// and the backward sweep keeps the push ring there, so the diagonal-to-
// diagonal dependency costs shared-memory latency instead of an L2 round trip.
// Ring layout [diag % 3][field][slot], slot = i - max(0, d - L2).
template <int NS>
__host__ __device__ constexpr int aux_ring_fields() {
  return (3 * NS > 2 * AuxShape<NS>::NPUSH) ? 3 * NS : 2 * AuxShape<NS>::NPUSH;
}

template <int NS, int MODE, bool SM>
__global__ void __launch_bounds__(AUX_THREADS) aux_kernel(AuxArgs a) {
  constexpr int NP = AuxShape<NS>::NPUSH;
  constexpr bool TM = (MODE == AUX_PT);
  __shared__ float red[2 * (AUX_THREADS / 32) * 4];
  extern __shared__ float ring[];
  const int p = blockIdx.x;
  const int tid = threadIdx.x;
  int L1 = a.L1m, L2 = a.L2m;
  if (a.lengths) {
    L1 = min(max(a.lengths[2 * p], 0), a.L1m);
    L2 = min(max(a.lengths[2 * p + 1], 0), a.L2m);
  }
  if (L1 == 0 || L2 == 0) {
    if (a.gt && tid < 4) a.gt[4 * p + tid] = 0.f;
    return;
  }
  const size_t slab = (size_t)p * a.L1m * a.L2m;
  const float* S_ = a.scores + slab;
  const float* V_ = (MODE == AUX_HVP) ? a.v + slab : nullptr;
  float* O_ = a.out + slab;
  const int ld = a.L2m;
  const DiagIx ix{L1, L2};
  const size_t nc = aux_cells(L1, L2);
  float* tab = a.tab + (size_t)p * a.tab_pair;
  float* AH = tab;                  // NS planes
  float* AL = tab + NS * nc;        // NS planes
  float* UU = tab + 2 * NS * nc;    // NS planes
  float* roll = a.roll + (size_t)p * a.roll_pair;
  const size_t rstride = (size_t)(L1 + 1) * 2 * NP;   // floats per rolling diagonal
  const float k = a.k, g0 = a.go * k, g1 = a.ge * k, T = a.T, iT = 1.f / a.T;
  const int DLm = min(a.L1m, a.L2m) + 1;               // ring slots per diagonal (SM)
  auto slot = [&](int i, int d) { return i - max(0, d - L2); };
  // forward-sweep reads of alpha (hi, lo) and tangent of cell (i, j), state st
  auto rd = [&](int st, int i, int j, float& h, float& l, float& u) {
    if constexpr (SM) {
      const int d = i + j;
      const float* r = ring + (size_t)(d % 3) * 3 * NS * DLm + slot(i, d);
      h = r[(size_t)st * DLm]; l = r[(size_t)(NS + st) * DLm]; u = r[(size_t)(2 * NS + st) * DLm];
    } else {
      const long long o = ix.at(i, j);
      h = AH[st * nc + o]; l = AL[st * nc + o]; u = UU[st * nc + o];
    }
  };
  auto wr = [&](int st, int i, int j, float h, float l, float u) {
    const long long o = ix.at(i, j);
    AH[st * nc + o] = h; AL[st * nc + o] = l; UU[st * nc + o] = u;
    if constexpr (SM) {
      const int d = i + j;
      float* r = ring + (size_t)(d % 3) * 3 * NS * DLm + slot(i, d);
      r[(size_t)st * DLm] = h; r[(size_t)(NS + st) * DLm] = l; r[(size_t)(2 * NS + st) * DLm] = u;
    }
  };

  // boundary cells: alpha = NEG, tangent 0
  for (int q = tid; q <= L1 + L2; q += AUX_THREADS) {
    const int i = q <= L2 ? 0 : q - L2, j = q <= L2 ? q : 0;
    const long long o = ix.at(i, j);
#pragma unroll
    for (int st = 0; st < NS; ++st) { AH[st * nc + o] = NEG; AL[st * nc + o] = 0.f; UU[st * nc + o] = 0.f; }
  }
  __syncthreads();

  // ---- forward sweep: alpha and its tangent ----
  // (SM: from diagonal 0, so the ring holds the boundary cells too)
  for (int d = SM ? 0 : 2; d <= L1 + L2; ++d) {
    const int i0 = max(SM ? 0 : 1, d - L2), i1 = min(L1, SM ? d : d - 1);
    for (int i = i0 + tid; i <= i1; i += AUX_THREADS) {
      const int j = d - i;
      if (SM && (i == 0 || j == 0)) {
#pragma unroll
        for (int st = 0; st < NS; ++st) {
          float* r = ring + (size_t)(d % 3) * 3 * NS * DLm + slot(i, d);
          r[(size_t)st * DLm] = NEG; r[(size_t)(NS + st) * DLm] = 0.f; r[(size_t)(2 * NS + st) * DLm] = 0.f;
        }
        continue;
      }
      const float sc = S_[(size_t)(i - 1) * ld + (j - 1)];
      const float s = __fmul_rn(sc, k);
      const float vv = (MODE == AUX_HVP) ? V_[(size_t)(i - 1) * ld + (j - 1)] : 0.f;
      if constexpr (NS == 3) {
        float dh[3], dl[3], du[3], uh[2], ul[2], uu[2], lh[2], ll[2], lu[2];
#pragma unroll
        for (int st = 0; st < 3; ++st) rd(st, i - 1, j - 1, dh[st], dl[st], du[st]);
        rd(0, i - 1, j, uh[0], ul[0], uu[0]);
        rd(1, i - 1, j, uh[1], ul[1], uu[1]);
        rd(0, i, j - 1, lh[0], ll[0], lu[0]);
        rd(2, i, j - 1, lh[1], ll[1], lu[1]);
        AffCell c;
        aff_cell(dh, dl, uh[0], ul[0], uh[1], ul[1], lh[0], ll[0], lh[1], ll[1], s, g0, g1, c);
        const float uM = c.wm[0] * du[0] + c.wm[1] * du[1] + c.wm[2] * du[2];
        float tu0 = uu[0], tu1 = uu[1], tl0 = lu[0], tl1 = lu[1];
        if (MODE == AUX_P0) { tu0 += 1.f; tl0 += 1.f; }
        if (MODE == AUX_P1) { tu1 += 1.f; tl1 += 1.f; }
        float m = uM, ii = c.wi[0] * tu0 + c.wi[1] * tu1, dd = c.wd[0] * tl0 + c.wd[1] * tl1;
        if (MODE == AUX_HVP) m += vv;
        if (TM) { m += ent<4>(c.wm); ii += ent<2>(c.wi); dd += ent<2>(c.wd); }
        wr(0, i, j, c.Mh, c.Ml, m);
        wr(1, i, j, c.Ih, c.Il, ii);
        wr(2, i, j, c.Dh, c.Dl, dd);
      } else {
        float dh, dl, du, uh, ul, uu, lh, ll, lu;
        rd(0, i - 1, j - 1, dh, dl, du);
        rd(0, i - 1, j, uh, ul, uu);
        rd(0, i, j - 1, lh, ll, lu);
        LinCell c;
        lin_cell(dh, dl, uh, ul, lh, ll, s, g0, c);
        float tu = uu, tl = lu;
        if (MODE == AUX_P0) { tu += 1.f; tl += 1.f; }
        float u = c.w[0] * du + c.w[1] * tu + c.w[2] * tl;
        if (MODE == AUX_HVP) u += (c.w[0] + c.w[3]) * vv;
        if (TM) u += ent<4>(c.w);
        wr(0, i, j, c.Ah, c.Al, u);
      }
    }
    __syncthreads();
  }

  // ---- S (scaled, double-float) and the tangent of S ----
  float ref = 0.f, sacc = (tid == 0) ? 1.f : 0.f;   // the M[0,0] = 0 origin term
  for (int d = 2; d <= L1 + L2; ++d) {
    const int i0 = max(1, d - L2), i1 = min(L1, d - 1);
    for (int i = i0 + tid; i <= i1; i += AUX_THREADS) {
      const long long o = ix.at(i, d - i);
#pragma unroll
      for (int st = 0; st < NS; ++st) {
        const float x = AH[st * nc + o] + AL[st * nc + o];
        if (x > ref + 8.f) { sacc *= ex2(ref - x); ref = x; }
        sacc += ex2((AH[st * nc + o] - ref) + AL[st * nc + o]);
      }
    }
  }
  aux_reduce_logsum(ref, sacc, red);
  float Sh, Sl;
  {
    const unsigned bits = __float_as_uint(sacc);
    const int e = (int)((bits >> 23) & 0xffu) - 127;
    float h, l;
    two_sum(ref, (float)e, h, l);
    Sh = h;
    Sl = l + lg2(__uint_as_float((bits & 0x7fffffu) | 0x3f800000u));
  }
  // sum P_end * U and (temperature) sum P_end * log2 P_end, P_end = 2^(x - S)
  float tsum[2] = {0.f, 0.f};
  if (tid == 0 && TM) {  // origin term: P = 2^(-S), U = 0
    const float lp = (0.f - Sh) - Sl;
    tsum[1] += ex2(lp) * lp;
  }
  for (int d = 2; d <= L1 + L2; ++d) {
    const int i0 = max(1, d - L2), i1 = min(L1, d - 1);
    for (int i = i0 + tid; i <= i1; i += AUX_THREADS) {
      const long long o = ix.at(i, d - i);
#pragma unroll
      for (int st = 0; st < NS; ++st) {
        const float lp = (AH[st * nc + o] - Sh) + (AL[st * nc + o] - Sl);
        const float pe = ex2(fminf(lp, 0.f));
        tsum[0] += pe * UU[st * nc + o];
        if (TM && pe > 0.f) tsum[1] += pe * lp;
      }
    }
  }
  aux_reduce_sum<2>(tsum, red);
  const float dS = tsum[0] - (TM ? tsum[1] * LN2 : 0.f);   // dS along the direction

  // ---- backward sweep: beta and its tangent, pulled from the successors ----
  float acc[4] = {0.f, 0.f, 0.f, 0.f};   // tangents of g0, g1; sum Pdot*s; sum P*v
  for (int d = L1 + L2; d >= 2; --d) {
    const int i0 = max(1, d - L2), i1 = min(L1, d - 1);
    // push rings: global [diag % 3][i][field] or shared [diag % 3][field][slot]
    float* rw = SM ? ring + (size_t)(d % 3) * 2 * NP * DLm : roll + (size_t)(d % 3) * rstride;
    const float* r1 = SM ? ring + (size_t)((d + 1) % 3) * 2 * NP * DLm
                         : roll + (size_t)((d + 1) % 3) * rstride;   // successors (i+1, j), (i, j+1)
    const float* r2 = SM ? ring + (size_t)((d + 2) % 3) * 2 * NP * DLm
                         : roll + (size_t)((d + 2) % 3) * rstride;   // successor (i+1, j+1)
    const size_t ps = SM ? (size_t)DLm : 1;   // stride between the fields of one cell
    auto at = [&](const float* r, int i_, int d_) {
      return SM ? r + slot(i_, d_) : r + (size_t)i_ * 2 * NP;
    };
    for (int i = i0 + tid; i <= i1; i += AUX_THREADS) {
      const int j = d - i;
      const bool sD = (i < L1 && j < L2), sU = (i < L1), sL = (j < L2);
      const float* pD = at(r2, i + 1, d + 2);   // pushes of (i+1, j+1)
      const float* pU = at(r1, i + 1, d + 1);   // pushes of (i+1, j)
      const float* pL = at(r1, i, d + 1);       // pushes of (i, j+1)
      const float sc = S_[(size_t)(i - 1) * ld + (j - 1)];
      const float s = __fmul_rn(sc, k);
      const float vv = (MODE == AUX_HVP) ? V_[(size_t)(i - 1) * ld + (j - 1)] : 0.f;
      const long long od = ix.at(i - 1, j - 1), ou = ix.at(i - 1, j), ol = ix.at(i, j - 1), o = ix.at(i, j);
      float* w_out = const_cast<float*>(at(rw, i, d));
      if constexpr (NS == 3) {
        float dh[3], dl[3];
#pragma unroll
        for (int st = 0; st < 3; ++st) { dh[st] = AH[st * nc + od]; dl[st] = AL[st * nc + od]; }
        AffCell c;
        aff_cell(dh, dl, AH[ou], AL[ou], AH[nc + ou], AL[nc + ou], AH[ol], AL[ol], AH[2 * nc + ol],
                 AL[2 * nc + ol], s, g0, g1, c);
        // pushes layout: [MM, MI, MD, IM, II, DM, DD] then their tangents
        float bM = sD ? pD[(0) * ps] : 0.f, bI = sD ? pD[(1) * ps] : 0.f, bD = sD ? pD[(2) * ps] : 0.f;
        float tM = sD ? pD[(NP + 0) * ps] : 0.f, tI = sD ? pD[(NP + 1) * ps] : 0.f, tD = sD ? pD[(NP + 2) * ps] : 0.f;
        if (sU) { bM += pU[(3) * ps]; bI += pU[(4) * ps]; tM += pU[(NP + 3) * ps]; tI += pU[(NP + 4) * ps]; }
        if (sL) { bM += pL[(5) * ps]; bD += pL[(6) * ps]; tM += pL[(NP + 5) * ps]; tD += pL[(NP + 6) * ps]; }
        const float xs[3] = {(c.Mh - Sh) + (c.Ml - Sl), (c.Ih - Sh) + (c.Il - Sl), (c.Dh - Sh) + (c.Dl - Sl)};
        const float us[3] = {UU[o], UU[nc + o], UU[2 * nc + o]};
        float b[3] = {bM, bI, bD}, t[3] = {tM, tI, tD};
#pragma unroll
        for (int st = 0; st < 3; ++st) {
          const float e0 = ex2(fminf(xs[st], 0.f));
          b[st] += e0;
          float x = us[st] - dS;
          if (TM) x -= (e0 > 0.f ? xs[st] * LN2 : 0.f);
          t[st] += e0 * x * iT;
        }
        // weight tangents
        float cm[4], ci[2], cd[2], dwm[4], dwi[2], dwd[2];
        cm[0] = UU[od]; cm[1] = UU[nc + od]; cm[2] = UU[2 * nc + od]; cm[3] = 0.f;
        if (MODE == AUX_HVP) { cm[0] += vv; cm[1] += vv; cm[2] += vv; cm[3] = vv; }
        ci[0] = UU[ou]; ci[1] = UU[nc + ou];
        cd[0] = UU[ol]; cd[1] = UU[2 * nc + ol];
        if (MODE == AUX_P0) { ci[0] += 1.f; cd[0] += 1.f; }
        if (MODE == AUX_P1) { ci[1] += 1.f; cd[1] += 1.f; }
        wtan<4, TM>(c.wm, cm, iT, dwm);
        wtan<2, TM>(c.wi, ci, iT, dwi);
        wtan<2, TM>(c.wd, cd, iT, dwd);
        const float P = b[0], Pd = t[0];
        O_[(size_t)(i - 1) * ld + (j - 1)] = Pd;
        w_out[(0) * ps] = b[0] * c.wm[0]; w_out[(1) * ps] = b[0] * c.wm[1]; w_out[(2) * ps] = b[0] * c.wm[2];
        w_out[(3) * ps] = b[1] * c.wi[0]; w_out[(4) * ps] = b[1] * c.wi[1];
        w_out[(5) * ps] = b[2] * c.wd[0]; w_out[(6) * ps] = b[2] * c.wd[1];
        w_out[(NP + 0) * ps] = t[0] * c.wm[0] + b[0] * dwm[0];
        w_out[(NP + 1) * ps] = t[0] * c.wm[1] + b[0] * dwm[1];
        w_out[(NP + 2) * ps] = t[0] * c.wm[2] + b[0] * dwm[2];
        w_out[(NP + 3) * ps] = t[1] * c.wi[0] + b[1] * dwi[0];
        w_out[(NP + 4) * ps] = t[1] * c.wi[1] + b[1] * dwi[1];
        w_out[(NP + 5) * ps] = t[2] * c.wd[0] + b[2] * dwd[0];
        w_out[(NP + 6) * ps] = t[2] * c.wd[1] + b[2] * dwd[1];
        if (MODE == AUX_HVP) {
          acc[0] += w_out[(NP + 3) * ps] + w_out[(NP + 5) * ps];
          acc[1] += w_out[(NP + 4) * ps] + w_out[(NP + 6) * ps];
          acc[2] += Pd * sc;
          acc[3] += P * vv;
        }
      } else {
        LinCell c;
        lin_cell(AH[od], AL[od], AH[ou], AL[ou], AH[ol], AL[ol], s, g0, c);
        float b = (sD ? pD[(0) * ps] : 0.f) + (sU ? pU[(1) * ps] : 0.f) + (sL ? pL[(2) * ps] : 0.f);
        float t = (sD ? pD[(NP + 0) * ps] : 0.f) + (sU ? pU[(NP + 1) * ps] : 0.f) + (sL ? pL[(NP + 2) * ps] : 0.f);
        const float xs = (c.Ah - Sh) + (c.Al - Sl);
        const float e0 = ex2(fminf(xs, 0.f));
        b += e0;
        float x = UU[o] - dS;
        if (TM) x -= (e0 > 0.f ? xs * LN2 : 0.f);
        t += e0 * x * iT;
        float cv[4], dw[4];
        cv[0] = UU[od]; cv[1] = UU[ou]; cv[2] = UU[ol]; cv[3] = 0.f;
        if (MODE == AUX_HVP) { cv[0] += vv; cv[3] = vv; }
        if (MODE == AUX_P0) { cv[1] += 1.f; cv[2] += 1.f; }
        wtan<4, TM>(c.w, cv, iT, dw);
        const float P = b * (c.w[0] + c.w[3]);
        const float Pd = t * (c.w[0] + c.w[3]) + b * (dw[0] + dw[3]);
        O_[(size_t)(i - 1) * ld + (j - 1)] = Pd;
        w_out[(0) * ps] = b * c.w[0]; w_out[(1) * ps] = b * c.w[1]; w_out[(2) * ps] = b * c.w[2];
        w_out[(NP + 0) * ps] = t * c.w[0] + b * dw[0];
        w_out[(NP + 1) * ps] = t * c.w[1] + b * dw[1];
        w_out[(NP + 2) * ps] = t * c.w[2] + b * dw[2];
        if (MODE == AUX_HVP) {
          acc[0] += w_out[(NP + 1) * ps] + w_out[(NP + 2) * ps];
          acc[2] += Pd * sc;
          acc[3] += P * vv;
        }
      }
    }
    __syncthreads();
  }
  if (MODE == AUX_HVP && a.gt) {
    aux_reduce_sum<4>(acc, red);
    if (tid == 0) {
      const float g0t = acc[0], g1t = acc[1];
      const float gTt = (dS - (acc[2] + acc[3]) - (NS == 3 ? a.go * g0t + a.ge * g1t : a.go * g0t)) * iT;
      a.gt[4 * p + 0] = g0t;
      a.gt[4 * p + 1] = (NS == 3) ? g1t : gTt;
      a.gt[4 * p + 2] = (NS == 3) ? gTt : 0.f;
      a.gt[4 * p + 3] = dS;
    }
  }
  (void)T;
}

}  // namespace swb
