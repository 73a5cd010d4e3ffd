// Second-order soft Smith-Waterman ops as band wavefronts (sm_100a): the
// Hessian-vector product of the marginal map, the map's parameter Jacobians,
// and the tangents of the parameter gradients that the map's full VJP needs.
// Compiled as part of sw_capi.cu, after sw_kernels.cu (helpers, band
// geometry).
//
// Reference semantics (megure-labs/orihime):
//   affine  HVP          src/sw_affine/kernels_gpu.cu:623-785 (launcher :1566)
//           dP/dtheta    src/sw_affine/kernels_gpu.cu:1011-1473 (launcher :1638)
//           full VJP     src/sw_affine/torch_cuda.cpp:681-811
//   linear  HVP          src/sw/kernels_cpu.cpp:279-485 (CUDA twin src/sw/kernels_gpu.cu)
//           dP/dtheta    src/sw/kernels_cpu.cpp:491-710
//
// Decomposition: the first-order band wavefront.  A warp owns 32*R columns of
// one pair; lane l owns R adjacent columns and at step t works on row
// t - l + 1; bands hand their right edge to the next band through polled
// buffers.
//
// Forward (xfwd_kernel): alpha (double-float, scaled log2 domain) and its
// tangent U along the direction (the score direction V for the HVP, one
// parameter for a Jacobian) per state.  Each cell writes what the backward
// needs -- its normalised predecessor weights, their tangents, its alpha
// (hi, lo) and U -- to a wavefront-major table: per step, one float4 per
// lane per field group, so the warp's stores (and later loads) are whole
// contiguous lines.  Per band it accumulates the partition sum with its
// U-weighted and log-weighted sums, from which S and dS follow.
//
// Backward (xbwd_kernel): the same steps in reverse order, lane 31 leading
// as in the first-order adjoint.  A cell's beta and its tangent are its init
// terms plus the pushes of its successors; it pushes beta * w and
// tangent * w + beta * dw to each predecessor: in registers within a lane,
// by __shfl_down_sync to the left lane, through a polled buffer to the left
// band.  Fields stream in by cp.async through a shared-memory ring of
// XSTAGES steps; each lane copies, and later reads, only its own vectors.
//
// Tangents are in natural units.  A weight's tangent along a direction with
// candidate tangents c_k is w_k (c_k - sum_l w_l c_l) / T; the temperature
// direction adds w_k (-ln w_k - H) / T, H the entropy (nats) of the cell's
// softmax, and a cell's U is sum_l w_l c_l (+ H for the temperature).
namespace swb {

// Direction of the tangent pass: the score direction V (HVP), gap open (or
// the linear gap), gap extend, temperature.
enum : int { AUX_HVP = 0, AUX_P0 = 1, AUX_P1 = 2, AUX_PT = 3 };
constexpr float LN2 = 0.69314718055994531f;
// Weights below the smallest normal float count as 0 in the log terms: the
// MUFU lg2 flushes a subnormal input to 0 and would return -inf.
constexpr float W_TINY = 1.17549435e-38f;

template <int NS, int GM = 0> struct XShape;
// G: float4 field groups per cell; NE: floats per row crossing a band edge
// forward (hi, lo, tangent of each state); NP: value push channels crossing a
// lane or band edge backward (their tangents double it); NL of them are left
// pushes.  Global affine: nine weights and their tangents, no per-cell
// alpha (its only beta-init, at the terminal, travels in the partial slot).
// (GM: 0 local, 1 global, 2 Saigo-Vert; Saigo-Vert keeps only M's alpha and
// tangent per cell, the one state with a beta-init)
template <> struct XShape<3, 0> { static constexpr int G = 6, NE = 9, NP = 5, NL = 2; };
template <> struct XShape<3, 1> { static constexpr int G = 5, NE = 9, NP = 6, NL = 3; };
template <> struct XShape<3, 2> { static constexpr int G = 5, NE = 9, NP = 6, NL = 3; };
template <> struct XShape<1, 0> { static constexpr int G = 3, NE = 3, NP = 2, NL = 1; };
template <> struct XShape<1, 1> { static constexpr int G = 3, NE = 3, NP = 2, NL = 1; };
// floats of the forward's per-band partial slot: (ref or S hi, sum or S lo,
// U-sum or dS, log-sum), then the global affine terminal's beta-inits and
// their tangents (w_M, w_I, w_D, dw_M, dw_I, dw_D), padded to 12
constexpr int XPART = 12;

constexpr int XC = 4;   // steps per edge / push prefetch chunk
#ifndef SWB_XPF
#define SWB_XPF 2
#endif
constexpr int XPF = SWB_XPF;   // rows of scores (and direction) loaded ahead
static_assert(XC % XPF == 0, "the score prefetch distance must divide the chunk");
#ifndef SWB_XSTAGES
#define SWB_XSTAGES 2
#endif
constexpr int XSTAGES = SWB_XSTAGES;   // field steps in flight per backward warp
#ifndef SWB_XFWD_MINB
#define SWB_XFWD_MINB 1
#endif
#ifndef SWB_XBWD_MINB
#define SWB_XBWD_MINB 1
#endif

// floats of one step of fields for one warp
template <int NS, int R, int GM = 0>
__host__ __device__ constexpr int xstep_floats() { return R * XShape<NS, GM>::G * 128; }

struct XArgs {
  const float* scores;     // [B, L1m, L2m]
  const float* v;          // AUX_HVP: direction [B, L1m, L2m], else null
  const int* lengths;      // [B, 2] or null
  int B, L1m, L2m, nb;     // nb: bands per pair
  int nsteps;              // field steps per band slot (>= L1m + 31, multiple of XC)
  float go, ge, T, k;      // natural parameters (linear: go = gap), k = log2(e) / T
  float* out;              // [B, L1m, L2m], zero outside lengths (cleared by the host)
  float* gt;               // AUX_HVP: [B][4] tangents of (g0, g1, g_T, S), or null
  float* fld;              // per band slot: nsteps * xstep_floats floats
  float* edge;             // per band slot: NE * L1m floats (sentinel-filled)
  float* bpush;            // per band slot: 2 * NP * (L1m + 1) floats (sentinel-filled)
  float* part;             // per band slot: ref, sum, U-sum, log-sum
  float* cmax;             // per band slot: nsteps / XC floats, largest hi alpha of each chunk
  float* gpart;            // per band slot: HVP parameter-tangent partials
  unsigned* counters;      // [0] forward tasks, [1] backward tasks
  unsigned* pair_done;     // per pair: backward bands finished
  unsigned* status;
  unsigned long long spin_limit_ns;
};

__device__ __forceinline__ void xlengths(const XArgs& a, int p, int& L1, int& L2) {
  L1 = a.L1m;
  L2 = a.L2m;
  if (a.lengths) {  // never index outside the padded slab
    L1 = min(max(a.lengths[2 * p], 0), a.L1m);
    L2 = min(max(a.lengths[2 * p + 1], 0), a.L2m);
  }
}

// Row access to a padded [B, L1m, L2m] tensor (and optionally the output map)
// through the first-order band helpers load_row / store_row.
__device__ __forceinline__ Pair xpair_of(const XArgs& a, int p, int L1, int L2, const float* src,
                                         float* dst) {
  Pair r;
  const size_t base = (size_t)p * a.L1m * a.L2m;
  r.s = src + base;
  r.m = dst ? dst + base : nullptr;
  r.L1 = L1;
  r.L2 = L2;
  r.ld = a.L2m;
  r.vec = ((r.ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(r.s) & 15) == 0) &&
          (!dst || (reinterpret_cast<uintptr_t>(r.m) & 15) == 0);
  return r;
}

// Weight tangents dw_k = w_k (c_k - cbar [+ (-ln w_k - H)]) / T; returns the
// cell's tangent cbar [+ H].  The mean is taken as c_0 + sum w_k (c_k - c_0):
// the weights sum to 1 only up to the approximate reciprocal (~1e-7), and
// that error then scales the candidates' small differences instead of their
// magnitude (tangents along a gap grow with the number of gaps on a path,
// and a bias of ~1e-7 of them per cell accumulates along the DP).
template <int N, bool TM>
__device__ __forceinline__ float xwtan(const float (&w)[N], const float (&c)[N], float iT,
                                       float (&dw)[N]) {
  const float c0 = c[0];
  float d[N];
#pragma unroll
  for (int q = 0; q < N; ++q) d[q] = c[q] - c0;
  float cb = 0.f;   // sum w (c - c0)
#pragma unroll
  for (int q = 0; q < N; ++q) cb = fmaf(w[q], d[q], cb);
  float h = 0.f, nl[N];
  if (TM) {
#pragma unroll
    for (int q = 0; q < N; ++q) {
      nl[q] = w[q] > W_TINY ? -lg2(w[q]) * LN2 : 0.f;
      h = fmaf(w[q], nl[q], h);
    }
  }
#pragma unroll
  for (int q = 0; q < N; ++q) {
    float x = d[q] - cb;
    if (TM) x += nl[q] - h;
    dw[q] = w[q] * x * iT;
  }
  return TM ? (c0 + cb) + h : c0 + cb;
}

// One affine cell of the forward: new alpha pairs and tangents of M, I, D in
// o = (Mh, Ml, Mu, Ih, Il, Iu, Dh, Dl, Du) and its backward fields in f:
//   f0 = (wMM, wMI, wMD, wIM)   f1 = (wII, wDM, wDD, dwMM)
//   f2 = (dwMI, dwMD, dwIM, dwII)  f3 = (dwDM, dwDD, Mh, Ih)
//   f4 = (Dh, Ml, Il, Dl)       f5 = (uM, uI, uD, 0)
// Predecessors: diag (dh, dl, du) of M, I, D; up M and I; left M and D.
template <int MODE>
__device__ __forceinline__ void xcell3(const float (&dh)[3], const float (&dl)[3],
                                       const float (&du)[3], float uMh, float uMl, float uMu,
                                       float uIh, float uIl, float uIu, float lMh, float lMl,
                                       float lMu, float lDh, float lDl, float lDu, float s,
                                       float vv, float g0, float g1, float iT, float (&o)[9],
                                       float4 (&f)[6]) {
  constexpr bool TM = (MODE == AUX_PT);
  // M = s + LSE(M, I, D at diag, 0)
  const float r = fmaxf(fmaxf(dh[0], dh[1]), fmaxf(dh[2], 0.f));
  const float tM = ex2((dh[0] - r) + dl[0]), tI = ex2((dh[1] - r) + dl[1]);
  const float tD = ex2((dh[2] - r) + dl[2]), tZ = ex2(-r);
  const float sm = (tM + tI) + (tD + tZ);
  float Mh, Ml;
  two_sum(r, s, Mh, Ml);
  Ml += lg2(sm);
  const float vm = recip(sm);
  const float wm[4] = {tM * vm, tI * vm, tD * vm, tZ * vm};
  // I = LSE(M up + go, I up + ge)
  const float ru = fmaxf(uMh + g0, uIh + g1);
  const float ta = ex2(((uMh - ru) + g0) + uMl), tb = ex2(((uIh - ru) + g1) + uIl);
  const float si = ta + tb;
  float Ih, Il;
  fast2(ru, lg2(si), Ih, Il);
  const float vi = recip(si);
  const float wi[2] = {ta * vi, tb * vi};
  // D = LSE(M left + go, D left + ge)
  const float rl = fmaxf(lMh + g0, lDh + g1);
  const float tc = ex2(((lMh - rl) + g0) + lMl), td = ex2(((lDh - rl) + g1) + lDl);
  const float sd = tc + td;
  float Dh, Dl;
  fast2(rl, lg2(sd), Dh, Dl);
  const float vd = recip(sd);
  const float wd[2] = {tc * vd, td * vd};
  // candidate tangents: predecessors' U, the score direction on M's terms,
  // 1 on the gap terms of the differentiated parameter
  float cm[4] = {du[0], du[1], du[2], 0.f};
  if (MODE == AUX_HVP) { cm[0] += vv; cm[1] += vv; cm[2] += vv; cm[3] = vv; }
  float ci[2] = {uMu, uIu}, cd[2] = {lMu, lDu};
  if (MODE == AUX_P0) { ci[0] += 1.f; cd[0] += 1.f; }
  if (MODE == AUX_P1) { ci[1] += 1.f; cd[1] += 1.f; }
  float dwm[4], dwi[2], dwd[2];
  const float uM = xwtan<4, TM>(wm, cm, iT, dwm);
  const float uI = xwtan<2, TM>(wi, ci, iT, dwi);
  const float uD = xwtan<2, TM>(wd, cd, iT, dwd);
  o[0] = Mh; o[1] = Ml; o[2] = uM;
  o[3] = Ih; o[4] = Il; o[5] = uI;
  o[6] = Dh; o[7] = Dl; o[8] = uD;
  f[0] = make_float4(wm[0], wm[1], wm[2], wi[0]);
  f[1] = make_float4(wi[1], wd[0], wd[1], dwm[0]);
  f[2] = make_float4(dwm[1], dwm[2], dwi[0], dwi[1]);
  f[3] = make_float4(dwd[0], dwd[1], Mh, Ih);
  f[4] = make_float4(Dh, Ml, Il, Dl);
  f[5] = make_float4(uM, uI, uD, 0.f);
}

// One global affine cell: M = s + LSE(M, I, D at diag); I = LSE(M + go,
// I + ge, D + go) from above; D = LSE(M + go, I + go, D + ge) from the left.
// o as xcell3; fields
//   f0 = (wMM, wMI, wMD, wIM)   f1 = (wII, wID, wDM, wDI)
//   f2 = (wDD, dwMM, dwMI, dwMD)  f3 = (dwIM, dwII, dwID, dwDM)  f4 = (dwDI, dwDD, 0, 0)
template <int MODE>
__device__ __forceinline__ void xcell3g(const float (&dh)[3], const float (&dl)[3],
                                        const float (&du)[3], const float (&uh)[3],
                                        const float (&ul)[3], const float (&uu)[3],
                                        const float (&lh)[3], const float (&ll)[3],
                                        const float (&lu)[3], float s, float vv, float g0, float g1,
                                        float iT, float (&o)[9], float4 (&f)[5]) {
  constexpr bool TM = (MODE == AUX_PT);
  const float r = fmaxf(fmaxf(dh[0], dh[1]), dh[2]);
  const float tM = ex2((dh[0] - r) + dl[0]), tI = ex2((dh[1] - r) + dl[1]);
  const float tD = ex2((dh[2] - r) + dl[2]);
  const float sm = (tM + tI) + tD;
  float Mh, Ml;
  two_sum(r, s, Mh, Ml);
  Ml += lg2(sm);
  const float vm = recip(sm);
  const float wm[3] = {tM * vm, tI * vm, tD * vm};
  const float ru = fmaxf(fmaxf(uh[0] + g0, uh[1] + g1), uh[2] + g0);
  const float ta = ex2(((uh[0] - ru) + g0) + ul[0]), tb = ex2(((uh[1] - ru) + g1) + ul[1]);
  const float tc = ex2(((uh[2] - ru) + g0) + ul[2]);
  const float si = (ta + tb) + tc;
  float Ih, Il;
  fast2(ru, lg2(si), Ih, Il);
  const float vi = recip(si);
  const float wi[3] = {ta * vi, tb * vi, tc * vi};
  const float rl = fmaxf(fmaxf(lh[0] + g0, lh[1] + g0), lh[2] + g1);
  const float td = ex2(((lh[0] - rl) + g0) + ll[0]), te = ex2(((lh[1] - rl) + g0) + ll[1]);
  const float tf = ex2(((lh[2] - rl) + g1) + ll[2]);
  const float sd = (td + te) + tf;
  float Dh, Dl;
  fast2(rl, lg2(sd), Dh, Dl);
  const float vd = recip(sd);
  const float wd[3] = {td * vd, te * vd, tf * vd};
  // candidate tangents: predecessors' U, the score direction on all of M's
  // terms (its weights sum to 1), 1 on the terms of the differentiated gap
  float cm[3] = {du[0], du[1], du[2]}, ci[3] = {uu[0], uu[1], uu[2]}, cd[3] = {lu[0], lu[1], lu[2]};
  if (MODE == AUX_HVP) { cm[0] += vv; cm[1] += vv; cm[2] += vv; }
  if (MODE == AUX_P0) { ci[0] += 1.f; ci[2] += 1.f; cd[0] += 1.f; cd[1] += 1.f; }
  if (MODE == AUX_P1) { ci[1] += 1.f; cd[2] += 1.f; }
  float dwm[3], dwi[3], dwd[3];
  const float uM = xwtan<3, TM>(wm, cm, iT, dwm);
  const float uI = xwtan<3, TM>(wi, ci, iT, dwi);
  const float uD = xwtan<3, TM>(wd, cd, iT, dwd);
  o[0] = Mh; o[1] = Ml; o[2] = uM;
  o[3] = Ih; o[4] = Il; o[5] = uI;
  o[6] = Dh; o[7] = Dl; o[8] = uD;
  f[0] = make_float4(wm[0], wm[1], wm[2], wi[0]);
  f[1] = make_float4(wi[1], wi[2], wd[0], wd[1]);
  f[2] = make_float4(wd[2], dwm[0], dwm[1], dwm[2]);
  f[3] = make_float4(dwi[0], dwi[1], dwi[2], dwd[0]);
  f[4] = make_float4(dwd[1], dwd[2], 0.f, 0.f);
}

// One Saigo-Vert cell: M as the local affine cell; I = LSE(M + go, I + ge)
// from above; D = LSE(M + go, I + go, D + ge) from the left.  o as xcell3;
// fields
//   f0 = (wMM, wMI, wMD, wIM)   f1 = (wII, wDM, wDI, wDD)
//   f2 = (dwMM, dwMI, dwMD, dwIM)  f3 = (dwII, dwDM, dwDI, dwDD)  f4 = (Mh, Ml, uM, 0)
template <int MODE>
__device__ __forceinline__ void xcell3v(const float (&dh)[3], const float (&dl)[3],
                                        const float (&du)[3], const float (&uh)[3],
                                        const float (&ul)[3], const float (&uu)[3],
                                        const float (&lh)[3], const float (&ll)[3],
                                        const float (&lu)[3], float s, float vv, float g0, float g1,
                                        float iT, float (&o)[9], float4 (&f)[5]) {
  constexpr bool TM = (MODE == AUX_PT);
  const float r = fmaxf(fmaxf(dh[0], dh[1]), fmaxf(dh[2], 0.f));
  const float tM = ex2((dh[0] - r) + dl[0]), tI = ex2((dh[1] - r) + dl[1]);
  const float tD = ex2((dh[2] - r) + dl[2]), tZ = ex2(-r);
  const float sm = (tM + tI) + (tD + tZ);
  float Mh, Ml;
  two_sum(r, s, Mh, Ml);
  Ml += lg2(sm);
  const float vm = recip(sm);
  const float wm[4] = {tM * vm, tI * vm, tD * vm, tZ * vm};
  const float ru = fmaxf(uh[0] + g0, uh[1] + g1);
  const float ta = ex2(((uh[0] - ru) + g0) + ul[0]), tb = ex2(((uh[1] - ru) + g1) + ul[1]);
  const float si = ta + tb;
  float Ih, Il;
  fast2(ru, lg2(si), Ih, Il);
  const float vi = recip(si);
  const float wi[2] = {ta * vi, tb * vi};
  const float rl = fmaxf(fmaxf(lh[0] + g0, lh[1] + g0), lh[2] + g1);
  const float tc = ex2(((lh[0] - rl) + g0) + ll[0]), te = ex2(((lh[1] - rl) + g0) + ll[1]);
  const float td = ex2(((lh[2] - rl) + g1) + ll[2]);
  const float sd = (tc + te) + td;
  float Dh, Dl;
  fast2(rl, lg2(sd), Dh, Dl);
  const float vd = recip(sd);
  const float wd[3] = {tc * vd, te * vd, td * vd};
  float cm[4] = {du[0], du[1], du[2], 0.f};
  if (MODE == AUX_HVP) { cm[0] += vv; cm[1] += vv; cm[2] += vv; cm[3] = vv; }
  float ci[2] = {uu[0], uu[1]}, cd[3] = {lu[0], lu[1], lu[2]};
  if (MODE == AUX_P0) { ci[0] += 1.f; cd[0] += 1.f; cd[1] += 1.f; }
  if (MODE == AUX_P1) { ci[1] += 1.f; cd[2] += 1.f; }
  float dwm[4], dwi[2], dwd[3];
  const float uM = xwtan<4, TM>(wm, cm, iT, dwm);
  const float uI = xwtan<2, TM>(wi, ci, iT, dwi);
  const float uD = xwtan<3, TM>(wd, cd, iT, dwd);
  o[0] = Mh; o[1] = Ml; o[2] = uM;
  o[3] = Ih; o[4] = Il; o[5] = uI;
  o[6] = Dh; o[7] = Dl; o[8] = uD;
  f[0] = make_float4(wm[0], wm[1], wm[2], wi[0]);
  f[1] = make_float4(wi[1], wd[0], wd[1], wd[2]);
  f[2] = make_float4(dwm[0], dwm[1], dwm[2], dwi[0]);
  f[3] = make_float4(dwi[1], dwd[0], dwd[1], dwd[2]);
  f[4] = make_float4(Mh, Ml, uM, 0.f);
}

// One linear cell: o = (Ah, Al, U); fields
//   f0 = (w_diag, w_up, w_left, w_diag + w_start)
//   f1 = (dw_diag, dw_up, dw_left, dw_diag + dw_start)   f2 = (Ah, Al, U, 0)
// GL (global alignment): no start term, map factor w_diag.
template <int MODE, bool GL = false>
__device__ __forceinline__ void xcell1(float dh, float dl, float du, float uh, float ul, float uu,
                                       float lh, float ll, float lu, float s, float vv, float g,
                                       float iT, float (&o)[3], float4 (&f)[3]) {
  constexpr bool TM = (MODE == AUX_PT);
  if constexpr (GL) {
    // A = LSE(diag + s, up + g, left + g)
    const float r = fmaxf(dh + s, fmaxf(uh + g, lh + g));
    const float ta = ex2(((dh - r) + s) + dl), tu = ex2(((uh - r) + g) + ul);
    const float tl = ex2(((lh - r) + g) + ll);
    const float sm = (ta + tu) + tl;
    float Ah, Al;
    fast2(r, lg2(sm), Ah, Al);
    const float v = recip(sm);
    const float w[3] = {ta * v, tu * v, tl * v};
    float c[3] = {du, uu, lu};
    if (MODE == AUX_HVP) c[0] += vv;
    if (MODE == AUX_P0) { c[1] += 1.f; c[2] += 1.f; }
    float dw[3];
    const float U = xwtan<3, TM>(w, c, iT, dw);
    o[0] = Ah; o[1] = Al; o[2] = U;
    f[0] = make_float4(w[0], w[1], w[2], w[0]);
    f[1] = make_float4(dw[0], dw[1], dw[2], dw[0]);
    f[2] = make_float4(Ah, Al, U, 0.f);
    return;
  }
  // A = LSE(diag + s, up + g, left + g, s)
  const float r = fmaxf(fmaxf(dh + s, uh + g), fmaxf(lh + g, s));
  const float ta = ex2(((dh - r) + s) + dl), tu = ex2(((uh - r) + g) + ul);
  const float tl = ex2(((lh - r) + g) + ll), ts = ex2(s - r);
  const float sm = (ta + tu) + (tl + ts);
  float Ah, Al;
  fast2(r, lg2(sm), Ah, Al);
  const float v = recip(sm);
  const float w[4] = {ta * v, tu * v, tl * v, ts * v};
  float c[4] = {du, uu, lu, 0.f};
  if (MODE == AUX_HVP) { c[0] += vv; c[3] = vv; }
  if (MODE == AUX_P0) { c[1] += 1.f; c[2] += 1.f; }
  float dw[4];
  const float U = xwtan<4, TM>(w, c, iT, dw);
  o[0] = Ah; o[1] = Al; o[2] = U;
  f[0] = make_float4(w[0], w[1], w[2], w[0] + w[3]);
  f[1] = make_float4(dw[0], dw[1], dw[2], dw[0] + dw[3]);
  f[2] = make_float4(Ah, Al, U, 0.f);
}

// (ref, sum 2^(x-ref), sum 2^(x-ref) U, sum 2^(x-ref) (x-ref)) merged into
// the first tuple at the larger reference.
__device__ __forceinline__ void xcombine(float& r1, float& s1, float& u1, float& x1, float r2,
                                         float s2, float u2, float x2) {
  const float m = fmaxf(r1, r2), d1 = r1 - m, d2 = r2 - m;
  const float f1 = ex2(d1), f2 = ex2(d2);
  x1 = f1 * fmaf(d1, s1, x1) + f2 * fmaf(d2, s2, x2);
  s1 = s1 * f1 + s2 * f2;
  u1 = u1 * f1 + u2 * f2;
  r1 = m;
}

// Tangents of a global alignment's row-0 values at column j along the
// differentiated direction: linear j * gap -> j (gap); affine D(0,j) =
// go + (j-1) ge -> 1 (gap open) or j - 1 (gap extend); 0 otherwise.
template <int NS, int MODE>
__device__ __forceinline__ void xrow0_tan(int j, float (&u)[NS]) {
#pragma unroll
  for (int q = 0; q < NS; ++q) u[q] = 0.f;
  if constexpr (NS == 1) {
    if (MODE == AUX_P0) u[0] = (float)j;
  } else {
    if (j >= 1 && MODE == AUX_P0) u[2] = 1.f;
    if (j >= 1 && MODE == AUX_P1) u[2] = (float)(j - 1);
  }
}

// Column-0 edge record at row i (hi, lo, tangent of each state): linear
// i * gap; affine I(i,0) = go + (i-1) ge, M and D NEG.
template <int NS, int MODE>
__device__ __forceinline__ void xcol0_edge(int i, float g0, float g1, float (&e)[3 * NS]) {
  float hl[2 * NS];
  col0_edge<NS>(i, g0, g1, hl);
#pragma unroll
  for (int f = 0; f < 2 * NS; ++f) e[f] = hl[f];
  if constexpr (NS == 1) {
    e[2] = MODE == AUX_P0 ? (float)i : 0.f;
  } else {
    e[6] = 0.f;
    e[7] = MODE == AUX_P0 ? 1.f : (MODE == AUX_P1 ? (float)(i - 1) : 0.f);
    e[8] = 0.f;
  }
}

// The terminal of a global alignment (column c of the lane): part = (S hi,
// S lo, dS, 0, then for the affine model the beta-inits w_q = 2^(x_q - S)
// of M, I, D and their tangents).
template <int NS, int MODE, int R>
__device__ __forceinline__ void xterminal(const float (&ph)[NS][R], const float (&pl)[NS][R],
                                          const float (&pu)[NS][R], int c, float iT, float* part) {
  if constexpr (NS == 1) {
    part[0] = ph[0][c]; part[1] = pl[0][c]; part[2] = pu[0][c]; part[3] = 0.f;
  } else {
    constexpr bool TM = (MODE == AUX_PT);
    const float r = fmaxf(fmaxf(ph[0][c], ph[1][c]), ph[2][c]);
    float e[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) e[q] = ex2((ph[q][c] - r) + pl[q][c]);
    const float sm = (e[0] + e[1]) + e[2];
    float Sh, Sl;
    fast2(r, lg2(sm), Sh, Sl);
    const float v = recip(sm);
    const float w[3] = {e[0] * v, e[1] * v, e[2] * v};
    const float u[3] = {pu[0][c], pu[1][c], pu[2][c]};
    float dw[3];
    const float dS = xwtan<3, TM>(w, u, iT, dw);
    part[0] = Sh; part[1] = Sl; part[2] = dS; part[3] = 0.f;
    part[4] = w[0]; part[5] = w[1]; part[6] = w[2];
    part[7] = dw[0]; part[8] = dw[1]; part[9] = dw[2];
  }
}

// ---------------------------------------------------------------------------
// forward band task
// ---------------------------------------------------------------------------

// GL: global alignment (NS == 1).  Rows start from the row-0 boundary j * gap
// (tangent j along the gap, else 0) and band 0 takes the column-0 boundary
// i * gap; a row before the lane's first keeps the boundary and writes zero
// fields.  The band holding the pair's last column writes the terminal
// (hi, lo, U) to its partial slot; the chunk maximum is a marker, +1e30 in
// the chunk holding the terminal and NEG elsewhere.
template <int NS, int R, int MODE, int GM = 0>
__device__ void xfwd_band(const XArgs& a, int p, int band, int lane, uint64_t deadline) {
  constexpr bool GL = GM == 1, SV = GM == 2;
  using XS = XShape<NS, GM>;
  constexpr int G = XS::G, NE = XS::NE;
  constexpr int XSTEP = xstep_floats<NS, R, GM>();
  constexpr bool HV = (MODE == AUX_HVP);
  int L1, L2;
  xlengths(a, p, L1, L2);
  const size_t slot = (size_t)p * a.nb + band;
  float* part = a.part + XPART * slot;
  const int col0 = band * 32 * R;
  if (!(L1 > 0 && col0 < L2)) {
    if (!GL && lane == 0) { part[0] = 0.f; part[1] = (band == 0) ? 1.f : 0.f; part[2] = 0.f; part[3] = 0.f; }
    return;
  }
  const Pair ps = xpair_of(a, p, L1, L2, a.scores, nullptr);
  const Pair pv = xpair_of(a, p, L1, L2, HV ? a.v : a.scores, nullptr);
  const int jl = col0 + lane * R;
  const float k = a.k, g0 = a.go * k, g1 = a.ge * k, iT = 1.f / a.T;
  const size_t Lm = (size_t)a.L1m;
  float* eout = a.edge + slot * NE * Lm;
  const float* ein = (band > 0) ? eout - NE * Lm : nullptr;
  float* F = a.fld + slot * (size_t)a.nsteps * XSTEP;
  const int nch = (L1 + 31 + XC - 1) / XC;

  float ph[NS][R], pl[NS][R], pu[NS][R], lh[NS], ll[NS], lu[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    lh[q] = NEG; ll[q] = 0.f; lu[q] = 0.f;
#pragma unroll
    for (int c = 0; c < R; ++c) { ph[q][c] = NEG; pl[q][c] = 0.f; pu[q][c] = 0.f; }
  }
  if constexpr (GL) {   // row 0 and its tangents (the boundaries' gap derivatives)
    row0<NS>(jl, g0, g1, lh, ll);
    xrow0_tan<NS, MODE>(jl, lu);
#pragma unroll
    for (int c = 0; c < R; ++c) {
      float h[NS], l[NS], u[NS];
      row0<NS>(jl + c + 1, g0, g1, h, l);
      xrow0_tan<NS, MODE>(jl + c + 1, u);
#pragma unroll
      for (int q = 0; q < NS; ++q) { ph[q][c] = h[q]; pl[q][c] = l[q]; pu[q][c] = u[q]; }
    }
  }
  const bool term_lane = GL && jl < L2 && L2 <= jl + R;   // holds the pair's last column
  float ref = 0.f, su = 0.f, sx = 0.f;
  KSum acc;
  if (!GL && band == 0 && lane == 0) acc.s = 1.f;  // origin M[0,0] = 0: weight 1, U 0, log term 0

  // Lane u < XC holds the left band's edge values that lane 0 needs at step u
  // of a chunk, loaded one chunk ahead; lane 0 takes them by shuffle.  Band 0
  // of a global alignment takes the column-0 boundary instead.
  const bool left_bnd = GL && band == 0;
  float eb[NE], ebn[NE];
  auto load_edge = [&](int kc, float (&dst)[NE]) {
    const int i = kc * XC + lane + 1;
    const bool ok = ein && lane < XC && i <= L1;
#pragma unroll
    for (int f = 0; f < NE; ++f) dst[f] = ok ? ld_poll(ein + f * Lm + (i - 1)) : 0.f;
    if (left_bnd) xcol0_edge<NS, MODE>(i, g0, g1, dst);
  };
  load_edge(0, eb);
  float sb[XPF][R], vb[XPF][R];
#pragma unroll
  for (int u = 0; u < XPF; ++u) {
    const int i = u - lane + 1;
    load_row<R>(ps, i, jl, i >= 1 && i <= L1, sb[u]);
    load_row<R>(pv, i, jl, HV && i >= 1 && i <= L1, vb[u]);
  }

  float* cm = a.cmax + slot * (size_t)(a.nsteps / XC);
  for (int kc = 0; kc < nch; ++kc) {
    if (kc + 1 < nch) load_edge(kc + 1, ebn);
    float cmx = NEG;   // largest hi alpha of the lane's live cells in this chunk
#pragma unroll 1
    for (int u0 = 0; u0 < XC; u0 += XPF)
#pragma unroll
      for (int u = 0; u < XPF; ++u) {
        const int cu = u0 + u;
        const int t = kc * XC + cu;
        const int i = t - lane + 1;
        const bool act = (i >= 1) && (i <= L1);
        float xh[NS], xl[NS], xu[NS], ev[NE];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          xh[q] = __shfl_up_sync(FULL, ph[q][R - 1], 1);
          xl[q] = __shfl_up_sync(FULL, pl[q][R - 1], 1);
          xu[q] = __shfl_up_sync(FULL, pu[q][R - 1], 1);
        }
#pragma unroll
        for (int f = 0; f < NE; ++f) ev[f] = __shfl_sync(FULL, eb[f], cu);
        // a value still at the sentinel (left band not there yet) is polled
        // on a warp-uniform slow path
        bool miss = false;
#pragma unroll
        for (int f = 0; f < NE; ++f) miss |= is_sentinel(ev[f]);
        miss = (lane == 0) && ein && act && miss;
        if (__any_sync(FULL, miss) && miss) {
          FieldVec<NE> x;
#pragma unroll
          for (int f = 0; f < NE; ++f) x.v[f] = ev[f];
          x = poll_fields_v<NE, NS>(x, ein + (i - 1), Lm, deadline, a.status, a.pair_done + p);
#pragma unroll
          for (int f = 0; f < NE; ++f) ev[f] = x.v[f];
        }
        if (lane == 0) {
          const bool take = act && (ein || left_bnd);
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            xh[q] = take ? ev[q] : NEG;
            xl[q] = take ? ev[NS + q] : 0.f;
            xu[q] = take ? ev[2 * NS + q] : 0.f;
          }
        }
        float dgh[NS], dgl[NS], dgu[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          dgh[q] = lh[q]; dgl[q] = ll[q]; dgu[q] = lu[q];
          lh[q] = xh[q]; ll[q] = xl[q]; lu[q] = xu[q];
        }
        float s[R], vv[R];
#pragma unroll
        for (int c = 0; c < R; ++c) {
          s[c] = i >= 1 ? __fmul_rn(sb[u][c], k) : NEG;
          vv[c] = HV ? vb[u][c] : 0.f;
        }
        {
          const int ip = i + XPF;
          load_row<R>(ps, ip, jl, ip >= 1 && ip <= L1, sb[u]);
          load_row<R>(pv, ip, jl, HV && ip >= 1 && ip <= L1, vb[u]);
        }
        float* Fs = F + (size_t)t * XSTEP;
        // left values inside the row: start from the left input, which itself
        // stays as the next step's diagonal of column 0
        float wh[NS], wl[NS], wu[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) { wh[q] = lh[q]; wl[q] = ll[q]; wu[q] = lu[q]; }
#pragma unroll
        for (int c = 0; c < R; ++c) {
          if constexpr (NS == 3 && (GL || SV)) {
            const float uh3[3] = {ph[0][c], ph[1][c], ph[2][c]};
            const float ul3[3] = {pl[0][c], pl[1][c], pl[2][c]};
            const float uu3[3] = {pu[0][c], pu[1][c], pu[2][c]};
            float o[9];
            float4 f[G];
            if constexpr (SV)
              xcell3v<MODE>(dgh, dgl, dgu, uh3, ul3, uu3, wh, wl, wu, s[c], vv[c], g0, g1, iT, o, f);
            else
              xcell3g<MODE>(dgh, dgl, dgu, uh3, ul3, uu3, wh, wl, wu, s[c], vv[c], g0, g1, iT, o, f);
            if (GL && i < 1) {   // boundary row: keep the values, no fields
#pragma unroll
              for (int q = 0; q < 3; ++q) { o[3 * q] = uh3[q]; o[3 * q + 1] = ul3[q]; o[3 * q + 2] = uu3[q]; }
#pragma unroll
              for (int g = 0; g < G; ++g) f[g] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int g = 0; g < G; ++g) reinterpret_cast<float4*>(Fs + (c * G + g) * 128)[lane] = f[g];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              dgh[q] = uh3[q]; dgl[q] = ul3[q]; dgu[q] = uu3[q];
              wh[q] = o[3 * q]; wl[q] = o[3 * q + 1]; wu[q] = o[3 * q + 2];
              ph[q][c] = o[3 * q]; pl[q][c] = o[3 * q + 1]; pu[q][c] = o[3 * q + 2];
            }
          } else if constexpr (NS == 3) {
            const float uMh = ph[0][c], uMl = pl[0][c], uMu = pu[0][c];
            const float uIh = ph[1][c], uIl = pl[1][c], uIu = pu[1][c];
            const float uDh = ph[2][c], uDl = pl[2][c], uDu = pu[2][c];
            float o[9];
            float4 f[6];
            xcell3<MODE>(dgh, dgl, dgu, uMh, uMl, uMu, uIh, uIl, uIu, wh[0], wl[0], wu[0], wh[2],
                         wl[2], wu[2], s[c], vv[c], g0, g1, iT, o, f);
#pragma unroll
            for (int g = 0; g < G; ++g) reinterpret_cast<float4*>(Fs + (c * G + g) * 128)[lane] = f[g];
            dgh[0] = uMh; dgl[0] = uMl; dgu[0] = uMu;
            dgh[1] = uIh; dgl[1] = uIl; dgu[1] = uIu;
            dgh[2] = uDh; dgl[2] = uDl; dgu[2] = uDu;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              wh[q] = o[3 * q]; wl[q] = o[3 * q + 1]; wu[q] = o[3 * q + 2];
              ph[q][c] = o[3 * q]; pl[q][c] = o[3 * q + 1]; pu[q][c] = o[3 * q + 2];
            }
          } else {
            const float uh = ph[0][c], ul = pl[0][c], uu = pu[0][c];
            float o[3];
            float4 f[3];
            xcell1<MODE, GL>(dgh[0], dgl[0], dgu[0], uh, ul, uu, wh[0], wl[0], wu[0], s[c], vv[c],
                             g0, iT, o, f);
            if (GL && i < 1) {   // boundary row: keep the values, no fields
              o[0] = uh; o[1] = ul; o[2] = uu;
#pragma unroll
              for (int g = 0; g < G; ++g) f[g] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int g = 0; g < G; ++g) reinterpret_cast<float4*>(Fs + (c * G + g) * 128)[lane] = f[g];
            dgh[0] = uh; dgl[0] = ul; dgu[0] = uu;
            wh[0] = o[0]; wl[0] = o[1]; wu[0] = o[2];
            ph[0][c] = o[0]; pl[0][c] = o[1]; pu[0][c] = o[2];
          }
        }
        if (GL && act) {
          if (term_lane && i == L1) {   // the terminal with its tangent (affine: LSE of M, I, D)
#pragma unroll
            for (int c = 0; c < R; ++c)
              if (jl + c == L2 - 1) xterminal<NS, MODE>(ph, pl, pu, c, iT, part);
            cmx = 1e30f;
          }
          if (lane == 31) {
#pragma unroll
            for (int q = 0; q < NS; ++q) {
              eout[q * Lm + (i - 1)] = ph[q][R - 1];
              eout[(NS + q) * Lm + (i - 1)] = pl[q][R - 1];
              eout[(2 * NS + q) * Lm + (i - 1)] = pu[q][R - 1];
            }
          }
        }
        if (!GL && act) {
          // partition with its U- and log-weighted sums, lazily rescaled:
          // exponents stay <= 8 so (hi - ref) + lo rounds at <= 2^-21
          constexpr int NT = SV ? 1 : NS;   // Saigo-Vert: S = LSE(0, M cells)
          float mx = NEG;
#pragma unroll
          for (int c = 0; c < R; ++c)
            if (jl + c < L2)
#pragma unroll
              for (int q = 0; q < NT; ++q) mx = fmaxf(mx, ph[q][c]);
          cmx = fmaxf(cmx, mx);
          if (mx > ref + 8.f) {
            const float d = ref - mx, f = ex2(d);
            sx = f * fmaf(d, acc.s, sx);
            acc.s *= f;
            acc.c *= f;
            su *= f;
            ref = mx;
          }
          float ts = 0.f, tu = 0.f, tx = 0.f;
#pragma unroll
          for (int c = 0; c < R; ++c)
            if (jl + c < L2)
#pragma unroll
              for (int q = 0; q < NT; ++q) {
                const float x = (ph[q][c] - ref) + pl[q][c];
                const float e = ex2(x);
                ts += e;
                tu = fmaf(e, pu[q][c], tu);
                tx = fmaf(e, x, tx);
              }
          acc.add(ts);
          su += tu;
          sx += tx;
          if (lane == 31) {
#pragma unroll
            for (int q = 0; q < NS; ++q) {
              eout[q * Lm + (i - 1)] = ph[q][R - 1];
              eout[(NS + q) * Lm + (i - 1)] = pl[q][R - 1];
              eout[(2 * NS + q) * Lm + (i - 1)] = pu[q][R - 1];
            }
          }
        }
      }
#pragma unroll
    for (int f = 0; f < NE; ++f) eb[f] = ebn[f];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cmx = fmaxf(cmx, __shfl_xor_sync(FULL, cmx, o));
    if (lane == 0) cm[kc] = cmx;
  }
  if constexpr (GL) return;
  // warp-combine the lanes' tuples (fixed shuffle tree: deterministic)
  float s_ = acc.s;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float r2 = __shfl_xor_sync(FULL, ref, o), s2 = __shfl_xor_sync(FULL, s_, o);
    const float u2 = __shfl_xor_sync(FULL, su, o), x2 = __shfl_xor_sync(FULL, sx, o);
    xcombine(ref, s_, su, sx, r2, s2, u2, x2);
  }
  if (lane == 0) { part[0] = ref; part[1] = s_; part[2] = su; part[3] = sx; }
}

template <int NS, int R, int MODE, int GM = 0>
__global__ void __launch_bounds__(128, SWB_XFWD_MINB) xfwd_kernel(XArgs a) {
  const int lane = threadIdx.x & 31;
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = a.B * a.nb;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 0, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    const int p = task / a.nb;
    xfwd_band<NS, R, MODE, GM>(a, p, task - p * a.nb, lane, deadline);
  }
}

// ---------------------------------------------------------------------------
// backward band task
// ---------------------------------------------------------------------------

// S' = Sh + Sl (scaled) and dS of pair p from its bands' forward tuples.
// GL: the terminal tuple of the band holding the last column; an empty side
// leaves the boundary (L1 + L2) * gap (the caller then returns early).
template <bool TM, int R = 0, bool GL = false>
__device__ __forceinline__ void xpair_stats(const XArgs& a, int p, int lane, float& Sh, float& Sl,
                                            float& dS) {
  if constexpr (GL) {
    int L1, L2;
    xlengths(a, p, L1, L2);
    if (L1 == 0 || L2 == 0) {
      nmul(L1 + L2, a.go * a.k, Sh, Sl);
      dS = 0.f;
      return;
    }
    const float* q = a.part + XPART * ((size_t)p * a.nb + (L2 - 1) / (32 * R));
    Sh = q[0];
    Sl = q[1];
    dS = q[2];
    return;
  }
  float ref = NEG, s = 0.f, su = 0.f, sx = 0.f;
  for (int b = lane; b < a.nb; b += 32) {
    const float* q = a.part + XPART * ((size_t)p * a.nb + b);
    const float r2 = q[0], s2 = q[1], u2 = q[2], x2 = q[3];
    if (s2 > 0.f) xcombine(ref, s, su, sx, r2, s2, u2, x2);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float r2 = __shfl_xor_sync(FULL, ref, o), s2 = __shfl_xor_sync(FULL, s, o);
    const float u2 = __shfl_xor_sync(FULL, su, o), x2 = __shfl_xor_sync(FULL, sx, o);
    xcombine(ref, s, su, sx, r2, s2, u2, x2);
  }
  // S = ref + log2(s) as a double-float: with s = m * 2^e, m in [1, 2), lg2
  // sees only the mantissa and the integer e joins ref by TwoSum
  const unsigned bits = __float_as_uint(s);
  const int e = (int)((bits >> 23) & 0xffu) - 127;
  float lgs;
  if (s > 0.f && e > -127 && e < 128) {
    const float lm = lg2(__uint_as_float((bits & 0x7fffffu) | 0x3f800000u));
    float h, l;
    two_sum(ref, (float)e, h, l);
    Sh = h;
    Sl = l + lm;
    lgs = (float)e + lm;
  } else {
    Sh = ref;
    Sl = lg2(s);
    lgs = Sl;
  }
  // dS = sum P U - [T] ln2 sum P log2 P, P = 2^(x - S):
  // sum P (x - S) = sx / s - log2(s)
  dS = su / s - (TM ? (sx / s - lgs) * LN2 : 0.f);
}

__device__ __forceinline__ void cp_async16(float* sdst, const float* gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Band partials of the HVP's parameter tangents; the last band of a pair to
// finish folds them (in band order: deterministic) into grad_tangents.  When
// a bounded wait of the pair expired (PAIR_TIMEOUT in its completion word),
// the last band fills the pair's output map (and grad_tangents) with NaN.
template <int NS, int MODE>
__device__ void xfinish(const XArgs& a, int p, int band, int lane, bool empty, float dS, float ga,
                        float gb, float gc, int L1, int L2) {
  const bool tangents = MODE == AUX_HVP && a.gt;
  unsigned done = 0;
  if (lane == 0) {
    if (tangents) {
      float* gp = a.gpart + 4 * ((size_t)p * a.nb + band);
      gp[0] = ga; gp[1] = gb; gp[2] = gc; gp[3] = 0.f;
      __threadfence();
    }
    done = atomicAdd(a.pair_done + p, 1u);
  }
  done = __shfl_sync(FULL, done, 0);
  if ((done & ~PAIR_TIMEOUT) == (unsigned)a.nb - 1 && (done & PAIR_TIMEOUT)) {
    const float nan = __int_as_float(0x7fc00000);
    float* o = a.out + (size_t)p * a.L1m * a.L2m;
    for (int i = 0; i < L1; ++i)
      for (int j = lane; j < L2; j += 32) o[(size_t)i * a.L2m + j] = nan;
    if (tangents && lane < 4) a.gt[4 * p + lane] = nan;
    return;
  }
  if (!tangents) return;
  if (lane == 0) {
    if ((done & ~PAIR_TIMEOUT) == (unsigned)a.nb - 1) {
      __threadfence();
      float o = 0.f, e = 0.f, c = 0.f;
      for (int b = 0; b < a.nb; ++b) {
        const float* q = a.gpart + 4 * ((size_t)p * a.nb + b);
        o += ld_poll(q + 0);
        e += ld_poll(q + 1);
        c += ld_poll(q + 2);
      }
      float* g = a.gt + 4 * p;
      if (empty) {
        g[0] = 0.f; g[1] = 0.f; g[2] = 0.f; g[3] = 0.f;
      } else {
        const float gTt = (dS - c - (NS == 3 ? a.go * o + a.ge * e : a.go * o)) * (1.f / a.T);
        g[0] = o;
        g[1] = (NS == 3) ? e : gTt;
        g[2] = (NS == 3) ? gTt : 0.f;
        g[3] = dS;
      }
    }
  }
}

// GL: the only beta-init is 1 at the terminal (tangent 0); pushes into the
// row-0 / column-0 boundary add index * tangent to the gap tangent (HVP).
template <int NS, int R, int MODE, int GM = 0>
__device__ void xbwd_band(const XArgs& a, int p, int band, int lane, float* ring,
                          uint64_t deadline) {
  constexpr bool GL = GM == 1, SV = GM == 2;
  using XS = XShape<NS, GM>;
  constexpr int G = XS::G, NP = XS::NP, NQ = 2 * NP, NL = XS::NL;
  constexpr int XSTEP = xstep_floats<NS, R, GM>();
  constexpr bool TM = (MODE == AUX_PT), HV = (MODE == AUX_HVP);
  int L1, L2;
  xlengths(a, p, L1, L2);
  const int col0 = band * 32 * R;
  float Sh, Sl, dS;
  xpair_stats<TM, R, GL>(a, p, lane, Sh, Sl, dS);
  if (!(L1 > 0 && col0 < L2)) {
    xfinish<NS, MODE>(a, p, band, lane, L1 == 0 || L2 == 0, dS, 0.f, 0.f, 0.f, L1, L2);
    return;
  }
  const size_t slot = (size_t)p * a.nb + band;
  const Pair po = xpair_of(a, p, L1, L2, a.scores, a.out);
  const Pair pv = xpair_of(a, p, L1, L2, HV ? a.v : a.scores, nullptr);
  const int jl = col0 + lane * R;
  const bool term_lane = GL && jl < L2 && L2 <= jl + R;   // holds the pair's last column
  // the terminal's beta-inits and their tangents (linear: 1 and 0)
  float tw[NS], tdw[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) { tw[q] = 1.f; tdw[q] = 0.f; }
  if (NS == 3 && term_lane) {
    const float* q = a.part + XPART * ((size_t)p * a.nb + band);
#pragma unroll
    for (int st = 0; st < NS; ++st) { tw[st] = q[4 + st]; tdw[st] = q[7 + st]; }
  }
  const float iT = 1.f / a.T;
  const size_t Lm = (size_t)a.L1m;
  float* pout = (band > 0) ? a.bpush + slot * NQ * (Lm + 1) : nullptr;
  const bool right_live = (col0 + 32 * R) < L2 && (band + 1) < a.nb;
  const float* pin = right_live ? a.bpush + (slot + 1) * NQ * (Lm + 1) : nullptr;
  const float* F = a.fld + slot * (size_t)a.nsteps * XSTEP;
  const int nch = (L1 + 31 + XC - 1) / XC;
  const int nst = nch * XC;   // steps, padded to whole chunks (padding steps find no row)

  // field ring: reverse step tt (forward step nst - 1 - tt) in stage tt % XSTAGES
  auto issue = [&](int tt, bool copy) {
    if (copy && tt < nst) {
      const float* src = F + (size_t)(nst - 1 - tt) * XSTEP;
      float* dst = ring + (size_t)(tt % XSTAGES) * XSTEP;
#pragma unroll
      for (int cg = 0; cg < R * G; ++cg) cp_async16(dst + (cg * 32 + lane) * 4, src + (cg * 32 + lane) * 4);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int q = 0; q < XSTAGES - 1; ++q) issue(q, true);

  // right-band pushes: lane u < XC holds those lane 31 needs at step u of a chunk
  float pbc[NQ], pbn[NQ];
  auto load_pb = [&](int kc, float (&dst)[NQ]) {
    const int i = kc * XC + XC - 1 - lane - 30;  // lane 31's row at chunk step lane
    const bool ok = pin && lane < XC && i >= 1 && i <= L1;
#pragma unroll
    for (int f = 0; f < NQ; ++f) {
      const int fc = f % NP;
      const bool left = fc < NL;
      dst[f] = (ok && (left || i < L1)) ? ld_poll(pin + f * (Lm + 1) + i) : 0.f;
    }
  };
  load_pb(nch - 1, pbc);
  // HVP: raw scores and direction of the rows XPF steps ahead
  float sb[XPF][R], vb[XPF][R];
#pragma unroll
  for (int u = 0; u < XPF; ++u) {
    const int i = (nst - 1 - u) - lane + 1;
    load_row<R>(po, i, jl, HV && i >= 1 && i <= L1, sb[u]);
    load_row<R>(pv, i, jl, HV && i >= 1 && i <= L1, vb[u]);
  }

  float ac[NS][R], at[NS][R], nx[NS][R], nt[NS][R];
#pragma unroll
  for (int q = 0; q < NS; ++q)
#pragma unroll
    for (int c = 0; c < R; ++c) { ac[q][c] = 0.f; at[q][c] = 0.f; nx[q][c] = 0.f; nt[q][c] = 0.f; }
  float hold[NS], holdt[NS], outp[NQ];
#pragma unroll
  for (int q = 0; q < NS; ++q) { hold[q] = 0.f; holdt[q] = 0.f; }
#pragma unroll
  for (int q = 0; q < NQ; ++q) outp[q] = 0.f;
  KSum kA, kB, kC;

  const float* cm = a.cmax + slot * (size_t)(a.nsteps / XC);
  float ckm = cm[nch - 1];   // the forward's largest hi alpha of the chunk about to run
  for (int kc = nch - 1; kc >= 0; --kc) {
    if (kc > 0) load_pb(kc - 1, pbn);
    const float ckm_next = kc > 0 ? cm[kc - 1] : NEG;
    // ---- quiet chunk: as in the first-order adjoint, every value inside a
    // chunk is bounded by the summed inflow (values and tangents, which a
    // cell's weights and weight tangents scale by bounded factors) plus its
    // inits.  With every entering push below kFlowTiny in magnitude and
    // every hi alpha kInitQuiet below S, the chunk computes nothing (its
    // output is already 0), pushes zeros to the left band and skips the
    // field copies of its later steps. ----
    {
      bool miss = false;
#pragma unroll
      for (int q = 0; q < NQ; ++q) miss |= is_sentinel(pbc[q]);
      if (__any_sync(FULL, miss) && miss) {
        const int ir = kc * XC + XC - 1 - lane - 30;   // as in load_pb
#pragma unroll
        for (int q = 0; q < NQ; ++q)
          if (is_sentinel(pbc[q]))
            pbc[q] = poll_value(pin + q * (Lm + 1) + ir, ld_poll(pin + q * (Lm + 1) + ir), deadline,
                                a.status, a.pair_done + p, 0.f);
      }
    }
    float inmax = 0.f;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      inmax = fmaxf(inmax, fmaxf(fabsf(hold[q]), fabsf(holdt[q])));
#pragma unroll
      for (int c = 0; c < R; ++c) inmax = fmaxf(inmax, fmaxf(fabsf(ac[q][c]), fabsf(at[q][c])));
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) inmax = fmaxf(inmax, fmaxf(fabsf(outp[q]), fabsf(pbc[q])));
    if (__all_sync(FULL, inmax < kFlowTiny && ckm - Sh < kInitQuiet)) {
      // no copy may still be landing in a stage this chunk refills
      asm volatile("cp.async.wait_all;" ::: "memory");
      for (int cu = 0; cu < XC; ++cu) {
        const int t = kc * XC + (XC - 1 - cu);
        const int tt = nst - 1 - t;
        // keep one commit group per step; copy only steps of later chunks
        issue(tt + XSTAGES - 1, nst - 1 - (tt + XSTAGES - 1) < kc * XC);
        const int i = t - lane + 1;
        if (lane == 0 && pout && i >= 1 && i <= L1) {
#pragma unroll
          for (int f = 0; f < NQ; ++f) {
            const int fc = f % NP;
            const bool left = fc < NL;
            pout[f * (Lm + 1) + (left ? i : i - 1)] = 0.f;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        hold[q] = 0.f;
        holdt[q] = 0.f;
#pragma unroll
        for (int c = 0; c < R; ++c) { ac[q][c] = 0.f; at[q][c] = 0.f; }
      }
#pragma unroll
      for (int q = 0; q < NQ; ++q) outp[q] = 0.f;
      if (HV && kc > 0) {   // the score ring for the next chunk's first steps
#pragma unroll
        for (int u = 0; u < XPF; ++u) {
          const int i = (kc - 1) * XC + (XC - 1 - u) - lane + 1;
          load_row<R>(po, i, jl, i >= 1 && i <= L1, sb[u]);
          load_row<R>(pv, i, jl, i >= 1 && i <= L1, vb[u]);
        }
      }
#pragma unroll
      for (int q = 0; q < NQ; ++q) pbc[q] = pbn[q];
      ckm = ckm_next;
      continue;
    }
#pragma unroll 1
    for (int u0 = 0; u0 < XC; u0 += XPF)
#pragma unroll
      for (int u = 0; u < XPF; ++u) {
        const int cu = u0 + u;
        const int t = kc * XC + (XC - 1 - cu);
        const int tt = nst - 1 - t;
        const int i = t - lane + 1;
        const bool act = (i >= 1) && (i <= L1);
        issue(tt + XSTAGES - 1, true);
        cp_async_wait<XSTAGES - 1>();
        const float* E = ring + (size_t)(tt % XSTAGES) * XSTEP + lane * 4;
        float r[NQ], pw[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          r[q] = __shfl_down_sync(FULL, outp[q], 1);
          pw[q] = __shfl_sync(FULL, pbc[q], cu);
        }
        {
          bool miss = false;
#pragma unroll
          for (int q = 0; q < NQ; ++q) miss |= is_sentinel(pw[q]);
          miss = miss && (lane == 31);
          if (__any_sync(FULL, miss) && miss) {
#pragma unroll
            for (int q = 0; q < NQ; ++q)
              if (is_sentinel(pw[q]))
                pw[q] = poll_value(pin + q * (Lm + 1) + i, ld_poll(pin + q * (Lm + 1) + i), deadline,
                                   a.status, a.pair_done + p, 0.f);
          }
        }
        // pushes arriving at column R-1 of row i: from the right lane (or band)
        // into the left of this cell, and into its diagonal from (i+1, j+1)
        if constexpr (NS == 3 && (GL || SV)) {
          float iL[3], tL[3], iD[3], tD[3];
          if (lane == 31) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              iL[q] = pw[q]; tL[q] = pw[NP + q]; iD[q] = pw[NL + q]; tD[q] = pw[NP + NL + q];
            }
          } else {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              iL[q] = r[q]; tL[q] = r[NP + q];
              iD[q] = hold[q]; hold[q] = r[NL + q];
              tD[q] = holdt[q]; holdt[q] = r[NP + NL + q];
            }
          }
#pragma unroll
          for (int q = 0; q < 3; ++q) { ac[q][R - 1] += iL[q] + iD[q]; at[q][R - 1] += tL[q] + tD[q]; }
          if (GL && term_lane && i == L1) {   // the terminal's beta-inits and their tangents
#pragma unroll
            for (int c = 0; c < R; ++c)
              if (jl + c == L2 - 1)
#pragma unroll
                for (int q = 0; q < 3; ++q) { ac[q][c] += tw[q]; at[q][c] += tdw[q]; }
          }
        } else if constexpr (NS == 3) {
          float iL0, iL1, tL0, tL1, iD[3], tD[3];
          if (lane == 31) {
            iL0 = pw[0]; iL1 = pw[1]; tL0 = pw[NP + 0]; tL1 = pw[NP + 1];
#pragma unroll
            for (int q = 0; q < 3; ++q) { iD[q] = pw[2 + q]; tD[q] = pw[NP + 2 + q]; }
          } else {
            iL0 = r[0]; iL1 = r[1]; tL0 = r[NP + 0]; tL1 = r[NP + 1];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              iD[q] = hold[q]; hold[q] = r[2 + q];
              tD[q] = holdt[q]; holdt[q] = r[NP + 2 + q];
            }
          }
          ac[0][R - 1] += iL0 + iD[0]; ac[1][R - 1] += iD[1]; ac[2][R - 1] += iL1 + iD[2];
          at[0][R - 1] += tL0 + tD[0]; at[1][R - 1] += tD[1]; at[2][R - 1] += tL1 + tD[2];
        } else {
          float iL, tL, iD, tD;
          if (lane == 31) {
            iL = pw[0]; iD = pw[1]; tL = pw[2]; tD = pw[3];
          } else {
            iL = r[0]; tL = r[2];
            iD = hold[0]; hold[0] = r[1];
            tD = holdt[0]; holdt[0] = r[3];
          }
          ac[0][R - 1] += iL + iD;
          at[0][R - 1] += tL + tD;
          if (GL && term_lane && i == L1) {   // beta = 1 at the terminal
#pragma unroll
            for (int c = 0; c < R; ++c)
              if (jl + c == L2 - 1) ac[0][c] += 1.f;
          }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) outp[q] = 0.f;
        float sc[R], vv[R];
#pragma unroll
        for (int c = 0; c < R; ++c) { sc[c] = sb[u][c]; vv[c] = vb[u][c]; }
        if (HV) {
          const int ip = i - XPF;
          load_row<R>(po, ip, jl, ip >= 1 && ip <= L1, sb[u]);
          load_row<R>(pv, ip, jl, ip >= 1 && ip <= L1, vb[u]);
        }
        float cA = 0.f, cB = 0.f, cC = 0.f;
        float pm[R];
#pragma unroll
        for (int c = R - 1; c >= 0; --c) {
          float4 f[G];
#pragma unroll
          for (int g = 0; g < G; ++g) f[g] = *reinterpret_cast<const float4*>(E + (c * G + g) * 128);
          const bool live = act && (jl + c < L2);
          if constexpr (NS == 3 && SV) {
            // f0 = (wMM, wMI, wMD, wIM) f1 = (wII, wDM, wDI, wDD) f2 = (dwMM, dwMI, dwMD, dwIM)
            // f3 = (dwII, dwDM, dwDI, dwDD) f4 = (Mh, Ml, uM, -); M's beta-init only
            const float xs = (f[4].x - Sh) + (f[4].y - Sl);
            const float e0 = live ? ex2(fminf(xs, 0.f)) : 0.f;
            float x = f[4].z - dS;
            if (TM) x -= (e0 > 0.f ? xs * LN2 : 0.f);
            const float bM = ac[0][c] + e0, tgM = at[0][c] + e0 * x * iT;
            const float bI = ac[1][c], tgI = at[1][c], bD = ac[2][c], tgD = at[2][c];
            const float qM = bM * f[0].x, qI = bM * f[0].y, qD = bM * f[0].z;
            const float tqM = fmaf(tgM, f[0].x, bM * f[2].x);
            const float tqI = fmaf(tgM, f[0].y, bM * f[2].y);
            const float tqD = fmaf(tgM, f[0].z, bM * f[2].z);
            const float pIM = bI * f[0].w, pII = bI * f[1].x;
            const float tIM = fmaf(tgI, f[0].w, bI * f[2].w);
            const float tII = fmaf(tgI, f[1].x, bI * f[3].x);
            const float pDM = bD * f[1].y, pDI = bD * f[1].z, pDD = bD * f[1].w;
            const float tDM = fmaf(tgD, f[1].y, bD * f[3].y);
            const float tDI = fmaf(tgD, f[1].z, bD * f[3].z);
            const float tDD = fmaf(tgD, f[1].w, bD * f[3].w);
            pm[c] = tgM;
            if (HV) {
              cA += (tIM + tDM) + tDI;
              cB += tII + tDD;
              cC = fmaf(tgM, sc[c], fmaf(bM, vv[c], cC));
            }
            nx[0][c] += pIM; nx[1][c] += pII;
            nt[0][c] += tIM; nt[1][c] += tII;
            if (c > 0) {
              nx[0][c - 1] += qM; nx[1][c - 1] += qI; nx[2][c - 1] += qD;
              nt[0][c - 1] += tqM; nt[1][c - 1] += tqI; nt[2][c - 1] += tqD;
              ac[0][c - 1] += pDM; ac[1][c - 1] += pDI; ac[2][c - 1] += pDD;
              at[0][c - 1] += tDM; at[1][c - 1] += tDI; at[2][c - 1] += tDD;
            } else {
              outp[0] = pDM; outp[1] = pDI; outp[2] = pDD; outp[3] = qM; outp[4] = qI; outp[5] = qD;
              outp[NP + 0] = tDM; outp[NP + 1] = tDI; outp[NP + 2] = tDD;
              outp[NP + 3] = tqM; outp[NP + 4] = tqI; outp[NP + 5] = tqD;
            }
          } else if constexpr (NS == 3 && GL) {
            // f0 = (wMM, wMI, wMD, wIM) f1 = (wII, wID, wDM, wDI) f2 = (wDD, dwMM, dwMI, dwMD)
            // f3 = (dwIM, dwII, dwID, dwDM) f4 = (dwDI, dwDD, -, -)
            const float bM = ac[0][c], bI = ac[1][c], bD = ac[2][c];
            const float tgM = at[0][c], tgI = at[1][c], tgD = at[2][c];
            const float qM = bM * f[0].x, qI = bM * f[0].y, qD = bM * f[0].z;
            const float tqM = fmaf(tgM, f[0].x, bM * f[2].y);
            const float tqI = fmaf(tgM, f[0].y, bM * f[2].z);
            const float tqD = fmaf(tgM, f[0].z, bM * f[2].w);
            const float pIM = bI * f[0].w, pII = bI * f[1].x, pID = bI * f[1].y;
            const float tIM = fmaf(tgI, f[0].w, bI * f[3].x);
            const float tII = fmaf(tgI, f[1].x, bI * f[3].y);
            const float tID = fmaf(tgI, f[1].y, bI * f[3].z);
            const float pDM = bD * f[1].z, pDI = bD * f[1].w, pDD = bD * f[2].x;
            const float tDM = fmaf(tgD, f[1].z, bD * f[3].w);
            const float tDI = fmaf(tgD, f[1].w, bD * f[4].x);
            const float tDD = fmaf(tgD, f[2].x, bD * f[4].y);
            pm[c] = tgM;
            if (HV) {
              cA += (tIM + tID) + (tDM + tDI);
              cB += tII + tDD;
              cC = fmaf(tgM, sc[c], fmaf(bM, vv[c], cC));
              // tangents pushed into the boundary states D(0, j) and I(i, 0)
              if (i == 1) {
                cA += tID + tqD;
                cB += (float)(jl + c) * tID + (float)(jl + c - 1) * tqD;
              }
              if (band == 0 && lane == 0 && c == 0) {
                cA += tDI + tqI;
                cB += (float)(i - 1) * tDI + (float)(i - 2) * tqI;
              }
            }
            nx[0][c] += pIM; nx[1][c] += pII; nx[2][c] += pID;
            nt[0][c] += tIM; nt[1][c] += tII; nt[2][c] += tID;
            if (c > 0) {
              nx[0][c - 1] += qM; nx[1][c - 1] += qI; nx[2][c - 1] += qD;
              nt[0][c - 1] += tqM; nt[1][c - 1] += tqI; nt[2][c - 1] += tqD;
              ac[0][c - 1] += pDM; ac[1][c - 1] += pDI; ac[2][c - 1] += pDD;
              at[0][c - 1] += tDM; at[1][c - 1] += tDI; at[2][c - 1] += tDD;
            } else {
              outp[0] = pDM; outp[1] = pDI; outp[2] = pDD; outp[3] = qM; outp[4] = qI; outp[5] = qD;
              outp[NP + 0] = tDM; outp[NP + 1] = tDI; outp[NP + 2] = tDD;
              outp[NP + 3] = tqM; outp[NP + 4] = tqI; outp[NP + 5] = tqD;
            }
          } else if constexpr (NS == 3) {
            const float xs[3] = {(f[3].z - Sh) + (f[4].y - Sl), (f[3].w - Sh) + (f[4].z - Sl),
                                 (f[4].x - Sh) + (f[4].w - Sl)};
            const float us[3] = {f[5].x, f[5].y, f[5].z};
            float b[3] = {ac[0][c], ac[1][c], ac[2][c]}, tg[3] = {at[0][c], at[1][c], at[2][c]};
#pragma unroll
            for (int st = 0; st < 3; ++st) {
              const float e0 = live ? ex2(fminf(xs[st], 0.f)) : 0.f;
              b[st] += e0;
              float x = us[st] - dS;
              if (TM) x -= (e0 > 0.f ? xs[st] * LN2 : 0.f);
              tg[st] += e0 * x * iT;
            }
            // f0 = (wMM, wMI, wMD, wIM) f1 = (wII, wDM, wDD, dwMM)
            // f2 = (dwMI, dwMD, dwIM, dwII) f3 = (dwDM, dwDD, ...)
            const float qM = b[0] * f[0].x, qI = b[0] * f[0].y, qD = b[0] * f[0].z;
            const float pIM = b[1] * f[0].w, pII = b[1] * f[1].x;
            const float pDM = b[2] * f[1].y, pDD = b[2] * f[1].z;
            const float tqM = fmaf(tg[0], f[0].x, b[0] * f[1].w);
            const float tqI = fmaf(tg[0], f[0].y, b[0] * f[2].x);
            const float tqD = fmaf(tg[0], f[0].z, b[0] * f[2].y);
            const float tIM = fmaf(tg[1], f[0].w, b[1] * f[2].z);
            const float tII = fmaf(tg[1], f[1].x, b[1] * f[2].w);
            const float tDM = fmaf(tg[2], f[1].y, b[2] * f[3].x);
            const float tDD = fmaf(tg[2], f[1].z, b[2] * f[3].y);
            pm[c] = tg[0];
            if (HV) {
              cA += tIM + tDM;
              cB += tII + tDD;
              cC = fmaf(tg[0], sc[c], fmaf(b[0], vv[c], cC));
            }
            nx[0][c] += pIM; nx[1][c] += pII;
            nt[0][c] += tIM; nt[1][c] += tII;
            if (c > 0) {
              nx[0][c - 1] += qM; nx[1][c - 1] += qI; nx[2][c - 1] += qD;
              nt[0][c - 1] += tqM; nt[1][c - 1] += tqI; nt[2][c - 1] += tqD;
              ac[0][c - 1] += pDM; ac[2][c - 1] += pDD;
              at[0][c - 1] += tDM; at[2][c - 1] += tDD;
            } else {
              outp[0] = pDM; outp[1] = pDD; outp[2] = qM; outp[3] = qI; outp[4] = qD;
              outp[NP + 0] = tDM; outp[NP + 1] = tDD;
              outp[NP + 2] = tqM; outp[NP + 3] = tqI; outp[NP + 4] = tqD;
            }
          } else {
            // f0 = (w_diag, w_up, w_left, map factor) f1 = their tangents
            // f2 = (Ah, Al, U, 0)
            const float xs = (f[2].x - Sh) + (f[2].y - Sl);
            const float e0 = (!GL && live) ? ex2(fminf(xs, 0.f)) : 0.f;
            const float b = ac[0][c] + e0;
            float x = f[2].z - dS;
            if (TM) x -= (e0 > 0.f ? xs * LN2 : 0.f);
            const float tg = at[0][c] + e0 * x * iT;
            const float P = b * f[0].w;
            const float Pd = fmaf(tg, f[0].w, b * f[1].w);
            const float pD = b * f[0].x, pU = b * f[0].y, pL = b * f[0].z;
            const float tpD = fmaf(tg, f[0].x, b * f[1].x);
            const float tpU = fmaf(tg, f[0].y, b * f[1].y);
            const float tpL = fmaf(tg, f[0].z, b * f[1].z);
            pm[c] = Pd;
            if (HV) {
              cA += tpU + tpL;
              cC = fmaf(Pd, sc[c], fmaf(P, vv[c], cC));
              if constexpr (GL) {   // tangents pushed into the boundary cells
                if (i == 1) cA += (float)(jl + c + 1) * tpU + (float)(jl + c) * tpD;
                if (band == 0 && lane == 0 && c == 0) cA += (float)i * tpL + (float)(i - 1) * tpD;
              }
            }
            nx[0][c] += pU;
            nt[0][c] += tpU;
            if (c > 0) {
              nx[0][c - 1] += pD; nt[0][c - 1] += tpD;
              ac[0][c - 1] += pL; at[0][c - 1] += tpL;
            } else {
              outp[0] = pL; outp[1] = pD; outp[2] = tpL; outp[3] = tpD;
            }
          }
        }
        if (act) {
          store_row<R>(po, i, jl, pm);
          if (lane == 0 && pout) {
#pragma unroll
            for (int f = 0; f < NQ; ++f) {
              const int fc = f % NP;
              const bool left = fc < NL;
              pout[f * (Lm + 1) + (left ? i : i - 1)] = outp[f];
            }
          }
        }
        if (HV) { kA.add(cA); kB.add(cB); kC.add(cC); }
#pragma unroll
        for (int q = 0; q < NS; ++q)
#pragma unroll
          for (int c = 0; c < R; ++c) {
            ac[q][c] = nx[q][c]; nx[q][c] = 0.f;
            at[q][c] = nt[q][c]; nt[q][c] = 0.f;
          }
      }
#pragma unroll
    for (int q = 0; q < NQ; ++q) pbc[q] = pbn[q];
    ckm = ckm_next;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncwarp();
  float v0 = kA.s, v1 = kB.s, v2 = kC.s;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_xor_sync(FULL, v0, o);
    v1 += __shfl_xor_sync(FULL, v1, o);
    v2 += __shfl_xor_sync(FULL, v2, o);
  }
  xfinish<NS, MODE>(a, p, band, lane, false, dS, v0, v1, v2, L1, L2);
}

template <int NS, int R, int MODE, int GM = 0>
__global__ void __launch_bounds__(32, SWB_XBWD_MINB) xbwd_kernel(XArgs a) {
  extern __shared__ __align__(16) float xring[];
  const int lane = threadIdx.x & 31;
  const uint64_t deadline = gtimer() + a.spin_limit_ns;
  const int ntasks = a.B * a.nb;
  while (true) {
    int task = 0;
    if (lane == 0) task = (int)atomicAdd(a.counters + 1, 1u);
    task = __shfl_sync(FULL, task, 0);
    if (task >= ntasks) break;
    const int p = task / a.nb;
    xbwd_band<NS, R, MODE, GM>(a, p, a.nb - 1 - (task - p * a.nb), lane, xring, deadline);
  }
}

}  // namespace swb
