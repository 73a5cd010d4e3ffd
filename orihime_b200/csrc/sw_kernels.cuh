// Soft Smith-Waterman wavefront kernels for sm_100a (linear and affine gaps).
//
// Work decomposition
// ------------------
// A pair (L1 x L2 scores) is cut into column *bands* of 32*R columns.  One
// warp owns one band: lane l owns the R consecutive columns
// [band*32R + l*R, +R) and the warp sweeps the rows top to bottom as a skewed
// wavefront -- at step t lane l works on row i = t - l + 1 (1-based), so the
// band takes L1 + 31 steps (padded to whole checkpoint chunks).  The values of
// a lane's last column reach lane l+1 one step later through __shfl_up_sync;
// the last lane of a band writes them to a global "edge" buffer that lane 0
// of the next band polls.
//
// Arithmetic
// ----------
// DP values live in a scaled log2 domain, x' = x * log2(e) / T, so every
// exp/log of the reference recurrence is one MUFU ex2/lg2.  Each value is a
// double-float pair (hi, lo) with value = hi + lo: the hi part is an exact
// copy of a predecessor's hi (or of a TwoSum), and every exponent is formed
// as ((hi - base) + edge) + lo.  FP32 rounding of the DP values therefore
// never accumulates along alignment paths, which is what limits the accuracy
// of a plain FP32 forward-backward (the reference included) on long pairs.
//
// Forward kernel (one launch per op call): alpha, the partition partials and,
// every C steps, a per-lane checkpoint of the DP state.  No alpha table is
// ever stored.
//
// Adjoint kernel: per band, time chunks in reverse.  Each chunk restores its
// checkpoint and recomputes C steps of alpha; every cell writes its adjoint
// fields to shared memory: the weights of its predecessors (the recurrence's
// own softmax terms divided by their sum, so they add up to 1 and the adjoint
// conserves probability flow whatever the MUFU rounding), its beta-init term
// exp2(min(x - S, 0)) and its scaled score.  The adjoint then runs the chunk
// backwards in "push" form with multiply-adds only: a finished cell pushes
// beta*w to its predecessors -- within the lane through registers, to the
// left lane through __shfl_down_sync, to the left band through a global
// buffer.  No atomics; the map is written row by row.
//
// Cross-band buffers are filled with a NaN sentinel before each call; a
// consumer polls the value itself until it is not the sentinel, so no memory
// fence is needed on the producer side.  Every poll is bounded by a
// globaltimer deadline; on expiry the kernel records SWB_STATUS_WAIT_TIMEOUT
// in the status word, substitutes a neutral value and carries on, so no warp
// can hang.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace swb {

constexpr float NEG = -1e30f;           // "no path" in the scaled domain
// Adjoint flows below this (2^-60) entering a chunk count as none.  A chunk
// whose inflow (at most ~660 values) and beta-inits (512 cells x 3 states) are
// all below it holds less than ~2e-15 of probability in total; summed over
// every such chunk of a pair, the dropped mass stays below ~1e-10.
constexpr float kFlowTiny = 8.6736173798840355e-19f;
// A chunk's beta-inits are all below kFlowTiny when every hi alpha in it lies
// this far below S (scaled log2 units; 3 of margin for the lo parts).
constexpr float kInitQuiet = -63.f;
constexpr unsigned FULL = 0xffffffffu;
#ifndef SWB_C_STEPS
#define SWB_C_STEPS 4
#endif
constexpr int C_STEPS = SWB_C_STEPS;    // checkpoint stride (steps)
#ifndef SWB_PF
#define SWB_PF 2
#endif
constexpr int PF = SWB_PF;              // score prefetch distance (steps); C_STEPS % PF == 0
constexpr uint32_t SENTINEL_BITS = 0xffffffffu;

// Ragged plan: per-pair words.  Offsets are in floats within the respective
// workspace array; score_off is the pair's element offset in the packed
// score/map buffers (row pitch = L2 rounded up to a multiple of 4).
enum PlanWord : int {
  PW_SCORE_OFF = 0, PW_L1 = 1, PW_L2 = 2, PW_SLOT0 = 3, PW_NB = 4,
  PW_CK0 = 5, PW_EDGE0 = 6, PW_BP0 = 7, PLAN_PAIR_WORDS = 8
};

enum : unsigned {
  ERR_WAIT_TIMEOUT = 1u,
  ERR_BAD_LENGTHS = 2u,      // a pair's lengths outside [0, padded size] (checked on the device)
  ERR_BAD_PARAMS = 4u,       // device parameters: temperature not finite > 0, or a positive gap
};

// Launch arguments shared by the forward and adjoint kernels.
struct Args {
  // problem
  const float* scores;        // layout 0: [B, Lmax1, Lmax2]; layout 1: flat ragged
  float* map;                 // same layout as scores
  const int* lengths;         // [B, 2] or null (= full padded lengths)
  const int* order;           // layout 0: optional pair order of the task queue (null = 0..B-1)
  const long long* plan_pairs;// layout 1: [B][PLAN_PAIR_WORDS] per-pair placement (see below)
  const int* plan_tasks;      // layout 1: [ntasks][2] (pair, band) in queue order
  int ntasks;                 // layout 1: number of band tasks
  int B, Lmax1, Lmax2;
  int layout;                 // 0 padded, 1 ragged packed via plan (row pitch = round4(L2))
  float go, ge, T, k;         // gaps in natural units, temperature, k = log2(e)/T
  float xgo, xge;             // linear-domain kernels: transition factors 2^(go k), 2^(ge k)
  const float* dparams;       // linear-domain kernels: (go, ge, T) or (gap, T) read on the device
                              // instead of go, ge, T (graph capture with tensor parameters), or null
  int nb;                     // bands per pair (uniform, >= ceil(max L2 / 32R))
  int nchunks;                // checkpoint chunks per band (>= ceil((max L1+31)/C))
  int ck_every;               // linear-domain kernels: a checkpoint every ck_every chunks (>= 1)
  size_t ck_band_floats;      // layout 0: checkpoint floats per band slot (0: nchunks records)
  // outputs [B]
  float* value;
  float* g_open;              // affine: dS/dgo ; linear: dS/dgap
  float* g_ext;               // affine: dS/dge ; linear: unused
  float* g_T;
  // workspace (see layout_for in sw_capi.cu)
  unsigned* counters;         // [0] forward task counter, [1] adjoint task counter
  unsigned* status;           // error bits
  unsigned* pair_done;        // [B]
  float* part;                // [B*nb][2] partition partials (ref, sum)
  float* gpart;               // [B*nb][4] gradient partials
  float* edge;                // [B*nb][2*NS][Lmax1] sentinel-initialised
  float* bpush;               // [B*nb][NP][Lmax1+1] sentinel-initialised
  float* ckpt;                // [B*nb][nchunks][CKF][32]
  unsigned long long spin_limit_ns;
  int fault_inject;           // 1: band>0 waits on a word nobody writes (tests only)
  float* never_written;       // target of fault_inject polls
  // tangent (second-order) kernels of the linear domain, layout 0 only
  const float* tdir;          // tmode 0: the score direction [B, Lmax1, Lmax2]
  float* tgt;                 // tmode 0: per pair tangents of (g0, g1, g_T, S) [B][4], or null
  float* zdot;                // [B*nb][2] per band: frame, tangent of the partition sum
  int tmode;                  // 0 score direction, 1 gap_open (linear: gap), 2 gap_ext, 3 temperature
};

}  // namespace swb
