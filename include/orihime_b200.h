/*
 * orihime_b200 — C ABI of the B200 (sm_100a) soft Smith–Waterman kernels.
 *
 * This is the drop-in boundary for the CUDA path of megure-labs/orihime's
 * soft Smith–Waterman operators.  Each entry point replaces one CUDA op body
 * of the reference (the C++ functions registered under
 * TORCH_LIBRARY_IMPL(orihime, CUDA)) together with the extern "C" launchers it
 * calls; references are to files of that project.
 *
 * Conventions
 *   - All pointers are device pointers unless stated; float32 data, int32
 *     lengths, row-major.
 *   - scores / map use the reference's padded layout [B, L1max, L2max].
 *     lengths is [B, 2] (rows, cols used by pair b) or NULL for full lengths;
 *     0 <= lengths[b][k] <= L{1,2}max is the caller's responsibility (the
 *     Python host checks it with the reference's error messages).
 *   - Every call is asynchronous on `stream` (a cudaStream_t, NULL = legacy
 *     default stream), allocates nothing and never synchronises, so it can be
 *     captured in a CUDA graph.  Device scratch is passed as `workspace`,
 *     at least *_workspace_bytes() bytes, 256-byte aligned; calls that share a
 *     workspace must be ordered on one stream.
 *   - Outputs: value [B] (soft alignment score S), map [B, L1max, L2max]
 *     (dS/dscores; exactly 0 outside lengths), and per-pair dS/dparameter [B].
 *   - Return value: SWB_OK or a negative SWB_ERR_* code (nothing launched).
 *     A bounded cross-warp wait that expires inside a kernel is reported in the
 *     workspace status word (swb_read_status), not by the return value, and
 *     the affected pairs' value and gradients come back NaN.
 */
#ifndef ORIHIME_B200_H
#define ORIHIME_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWB_ABI_VERSION 2

#define SWB_OK 0
#define SWB_ERR_ARG (-1)
#define SWB_ERR_WORKSPACE (-2)
#define SWB_ERR_CUDA (-3)

/* Status bits written by kernels into the workspace status word.  The pairs
 * concerned also come back NaN (value, dS/dparameters). */
#define SWB_STATUS_WAIT_TIMEOUT 1u
#define SWB_STATUS_BAD_LENGTHS 2u   /* lengths outside [0, padded size], checked on the device */
#define SWB_STATUS_BAD_PARAMS 4u    /* device parameters invalid (params_device) */

/* Optional launch knobs (pass NULL for defaults). */
typedef struct swb_options {
    int max_ctas;                      /* cap on persistent CTAs (0 = occupancy-derived) */
    unsigned long long spin_limit_ns;  /* bound on every cross-warp wait (0 = 20 s)      */
    int fault_inject;                  /* 1: band>0 waits on a word nobody writes (tests) */
    void* split_event;                 /* cudaEvent_t recorded between the forward and the
                                          adjoint kernel (per-kernel timing), or NULL     */
    int cols_per_lane;                 /* columns per lane of a band: 2, 4 or (local families,
                                          linear domain) 8; 0 = swb_cols_per_lane's default */
    int domain;                        /* local models: SWB_DOMAIN_AUTO (0), _LOG or _LINEAR */
    const float* params_device;        /* local models, linear domain: device array
                                          (gap_open, gap_ext, temp) or (gap, temp) that the
                                          kernels read at run time instead of the float
                                          arguments (a CUDA graph captured with tensor
                                          parameters reads their current values at each
                                          replay); NULL = use the floats.  The floats still
                                          choose the domain: keep the gaps <= 0.  Invalid
                                          device values give NaN results and
                                          SWB_STATUS_BAD_PARAMS. */
} swb_options;

/* Arithmetic of the local-alignment kernels (swb_options.domain).  AUTO runs
 * the scaled linear domain (one ex2 per cell, multiply-adds, power-of-two
 * frames per lane) whenever every gap parameter is <= 0, else the scaled log
 * domain (double-float log-sum-exp); LOG forces the latter; LINEAR requires
 * the former and returns SWB_ERR_ARG when a gap parameter is positive.  The
 * global and Saigo-Vert families always run in the log domain. */
#define SWB_DOMAIN_AUTO 0
#define SWB_DOMAIN_LOG 1
#define SWB_DOMAIN_LINEAR 2

/* Columns per lane the padded entry points use when swb_options does not
 * set one: for the local families (family 1 linear gap, 3 affine gaps) in
 * the linear domain, 8 on batches with L2max >= 256, 2 on batches with
 * L2max <= 64, else 4; in the log domain and for families 2, 4, 5 (the
 * global and Saigo-Vert models) always 4.  Results depend on it bit for
 * bit (the band decomposition orders each pair's sums), so a packed plan
 * built with the same value reproduces a padded call exactly.  No reference
 * counterpart. */
int swb_cols_per_lane(int family, int L2max, float gap_open, float gap_ext, float temp);

/* Workspace bytes for swb_sw_affine_forward on a [B, L1max, L2max] batch. */
size_t swb_sw_affine_workspace_bytes(int B, int L1max, int L2max);

/*
 * Soft Smith–Waterman, affine gaps: value, marginal map and dS/d(gap_open,
 * gap_ext, temp) in one call (forward wavefront + checkpointed adjoint).
 * Replaces orihime_sw_affine_forward_cuda / soft_sw_affine_cuda_float
 * (src/sw_affine/torch_cuda.cpp:820, :419 -> SoftSWAffineCUDAFunction::forward
 * :128-206) and orihime_sw_affine_value_grad_params_cuda (:842 ->
 * soft_sw_affine_cuda_with_grads :446), i.e. the launchers sw_affine_forward +
 * sw_affine_backward (src/sw_affine/kernels_gpu.cuh:165, :193).
 */
int swb_sw_affine_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp,
                          float* value, float* map,
                          float* grad_open, float* grad_ext, float* grad_temp,
                          void* workspace, size_t workspace_bytes, void* stream,
                          const swb_options* opt);

/* Size of the fixed device scratch of swb_sw_affine_forward_static (32 MiB). */
#define SWB_STATIC_SCRATCH_BYTES (32u * 1024u * 1024u)

/*
 * swb_sw_affine_forward without a workspace argument (no reference
 * counterpart: the reference allocates its scratch through torch inside each
 * op).  For callers that hold device pointers to their inputs and outputs but
 * no device allocator of their own, e.g. a plain C or FFI host: it needs no
 * workspace and makes no allocating call (no cudaMalloc/cudaFree, no library
 * allocator).  Scratch is one file-scope device array of
 * SWB_STATIC_SCRATCH_BYTES per device; whatever must start at zero or at the
 * sentinel is reset with cudaMemsetAsync on `stream` at every call.
 *   - Limit: returns SWB_ERR_WORKSPACE, before any CUDA call, when the
 *     batch's workspace at the chosen columns per lane exceeds
 *     SWB_STATIC_SCRATCH_BYTES.  Every batch whose
 *     swb_sw_affine_workspace_bytes(B, L1max, L2max) is within the limit
 *     fits (e.g. 8 x 512 x 512); at the default 4 columns per lane about
 *     12 x 512 x 512 or one 2048 x 2048 pair fit.
 *   - The first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress, which may load the module) and sets up the
 *     kernels; make that first call before any stream capture.  The address
 *     is cached per device and CUDA context: after cudaDeviceReset (or a
 *     re-created primary context) the next call looks it up again.
 *   - All calls of one process on one device share the array: calls that
 *     overlap in time (on different streams, or from several host threads,
 *     without ordering) race and corrupt each other's results.  Order them on
 *     one stream.
 *   - A bounded wait that expires makes the affected pairs' value and
 *     gradients NaN; the status word in the shared array records it too and
 *     is read with swb_static_read_status (not swb_read_status).
 * Arguments and outputs as swb_sw_affine_forward.
 */
int swb_sw_affine_forward_static(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp,
                                 float* value, float* map,
                                 float* grad_open, float* grad_ext, float* grad_temp,
                                 void* stream, const swb_options* opt);

/* Workspace bytes for swb_sw_forward on a [B, L1max, L2max] batch. */
size_t swb_sw_workspace_bytes(int B, int L1max, int L2max);

/*
 * Soft Smith–Waterman, linear gap: value, marginal map, dS/dgap, dS/dT.
 * Replaces orihime_sw_forward_cuda / soft_sw_cuda_float and
 * orihime_sw_value_grad_params_cuda (src/sw/torch_cuda.cpp:364-450,
 * :803-830 registration), i.e. the launchers sw_regular_forward +
 * sw_regular_backward (src/sw/kernels_gpu.cuh:139, :165).
 */
int swb_sw_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                   float gap, float temp,
                   float* value, float* map, float* grad_gap, float* grad_temp,
                   void* workspace, size_t workspace_bytes, void* stream,
                   const swb_options* opt);

/*
 * Value only: S per pair, without the marginal map or gradients.  Runs the
 * forward wavefront alone (no checkpoints, no adjoint) and folds each pair's
 * band partials, so scoring costs about half a full call; the values equal
 * those of swb_sw_affine_forward / swb_sw_forward bit for bit.  No reference
 * counterpart: the reference's forward ops always run forward and backward.
 * Workspace from swb_sw_affine_value_workspace_bytes / swb_sw_value_workspace_bytes.
 */
size_t swb_sw_affine_value_workspace_bytes(int B, int L1max, int L2max);
int swb_sw_affine_value(const float* scores, const int* lengths, int B, int L1max, int L2max,
                        float gap_open, float gap_ext, float temp, float* value, void* workspace,
                        size_t workspace_bytes, void* stream);
size_t swb_sw_value_workspace_bytes(int B, int L1max, int L2max);
int swb_sw_value(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                 float temp, float* value, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Soft Needleman–Wunsch (global alignment), linear gap: value S = A[L1, L2],
 * marginal map (posterior of each aligned cell), dS/dgap, dS/dT.  Boundaries
 * A[i,0] = i*gap, A[0,j] = j*gap, no local start.  Replaces nw_forward_cuda /
 * soft_nw_cuda_float and nw_value_grad_params_cuda (src/nw/torch_cuda.cpp:364,
 * :716-745, registration :795-821), i.e. the launchers nw_forward +
 * nw_backward (src/nw/kernels_gpu.cuh:209, :232).  Same band wavefront as swb_sw_forward;
 * workspace from swb_nw_workspace_bytes.
 */
size_t swb_nw_workspace_bytes(int B, int L1max, int L2max);
int swb_nw_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                   float gap, float temp,
                   float* value, float* map, float* grad_gap, float* grad_temp,
                   void* workspace, size_t workspace_bytes, void* stream,
                   const swb_options* opt);
/*
 * Soft Needleman–Wunsch with affine gaps: value S = LSE(M, I, D at (L1, L2)),
 * marginal map (posterior of M), dS/dgap_open, dS/dgap_ext, dS/dT.  Three
 * states with I <- (M, I, D) from above and D <- (M, I, D) from the left;
 * boundaries M(0,0) = 0, I(i,0) = go + (i-1) ge, D(0,j) = go + (j-1) ge.
 * Replaces soft_nw_affine_cuda_float / soft_nw_affine_cuda_with_grads
 * (src/nw_affine/torch_cuda.cpp:364, :387; registration :763-786), i.e. the reference
 * launchers nw_affine_forward + nw_affine_backward
 * (src/nw_affine/kernels_cpu.cpp:100-347 restated).  Workspace from
 * swb_nw_affine_workspace_bytes; the value-only call and the packed ragged
 * calls (plan family 4) follow the linear global ones.
 */
size_t swb_nw_affine_workspace_bytes(int B, int L1max, int L2max);
int swb_nw_affine_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, float* value, float* map,
                          float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                          size_t workspace_bytes, void* stream, const swb_options* opt);
size_t swb_nw_affine_value_workspace_bytes(int B, int L1max, int L2max);
int swb_nw_affine_value(const float* scores, const int* lengths, int B, int L1max, int L2max,
                        float gap_open, float gap_ext, float temp, float* value, void* workspace,
                        size_t workspace_bytes, void* stream);
int swb_nw_affine_ragged(const float* scores, const void* host_plan, const void* dev_plan,
                         float gap_open, float gap_ext, float temp, float* value, float* map,
                         float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                         size_t workspace_bytes, void* stream, const swb_options* opt);
int swb_nw_affine_ragged_value(const float* scores, const void* host_plan, const void* dev_plan,
                               float gap_open, float gap_ext, float temp, float* value,
                               void* workspace, size_t workspace_bytes, void* stream);

/*
 * Saigo–Vert local alignment, affine gaps: value S = LSE(0, M cells), marginal
 * map (posterior of M), dS/dgap_open, dS/dgap_ext, dS/dT.  The local affine
 * model with one more transition, D <- I (gap open) from the left; only M
 * ends an alignment.  Replaces soft_sv_affine_cuda_float /
 * soft_sv_affine_cuda_with_grads (src/sv_affine/torch_cuda.cpp), restating
 * src/sv_affine/kernels_cpu.cpp:81-365.  The linear model
 * (src/sv_linear) is this one with gap_open = gap_ext = gap and
 * dS/dgap = dS/dgap_open + dS/dgap_ext.  Value-only and packed ragged calls
 * (plan family 5) as for the other families.
 */
size_t swb_sv_affine_workspace_bytes(int B, int L1max, int L2max);
int swb_sv_affine_forward(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, float* value, float* map,
                          float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                          size_t workspace_bytes, void* stream, const swb_options* opt);
size_t swb_sv_affine_value_workspace_bytes(int B, int L1max, int L2max);
int swb_sv_affine_value(const float* scores, const int* lengths, int B, int L1max, int L2max,
                        float gap_open, float gap_ext, float temp, float* value, void* workspace,
                        size_t workspace_bytes, void* stream);
int swb_sv_affine_ragged(const float* scores, const void* host_plan, const void* dev_plan,
                         float gap_open, float gap_ext, float temp, float* value, float* map,
                         float* grad_open, float* grad_ext, float* grad_temp, void* workspace,
                         size_t workspace_bytes, void* stream, const swb_options* opt);
int swb_sv_affine_ragged_value(const float* scores, const void* host_plan, const void* dev_plan,
                               float gap_open, float gap_ext, float temp, float* value,
                               void* workspace, size_t workspace_bytes, void* stream);

/* Value only (forward wavefront alone; equals swb_nw_forward's value bit for bit). */
size_t swb_nw_value_workspace_bytes(int B, int L1max, int L2max);
int swb_nw_value(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                 float temp, float* value, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Packed ragged batch (no reference counterpart: the reference pads every
 * pair to one shape; this is the batched path beside its drop-in).
 *
 * Packing: pair b's scores are an L1_b x L2_b row-major block with row pitch
 * P_b = L2_b rounded up to a multiple of 4, starting at element offsets[b]
 * (a multiple of 4) of one flat float buffer; offsets has B+1 entries and
 * offsets[b+1] - offsets[b] >= L1_b * P_b.  The map uses the same packing;
 * its pitch padding is written as 0.
 *
 * swb_ragged_plan runs on the host: it validates the packing, orders the
 * pairs by critical path (L1 + 31 x bands wavefront steps, then cells) for
 * the persistent task queue and places every band's workspace slice.  Call
 * it once with plan = NULL to get
 * *plan_bytes (and *workspace_bytes), then with a buffer of that size; copy
 * the plan bytes to the device unchanged and pass both copies to the launch.
 * family: 3 = affine, 1 = linear, 2 = global alignment (soft Needleman–Wunsch,
 * linear gap), 4 = global alignment with affine gaps, 5 = Saigo–Vert;
 * cols_per_lane: 2 or 4 (0 = default).
 * host lengths [B, 2], host offsets [B+1].
 */
int swb_ragged_plan(int family, int cols_per_lane, const int* lengths, const long long* offsets,
                    int B, void* plan, size_t plan_capacity, size_t* plan_bytes,
                    size_t* workspace_bytes);

/* Affine soft Smith–Waterman over a packed ragged batch; outputs as
 * swb_sw_affine_forward, map in the packed layout. */
int swb_sw_affine_ragged(const float* scores, const void* host_plan, const void* dev_plan,
                         float gap_open, float gap_ext, float temp,
                         float* value, float* map,
                         float* grad_open, float* grad_ext, float* grad_temp,
                         void* workspace, size_t workspace_bytes, void* stream,
                         const swb_options* opt);

/* Linear-gap soft Smith–Waterman over a packed ragged batch. */
int swb_sw_ragged(const float* scores, const void* host_plan, const void* dev_plan,
                  float gap, float temp,
                  float* value, float* map, float* grad_gap, float* grad_temp,
                  void* workspace, size_t workspace_bytes, void* stream,
                  const swb_options* opt);

/*
 * Value only for a packed ragged batch (no map, no gradients): the forward
 * wavefront and a per-pair fold, with the same plan and workspace as
 * swb_sw_affine_ragged / swb_sw_ragged (its checkpoint part goes unused).
 * The values equal the full call's bit for bit.  No reference counterpart.
 */
int swb_sw_affine_ragged_value(const float* scores, const void* host_plan, const void* dev_plan,
                               float gap_open, float gap_ext, float temp, float* value,
                               void* workspace, size_t workspace_bytes, void* stream);
int swb_sw_ragged_value(const float* scores, const void* host_plan, const void* dev_plan, float gap,
                        float temp, float* value, void* workspace, size_t workspace_bytes,
                        void* stream);
/* Global alignment over a family-2 plan: as swb_sw_ragged / swb_sw_ragged_value. */
int swb_nw_ragged(const float* scores, const void* host_plan, const void* dev_plan, float gap,
                  float temp, float* value, float* map, float* grad_gap, float* grad_temp,
                  void* workspace, size_t workspace_bytes, void* stream, const swb_options* opt);
int swb_nw_ragged_value(const float* scores, const void* host_plan, const void* dev_plan, float gap,
                        float temp, float* value, void* workspace, size_t workspace_bytes,
                        void* stream);

/*
 * Second-order ops (band wavefronts: a forward kernel carrying alpha and its
 * tangent, then a backward kernel carrying beta and its tangent).  Two kernel
 * pairs serve them, chosen per call from the parameters:
 *   - every gap <= 0 and 0 < T < inf: the scaled linear-domain dual-number
 *     kernels, whose workspace holds per-chunk checkpoints of values and
 *     tangents plus per-band edge, push and partial buffers (about 7 B per
 *     cell of the padded batch at 4 columns per lane);
 *   - otherwise the log-domain kernels, whose workspace holds, for every cell
 *     the wavefront visits, the fields the backward reads: 24 floats affine
 *     (weights, weight tangents, alpha hi/lo, tangents), 12 linear; about 100
 *     (affine) or 50 (linear) bytes per cell.
 * swb_sw_affine_aux_workspace_bytes is enough for any parameters (the larger
 * of the two); swb_sw_affine_aux_workspace_bytes_for is enough for the given
 * ones (what the call with them launches).  Callers that bound memory split
 * the batch into pair groups.
 */
size_t swb_sw_affine_aux_workspace_bytes(int B, int L1max, int L2max);
size_t swb_sw_affine_aux_workspace_bytes_for(int B, int L1max, int L2max, float gap_open,
                                             float gap_ext, float temp);

/*
 * Hessian-vector product of the marginal map: out = d(map)/d(scores) . v
 * [B, L1max, L2max], zero outside lengths.  Replaces soft_sw_affine_hvp_cuda
 * (src/sw_affine/torch_cuda.cpp:508 -> sw_affine_hvp, kernels_gpu.cu:1566).
 * grad_tangents (optional, device [B][4]): per pair the tangents along v of
 * (dS/dgap_open, dS/dgap_ext, dS/dT, S); their batch sums are the parameter
 * part of the map's VJP with cotangent v, which
 * orihime_sw_affine_marginals_backward_cuda (torch_cuda.cpp:681-811) gets from
 * three parameter-Jacobian passes.
 */
int swb_sw_affine_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
                      int L2max, float gap_open, float gap_ext, float temp, float* out,
                      float* grad_tangents, void* workspace, size_t workspace_bytes, void* stream);

/*
 * d(map)/d(theta) [B, L1max, L2max], param 0 = gap_open, 1 = gap_ext, 2 = temp.
 * Replaces soft_sw_affine_param_jacobian_cuda (src/sw_affine/torch_cuda.cpp:580
 * -> sw_affine_param_grad, kernels_gpu.cu:1638).
 */
int swb_sw_affine_param_jacobian(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp, int param,
                                 float* out, void* workspace, size_t workspace_bytes, void* stream);

size_t swb_sw_aux_workspace_bytes(int B, int L1max, int L2max);
size_t swb_sw_aux_workspace_bytes_for(int B, int L1max, int L2max, float gap, float temp);

/* Linear-gap HVP (src/sw/torch_cuda.cpp marginals_hvp body); grad_tangents
 * [B][4] = tangents of (dS/dgap, dS/dT, 0, S). */
int swb_sw_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
               int L2max, float gap, float temp, float* out, float* grad_tangents,
               void* workspace, size_t workspace_bytes, void* stream);

/* Linear-gap d(map)/d(theta), param 0 = gap, 1 = temp
 * (src/sw/torch_cuda.cpp param-Jacobian body, kernels_cpu.cpp:491-710). */
int swb_sw_param_jacobian(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap, float temp, int param, float* out, void* workspace,
                          size_t workspace_bytes, void* stream);

/*
 * Global alignment (soft Needleman–Wunsch, linear gap) second-order ops on the
 * same band wavefront; workspace from swb_nw_aux_workspace_bytes.
 * swb_nw_hvp replaces soft_nw_hvp_cuda (src/nw/torch_cuda.cpp:442, launcher
 * nw_hvp src/nw/kernels_gpu.cuh:258); grad_tangents [B][4] = tangents of
 * (dS/dgap, dS/dT, 0, S), dS/dgap including the boundary cells, for
 * soft_nw_backward_full_cuda (:603).  swb_nw_param_jacobian (param 0 = gap,
 * 1 = temp) replaces soft_nw_param_jacobian_cuda (:509, launcher nw_param_grad
 * src/nw/kernels_gpu.cuh:285).
 */
size_t swb_nw_aux_workspace_bytes(int B, int L1max, int L2max);
/* Affine global alignment: the same two ops (param 0 = gap_open, 1 = gap_ext,
 * 2 = temp; grad_tangents [B][4] = tangents of (dS/dgo, dS/dge, dS/dT, S)),
 * replacing soft_nw_affine_hvp_cuda and soft_nw_affine_param_jacobian_cuda
 * (src/nw_affine/torch_cuda.cpp:435, :484; backward_full :555). */
size_t swb_nw_affine_aux_workspace_bytes(int B, int L1max, int L2max);
/* Saigo–Vert: the same two ops (param 0 / 1 / 2 = gap_open / gap_ext / temp;
 * the linear model's gap direction is the sum of 0 and 1), replacing
 * soft_sv_affine_hvp_cuda and soft_sv_affine_param_jacobian_cuda
 * (src/sv_affine/torch_cuda.cpp; restating src/sv_affine/kernels_cpu.cpp:369-934). */
size_t swb_sv_affine_aux_workspace_bytes(int B, int L1max, int L2max);
int swb_sv_affine_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
                      int L2max, float gap_open, float gap_ext, float temp, float* out,
                      float* grad_tangents, void* workspace, size_t workspace_bytes, void* stream);
int swb_sv_affine_param_jacobian(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp, int param,
                                 float* out, void* workspace, size_t workspace_bytes, void* stream);
int swb_nw_affine_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
                      int L2max, float gap_open, float gap_ext, float temp, float* out,
                      float* grad_tangents, void* workspace, size_t workspace_bytes, void* stream);
int swb_nw_affine_param_jacobian(const float* scores, const int* lengths, int B, int L1max,
                                 int L2max, float gap_open, float gap_ext, float temp, int param,
                                 float* out, void* workspace, size_t workspace_bytes, void* stream);
int swb_nw_hvp(const float* scores, const float* v, const int* lengths, int B, int L1max,
               int L2max, float gap, float temp, float* out, float* grad_tangents,
               void* workspace, size_t workspace_bytes, void* stream);
int swb_nw_param_jacobian(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap, float temp, int param, float* out, void* workspace,
                          size_t workspace_bytes, void* stream);

/*
 * One pass over a [B, per_item] fp32 tensor for the Python prelude's input
 * checks (replaces the reference's separate full-tensor passes in
 * orihime/operator.py:249-386: isposinf().any(), the domain mask .all(),
 * isneginf().any() and amax).  words (device, 1 + B unsigned): words[0] gets
 * flag 1 if some cell is +inf, 2 if some cell is NaN or is finite, not
 * -sentinel and |x| > limit, 4 if some cell is -inf.  amax (device, B floats)
 * gets each item's largest cell (-inf if all are -inf).  Asynchronous.
 */
int swb_scan_scores(const float* x, int B, long long per_item, float limit, float sentinel,
                    unsigned* words, float* amax, void* stream);

/*
 * Checkpointed value, in two launches (no reference counterpart: the
 * reference's forward op runs the forward and the backward together and
 * keeps the full alpha table for the map).  swb_*_checkpoint runs the
 * forward wavefront alone: it writes the value and leaves in the workspace
 * the DP state of every `ck_every`-th checkpoint chunk (4 wavefront steps
 * per chunk), the band partials and the cross-band edge records; nothing
 * else is kept.  swb_*_adjoint, later, on the same workspace, scores,
 * lengths and parameters, runs the checkpointed adjoint: the marginal map
 * and dS/dparameters (and the value again).  It can run more than once.
 * ck_every in [1, 16]: 1 keeps a checkpoint per chunk (the fastest
 * adjoint); 4 keeps about 0.93 bytes per cell of a large padded batch, and the
 * adjoint recomputes the chunks in between from the nearest checkpoint.
 * The local families in the linear domain only: gaps must be <= 0, else
 * SWB_ERR_ARG.  Columns per lane as swb_cols_per_lane gives for L2max (8 at
 * L2max >= 256, 2 at L2max <= 64, else 4).  Workspace from
 * swb_*_checkpoint_workspace_bytes(B, L1max, L2max, ck_every).
 */
size_t swb_sw_affine_checkpoint_workspace_bytes(int B, int L1max, int L2max, int ck_every);
int swb_sw_affine_checkpoint(const float* scores, const int* lengths, int B, int L1max, int L2max,
                             float gap_open, float gap_ext, float temp, int ck_every, float* value,
                             void* workspace, size_t workspace_bytes, void* stream);
int swb_sw_affine_adjoint(const float* scores, const int* lengths, int B, int L1max, int L2max,
                          float gap_open, float gap_ext, float temp, int ck_every, float* value,
                          float* map, float* grad_open, float* grad_ext, float* grad_temp,
                          void* workspace, size_t workspace_bytes, void* stream);
size_t swb_sw_checkpoint_workspace_bytes(int B, int L1max, int L2max, int ck_every);
int swb_sw_checkpoint(const float* scores, const int* lengths, int B, int L1max, int L2max,
                      float gap, float temp, int ck_every, float* value, void* workspace,
                      size_t workspace_bytes, void* stream);
int swb_sw_adjoint(const float* scores, const int* lengths, int B, int L1max, int L2max, float gap,
                   float temp, int ck_every, float* value, float* map, float* grad_gap,
                   float* grad_temp, void* workspace, size_t workspace_bytes, void* stream);

/* Copies the workspace status word to *status (synchronises `stream`).
 * No reference counterpart: the reference synchronises inside every op.
 * A bounded wait that expires also shows in the results without this call:
 * the affected pairs' value and dS/dparameters (second-order ops: their
 * output map) are NaN. */
int swb_read_status(const void* workspace, void* stream, unsigned* status);

/* The status word of swb_sw_affine_forward_static's shared scratch on the
 * current device (synchronises `stream`; allocates nothing).  No reference
 * counterpart. */
int swb_static_read_status(void* stream, unsigned* status);

/* Human-readable text for a SWB_ERR_* code. */
const char* swb_error_string(int code);

/* SWB_ABI_VERSION of the loaded library. */
int swb_abi_version(void);

/* Roofline probe (no reference counterpart): launches `blocks` x 256 threads,
 * each issuing iters * 8 dependent-chain ex2.approx operations on the MUFU
 * pipe; `scratch` needs blocks * 256 floats.  Time it with events on `stream`. */
int swb_mufu_probe(float* scratch, int blocks, int iters, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ORIHIME_B200_H */
