// Fused input scan of the Python prelude (sm_100a): one pass over the scores
// that answers what the reference's domain validation and mask normalisation
// ask of the whole tensor (orihime/operator.py:249-386):
//   flag 1: some cell is +inf;
//   flag 2: some cell is NaN, or finite, not the mask sentinel
//           -sentinel and |x| > limit;
//   flag 4: some cell is -inf (a masked cell);
// and, per batch item, the largest cell (amax over dims 1.., -inf when every
// cell is -inf), which the mask normalisation uses.  Comparisons are the
// torch expressions' own fp32 comparisons, so the decisions are identical.
// Compiled as part of sw_capi.cu.
namespace swb {

// float <-> unsigned with the order of the floats (for atomicMax)
__device__ __forceinline__ unsigned ord_bits(float v) {
  const unsigned u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unord_bits(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ void scan_cell(float v, float limit, float sent, unsigned& f, float& mx) {
  const bool ninf = v == -INFINITY;
  if (v == INFINITY) f |= 1u;
  if (ninf) f |= 4u;
  if (v != v || !(ninf || v == -sent || fabsf(v) <= limit)) f |= 2u;
  mx = fmaxf(mx, v);
}

__global__ void scan_init_kernel(unsigned* words, int B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) words[0] = 0u;
  if (i < B) words[1 + i] = ord_bits(-INFINITY);
}

// grid B * bpi blocks (bpi per item); words[0] = flags, words[1 + b] = ordered amax
__global__ void __launch_bounds__(256) scan_kernel(const float* x, long long per, int bpi,
                                                    float limit, float sent, unsigned* words) {
  const int b = blockIdx.x / bpi, blk = blockIdx.x - b * bpi;
  const float* xb = x + (size_t)b * per;
  unsigned f = 0u;
  float mx = -INFINITY;
  const long long stride = (long long)bpi * blockDim.x;
  const long long t0 = (long long)blk * blockDim.x + threadIdx.x;
  if ((per & 3) == 0 && (reinterpret_cast<uintptr_t>(xb) & 15) == 0) {
    const float4* x4 = reinterpret_cast<const float4*>(xb);
    for (long long i = t0; i < per / 4; i += stride) {
      const float4 v = __ldcs(x4 + i);   // streamed once
      scan_cell(v.x, limit, sent, f, mx);
      scan_cell(v.y, limit, sent, f, mx);
      scan_cell(v.z, limit, sent, f, mx);
      scan_cell(v.w, limit, sent, f, mx);
    }
  } else {
    for (long long i = t0; i < per; i += stride) scan_cell(__ldcs(xb + i), limit, sent, f, mx);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    f |= __shfl_xor_sync(FULL, f, o);
    mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
  }
  __shared__ unsigned sf[8];
  __shared__ float smx[8];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { sf[w] = f; smx[w] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < 8; ++k) { f |= sf[k]; mx = fmaxf(mx, smx[k]); }
    if (f) atomicOr(words, f);
    atomicMax(words + 1 + b, ord_bits(mx));
  }
}

__global__ void scan_finish_kernel(unsigned* words, float* amax, int B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B) amax[i] = unord_bits(words[1 + i]);
}

}  // namespace swb
