// Peak-rate probes used as roofline denominators by bench.py.
//
// mufu_probe: every thread runs 8 independent chains x <- ex2(-x), so the
// SFU (MUFU) pipe is the only busy unit; ops = threads * iters * 8.
#pragma once
#include <cuda_runtime.h>

namespace swb {

__global__ void __launch_bounds__(256) mufu_probe_kernel(float* out, int iters) {
  float x0 = 0.50f + threadIdx.x * 1e-6f, x1 = 0.51f, x2 = 0.52f, x3 = 0.53f;
  float x4 = 0.54f, x5 = 0.55f, x6 = 0.56f, x7 = 0.57f + blockIdx.x * 1e-7f;
  for (int it = 0; it < iters; ++it) {
#define SWB_EX2N(v) asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(v) : "f"(-(v)))
    SWB_EX2N(x0); SWB_EX2N(x1); SWB_EX2N(x2); SWB_EX2N(x3);
    SWB_EX2N(x4); SWB_EX2N(x5); SWB_EX2N(x6); SWB_EX2N(x7);
#undef SWB_EX2N
  }
  float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 123.f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains alive
}

}  // namespace swb
