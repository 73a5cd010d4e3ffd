/*
 * TEST INFRASTRUCTURE ONLY.  CPU oracle for the soft Smith-Waterman path
 * (linear and affine gaps) and the soft Needleman-Wunsch path (linear gap) of
 * megure-labs/orihime: value, marginal map, parameter gradients,
 * Hessian-vector product and parameter Jacobians.
 *
 * The product (orihime_b200) never loads this library: only tests/, the CPU
 * legs of bench.py and __graft_entry__.smoke() do, as the oracle.
 *
 * Symbols ending in _f32 follow the reference CPU kernels
 * (src/sw/kernels_cpu.cpp, src/sw_affine/kernels_cpu.cpp,
 * src/nw/kernels_cpu.cpp) operation by
 * operation in float, so that they reproduce the reference bit for bit when
 * built without FMA contraction (gcc -std=c11 implies -ffp-contract=off).
 * Symbols ending in _f64 run the same recurrences in double: the FP64 truth.
 */
#include <math.h>
#include <stdlib.h>
#include <stddef.h>

#define NEG_BIG -1e30

#define REAL float
#define SFX _f32
#define EXPF expf
#define LOGF logf
#define FABS fabsf
#include "sw_oracle_impl.h"
#undef REAL
#undef SFX
#undef EXPF
#undef LOGF
#undef FABS

#define REAL double
#define SFX _f64
#define EXPF exp
#define LOGF log
#define FABS fabs
#include "sw_oracle_impl.h"
