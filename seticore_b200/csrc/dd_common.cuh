// Shared definitions for the seticore-b200 dedoppler kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "seticore_b200.h"

namespace scb {

constexpr int kWarp = 32;

// Three-input maximum (PTX max.f32 with three sources, sm_100+).  Like fmaxf it
// returns the non-NaN operand when one operand is NaN, so a NaN path sum never becomes
// a top sum -- the reference's `path_sum > top` is false for NaN (dedoppler.cu:49).
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

// Channel offset, at row t, of the Taylor path with in-block offset `off` over L rows:
// both halves of a path carry offset off/2 and the second half starts (off+1)/2 to the
// right (the recursion of taylor.h:48-54).
__host__ __device__ __forceinline__ int path_pos(int off, int L, int t) {
  int p = 0;
  while (L > 1) {
    const int half = L >> 1;
    if (t >= half) {
      p += (off + 1) >> 1;
      t -= half;
    }
    off >>= 1;
    L = half;
  }
  return p;
}

// Pairwise (tree-order) sum of one path of L rows: bit-identical to the value the
// Taylor tree produces for that path.  get(t, pos) returns row t at channel offset pos.
template <typename Get>
__device__ __forceinline__ float path_sum_pairwise(int L, int off, Get get) {
  float stack[12];
  int depth = 0;
  for (int t = 0; t < L; ++t) {
    float v = get(t, path_pos(off, L, t));
    int k = t;
    while (k & 1) {
      v = stack[--depth] + v;
      k >>= 1;
    }
    stack[depth++] = v;
  }
  return stack[0];
}

// The same sum for L = 2^n rows with the channel offset advanced incrementally: going from
// row t to t + 1 clears the trailing one bits of t (the blocks whose second halves end
// there, which the pairwise merges close in the same loop) and sets the next bit, so the
// offset drops the shifts of the cleared levels and gains the shift of the set one
// (level m shifts a block's second half by ((off >> (n-1-m)) + 1) >> 1).  Bit-identical to
// path_sum_pairwise; about two loop steps per row instead of n.
template <typename Get>
__device__ __forceinline__ float path_sum_pow2(int n, int off, Get get) {
  float stack[12];
  int depth = 0, p = 0;
  const int L = 1 << n;
  for (int t = 0; t < L; ++t) {
    float v = get(t, p);
    int k = t, m = 0, sub = 0;
    while (k & 1) {
      v = stack[--depth] + v;
      sub += ((off >> (n - 1 - m)) + 1) >> 1;
      k >>= 1;
      ++m;
    }
    stack[depth++] = v;
    if (m < n) p += (((off >> (n - 1 - m)) + 1) >> 1) - sub;
  }
  return stack[0];
}

// Float -> unsigned key with the same order as the float values (non-NaN).
__device__ __forceinline__ uint32_t float_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Key of the order statistics: -0 is keyed as +0, so that key order is float order and
// equal floats have equal keys (for every non-NaN value).
__device__ __forceinline__ uint32_t sel_key(float f) { return float_key(f == 0.0f ? 0.0f : f); }

// Floor division for possibly negative numerators, positive divisor.
__host__ __device__ __forceinline__ long long floor_div(long long a, long long b) {
  return (a >= 0) ? a / b : -((-a + b - 1) / b);
}

}  // namespace scb
