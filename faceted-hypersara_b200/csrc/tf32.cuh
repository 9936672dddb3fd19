// 3xTF32 tensor-core products (mma.sync m16n8k8, FP32 accumulate).
//
// A float x is split into x = hi + lo with hi = tf32(x) and lo = tf32(x - hi);
// a*b ~ hi_a hi_b + hi_a lo_b + lo_a hi_b keeps the product to about FP32
// accuracy (the dropped lo_a lo_b is below 2^-22 of |a b|).
#pragma once

#include <cstdint>

namespace fhs {

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// d += a b for one m16n8k8 tile (row-major A 16x8, column-major B 8x8)
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Fragments with their hi and lo parts.  A: a0 (row g, col t), a1 (g+8, t),
// a2 (g, t+4), a3 (g+8, t+4); B: b0 (row t, col g), b1 (t+4, g); D: d0 (g, 2t),
// d1 (g, 2t+1), d2 (g+8, 2t), d3 (g+8, 2t+1), with g = lane / 4, t = lane % 4.
struct FragA3 {
  uint32_t h[4], l[4];
};
struct FragB3 {
  uint32_t h[2], l[2];
};

__device__ __forceinline__ FragA3 frag_a3(float a0, float a1, float a2, float a3) {
  FragA3 f;
  split_tf32(a0, f.h[0], f.l[0]);
  split_tf32(a1, f.h[1], f.l[1]);
  split_tf32(a2, f.h[2], f.l[2]);
  split_tf32(a3, f.h[3], f.l[3]);
  return f;
}

__device__ __forceinline__ FragB3 frag_b3(float b0, float b1) {
  FragB3 f;
  split_tf32(b0, f.h[0], f.l[0]);
  split_tf32(b1, f.h[1], f.l[1]);
  return f;
}

// d += a b in 3xTF32 (small terms first)
__device__ __forceinline__ void mma3xtf32(float (&d)[4], const FragA3& a, const FragB3& b) {
  mma_tf32(d, a.l[0], a.l[1], a.l[2], a.l[3], b.h[0], b.h[1]);
  mma_tf32(d, a.h[0], a.h[1], a.h[2], a.h[3], b.l[0], b.l[1]);
  mma_tf32(d, a.h[0], a.h[1], a.h[2], a.h[3], b.h[0], b.h[1]);
}

}  // namespace fhs
