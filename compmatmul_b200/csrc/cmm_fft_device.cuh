// Device helpers shared by the sketch kernels: complex arithmetic, radix-4
// and radix-8 decimation-in-time steps, Walsh-Hadamard butterflies and the
// two-sum used by the compensated FP32 accumulation.
#pragma once
#include <cuda_runtime.h>

namespace cmm {
namespace dev {

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return mk(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
template <typename C>
__device__ __forceinline__ void bf(C& a, C& b, C w) {
  const C t = cmul(b, w);
  b = mk(a.x - t.x, a.y - t.y);
  a = mk(a.x + t.x, a.y + t.y);
}
template <typename C>
__device__ __forceinline__ C csq(C a) {
  return mk(a.x * a.x - a.y * a.y, (a.x + a.x) * a.y);
}
// radix-4 / radix-8 decimation-in-time steps on points base + e * half;
// W = w_{K half}^kk (K = 4 or 8)
template <typename C>
__device__ __forceinline__ void r4(C (&x)[4], C W) {
  const C W2 = csq(W);
  bf(x[0], x[1], W2);
  bf(x[2], x[3], W2);
  bf(x[0], x[2], W);
  bf(x[1], x[3], mk(W.y, -W.x));  // W * (-i)
}
template <typename C>
__device__ __forceinline__ void r8(C (&x)[8], C W) {
  using R = decltype(W.x);
  const R h = (R)0.70710678118654752440;
  const C W2 = csq(W), W4 = csq(W2);
  bf(x[0], x[1], W4); bf(x[2], x[3], W4); bf(x[4], x[5], W4); bf(x[6], x[7], W4);
  const C W2m = mk(W2.y, -W2.x);
  bf(x[0], x[2], W2); bf(x[4], x[6], W2); bf(x[1], x[3], W2m); bf(x[5], x[7], W2m);
  const C W1 = cmul(W, mk(h, -h));
  const C Wi = mk(W.y, -W.x);
  const C W3 = cmul(W, mk(-h, -h));
  bf(x[0], x[4], W); bf(x[1], x[5], W1); bf(x[2], x[6], Wi); bf(x[3], x[7], W3);
}
// the same steps for kk = 0 (W = 1): the twiddles are 1, -i and w_8^{1,3}
template <typename C>
__device__ __forceinline__ void add_sub(C& a, C& b) {
  const C t = b;
  b = mk(a.x - t.x, a.y - t.y);
  a = mk(a.x + t.x, a.y + t.y);
}
template <typename C>
__device__ __forceinline__ C mul_mi(C a) { return mk(a.y, -a.x); }  // a * (-i)
template <typename C>
__device__ __forceinline__ void r4_first(C (&x)[4]) {
  add_sub(x[0], x[1]);
  add_sub(x[2], x[3]);
  add_sub(x[0], x[2]);
  x[3] = mul_mi(x[3]);
  add_sub(x[1], x[3]);
}
template <typename C>
__device__ __forceinline__ void r8_first(C (&x)[8]) {
  using R = decltype(x[0].x);
  const R h = (R)0.70710678118654752440;
  add_sub(x[0], x[1]); add_sub(x[2], x[3]); add_sub(x[4], x[5]); add_sub(x[6], x[7]);
  add_sub(x[0], x[2]); add_sub(x[4], x[6]);
  x[3] = mul_mi(x[3]); x[7] = mul_mi(x[7]);
  add_sub(x[1], x[3]); add_sub(x[5], x[7]);
  add_sub(x[0], x[4]);
  x[5] = mk((x[5].x + x[5].y) * h, (x[5].y - x[5].x) * h);    // * w_8
  add_sub(x[1], x[5]);
  x[6] = mul_mi(x[6]);
  add_sub(x[2], x[6]);
  x[7] = mk((x[7].y - x[7].x) * h, -(x[7].x + x[7].y) * h);   // * w_8^3
  add_sub(x[3], x[7]);
}
template <typename R, int M>
__device__ __forceinline__ void whtr(R (&x)[M]) {
#pragma unroll
  for (int h = 1; h < M; h <<= 1)
#pragma unroll
    for (int e = 0; e < M; ++e)
      if (!(e & h)) {
        const R a = x[e], b = x[e + h];
        x[e] = a + b;
        x[e + h] = a - b;
      }
}
__device__ __forceinline__ void tsum(float& hi, float& lo, float x) {
  const float s = hi + x;
  const float bp = s - hi;
  lo += (hi - (s - bp)) + (x - bp);
  hi = s;
}
}  // namespace dev
}  // namespace cmm
