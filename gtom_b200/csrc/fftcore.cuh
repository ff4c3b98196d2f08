// Complex arithmetic and small in-register DFTs shared by the gridding
// reconstructor's own FFT kernels (gridfft.cu, gridsym.cu).
#pragma once

#include <cuda_runtime.h>

namespace gtomrln {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}
// Complex sums as one packed f32x2 instruction each (two IEEE round-to-
// nearest operations, one per component, as the scalar forms).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  unsigned long long av, bv, r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(av) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(bv) : "f"(b.x), "f"(b.y));
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(av), "l"(bv));
  float2 o;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
  return o;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  unsigned long long av, bv, r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(av) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(bv) : "f"(b.x), "f"(b.y));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(av), "l"(bv));
  float2 o;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
  return o;
}
// times -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// In-register DFT of length R, forward (exp(-2 pi i nk/R)) or inverse.
template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
  if (R == 2) {
    const float2 t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
  } else if (R == 4) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 a2 = cadd(v[1], v[3]), a3 = mul_mi<INV>(csub(v[1], v[3]));
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
  } else {  // R == 8: two DFT-4 of the even and odd elements, then W8^k
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft<4, INV>(e);
    dft<4, INV>(o);
    const float h = 0.70710678118654752440f;
    // W8^1, W8^2, W8^3 (forward: (1-i)/sqrt2, -i, (-1-i)/sqrt2; inverse: conjugates)
    const float2 o1 = INV ? make_float2((o[1].x - o[1].y) * h, (o[1].x + o[1].y) * h)
                          : make_float2((o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h);
    const float2 o2 = mul_mi<INV>(o[2]);
    const float2 o3 = INV ? make_float2(-(o[3].x + o[3].y) * h, (o[3].x - o[3].y) * h)
                          : make_float2((o[3].y - o[3].x) * h, -(o[3].x + o[3].y) * h);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
}

}  // namespace gtomrln
