// Row segments: the pixels of a slice whose sample position falls in a box,
// found analytically instead of by a per-pixel binning pass.
//
// A slice pixel (u, v) sits at u * c0 + v * c1 in the volume (c0, c1 the
// first two matrix columns; the third column meets z = 0 for 2D slices).
// For a box [lo, hi] each axis r bounds u in row v to the interval
//   lo_r <= u * c0_r + v * c1_r <= hi_r,
// and the rows that can hold such a pixel lie between the extremes over the
// box of the linear function v(p) that recovers v from a point of the plane.
// A warp walks one (slice, box) pair: 32 rows at a time, one lane per row
// computes the row's u interval (clipped to the slice's pixel set), the
// lanes scan the interval lengths, and the pixels are dealt out 32 per wave,
// each lane finding its row by a binary search over the scan.  The boxes
// are widened by a margin well above the float error of both the positions
// and these bounds, so the candidates are a superset of the pixels the box
// holds; the caller applies the exact test with the kernels' own
// arithmetic (project_sample / backproject_sample), which decides alone.
#pragma once

#include "brick.cuh"

namespace gtomrln {

// Margin (voxels) by which callers widen a box: above the float error of a
// sample position (|pos| < 2^14 voxels: a few ulp, ~1e-3) and of the
// interval bounds below (relative 1e-6 of the same magnitudes).
constexpr float kSegMargin = 0.01f;

// The box and the pixel -> position map of one (slice, brick, side): the
// columns are read from the slice matrix (negated for the mirror side) and
// the box from the brick origin when needed, so that nothing beyond the
// matrix and the origin stays live in registers.
struct SegBox {
  const float* m;  // slice matrix (9 floats, column-major)
  float sg;        // +1: positions; -1: negated positions
  int3 o;          // brick origin
  float below;     // widening below the brick, before the margin
  float above;     // brick edge plus the margin
  __device__ __forceinline__ float c0(int r) const { return sg * m[r]; }
  __device__ __forceinline__ float c1(int r) const { return sg * m[3 + r]; }
  __device__ __forceinline__ float org(int r) const { return (float)(r == 0 ? o.x : (r == 1 ? o.y : o.z)); }
  __device__ __forceinline__ float lo(int r) const { return org(r) - below; }
  __device__ __forceinline__ float hi(int r) const { return org(r) + above; }
};

// Largest u with u^2 <= rem (0 <= rem < 2^24: radii below 4 096), exactly:
// the approximate square root is within a unit of the truth there, which the
// two integer corrections absorb.
__device__ __forceinline__ int seg_isqrt(int rem) {
  float f;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(f) : "f"((float)rem));
  int r = (int)f;
  r -= r * r > rem;
  r += (r + 1) * (r + 1) <= rem;
  return r;
}

// Approximate reciprocal (a few ulp), for bounds that a margin widens.
__device__ __forceinline__ float seg_rcp(float a) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
}

// Row range [vlo, vhi] (signed v) that can hold a pixel of the box, clipped
// to the slice rows within the pixel set's radius.  Returns false if empty.
__device__ __forceinline__ bool seg_rows(const SegBox& b, const PixelSet& px, int& vlo, int& vhi) {
  const int rlim = seg_isqrt(px.strict ? px.rmax2 - 1 : px.rmax2);
  vlo = max(px.n / 2 + 1 - px.n, -rlim);  // rows idy > n/2 hold v = idy - n
  vhi = min(px.n / 2, rlim);
  const float g00 = b.c0(0) * b.c0(0) + b.c0(1) * b.c0(1) + b.c0(2) * b.c0(2);
  const float g11 = b.c1(0) * b.c1(0) + b.c1(1) * b.c1(1) + b.c1(2) * b.c1(2);
  const float g01 = b.c0(0) * b.c1(0) + b.c0(1) * b.c1(1) + b.c0(2) * b.c1(2);
  const float det = g00 * g11 - g01 * g01;
  // v(p) = w . p and u(p) = w' . p on the plane, w = (g00 c1 - g01 c0) / det,
  // w' = (g11 c0 - g01 c1) / det: their extremes over the box bound the rows
  // and reject a box that lies wholly at u < 0 (the other side's pixels).
  // Near-parallel columns (det small against g00 g11) keep the full range.
  if (det > 1e-3f * g00 * g11 && g00 > 0.f) {
    const float inv = 1.f / det;
    float vc = 0.f, vh = 0.f, uc = 0.f, uh = 0.f;
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const float w = (g00 * b.c1(r) - g01 * b.c0(r)) * inv;
      const float wu = (g11 * b.c0(r) - g01 * b.c1(r)) * inv;
      const float c = 0.5f * (b.lo(r) + b.hi(r)), h = 0.5f * (b.hi(r) - b.lo(r));
      vc = fmaf(w, c, vc);
      vh = fmaf(fabsf(w), h, vh);
      uc = fmaf(wu, c, uc);
      uh = fmaf(fabsf(wu), h, uh);
    }
    const float upad = 0.5f + 1e-3f * (fabsf(uc) + uh);
    if (uc + uh + upad < 0.f || uc - uh - upad > (float)(px.dimft - 1)) return false;
    const float pad = 0.5f + 1e-3f * (fabsf(vc) + vh);
    const float flo = fmaxf(vc - vh - pad, -1e6f), fhi = fminf(vc + vh + pad, 1e6f);
    vlo = max(vlo, (int)floorf(flo));
    vhi = min(vhi, (int)ceilf(fhi));
  }
  return vlo <= vhi;
}

// Pixel interval [ua, ub] of row v holding the box, clipped to the pixel set
// (ub < ua when empty).  The bounds multiply by the approximate reciprocal of
// the column entry: a few more ulp, far inside the margin.
__device__ __forceinline__ void seg_row(const SegBox& b, const PixelSet& px, int v, int& ua, int& ub) {
  float umin = -1.f, umax = (float)px.dimft;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float a = b.c0(r), t = (float)v * b.c1(r);
    const float l = b.lo(r) - t, h = b.hi(r) - t;
    // |a| <= 1e-20 moves a * u by < 1e-16 over the row: a u-free test, which
    // the margin keeps conservative (and 1 / a stays finite otherwise)
    if (fabsf(a) > 1e-20f) {
      const float ra = seg_rcp(a);
      const float e0 = l * ra, e1 = h * ra;
      umin = fmaxf(umin, fminf(e0, e1));
      umax = fminf(umax, fmaxf(e0, e1));
    } else if (l > 0.f || h < 0.f) {
      umin = 1.f;
      umax = 0.f;
    }
  }
  const int rem = (px.strict ? px.rmax2 - 1 : px.rmax2) - v * v;
  if (rem < 0 || !(umin <= umax)) {
    ua = 1;
    ub = 0;
    return;
  }
  ua = max((int)ceilf(umin), (px.strict && v < 0) ? 1 : 0);
  ub = min((int)floorf(umax), min(seg_isqrt(rem), px.dimft - 1));
}

// Row range of a (slice, brick, side) as the plan stores it: vlo in the low
// and vhi in the high 16 bits; an empty side as vlo = 1, vhi = 0.
__host__ __device__ __forceinline__ int seg_pack_rows(int vlo, int vhi) {
  return (int)(((unsigned)vlo & 0xffffu) | ((unsigned)vhi << 16));
}
__device__ __forceinline__ void seg_unpack_rows(int packed, int& vlo, int& vhi) {
  vlo = (int)(short)(packed & 0xffff);
  vhi = packed >> 16;
}
constexpr int kSegNoRows = (int)(1u | (0u << 16));

// A segment plan's pair k: (slice, packed rows of side 0, of side 1, brick).
__device__ __forceinline__ int4 seg_pair(const PixelBin* __restrict__ bins, const int* __restrict__ pairs,
                                         int k) {
  return __ldg(reinterpret_cast<const int4*>(bins + __ldg(pairs + k)));
}

// Calls f(u, v, valid) once per lane per wave of 32 candidate pixels of the
// box in rows vlo .. vhi (from seg_rows; valid false on idle lanes of the
// last wave).  Warp-synchronous: all 32 lanes must call it together with the
// same box; f may use warp collectives.
template <class F>
__device__ __forceinline__ void seg_for_each_pixel_rows(const SegBox& b, const PixelSet& px, int vlo, int vhi,
                                                        F&& f) {
  const int lane = threadIdx.x & 31;
  for (int vb = vlo; vb <= vhi; vb += 32) {
    const int v = vb + lane;
    int ua = 1, ub = 0;
    if (v <= vhi) seg_row(b, px, v, ua, ub);
    const int cnt = max(0, ub - ua + 1);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int start = incl - cnt;
    for (int base = 0; base < total; base += 32) {
      const int k = base + lane;
      // row of candidate k: the number of rows whose inclusive end is <= k
      int r = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int t = __shfl_sync(0xffffffffu, incl, r + step - 1);
        if (t <= k) r += step;
      }
      const int rv = __shfl_sync(0xffffffffu, v, r & 31);
      const int ra = __shfl_sync(0xffffffffu, ua, r & 31);
      const int rs = __shfl_sync(0xffffffffu, start, r & 31);
      const bool valid = k < total;
      f(valid ? ra + (k - rs) : 0, valid ? rv : 0, valid);
    }
  }
}

// The same, finding the row range first.
template <class F>
__device__ __forceinline__ void seg_for_each_pixel(const SegBox& b, const PixelSet& px, F&& f) {
  int vlo, vhi;
  if (!seg_rows(b, px, vlo, vhi)) return;
  seg_for_each_pixel_rows(b, px, vlo, vhi, f);
}

// The box of brick origin o, edge B, widened by `below` voxels on the low
// side, by `widen` (a bound on how far samples leave the flat map, e.g. by
// the Ewald curvature) and the margin on both, for side 0 (positions) or
// side 1 (negated positions) of matrix m.
__device__ __forceinline__ SegBox seg_box(const float* m, int side, int3 o, int B, float below,
                                          float widen = 0.f) {
  SegBox b;
  b.m = m;
  b.sg = side ? -1.f : 1.f;
  b.o = o;
  b.below = below + widen + kSegMargin;
  b.above = (float)B + widen + kSegMargin;
  return b;
}

}  // namespace gtomrln
