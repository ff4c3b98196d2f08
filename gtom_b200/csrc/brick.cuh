// Brick decomposition shared by the privatised projector and backprojector.
//
// The half-complex volume is cut into cubic bricks in SIGNED Fourier
// coordinates: x in [0, V/2 + ...], y and z in [-V/2, V/2].  A brick-major
// kernel owns one brick at a time in shared memory and visits only the
// slices whose central plane crosses that brick, and within each slice only
// the pixels whose sample — or whose Friedel mate's sample, since the
// reference mirrors neighbours with x < 0 — falls into the brick dilated by
// one voxel.  Which slices cross which brick is decided by a plan built per
// call (count -> host prefix sum -> fill), so the main kernels never test a
// slice that has nothing to contribute.
#pragma once

#include "common.cuh"

namespace gtomrln {

struct BrickGrid {
  int V;      // volume dimension (dimsvolume.x)
  int B;      // brick edge in voxels
  int nbx, nby, nbz;
  int ylo, zlo;  // signed coordinate of brick row/plane 0 (= -V/2)
  int nbricks;
};

struct BrickItem {
  int brick;      // brick index
  int offset;     // first entry of the brick's slice list
  int count;      // slices in this item
  int exclusive;  // 1 if this is the brick's only item (no other CTA writes it)
};

__host__ __device__ inline int3 brick_origin(const BrickGrid& g, int b) {
  int bx = b % g.nbx;
  int t = b / g.nbx;
  int by = t % g.nby;
  int bz = t / g.nby;
  return make_int3(bx * g.B, g.ylo + by * g.B, g.zlo + bz * g.B);
}

// Candidate box Q of a brick: the brick [lo, lo+B-1] dilated by one voxel
// plus a small guard on each side.
__device__ __forceinline__ void brick_box(const BrickGrid& g, int b, float3& qlo, float3& qhi) {
  int3 o = brick_origin(g, b);
  const float guard = 1.0f + 1e-2f;
  qlo = make_float3(o.x - guard, o.y - guard, o.z - guard);
  qhi = make_float3(o.x + g.B - 1 + guard, o.y + g.B - 1 + guard, o.z + g.B - 1 + guard);
}

// Does the plane spanned by the first two matrix columns, restricted to the
// disk |pos| <= rdisk, touch box Q?
__device__ __forceinline__ bool plane_hits_box(const float* m, float3 qlo, float3 qhi, float rdisk) {
  float3 c0 = make_float3(m[0], m[1], m[2]), c1 = make_float3(m[3], m[4], m[5]);
  float3 nrm = make_float3(c0.y * c1.z - c0.z * c1.y, c0.z * c1.x - c0.x * c1.z,
                           c0.x * c1.y - c0.y * c1.x);
  float3 c = make_float3(0.5f * (qlo.x + qhi.x), 0.5f * (qlo.y + qhi.y), 0.5f * (qlo.z + qhi.z));
  float3 h = make_float3(0.5f * (qhi.x - qlo.x), 0.5f * (qhi.y - qlo.y), 0.5f * (qhi.z - qlo.z));
  float d = fabsf(nrm.x * c.x + nrm.y * c.y + nrm.z * c.z);
  float e = fabsf(nrm.x) * h.x + fabsf(nrm.y) * h.y + fabsf(nrm.z) * h.z;
  float nn = sqrtf(nrm.x * nrm.x + nrm.y * nrm.y + nrm.z * nrm.z);
  if (d > e + 1e-3f * nn * (1.f + fabsf(c.x) + fabsf(c.y) + fabsf(c.z))) return false;
  // nearest point of the box to the origin, against the disk radius
  float px = fminf(fmaxf(0.f, qlo.x), qhi.x), py = fminf(fmaxf(0.f, qlo.y), qhi.y),
        pz = fminf(fmaxf(0.f, qlo.z), qhi.z);
  return px * px + py * py + pz * pz <= rdisk * rdisk;
}

// In-plane coordinates: pos = u * c0 + v * c1.  The dual vector d1 gives
// v = pos . d1 for points on the plane; r0 holds 1 / c0 per axis (0 where
// that component is negligible).
struct PlaneFrame {
  float3 c0, c1, d1, r0;
};

__device__ __forceinline__ float safe_rcp(float a) { return fabsf(a) > 1e-6f ? 1.f / a : 0.f; }

__device__ __forceinline__ PlaneFrame plane_frame(const float* m) {
  PlaneFrame f;
  f.c0 = make_float3(m[0], m[1], m[2]);
  f.c1 = make_float3(m[3], m[4], m[5]);
  float g00 = f.c0.x * f.c0.x + f.c0.y * f.c0.y + f.c0.z * f.c0.z;
  float g01 = f.c0.x * f.c1.x + f.c0.y * f.c1.y + f.c0.z * f.c1.z;
  float g11 = f.c1.x * f.c1.x + f.c1.y * f.c1.y + f.c1.z * f.c1.z;
  float inv = 1.f / (g00 * g11 - g01 * g01);
  f.d1 = make_float3((f.c1.x * g00 - f.c0.x * g01) * inv, (f.c1.y * g00 - f.c0.y * g01) * inv,
                     (f.c1.z * g00 - f.c0.z * g01) * inv);
  f.r0 = make_float3(safe_rcp(f.c0.x), safe_rcp(f.c0.y), safe_rcp(f.c0.z));
  return f;
}

// Narrows [ua, ub] to the u with lo <= u * a + b <= hi (ra = 1/a, or 0 when
// a is negligible: then b alone decides).
__device__ __forceinline__ void slab(float ra, float b, float lo, float hi, float& ua, float& ub) {
  if (ra != 0.f) {
    float t0 = (lo - b) * ra, t1 = (hi - b) * ra;
    ua = fmaxf(ua, fminf(t0, t1));
    ub = fminf(ub, fmaxf(t0, t1));
  } else if (b < lo || b > hi) {
    ua = 1.f;
    ub = 0.f;
  }
}

// Integer u interval of row v inside Q and inside the disk u^2 + v^2 <= r2max.
// Deterministic: the same (v, frame, box) always gives the same interval,
// which the mate de-duplication below relies on.
__device__ __forceinline__ void row_interval(const PlaneFrame& f, int v, float3 qlo, float3 qhi,
                                             int r2max, int& ua, int& ub) {
  int rem = r2max - v * v;
  if (rem < 0) {
    ua = 1;
    ub = 0;
    return;
  }
  int umax = (int)sqrtf((float)rem);
  while (umax * umax > rem) umax--;
  while ((umax + 1) * (umax + 1) <= rem) umax++;
  float fa = -1e30f, fb = 1e30f;
  float fv = (float)v;
  slab(f.r0.x, fv * f.c1.x, qlo.x, qhi.x, fa, fb);
  slab(f.r0.y, fv * f.c1.y, qlo.y, qhi.y, fa, fb);
  slab(f.r0.z, fv * f.c1.z, qlo.z, qhi.z, fa, fb);
  if (fa > fb) {
    ua = 1;
    ub = 0;
    return;
  }
  ua = max(-umax, (int)ceilf(fa - 1e-3f));
  ub = min(umax, (int)floorf(fb + 1e-3f));
}

__device__ __forceinline__ void v_range(const PlaneFrame& f, float3 qlo, float3 qhi, int rmax, int& v0,
                                        int& v1) {
  float vmin = fminf(qlo.x * f.d1.x, qhi.x * f.d1.x) + fminf(qlo.y * f.d1.y, qhi.y * f.d1.y) +
               fminf(qlo.z * f.d1.z, qhi.z * f.d1.z);
  float vmax = fmaxf(qlo.x * f.d1.x, qhi.x * f.d1.x) + fmaxf(qlo.y * f.d1.y, qhi.y * f.d1.y) +
               fmaxf(qlo.z * f.d1.z, qhi.z * f.d1.z);
  v0 = max(-rmax, (int)ceilf(vmin - 1e-3f));
  v1 = min(rmax, (int)floorf(vmax + 1e-3f));
}

// Stored pixels of a half-complex slice: rows v in [vlo, vhi] (FFT order
// holds y = n/2 but not -n/2 for even n), columns u >= 0.  The projector
// evaluates the whole u = 0 column; the backprojector skips u = 0, v < 0
// (Backproject.cu:177), whose samples are the mirrors of u = 0, v > 0.
template <bool FULL_X0>
__device__ __forceinline__ bool stored_pixel(int u, int v, int vlo, int vhi) {
  if (v < vlo || v > vhi) return false;
  return FULL_X0 ? u >= 0 : (u > 0 || (u == 0 && v >= 0));
}

// Warp-cooperative walk over the stored pixels p = (u, v) with
// u^2 + v^2 <= r2max whose sample M p, or whose Friedel mate's sample
// M(-p), lies in Q.  Each such pixel is visited exactly once per call.  All
// 32 lanes must call this; visit(u, v) runs on the lane that owns the pixel.
template <bool FULL_X0, class Visit>
__device__ __forceinline__ void for_each_footprint_pixel(const float* m, float3 qlo, float3 qhi,
                                                         int r2max, int vlo, int vhi, Visit&& visit) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  PlaneFrame f = plane_frame(m);
  int rmax = (int)sqrtf((float)r2max) + 1;
  int v0, v1;
  v_range(f, qlo, qhi, rmax, v0, v1);
  // A pixel and its mate can both lie on the walk only if Q and -Q overlap,
  // i.e. Q straddles the origin on every axis (the few central bricks).
  const bool dedupe = qlo.x <= 0.5f && qhi.x >= -0.5f && qlo.y <= 0.5f && qhi.y >= -0.5f &&
                      qlo.z <= 0.5f && qhi.z >= -0.5f;
  for (int vb = v0; vb <= v1; vb += 32) {
    int v = vb + lane;
    int ua = 1, ub = 0;
    if (v <= v1) row_interval(f, v, qlo, qhi, r2max, ua, ub);
    int len = max(0, ub - ua + 1);
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    int total = __shfl_sync(FULL, incl, 31);
    for (int base = 0; base < total; base += 32) {
      int t = base + lane;
      int r = 0;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        int probe = __shfl_sync(FULL, incl, r + s - 1);
        if (probe <= t) r += s;
      }
      int incl_r = __shfl_sync(FULL, incl, r);
      int len_r = __shfl_sync(FULL, len, r);
      int ua_r = __shfl_sync(FULL, ua, r);
      if (t < total) {
        // q = (qu, qv) has M q in Q.  Visit q if it is stored, and its
        // Friedel mate p = -q (whose mirrored sample M q lies in Q) if that is
        // stored and is not itself on the walk (it is then visited as a q).
        int qu = ua_r + (t - (incl_r - len_r));
        int qv = vb + r;
        if (stored_pixel<FULL_X0>(qu, qv, vlo, vhi)) visit(qu, qv);
        int pu = -qu, pv = -qv;
        if ((pu != qu || pv != qv) && stored_pixel<FULL_X0>(pu, pv, vlo, vhi)) {
          bool direct = false;
          if (dedupe && pv >= v0 && pv <= v1) {
            int a, bnd;
            row_interval(f, pv, qlo, qhi, r2max, a, bnd);
            direct = pu >= a && pu <= bnd;
          }
          if (!direct) visit(pu, pv);
        }
      }
    }
  }
}

// Per-call plan, all in device memory: slice lists per brick, the work items
// over them, and the slices left to the direct kernels.
struct BrickPlan {
  BrickGrid g;
  int batch = 0;
  int max_items = 0;
  BrickItem* items = nullptr;
  int* nitems = nullptr;     // number of valid items
  int* lists = nullptr;
  int* counter = nullptr;    // work counter of the persistent kernel (starts at 0)
  int* fallback = nullptr;   // slices for the direct kernels
  int* nfallback = nullptr;
  void* scratch = nullptr;   // one pool allocation holding all of the above
};

// Enqueues the construction of the plan for `batch` matrices (device, 9
// floats each) on `stream`; nothing is synchronised.  pmax is the largest
// pixel radius of a slice: its samples lie within sigma * pmax of the origin
// (sigma = largest singular value of the matrix's first two columns).  A
// slice whose bound reaches `limit` is not planned but listed in
// plan->fallback, for the direct kernels, whose clamps and wraps cover every
// geometry.  chunk caps the slices per work item.
int build_brick_plan(const float* d_mats, int batch, const BrickGrid& g, float pmax, float limit,
                     int chunk, cudaStream_t stream, BrickPlan* plan);
int free_brick_plan(BrickPlan* plan, cudaStream_t stream);

// Largest singular value of the first two columns of a matrix.
__device__ __forceinline__ float plane_scale(const float* m) {
  float g00 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
  float g01 = m[0] * m[3] + m[1] * m[4] + m[2] * m[5];
  float g11 = m[3] * m[3] + m[4] * m[4] + m[5] * m[5];
  float h = 0.5f * (g00 - g11);
  return sqrtf(0.5f * (g00 + g11) + sqrtf(h * h + g01 * g01)) * (1.f + 1e-6f);
}

inline BrickGrid make_brick_grid(int V, int B, int xhi, int ylo, int yhi) {
  BrickGrid g;
  g.V = V;
  g.B = B;
  g.nbx = (xhi + 1 + B - 1) / B;
  g.nby = (yhi - ylo + 1 + B - 1) / B;
  g.nbz = g.nby;
  g.ylo = ylo;
  g.zlo = ylo;
  g.nbricks = g.nbx * g.nby * g.nbz;
  return g;
}

}  // namespace gtomrln
