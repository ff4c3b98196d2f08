// Brick decomposition shared by the privatised projector and backprojector.
//
// The half-complex volume is cut into cubic bricks in SIGNED Fourier
// coordinates: x in [0, V/2 + ...], y and z in [-V/2, V/2 + ...].  A
// brick-major kernel owns one brick at a time in shared memory (the
// projector stages the brick's voxels, the backprojector accumulates into
// it) and processes exactly the slice pixels that read from, or add to, that
// brick.  Which pixels those are is decided per call by a binning plan
// (brick_plan.cu), built on the device:
//
//  1. one CTA per slice evaluates every pixel's sample position with the
//     reference's arithmetic and finds the brick(s) it reads from (the
//     projector: the brick of its interpolation base voxel) or adds to (the
//     backprojector: the bricks of its up to 16 target voxels, after Friedel
//     mirroring and the x = 0 plane's second insertion), and counting-sorts
//     its pixel ids by brick: one "bin" per (slice, brick);
//  2. the bins are grouped by brick and cut into work items.
#pragma once

#include "common.cuh"

namespace gtomrln {

struct BrickGrid {
  int V;      // volume dimension (dimsvolume.x)
  int B;      // brick edge in voxels
  int nbx, nby, nbz;
  int ylo, zlo;  // signed coordinate of brick row/plane 0
  int nbricks;
};

struct BrickItem {
  int brick;      // brick index
  int offset;     // first entry in the pair list
  int count;      // bins (slice, pixel run) in this item
  int exclusive;  // 1 if this is the brick's only item (no other CTA writes it)
};

// A (slice, brick) bin: `count` pixel ids starting at entries[start]; the
// first `interior` of them are pixels whose whole 2x2x2 target cube (direct
// or mirrored, away from the x = 0 plane) lies inside the brick, so a warp
// can treat them with one branch-free path.  In a segment plan the bin
// lists no pixels: start and count hold the packed row ranges of the
// pair's side 0 and side 1 (seg_pack_rows).
struct PixelBin {
  int slice, start, count, brick, interior, pad0, pad1, pad2;
};

__host__ __device__ inline int3 brick_origin(const BrickGrid& g, int b) {
  int bx = b % g.nbx;
  int t = b / g.nbx;
  int by = t % g.nby;
  int bz = t / g.nby;
  return make_int3(bx * g.B, g.ylo + by * g.B, g.zlo + bz * g.B);
}

// floor(x / B) for 0 <= x < 2^20 without an integer division: a float
// estimate corrected by one step either way.
__device__ __forceinline__ int div_brick(int x, int B, float invB) {
  int q = (int)((float)x * invB);
  q -= q * B > x;
  q += (q + 1) * B <= x;
  return q;
}

// Brick holding signed voxel (x, y, z), or -1 outside the grid.
__device__ __forceinline__ int brick_of(const BrickGrid& g, int x, int y, int z) {
  int dy = y - g.ylo, dz = z - g.zlo;
  if (x < 0 || dy < 0 || dz < 0) return -1;
  const float inv = 1.f / (float)g.B;
  int bx = div_brick(x, g.B, inv), by = div_brick(dy, g.B, inv), bz = div_brick(dz, g.B, inv);
  if (bx >= g.nbx || by >= g.nby || bz >= g.nbz) return -1;
  return (bz * g.nby + by) * g.nbx + bx;
}

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

// Which slice pixels a plan covers and how their samples are formed.
struct PixelSet {
  int n, dimft;      // slice size and its half width n/2 + 1
  int64_t elements;  // pixels per slice
  int rmax2;
  int strict;        // 1: r^2 < rmax^2 and x == 0, y < 0 skipped (backprojector)
                     // 0: r^2 <= rmax^2, all x (projector)
  float pmax;        // largest |pixel| in the set
};

// Slice geometry beyond a plain matrix (the backprojector's general case,
// Backproject.cu:57-63, 145-152, 183-189): an in-plane magnification applied
// to the pixel coordinates before the matrix, the Ewald-sphere curvature
// z = curve * (x^2 + y^2) along the matrix's third column, and a target
// volume per slice.  Defaults describe the plain case.
struct SliceGeom {
  float4 mag = make_float4(1.f, 0.f, 0.f, 1.f);  // columns of the 2x2 magnification
  float curve = 0.f;            // 1 / (2 R); 0 = flat slices
  const int* ivolume = nullptr;  // per-slice volume index (device), or none
  int nvol = 1;                  // volumes the plan spans (ivolume values in [0, nvol))
  float qmax = -1.f;  // bound on |q| of the samples kept (magnified radius test); < 0: the pixel set's pmax
};

// The map pixel (u, v) -> u c0' + v c1' of the enumeration: the matrix's
// first two columns through the magnification (c0' = mag.x c0 + mag.y c1,
// c1' = mag.z c0 + mag.w c1), third column unchanged.
__device__ __forceinline__ void effective_matrix(const float* m, const SliceGeom& gm, float* me) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    me[r] = fmaf(gm.mag.x, m[r], gm.mag.y * m[3 + r]);
    me[3 + r] = fmaf(gm.mag.z, m[r], gm.mag.w * m[3 + r]);
    me[6 + r] = m[6 + r];
  }
}

// Largest displacement (voxels, any axis) of a sample from the flat map by
// the curvature, over pixels of radius <= pmax: curve pmax^2 max|c2_r|.
__device__ __forceinline__ float curvature_reach(const float* m, const SliceGeom& gm, float pmax) {
  if (gm.curve == 0.f) return 0.f;
  const float c2 = fmaxf(fabsf(m[6]), fmaxf(fabsf(m[7]), fabsf(m[8])));
  return fabsf(gm.curve) * pmax * pmax * c2 * (1.f + 1e-5f) + 1e-4f;
}

// Per-call plan, all in device memory.
struct BrickPlan {
  BrickGrid g;
  int nvol = 1;  // work-item keys are volume * g.nbricks + brick
  int batch = 0;
  int max_items = 0;
  BrickItem* items = nullptr;
  int* nitems = nullptr;      // number of valid items
  int* pairs = nullptr;       // per brick: indices into bins
  PixelBin* bins = nullptr;
  int* entries = nullptr;     // pixel ids, grouped by bin
  int* counter = nullptr;     // work counter of the persistent kernel (starts at 0)
  int* fallback = nullptr;    // slices for the direct kernels
  int* nfallback = nullptr;
  void* scratch = nullptr;    // one pool allocation holding all of the above
};

// Enqueues the plan for `batch` matrices (device, 9 floats each) on
// `stream`; nothing is synchronised.  op is GTOMRLN_OP_PROJECT (bin by the
// interpolation base voxel) or GTOMRLN_OP_BACKPROJECT (bin by every target
// voxel).  A slice whose samples could reach radius `limit` (beyond which
// the brick kernels would need the reference's clamps) is not planned but
// listed in plan->fallback for the direct kernels.  chunk caps the bins per
// work item.  segments = 1 builds the segment plan instead: bins without
// entries, one per (slice, brick) pair whose brick the slice's plane
// crosses, and the kernels enumerate the pixels themselves (segment.cuh).
// With a segment plan, zero_out (the projector's output, complex, elements
// per slice as px) receives the zeros outside px's radius for every planned
// slice, in the plan's own per-slice pass.
// geom (segment plans only): magnification, curvature and per-slice volumes
// of the backprojector's general case; the plan then lists one pair per
// (slice, volume-brick key) and its enumeration boxes are widened by the
// curvature's reach.
int build_brick_plan(int op, const float* d_mats, int batch, const BrickGrid& g, const PixelSet& px,
                     float limit, int chunk, cudaStream_t stream, BrickPlan* plan, int segments = 0,
                     void* zero_out = nullptr, const SliceGeom& geom = SliceGeom());
int free_brick_plan(BrickPlan* plan, cudaStream_t stream);

// Pixel id -> signed slice coordinates (FFT order in y).
__device__ __forceinline__ void pixel_uv(int id, int n, int dimft, int& u, int& v) {
  int idy = id / dimft;
  u = id - idy * dimft;
  v = idy <= n / 2 ? idy : idy - n;
}

}  // namespace gtomrln
