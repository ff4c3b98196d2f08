// Backprojector: trilinear scatter-insert of half-complex slices and their
// weights into a half-complex volume, the B200 replacement of
// Backproject3DtoNDKernel (src/Relion/Backproject.cu:126-322).
//
// Direct kernel: one thread per slice element, all slices of a batch in one
// flattened launch.  Per sample and neighbour the (re, im) pair goes to L2 as
// one vector reduction (red.global.add.v2.f32) instead of two scalar
// atomics; the weight as one scalar reduction.  Geometry, binary16 rounding
// of the trilinear weights, Friedel mirroring, the second insertion on the
// x = 0 plane and the clamps are the reference's, step for step.
#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>

#include "brick.cuh"
#include "common.cuh"
#include "sample.cuh"
#include "segment.cuh"

namespace gtomrln {

constexpr int kBpThreads = 256;
constexpr int kBpPerThread = 2;
constexpr int kBpTile = kBpThreads * kBpPerThread;

struct BpArgs {
  int n, dimft;
  int64_t area, elements;
  int tiles;
  int rmax2;
  int P, rowlen;
  int64_t nvox;
  float4 mag;            // columns of the 2x2 magnification
  float ewalddiaminv;    // 1 / (2 R), R = ewald radius * supersample; 0 = flat
};

// Stored location of neighbour (x, y, z) (Backproject.cu:261-274).  The
// clamps compare as unsigned like the reference's tmin(uint, short), so a
// negative coordinate clamps to the upper bound.
template <bool DECENTERED>
__device__ __forceinline__ int64_t place(int x, int y, int z, int P, int rowlen) {
  if (DECENTERED) {
    y = y < 0 ? y + P : y;
    z = z < 0 ? z + P : z;
  } else {
    y += P / 2;
    z += P / 2;
  }
  unsigned half = (unsigned)(P / 2), last = (unsigned)(P - 1);
  x = (unsigned)x > half ? (int)half : x;
  y = (unsigned)y > last ? (int)last : y;
  z = (unsigned)z > last ? (int)last : z;
  return ((int64_t)z * P + y) * rowlen + x;
}

template <int NDIMS, bool DECENTERED, bool SQUARE>
__global__ void __launch_bounds__(kBpThreads)
backproject_direct_kernel(float2* __restrict__ volft_base, float* __restrict__ volw_base,
                          const float2* __restrict__ projft, const float* __restrict__ projw,
                          const float* __restrict__ mats, const int* __restrict__ ivolume,
                          BpArgs a, const int* __restrict__ list, const int* __restrict__ nlist) {
  // Without a list the grid covers every (slice, tile) once; with one (the
  // slices a brick plan left over) a persistent grid strides over them.
  const int64_t total = list ? (int64_t)(*nlist) * a.tiles : (int64_t)gridDim.x;
  for (int64_t work = blockIdx.x; work < total; work += gridDim.x) {
  const int entry = (int)(work / a.tiles);
  const int tile = (int)(work - (int64_t)entry * a.tiles);
  const int slice = list ? __ldg(list + entry) : entry;
  float2* volft = volft_base;
  float* volw = volw_base;
  float m[9];
#pragma unroll
  for (int i = 0; i < 9; i++) m[i] = __ldg(mats + 9 * (int64_t)slice + i);
  if (ivolume) {
    // a negative index would address memory before the volumes (the
    // reference writes there); such a slice is skipped
    const int iv = __ldg(ivolume + slice);
    if (iv < 0) continue;
    int64_t off = (int64_t)iv * a.nvox;
    if (volft) volft += off;
    if (volw) volw += off;
  }
  const int half = a.n / 2;

  for (int k = 0; k < kBpPerThread; k++) {
    int64_t id = (int64_t)tile * kBpTile + k * kBpThreads + threadIdx.x;
    if (id >= a.elements) break;
    int idx, idy, idz;
    split_index(id, a.dimft, NDIMS == 3 ? a.area : a.elements, a.elements, idx, idy, idz);
    int x = idx;
    int y = idy <= half ? idy : idy - a.n;
    int z = NDIMS == 3 ? (idz <= half ? idz : idz - a.n) : 0;
    if (NDIMS == 3) {
      if (x == 0 && y < 0 && z < 0) continue;
    } else {
      if (x == 0 && y < 0) continue;
    }
    float qx = (float)x, qy = (float)y, qz = (float)z;
    if (NDIMS == 2) {  // glm mat2 * vec2, contracted like mat_apply
      qx = fmaf(a.mag.x, (float)x, a.mag.z * (float)y);
      qy = fmaf(a.mag.y, (float)x, a.mag.w * (float)y);
      qz = a.ewalddiaminv * (float)(x * x + y * y);
    }
    int r2 = NDIMS == 3 ? (z * z + y * y + x * x) : (int)fmaf(qz, qz, fmaf(qx, qx, qy * qy));
    if (r2 >= a.rmax2) continue;

    float3 pos = mat_apply(m, qx, qy, qz);
    int x0 = (short)floorf(pos.x + 1e-5f);
    int y0 = (short)floorf(pos.y);
    int z0 = (short)floorf(pos.z);
    float fx = pos.x - (float)x0, fy = pos.y - (float)y0, fz = pos.z - (float)z0;

    // Trilinear weights rounded through binary16 (Backproject.cu:221-238).
    float c0 = 1.f - fz, c1 = fz;
    float c00 = half_round((1.f - fy) * c0), c10 = half_round(fy * c0);
    float c01 = half_round((1.f - fy) * c1), c11 = half_round(fy * c1);
    float w[8];
    w[0] = half_round((1.f - fx) * c00); w[1] = half_round(fx * c00);
    w[2] = half_round((1.f - fx) * c10); w[3] = half_round(fx * c10);
    w[4] = half_round((1.f - fx) * c01); w[5] = half_round(fx * c01);
    w[6] = half_round((1.f - fx) * c11); w[7] = half_round(fx * c11);

    float2 v = projft ? __ldg(projft + a.elements * slice + id) : make_float2(1.f, 0.f);
    float pw = projw ? __ldg(projw + a.elements * slice + id) : 1.f;

#pragma unroll
    for (int i = 0; i < 8; i++) {
      int nx = x0 + (i & 1), ny = y0 + ((i >> 1) & 1), nz = z0 + ((i >> 2) & 1);
      float iw = w[i];
      if (SQUARE) iw *= iw;
      float sre = v.x, sim = v.y;
      int tx = nx, ty = ny, tz = nz;
      if (tx < 0) {
        tx = -tx; ty = -ty; tz = -tz;
        sim = -sim;
      }
      int64_t o = place<DECENTERED>(tx, ty, tz, a.P, a.rowlen);
      if (volft) red_add2((float*)(volft + o), iw * sre, iw * sim);
      if (volw) red_add(volw + o, iw * pw);
      if (nx == 0 && (ny != 0 || nz != 0)) {  // x = 0 plane (Backproject.cu:289-319)
        o = place<DECENTERED>(0, -ny, -nz, a.P, a.rowlen);
        if (volft) red_add2((float*)(volft + o), iw * sre, iw * -sim);
        if (volw) red_add(volw + o, iw * pw);
      }
    }
  }
  }  // work loop
}

// ---------------------------------------------------------------------------
// Brick-major backprojector: insertion privatised per shared-memory brick.
// A work item owns one edge^3 brick of the (signed-coordinate) volume as
// three FP32 accumulators (re, im, weight) in shared memory.  The warps take
// the item's bins (slice, pixel run) one at a time: the plan binned every
// pixel under each brick one of its targets falls into.  Per pixel a lane
// evaluates the reference's eight binary16-rounded trilinear weights,
// Friedel mirroring and the second insertion on the x = 0 plane, and adds
// the targets inside the brick to shared memory (a whole 2x2x2 cube inside
// the brick takes a path without per-target tests).  At the end of the item the brick
// is added to the volume once: with plain read-add-write when the item is
// the brick's only one and the voxel has no alias (decentred y or z = +-V/2
// share storage), otherwise with vector L2 reductions.
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Fixed-point accumulation of the segment backprojector.  Shared-memory
// int32 atomics run ~3.3x faster than FP32 ones on B200 (8.9 against 2.6
// per SM clock, measured), so a work item first accumulates every term as
// round(w v S) in int32, with S a power of two per item from a radial table
// of sampled magnitudes: S = 2^25 / (largest sampled |value| in the bands
// the brick's pixels come from), so a term at that magnitude is 2^25 steps
// (the terms themselves are formed in FP32 and rounded once).  Every atomic
// returns the sum before it; if any sum reaches 2^30 in magnitude, or a
// term exceeds 2^29 (a value 16x above the sampled maximum, or not finite),
// the item is accumulated again with FP32 atomics, so the result never
// depends on the sample.  The flush converts the integers with the exact
// inverse scale.  Squared interpolation weights stay in FP32.
// ---------------------------------------------------------------------------
constexpr float kFxBand = 16.f;  // voxels of sample radius per band
constexpr int kFxMaxBands = 128;

struct FxBands {
  const unsigned* vmax = nullptr;  // per band: largest sampled |re| or |im| (float bits); nullptr: FP32 only
  const unsigned* wmax = nullptr;  // per band: largest sampled |weight|
  const float* vsum = nullptr;     // per band: sum of the sampled max(|re|, |im|)
  const float* wsum = nullptr;     // per band: sum of the sampled |weight|
  const unsigned* count = nullptr;  // per band: pixels sampled
  int nbands = 0;
};
// A band whose largest sampled magnitude exceeds this multiple of its mean
// sampled magnitude keeps FP32: its typical terms would get fewer than 19 bits.
constexpr float kFxMaxSpread = 64.f;

__device__ __forceinline__ uint32_t fx_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// Samples pixels of the batch (uniformly over slices and elements, kept if
// inside rmax) and records per band of their sample radius the largest
// magnitudes.  The radius ignores magnification and curvature, which move a
// sample by far less than a band.
__global__ void fx_band_sample_kernel(const float2* __restrict__ projft, const float* __restrict__ projw,
                                      const float* __restrict__ mats, unsigned batch, int n, int dimft,
                                      int64_t elements, int rmax2, int nbands, int per_thread,
                                      unsigned* __restrict__ vmax, unsigned* __restrict__ wmax,
                                      float* __restrict__ vsum, float* __restrict__ wsum,
                                      unsigned* __restrict__ count) {
  __shared__ unsigned sv[kFxMaxBands], sw[kFxMaxBands], sc[kFxMaxBands];
  __shared__ float ssv[kFxMaxBands], ssw[kFxMaxBands];
  for (int b = threadIdx.x; b < nbands; b += blockDim.x) {
    sv[b] = sw[b] = sc[b] = 0u;
    ssv[b] = ssw[b] = 0.f;
  }
  __syncthreads();
  uint32_t h = fx_hash(blockIdx.x * blockDim.x + threadIdx.x + 0x9e3779b9u);
  for (int k = 0; k < per_thread; k++) {
    h = fx_hash(h + (uint32_t)k);
    const unsigned slice = h % batch;
    h = fx_hash(h ^ 0x85ebca6bu);
    const int id = (int)(h % (unsigned)elements);
    int u, v;
    pixel_uv(id, n, dimft, u, v);
    if (u * u + v * v >= rmax2) continue;
    const float* m = mats + 9 * (int64_t)slice;
    const float px0 = fmaf((float)u, __ldg(m), (float)v * __ldg(m + 3));
    const float px1 = fmaf((float)u, __ldg(m + 1), (float)v * __ldg(m + 4));
    const float px2 = fmaf((float)u, __ldg(m + 2), (float)v * __ldg(m + 5));
    const float r = sqrtf(px0 * px0 + px1 * px1 + px2 * px2);
    // clamped both ways: a non-finite matrix gives a NaN radius
    const int b = max(0, min(nbands - 1, (int)(r * (1.f / kFxBand))));
    const int64_t off = elements * slice + id;
    const float2 val = projft ? __ldg(projft + off) : make_float2(1.f, 0.f);
    const float pwv = projw ? __ldg(projw + off) : 1.f;
    const float mv = fmaxf(fabsf(val.x), fabsf(val.y)), mw = fabsf(pwv);
    atomicMax(&sv[b], __float_as_uint(mv));
    atomicMax(&sw[b], __float_as_uint(mw));
    atomicAdd(&ssv[b], mv);
    atomicAdd(&ssw[b], mw);
    atomicAdd(&sc[b], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbands; b += blockDim.x) {
    if (!sc[b]) continue;
    atomicMax(vmax + b, sv[b]);
    atomicMax(wmax + b, sw[b]);
    atomicAdd(vsum + b, ssv[b]);
    atomicAdd(wsum + b, ssw[b]);
    atomicAdd(count + b, sc[b]);
  }
}

// Power-of-two scale S with m S <= 2^25 for magnitude m; false when m is not
// finite or so small that S would leave the normal range.
__device__ __forceinline__ bool fx_scale(float m, float& s) {
  if (!(m < 3.0e38f)) return false;
  if (m == 0.f) {
    s = 1.f;
    return true;
  }
  int e;
  frexpf(m, &e);  // m < 2^e
  if (e < -100) return false;
  s = ldexpf(1.f, 25 - e);
  return true;
}

// The item's scales: the largest sampled magnitudes over the bands its
// pixels can come from (the brick widened by its neighbours' reach, one band
// of margin either way).  False (FP32) where those bands hold no non-zero
// sample or magnitudes too spread out.
__device__ __forceinline__ bool fx_item_scales(const FxBands& f, int3 o, int B, float& sv, float& sw) {
  const float lo[3] = {(float)o.x - 2.f, (float)o.y - 2.f, (float)o.z - 2.f};
  const float hi[3] = {(float)(o.x + B) + 1.f, (float)(o.y + B) + 1.f, (float)(o.z + B) + 1.f};
  float dmin2 = 0.f, dmax2 = 0.f;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float d = fmaxf(0.f, fmaxf(lo[r], -hi[r]));
    dmin2 += d * d;
    dmax2 += fmaxf(lo[r] * lo[r], hi[r] * hi[r]);
  }
  const int b0 = max(0, (int)(sqrtf(dmin2) * (1.f / kFxBand)) - 1);
  const int b1 = min(f.nbands - 1, (int)(sqrtf(dmax2) * (1.f / kFxBand)) + 1);
  unsigned mv = 0u, mw = 0u;
  for (int b = b0; b <= b1; b++) {
    mv = max(mv, f.vmax[b]);
    mw = max(mw, f.wmax[b]);
    const unsigned c = f.count[b];
    if (c && (__uint_as_float(f.vmax[b]) * (float)c > kFxMaxSpread * f.vsum[b] ||
              __uint_as_float(f.wmax[b]) * (float)c > kFxMaxSpread * f.wsum[b]))
      return false;  // magnitudes too spread out in this band for fixed point
  }
  // no magnitude sampled where this brick's pixels come from: FP32
  if (mv == 0u || mw == 0u) return false;
  return fx_scale(__uint_as_float(mv), sv) && fx_scale(__uint_as_float(mw), sw);
}

// Adds a brick's shared-memory accumulators to the volume: plain
// read-add-write when the work item is the brick's only one and the voxel has
// no alias (decentred y or z = +-V/2 share storage), else vector L2
// reductions.  Voxels that received nothing are skipped.  CLAMP (centred
// only): voxels beyond the volume are folded onto its edge with the clamps
// of place<false> (unsigned compares) instead of being skipped, and every
// voxel of the faces they fold onto counts as an alias.
//
// fx: the accumulators hold fixed-point integers (the segment kernel's
// fixed-point mode), turned into FP32 by the exact powers of two inv_v (data)
// and inv_w (weights).
template <bool DECENTERED, bool CLAMP = false>
__device__ __forceinline__ void bp_flush_brick(float2* __restrict__ volft, float* __restrict__ volw,
                                               const float* are, const float* aim, const float* aw, int B,
                                               int RS, int PS, int3 o, int V, int rowlen, bool exclusive,
                                               bool fx = false, float inv_v = 1.f, float inv_w = 1.f) {
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int row = threadIdx.x >> 5; row < B * B; row += nwarps) {  // one warp per (y, z) row
    const int ly = row % B, lz = row / B;
    for (int lx = lane; lx < B; lx += 32) {
      int k = lz * PS + ly * RS + lx;
      float r = are[k], im = aim[k], ww = aw[k];
      if (fx) {
        r = (float)__float_as_int(r) * inv_v;
        im = (float)__float_as_int(im) * inv_v;
        ww = (float)__float_as_int(ww) * inv_w;
      }
      if (r == 0.f && im == 0.f && ww == 0.f) continue;
      int x = o.x + lx, y = o.y + ly, z = o.z + lz;
      int ys, zs;
      bool alias;
      if (DECENTERED) {
        ys = y < 0 ? y + V : y;
        zs = z < 0 ? z + V : z;
        alias = (y == V / 2 || y == -(V / 2) || z == V / 2 || z == -(V / 2));
      } else {
        ys = y + V / 2;
        zs = z + V / 2;
        alias = false;
      }
      if (CLAMP && !DECENTERED) {
        const unsigned cx = min((unsigned)x, (unsigned)(V / 2)), cy = min((unsigned)ys, (unsigned)(V - 1)),
                       cz = min((unsigned)zs, (unsigned)(V - 1));
        // every voxel on a face the clamps fold onto, not only the folded
        // ones: a plain read-add-write there would race with their reductions
        alias = cx == (unsigned)(V / 2) || cy == (unsigned)(V - 1) || cz == (unsigned)(V - 1);
        x = (int)cx;
        ys = (int)cy;
        zs = (int)cz;
      } else if ((unsigned)x > (unsigned)(V / 2) || (unsigned)ys >= (unsigned)V || (unsigned)zs >= (unsigned)V) {
        continue;  // outside the volume: nothing can have been added here
      }
      int64_t idx = ((int64_t)zs * V + ys) * rowlen + x;
      if (exclusive && !alias) {
        if (volft) {
          float2 c = volft[idx];
          volft[idx] = make_float2(c.x + r, c.y + im);
        }
        if (volw) volw[idx] += ww;
      } else {
        if (volft) red_add2((float*)(volft + idx), r, im);
        if (volw) red_add(volw + idx, ww);
      }
    }
  }
}

template <bool DECENTERED, bool SQUARE>
__global__ void __launch_bounds__(1024)
backproject_brick_kernel(float2* __restrict__ volft, float* __restrict__ volw,
                         const float2* __restrict__ projft, const float* __restrict__ projw,
                         const float* __restrict__ mats, BpArgs a, BrickGrid g,
                         const BrickItem* __restrict__ items, const int* __restrict__ nitems_ptr,
                         const int* __restrict__ pairs, const PixelBin* __restrict__ bins,
                         const int* __restrict__ entries, int* __restrict__ counter) {
  extern __shared__ float acc[];
  __shared__ int item_s, next_s;
  const int nitems = *nitems_ptr;
  // Accumulator layout: rows padded to B+1 and planes to (B+1)^2 floats, so
  // that the lanes of a warp, whose samples step along an arbitrary
  // direction, spread over the banks (unpadded, steps along y or z would
  // land every lane in the same bank).
  const int B = g.B, RS = g.B + 1, PS = (g.B + 1) * (g.B + 1), NA = g.B * PS;
  float* are = acc;
  float* aim = acc + NA;
  float* aw = acc + 2 * NA;
  const int lane = threadIdx.x & 31;
  const int V = a.P;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      item_s = atomicAdd(counter, 1);
      next_s = 0;
    }
    for (int k = threadIdx.x; k < 3 * NA; k += blockDim.x) acc[k] = 0.f;
    __syncthreads();
    const int w = item_s;
    if (w >= nitems) break;
    const BrickItem it = items[w];
    const int3 o = brick_origin(g, it.brick);

    for (;;) {  // warps take the item's bins one at a time
      int j = 0;
      if (lane == 0) j = atomicAdd(&next_s, 1);
      j = __shfl_sync(0xffffffffu, j, 0);
      if (j >= it.count) break;
      const PixelBin bn = bins[__ldg(pairs + it.offset + j)];
      float m[9];
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)bn.slice + k);
      // Interior entries: the whole target cube lies in this brick, either
      // direct (x0 >= 1) or mirrored to -n and conjugated (x0 <= -2).  One
      // branch-free path: corner kb and direction sg (+1 or -1).
      for (int e = lane; e < bn.interior; e += 32) {
        const int pid = __ldg(entries + bn.start + e);
        int u, v;
        pixel_uv(pid, a.n, a.dimft, u, v);
        const int64_t id = a.elements * bn.slice + pid;
        BpSample s = backproject_sample(m, (float)u, (float)v, 0.f);
        float2 val = projft ? __ldg(projft + id) : make_float2(1.f, 0.f);
        float pw = projw ? __ldg(projw + id) : 1.f;
        const int sg = s.x0 >= 1 ? 1 : -1;
        const int kb = (sg * s.z0 - o.z) * PS + (sg * s.y0 - o.y) * RS + (sg * s.x0 - o.x);
        const float im = sg * val.y;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          float w = SQUARE ? s.w[i] * s.w[i] : s.w[i];
          int k = kb + sg * ((i & 1) + ((i >> 1) & 1) * RS + ((i >> 2) & 1) * PS);
          atomicAdd(are + k, w * val.x);
          atomicAdd(aim + k, w * im);
          atomicAdd(aw + k, w * pw);
        }
      }
      // Boundary entries: the cube crosses a brick face or the x = 0 plane;
      // every target is tested.
      for (int e = bn.interior + lane; e < bn.count; e += 32) {
        const int pid = __ldg(entries + bn.start + e);
        int u, v;
        pixel_uv(pid, a.n, a.dimft, u, v);
        const int64_t id = a.elements * bn.slice + pid;
        BpSample s = backproject_sample(m, (float)u, (float)v, 0.f);
        float2 val = projft ? __ldg(projft + id) : make_float2(1.f, 0.f);
        float pw = projw ? __ldg(projw + id) : 1.f;
        for_each_target(s.x0, s.y0, s.z0, [&](int i, int x, int y, int z, bool conj) {
          int lx = x - o.x, ly = y - o.y, lz = z - o.z;
          if ((unsigned)lx < (unsigned)B && (unsigned)ly < (unsigned)B && (unsigned)lz < (unsigned)B) {
            float w = SQUARE ? s.w[i] * s.w[i] : s.w[i];
            int k = lz * PS + ly * RS + lx;
            atomicAdd(are + k, w * val.x);
            atomicAdd(aim + k, w * (conj ? -val.y : val.y));
            atomicAdd(aw + k, w * pw);
          }
        });
      }
    }
    __syncthreads();

    // flush the brick into the volume
    bp_flush_brick<DECENTERED>(volft, volw, are, aim, aw, B, RS, PS, o, V, a.rowlen, it.exclusive != 0);
  }
}

// Segment variant of the brick backprojector: the same accumulators and
// flush, but a warp takes a (slice, brick) pair of the segment plan and finds
// the pixels itself, by row segments (segment.cuh).  Side 0 walks the pixels
// whose position lies in the brick widened by one voxel below (where their
// neighbours can reach it) and adds their unconjugated targets, the
// neighbours with x >= 0; side 1 walks the pixels whose mirrored position
// does and adds their conjugated targets, the mirrored neighbours (x < 0)
// and the second insertions on the x = 0 plane.  Each target of each pixel
// is added once, by the pair of its brick on the side of its conjugation,
// with the weights and values of the binned variant.
//
// GEN (centred output only): the general geometry of the reference's
// insertion — a magnification of the pixel coordinates, the Ewald curvature
// and a target volume per slice (Backproject.cu:57-63, 145-152, 183-189).
// A work item's key is volume * nbricks + brick; the row segments walk the
// magnified map u c0' + v c1' with every box widened by the curvature's
// reach, and each candidate is kept only if the reference's magnified
// radius test passes, so the samples and targets are the direct kernel's.
// The grid reaches one voxel past the volume (kept samples come within
// rmax * scale of the origin) and the flush folds those voxels onto the
// edge faces with the reference's clamps.
template <bool DECENTERED, bool SQUARE, bool GEN>
__global__ void __launch_bounds__(1024)
backproject_segment_kernel(float2* __restrict__ volft_base, float* __restrict__ volw_base,
                           const float2* __restrict__ projft, const float* __restrict__ projw,
                           const float* __restrict__ mats, BpArgs a, BrickGrid g, PixelSet px, SliceGeom gm,
                           const BrickItem* __restrict__ items, const int* __restrict__ nitems_ptr,
                           const int* __restrict__ pairs, const PixelBin* __restrict__ bins, int* __restrict__ counter,
                           FxBands fxb) {
  extern __shared__ float acc[];
  __shared__ int item_s, next_s, danger_s;
  __shared__ float sv_s, sw_s;
  const int nitems = *nitems_ptr;
  // Accumulator layout as in backproject_brick_kernel (rows padded to B+1,
  // planes to (B+1)^2 floats).
  const int B = g.B, RS = g.B + 1, PS = (g.B + 1) * (g.B + 1), NA = g.B * PS;
  float* are = acc;
  float* aim = acc + NA;
  float* aw = acc + 2 * NA;
  const int lane = threadIdx.x & 31;
  const int V = a.P;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item_s = atomicAdd(counter, 1);
    __syncthreads();
    const int w = item_s;
    if (w >= nitems) break;
    const BrickItem it = items[w];
    const int vol = GEN ? it.brick / g.nbricks : 0;
    const int3 o = brick_origin(g, it.brick - vol * g.nbricks);
    float2* volft = volft_base && GEN ? volft_base + (int64_t)vol * a.nvox : volft_base;
    float* volw = volw_base && GEN ? volw_base + (int64_t)vol * a.nvox : volw_base;

    // warps take the item's pairs one at a time, the next one's slice
    // fetched before the current one is processed; FXM: fixed-point
    // accumulation (int32 shared atomics of round(w v S)), else FP32
    // atomics.  Returns with `danger` holding, in its sign bit, whether any
    // fixed-point sum came within a factor two of overflowing.
    auto run_pairs = [&](auto fxtag, float sv, float sw, unsigned& danger) {
      constexpr bool FXM = decltype(fxtag)::value;
      auto add3 = [&](int k, float wt, float re, float im, float pwv) {
        if constexpr (FXM) {
          const int o1 = atomicAdd(reinterpret_cast<int*>(are) + k, __float2int_rn(wt * re));
          const int o2 = atomicAdd(reinterpret_cast<int*>(aim) + k, __float2int_rn(wt * im));
          const int o3 = atomicAdd(reinterpret_cast<int*>(aw) + k, __float2int_rn(wt * pwv));
          // |old| >= 2^30 sets the sign bit of old + 2^30 (every term is
          // below 2^29, so no sum can have wrapped while this stays clear)
          danger |= (unsigned)(o1 + 0x40000000) | (unsigned)(o2 + 0x40000000) | (unsigned)(o3 + 0x40000000);
        } else {
          atomicAdd(are + k, wt * re);
          atomicAdd(aim + k, wt * im);
          atomicAdd(aw + k, wt * pwv);
        }
      };
      auto take = [&]() {
        int j = 0;
        if (lane == 0) j = atomicAdd(&next_s, 1);
        return __shfl_sync(0xffffffffu, j, 0);
      };
      int j = take();
      int4 pr = j < it.count ? seg_pair(bins, pairs, it.offset + j) : make_int4(0, kSegNoRows, kSegNoRows, 0);
      while (j < it.count) {
        const int jn = take();
        const int4 nx =
            jn < it.count ? seg_pair(bins, pairs, it.offset + jn) : make_int4(0, kSegNoRows, kSegNoRows, 0);
        const int slice = pr.x;
        float m[9];
#pragma unroll
        for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)slice + k);
        float me[9];
        if (GEN) effective_matrix(m, gm, me);
        const float widen = GEN ? curvature_reach(m, gm, px.pmax) : 0.f;
        const int64_t sbase = a.elements * slice;
#pragma unroll 1
        for (int side = 0; side < 2; side++) {
          int vlo, vhi;
          seg_unpack_rows(side ? pr.z : pr.y, vlo, vhi);
          if (vlo > vhi) continue;  // no pixel of this side
          const SegBox box = seg_box(GEN ? me : m, side, o, B, 1.f, widen);
          const bool plane0 = side == 1 && o.x == 0;  // second insertions can land in this brick
          seg_for_each_pixel_rows(box, px, vlo, vhi, [&](int u, int v, bool valid) {
            if (!valid) return;
            float qx = (float)u, qy = (float)v, qz = 0.f;
            if (GEN) {  // Backproject.cu:176-192, as backproject_direct_kernel
              qx = fmaf(a.mag.x, (float)u, a.mag.z * (float)v);
              qy = fmaf(a.mag.y, (float)u, a.mag.w * (float)v);
              qz = a.ewalddiaminv * (float)(u * u + v * v);
              if ((int)fmaf(qz, qz, fmaf(qx, qx, qy * qy)) >= a.rmax2) return;
            }
            const int idy = v < 0 ? v + a.n : v;
            const int64_t id = sbase + (int64_t)idy * a.dimft + u;
            BpSample s = backproject_sample(m, qx, qy, qz);
            float2 val = projft ? __ldg(projft + id) : make_float2(1.f, 0.f);
            float pw = projw ? __ldg(projw + id) : 1.f;
            if (FXM) {  // values in units of the item's fixed-point step
              val.x *= sv;
              val.y *= sv;
              pw *= sw;
              // larger terms (or non-finite ones) than the scale allows: the
              // item is redone in FP32
              if (!(fmaxf(fabsf(val.x), fmaxf(fabsf(val.y), fabsf(pw))) < 536870912.f)) danger |= 0x80000000u;
            }
            if (side == 0) {
              const int lx0 = s.x0 - o.x, ly0 = s.y0 - o.y, lz0 = s.z0 - o.z;
#pragma unroll
              for (int i = 0; i < 8; i++) {
                const int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
                const int lx = lx0 + dx, ly = ly0 + dy, lz = lz0 + dz;
                if (s.x0 + dx >= 0 && (unsigned)lx < (unsigned)B && (unsigned)ly < (unsigned)B &&
                    (unsigned)lz < (unsigned)B) {
                  const float wt = SQUARE ? s.w[i] * s.w[i] : s.w[i];
                  add3(lz * PS + ly * RS + lx, wt, val.x, val.y, pw);
                }
              }
            } else {
              // mirrored neighbour -n of n = base + (dx, dy, dz), local coordinates
              const int lx0 = -s.x0 - o.x, ly0 = -s.y0 - o.y, lz0 = -s.z0 - o.z;
#pragma unroll
              for (int i = 0; i < 8; i++) {
                const int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
                const int lx = lx0 - dx, ly = ly0 - dy, lz = lz0 - dz;
                if (s.x0 + dx < 0 && (unsigned)lx < (unsigned)B && (unsigned)ly < (unsigned)B &&
                    (unsigned)lz < (unsigned)B) {
                  const float wt = SQUARE ? s.w[i] * s.w[i] : s.w[i];
                  add3(lz * PS + ly * RS + lx, wt, val.x, -val.y, pw);
                }
              }
              if (plane0) {
                // second insertion at (0, -ny, -nz) of each neighbour with
                // nx == 0 and (ny, nz) != 0; here o.x == 0, so local x is 0
#pragma unroll
                for (int i = 0; i < 8; i++) {
                  const int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
                  const int ny = s.y0 + dy, nz = s.z0 + dz;
                  const int ly = -ny - o.y, lz = -nz - o.z;
                  if (s.x0 + dx == 0 && (ny != 0 || nz != 0) && (unsigned)ly < (unsigned)B &&
                      (unsigned)lz < (unsigned)B) {
                    const float wt = SQUARE ? s.w[i] * s.w[i] : s.w[i];
                    add3(lz * PS + ly * RS, wt, val.x, -val.y, pw);
                  }
                }
              }
            }
          });
        }
        j = jn;
        pr = nx;
      }
    };

    // Fixed point first where a scale is known; if any sum of the item came
    // near overflow, the item is accumulated again in FP32.
    bool fx = !SQUARE && fxb.vmax != nullptr;
    for (;;) {
      for (int k = threadIdx.x; k < 3 * NA; k += blockDim.x) acc[k] = 0.f;
      if (threadIdx.x == 0) {
        next_s = 0;
        danger_s = 0;
        if (fx) {
          float svv, sww;
          if (fx_item_scales(fxb, o, B, svv, sww)) {
            sv_s = svv;
            sw_s = sww;
          } else {
            danger_s = 1;  // no usable scale: FP32
          }
        }
      }
      __syncthreads();
      if (fx && danger_s) {  // uniform: every thread read it after the barrier
        fx = false;
        __syncthreads();
        continue;
      }
      unsigned danger = 0;
      if (fx)
        run_pairs(std::true_type(), sv_s, sw_s, danger);
      else
        run_pairs(std::false_type(), 1.f, 1.f, danger);
      if (fx && __any_sync(0xffffffffu, (int)danger < 0) && lane == 0) danger_s = 1;
      __syncthreads();
      if (fx && danger_s) {
        fx = false;
        __syncthreads();
        continue;
      }
      break;
    }

    // flush the brick into the volume
    bp_flush_brick<DECENTERED, GEN>(volft, volw, are, aim, aw, B, RS, PS, o, V, a.rowlen, it.exclusive != 0, fx,
                                    fx ? 1.f / sv_s : 1.f, fx ? 1.f / sw_s : 1.f);
  }
}

template <bool DEC, bool SQ>
static void launch_bp_direct(dim3 grid, cudaStream_t stream, float2* vf, float* vw, const float2* pf,
                             const float* pw, const float* mats, const int* ivol, const BpArgs& a,
                             const int* list, const int* nlist, int ndp) {
  if (ndp == 2)
    backproject_direct_kernel<2, DEC, SQ><<<grid, kBpThreads, 0, stream>>>(vf, vw, pf, pw, mats, ivol, a, list, nlist);
  else
    backproject_direct_kernel<3, DEC, SQ><<<grid, kBpThreads, 0, stream>>>(vf, vw, pf, pw, mats, ivol, a, list, nlist);
}

static void launch_bp_direct_any(dim3 grid, cudaStream_t stream, float2* vf, float* vw, const float2* pf,
                                 const float* pw, const float* mats, const int* ivol, const BpArgs& a,
                                 const int* list, const int* nlist, int ndp, int decentered, int square) {
  if (decentered) {
    if (square) launch_bp_direct<true, true>(grid, stream, vf, vw, pf, pw, mats, ivol, a, list, nlist, ndp);
    else launch_bp_direct<true, false>(grid, stream, vf, vw, pf, pw, mats, ivol, a, list, nlist, ndp);
  } else {
    if (square) launch_bp_direct<false, true>(grid, stream, vf, vw, pf, pw, mats, ivol, a, list, nlist, ndp);
    else launch_bp_direct<false, false>(grid, stream, vf, vw, pf, pw, mats, ivol, a, list, nlist, ndp);
  }
}

// Square of the smallest singular value of the 2x2 magnification (columns
// (x, y) and (z, w)).
static double mag_smin2(float4 mag) {
  const double m00 = mag.x, m10 = mag.y, m01 = mag.z, m11 = mag.w;
  const double p = m00 * m00 + m10 * m10, q = m01 * m01 + m11 * m11, r = m00 * m01 + m10 * m11;
  return 0.5 * (p + q) - std::sqrt(0.25 * (p - q) * (p - q) + r * r);
}

// Largest volume index of a device array, through the pool (one small
// kernel and a read-back that waits for the stream).
__global__ void max_index_kernel(const int* __restrict__ iv, unsigned n, int* __restrict__ out) {
  int m = INT_MIN;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, iv[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

static int device_max_index(const int* d_iv, unsigned n, cudaStream_t stream, int* out) {
  int* d = nullptr;
  int st = pool_alloc((void**)&d, sizeof(int), stream);
  if (st) return st;
  const int init = INT_MIN;
  int h = INT_MIN;
  cudaError_t e = cudaMemcpyAsync(d, &init, sizeof(int), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) {
    max_index_kernel<<<std::min(1024u, (n + 255) / 256), 256, 0, stream>>>(d_iv, n, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  pool_free(d, stream);
  if (e != cudaSuccess) return set_error(GTOMRLN_ERR_CUDA, "volume index read-back: %s", cudaGetErrorString(e));
  *out = h;
  return GTOMRLN_OK;
}

// The brick path: plan, brick kernel, and the direct kernel for any slice the
// plan could not take.  Nothing synchronises.  gen: magnification, Ewald
// curvature or per-slice volumes (centred output, row segments only;
// d_ivolume values in [0, nvol)).
static int backproject_brick(float* d_volumeft, float* d_volumeweights, const float* d_projft,
                             const float* d_projweights, const float* d_mats, const BpArgs& a,
                             int rmax, int decentered, int square, unsigned batch, cudaStream_t stream,
                             int segments, bool gen = false, const int* d_ivolume = nullptr, int nvol = 1,
                             bool fixed_point = true) {
  const int V = a.P;
  // Neighbours stay inside x [0, V/2] and y, z [-V/2, yhi] (no clamp, no
  // wrap beyond the reference's) while every sample radius is below limit;
  // the general geometry's grid reaches one voxel further and its flush
  // folds that voxel onto the edge with the reference's clamps.
  const int yhi = decentered ? V / 2 : V - 1 - V / 2;
  const int ext = gen ? 1 : 0;
  const float limit = (float)(std::min(V / 2, yhi) + ext) - 1e-4f;
  const BrickTuning tune = brick_tuning(GTOMRLN_OP_BACKPROJECT);
  BrickGrid g = make_brick_grid(V, tune.edge, V / 2 + ext, -(V / 2) - ext, yhi + ext);
  size_t smem = sizeof(float) * 3 * (size_t)tune.edge * (tune.edge + 1) * (tune.edge + 1);
  auto kern = decentered ? (square ? backproject_brick_kernel<true, true> : backproject_brick_kernel<true, false>)
                         : (square ? backproject_brick_kernel<false, true> : backproject_brick_kernel<false, false>);
  auto skern = gen ? (square ? backproject_segment_kernel<false, true, true>
                             : backproject_segment_kernel<false, false, true>)
               : decentered
                   ? (square ? backproject_segment_kernel<true, true, false> : backproject_segment_kernel<true, false, false>)
                   : (square ? backproject_segment_kernel<false, true, false> : backproject_segment_kernel<false, false, false>);
  cudaError_t e = segments ? cudaFuncSetAttribute(skern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                           : cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return set_error(GTOMRLN_ERR_CUDA, "brick backprojector: %zu B of shared memory refused: %s", smem,
                     cudaGetErrorString(e));
  int dev = 0, sms = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (segments)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, skern, tune.threads, smem);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, tune.threads, smem);
  PixelSet px;
  px.n = a.n;
  px.dimft = a.dimft;
  px.elements = a.elements;
  px.rmax2 = a.rmax2;
  px.strict = 1;
  px.pmax = std::sqrt((float)std::max(0, rmax * rmax - 1));
  SliceGeom gm;
  if (gen) {
    // The samples kept have |q| < rmax with q the magnified coordinates, so
    // the pixels to visit lie within rmax / (smallest singular value of the
    // magnification); the kernel applies the exact test.
    const double rp = (double)rmax / std::sqrt(mag_smin2(a.mag));
    const double lim2 = 2.0 * (double)(a.n / 2 + 1) * (a.n / 2 + 1);  // beyond every pixel of the slice
    px.rmax2 = (int)std::min(lim2, std::floor(rp * rp * (1.0 + 1e-6)) + 2.0);
    px.pmax = (float)std::sqrt((double)px.rmax2) * (1.f + 1e-6f);
    gm.mag = a.mag;
    gm.curve = a.ewalddiaminv;
    gm.ivolume = d_ivolume;
    gm.nvol = nvol;
    gm.qmax = std::sqrt((float)a.rmax2) * (1.f + 1e-6f);
  }
  BrickPlan plan;
  int st = build_brick_plan(GTOMRLN_OP_BACKPROJECT, d_mats, (int)batch, g, px, limit, tune.chunk, stream, &plan,
                            segments, nullptr, gm);
  if (st) return st;
  // the radial magnitude table of the fixed-point mode (a sampled pass over
  // the batch, ~0.6 M pixels)
  FxBands fxb;
  unsigned* d_bands = nullptr;
  if (segments && !square && fixed_point) {
    const int nb = std::min(kFxMaxBands, (int)((V / 2 + 8) / kFxBand) + 2);
    const size_t bytes = 5 * sizeof(unsigned) * (size_t)nb;  // vmax, wmax, vsum, wsum, count
    st = pool_alloc((void**)&d_bands, bytes, stream);
    if (st) {
      free_brick_plan(&plan, stream);
      return st;
    }
    e = cudaMemsetAsync(d_bands, 0, bytes, stream);
    if (e == cudaSuccess) {
      unsigned* vmax = d_bands;
      unsigned* wmax = d_bands + nb;
      float* vsum = reinterpret_cast<float*>(d_bands + 2 * nb);
      float* wsum = reinterpret_cast<float*>(d_bands + 3 * nb);
      unsigned* count = d_bands + 4 * nb;
      fx_band_sample_kernel<<<sms * 2, 256, 0, stream>>>((const float2*)d_projft, d_projweights, d_mats, batch,
                                                         a.n, a.dimft, a.elements, a.rmax2, nb, 8, vmax, wmax, vsum,
                                                         wsum, count);
      fxb.vmax = vmax;
      fxb.wmax = wmax;
      fxb.vsum = vsum;
      fxb.wsum = wsum;
      fxb.count = count;
      fxb.nbands = nb;
    }
  }
  if (segments)
    skern<<<sms * std::max(occ, 1), tune.threads, smem, stream>>>(
        (float2*)d_volumeft, d_volumeweights, (const float2*)d_projft, d_projweights, d_mats, a, g, px, gm,
        plan.items, plan.nitems, plan.pairs, plan.bins, plan.counter, fxb);
  else
    kern<<<sms * std::max(occ, 1), tune.threads, smem, stream>>>(
        (float2*)d_volumeft, d_volumeweights, (const float2*)d_projft, d_projweights, d_mats, a, g, plan.items,
        plan.nitems, plan.pairs, plan.bins, plan.entries, plan.counter);
  launch_bp_direct_any(dim3(sms * 4), stream, (float2*)d_volumeft, d_volumeweights, (const float2*)d_projft,
                       d_projweights, d_mats, d_ivolume, a, plan.fallback, plan.nfallback, 2, decentered, square);
  if (e == cudaSuccess) e = cudaGetLastError();
  pool_free(d_bands, stream);
  free_brick_plan(&plan, stream);
  if (e != cudaSuccess)
    return set_error(GTOMRLN_ERR_CUDA, "launch of the brick backprojector failed: %s", cudaGetErrorString(e));
  return GTOMRLN_OK;
}

// d_rlnBackprojectShifted (BackprojectShifted.cu:67-186): a different
// insertion from Backproject3DtoNDKernel in the reference itself, kept as it
// is: r^2 <= rmax^2 (y, z signed by comparing with rmax), the whole x = 0
// column inserted, Friedel flip of the position only (no mirrored
// neighbours, no second insertion on x = 0), plain FP32 trilinear weights,
// centred output, the sample times exp(i phi), phi = -(x sx + y sy [+ z sz])
// with the slice's 2 pi / n-scaled shift, and the value and weight times the
// slice's global weight.  The reference writes without bounds checks; the
// indices here are clamped like place<false> (unsigned compares).
template <int NDIMS>
__global__ void __launch_bounds__(kBpThreads)
backproject_shifted_kernel(float2* __restrict__ volft, float* __restrict__ volw,
                           const float2* __restrict__ projft, const float* __restrict__ projw,
                           const float* __restrict__ mats, const float* __restrict__ shifts,
                           const float* __restrict__ gweights, BpArgs a, int rmax,
                           const int* __restrict__ list = nullptr, const int* __restrict__ nlist = nullptr) {
  // Without a list the grid covers every (slice, tile) once; with one (the
  // slices a brick plan left over) a persistent grid strides over them.
  const int64_t total = list ? (int64_t)(*nlist) * a.tiles : (int64_t)gridDim.x;
  for (int64_t work = blockIdx.x; work < total; work += gridDim.x) {
  const int entry = (int)(work / a.tiles);
  const int tile = (int)(work - (int64_t)entry * a.tiles);
  const int slice = list ? __ldg(list + entry) : entry;
  float m[9];
#pragma unroll
  for (int i = 0; i < 9; i++) m[i] = __ldg(mats + 9 * (int64_t)slice + i);
  const float sx = __ldg(shifts + 3 * (int64_t)slice), sy = __ldg(shifts + 3 * (int64_t)slice + 1);
  const float sz = __ldg(shifts + 3 * (int64_t)slice + 2);
  const float gw = __ldg(gweights + slice);
  const int V = a.P;
  for (int k = 0; k < kBpPerThread; k++) {
    int64_t id = (int64_t)tile * kBpTile + k * kBpThreads + threadIdx.x;
    if (id >= a.elements) break;
    int idx, idy, idz;
    split_index(id, a.dimft, NDIMS == 3 ? a.area : a.elements, a.elements, idx, idy, idz);
    int x = idx;
    int y = idy <= rmax ? idy : idy - a.n;
    int z = NDIMS == 3 ? (idz <= rmax ? idz : idz - a.n) : 0;
    int r2 = NDIMS == 3 ? z * z + y * y + x * x : y * y + x * x;
    if (r2 > a.rmax2) continue;
    float3 pos = mat_apply(m, (float)x, (float)y, (float)z);
    float sign = 1.f;
    if (pos.x + 1e-5f < 0.f) {
      pos.x = fabsf(pos.x);
      pos.y = -pos.y;
      pos.z = -pos.z;
      sign = -1.f;
    }
    int x0 = (int)floorf(pos.x + 1e-5f);
    float fx = pos.x - (float)x0;
    int y0 = (int)floorf(pos.y);
    float fy = pos.y - (float)y0;
    int z0 = (int)floorf(pos.z);
    float fz = pos.z - (float)z0;
    y0 += V / 2;
    z0 += V / 2;
    float c0 = 1.f - fz, c1 = fz;
    float c00 = (1.f - fy) * c0, c10 = fy * c0, c01 = (1.f - fy) * c1, c11 = fy * c1;
    float w[8] = {(1.f - fx) * c00, fx * c00, (1.f - fx) * c10, fx * c10,
                  (1.f - fx) * c01, fx * c01, (1.f - fx) * c11, fx * c11};
    float2 v = projft ? __ldg(projft + a.elements * slice + id) : make_float2(1.f, 0.f);
    float phase = fmaf((float)x, sx, (float)y * sy);
    if (NDIMS == 3) phase = fmaf((float)z, sz, phase);
    phase = -phase;
    float c = __cosf(phase), s = __sinf(phase);
    float re = fmaf(v.x, c, -(v.y * s)), im = fmaf(v.x, s, v.y * c);
    im *= sign;
    re *= gw;
    im *= gw;
    float pw = (projw ? __ldg(projw + a.elements * slice + id) : 1.f) * gw;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      unsigned tx = (unsigned)(x0 + (i & 1)), ty = (unsigned)(y0 + ((i >> 1) & 1));
      unsigned tz = (unsigned)(z0 + ((i >> 2) & 1));
      tx = tx > (unsigned)(V / 2) ? (unsigned)(V / 2) : tx;
      ty = ty > (unsigned)(V - 1) ? (unsigned)(V - 1) : ty;
      tz = tz > (unsigned)(V - 1) ? (unsigned)(V - 1) : tz;
      int64_t o = ((int64_t)tz * V + ty) * a.rowlen + tx;
      if (volft) red_add2((float*)(volft + o), w[i] * re, w[i] * im);
      if (volw) red_add(volw + o, w[i] * pw);
    }
  }
  }  // work loop
}

// Segment variant of the shifted insertion for 2D slices: per sample the
// arithmetic of backproject_shifted_kernel (Friedel flip of the position when
// pos.x + 1e-5 < 0, plain trilinear weights on the 2x2x2 cube at the flipped
// position's base voxel, the sample times exp(i phi) and the slice's weight),
// with the targets accumulated per shared-memory brick as in
// backproject_segment_kernel.  Side 0 walks the unflipped samples, side 1
// the flipped ones (negated positions), each over the brick widened by one
// voxel below; a sample's eight targets are added by the pairs of their
// bricks on the side of its flip.  Centred output.  The brick grid reaches one
// voxel past the volume (the insertion takes the whole rmax disk, so at
// padding 2 the rim's cubes reach x = V/2 + 1), and the flush folds those
// voxels onto the edge with the direct kernel's clamps.
__global__ void __launch_bounds__(1024)
backproject_shifted_segment_kernel(float2* __restrict__ volft, float* __restrict__ volw,
                                   const float2* __restrict__ projft, const float* __restrict__ projw,
                                   const float* __restrict__ mats, const float* __restrict__ shifts,
                                   const float* __restrict__ gweights, BpArgs a, BrickGrid g, PixelSet px,
                                   const BrickItem* __restrict__ items, const int* __restrict__ nitems_ptr,
                                   const int* __restrict__ pairs, const PixelBin* __restrict__ bins, int* __restrict__ counter) {
  extern __shared__ float acc[];
  __shared__ int item_s, next_s;
  const int nitems = *nitems_ptr;
  const int B = g.B, RS = g.B + 1, PS = (g.B + 1) * (g.B + 1), NA = g.B * PS;
  float* are = acc;
  float* aim = acc + NA;
  float* aw = acc + 2 * NA;
  const int lane = threadIdx.x & 31;
  const int V = a.P;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      item_s = atomicAdd(counter, 1);
      next_s = 0;
    }
    for (int k = threadIdx.x; k < 3 * NA; k += blockDim.x) acc[k] = 0.f;
    __syncthreads();
    const int w = item_s;
    if (w >= nitems) break;
    const BrickItem it = items[w];
    const int3 o = brick_origin(g, it.brick);
    auto take = [&]() {
      int j = 0;
      if (lane == 0) j = atomicAdd(&next_s, 1);
      return __shfl_sync(0xffffffffu, j, 0);
    };
    int j = take();
    int4 pr = j < it.count ? seg_pair(bins, pairs, it.offset + j) : make_int4(0, kSegNoRows, kSegNoRows, 0);
    while (j < it.count) {
      const int jn = take();
      const int4 nx = jn < it.count ? seg_pair(bins, pairs, it.offset + jn) : make_int4(0, kSegNoRows, kSegNoRows, 0);
      const int slice = pr.x;
      float m[9];
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)slice + k);
      const float sx = __ldg(shifts + 3 * (int64_t)slice), sy = __ldg(shifts + 3 * (int64_t)slice + 1);
      const float gw = __ldg(gweights + slice);
      const int64_t sbase = a.elements * slice;
#pragma unroll 1
      for (int side = 0; side < 2; side++) {
        int vlo, vhi;
        seg_unpack_rows(side ? pr.z : pr.y, vlo, vhi);
        if (vlo > vhi) continue;  // no pixel of this side
        const SegBox box = seg_box(m, side, o, B, 1.f);
        seg_for_each_pixel_rows(box, px, vlo, vhi, [&](int u, int v, bool valid) {
          if (!valid) return;
          float3 pos = mat_apply(m, (float)u, (float)v, 0.f);
          const bool flip = pos.x + 1e-5f < 0.f;
          if (flip != (side == 1)) return;  // the other side's sample
          float sign = 1.f;
          if (flip) {
            pos.x = fabsf(pos.x);
            pos.y = -pos.y;
            pos.z = -pos.z;
            sign = -1.f;
          }
          const int x0 = (int)floorf(pos.x + 1e-5f);
          const float fx = pos.x - (float)x0;
          const int y0 = (int)floorf(pos.y);
          const float fy = pos.y - (float)y0;
          const int z0 = (int)floorf(pos.z);
          const float fz = pos.z - (float)z0;
          const int lx0 = x0 - o.x, ly0 = y0 - o.y, lz0 = z0 - o.z;
          if (lx0 < -1 || lx0 >= B || ly0 < -1 || ly0 >= B || lz0 < -1 || lz0 >= B) return;
          const float c0 = 1.f - fz, c1 = fz;
          const float c00 = (1.f - fy) * c0, c10 = fy * c0, c01 = (1.f - fy) * c1, c11 = fy * c1;
          const float wt[8] = {(1.f - fx) * c00, fx * c00, (1.f - fx) * c10, fx * c10,
                               (1.f - fx) * c01, fx * c01, (1.f - fx) * c11, fx * c11};
          const int idy = v < 0 ? v + a.n : v;
          const int64_t id = sbase + (int64_t)idy * a.dimft + u;
          const float2 val = projft ? __ldg(projft + id) : make_float2(1.f, 0.f);
          float phase = fmaf((float)u, sx, (float)v * sy);
          phase = -phase;
          const float c = __cosf(phase), sn = __sinf(phase);
          float re = fmaf(val.x, c, -(val.y * sn)), im = fmaf(val.x, sn, val.y * c);
          im *= sign;
          re *= gw;
          im *= gw;
          const float pw = (projw ? __ldg(projw + id) : 1.f) * gw;
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int lx = lx0 + (i & 1), ly = ly0 + ((i >> 1) & 1), lz = lz0 + ((i >> 2) & 1);
            if ((unsigned)lx < (unsigned)B && (unsigned)ly < (unsigned)B && (unsigned)lz < (unsigned)B) {
              const int k = lz * PS + ly * RS + lx;
              atomicAdd(are + k, wt[i] * re);
              atomicAdd(aim + k, wt[i] * im);
              atomicAdd(aw + k, wt[i] * pw);
            }
          }
        });
      }
      j = jn;
      pr = nx;
    }
    __syncthreads();
    bp_flush_brick<false, true>(volft, volw, are, aim, aw, B, RS, PS, o, V, a.rowlen, it.exclusive != 0);
  }
}

// The segment path of the shifted insertion: plan, segment kernel, and the
// direct kernel for any slice the plan could not take.  Nothing synchronises.
static int backproject_shifted_brick(float* d_volumeft, float* d_volumeweights, const float* d_projft,
                                     const float* d_projweights, const float* d_mats, const float* d_shifts,
                                     const float* d_gweights, const BpArgs& a, int rmax, unsigned batch,
                                     cudaStream_t stream) {
  const int V = a.P;
  // While every sample radius stays below V/2 + 0.99, the cubes' voxels lie
  // in x [0, V/2 + 1] and y, z [-V/2 - 1, V/2 + 1] (centred, before clamps).
  const float limit = (float)(V / 2) + 0.99f;
  const BrickTuning tune = brick_tuning(GTOMRLN_OP_BACKPROJECT);
  BrickGrid g = make_brick_grid(V, tune.edge, V / 2 + 1, -(V / 2) - 1, V / 2 + 1);
  size_t smem = sizeof(float) * 3 * (size_t)tune.edge * (tune.edge + 1) * (tune.edge + 1);
  cudaError_t e = cudaFuncSetAttribute(backproject_shifted_segment_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return set_error(GTOMRLN_ERR_CUDA, "shifted brick backprojector: %zu B of shared memory refused: %s", smem,
                     cudaGetErrorString(e));
  int dev = 0, sms = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, backproject_shifted_segment_kernel, tune.threads, smem);
  PixelSet px;
  px.n = a.n;
  px.dimft = a.dimft;
  px.elements = a.elements;
  px.rmax2 = a.rmax2;
  px.strict = 0;  // r^2 <= rmax^2, the whole x = 0 column
  px.pmax = (float)rmax;
  BrickPlan plan;
  int st = build_brick_plan(GTOMRLN_OP_BACKPROJECT, d_mats, (int)batch, g, px, limit, tune.chunk, stream, &plan,
                            1);
  if (st) return st;
  backproject_shifted_segment_kernel<<<sms * std::max(occ, 1), tune.threads, smem, stream>>>(
      (float2*)d_volumeft, d_volumeweights, (const float2*)d_projft, d_projweights, d_mats, d_shifts, d_gweights,
      a, g, px, plan.items, plan.nitems, plan.pairs, plan.bins, plan.counter);
  backproject_shifted_kernel<2><<<sms * 4, kBpThreads, 0, stream>>>(
      (float2*)d_volumeft, d_volumeweights, (const float2*)d_projft, d_projweights, d_mats, d_shifts, d_gweights,
      a, rmax, plan.fallback, plan.nfallback);
  e = cudaGetLastError();
  free_brick_plan(&plan, stream);
  if (e != cudaSuccess)
    return set_error(GTOMRLN_ERR_CUDA, "launch of the shifted brick backprojector failed: %s",
                     cudaGetErrorString(e));
  return GTOMRLN_OK;
}

// nvol_hint: the number of volumes d_ivolume indexes when the caller knows it
// (the host-array overload), <= 0 when not.
static int backproject_launch(float* d_volumeft, float* d_volumeweights, int vx, int vy, int vz,
                              const float* d_projft, const float* d_projweights, int px, int py,
                              int pz, unsigned rmax, const float* d_matrices, const int* d_ivolume,
                              float4 mag, float ewaldradiussuper, int decentered, int square,
                              unsigned batch, cudaStream_t stream, int nvol_hint = 0) {
  int ndv = dimension_count(vx, vy, vz), ndp = dimension_count(px, py, pz);
  if (ndv < ndp)
    return set_error(GTOMRLN_ERR_INVALID,
                     "backproject: volume has %d dimensions, projections %d (reference throws)",
                     ndv, ndp);
  if (vx <= 0 || px <= 0) return set_error(GTOMRLN_ERR_INVALID, "backproject: non-positive dimension");
  // A 2D volume is a silent no-op in the reference (Backproject.cu:105-123).
  if (ndv != 3 || batch == 0) return GTOMRLN_OK;
  if (ndp != 2 && ndp != 3)
    return set_error(GTOMRLN_ERR_INVALID, "backproject: projections must be 2D or 3D");
  if (!d_matrices) return set_error(GTOMRLN_ERR_INVALID, "backproject: d_matrices is NULL");
  if (rmax > (unsigned)(px / 2)) rmax = px / 2;

  BpArgs a;
  a.n = px;
  a.dimft = px / 2 + 1;
  a.area = (int64_t)a.dimft * px;
  a.elements = ndp == 3 ? a.area * px : a.area;
  a.tiles = (int)((a.elements + kBpTile - 1) / kBpTile);
  a.rmax2 = (int)(rmax * rmax);
  a.P = vx;
  a.rowlen = vx / 2 + 1;
  a.nvox = (int64_t)a.rowlen * vx * vx;
  a.mag = mag;
  a.ewalddiaminv = ewaldradiussuper == 0 ? 0.f : 1.0f / (2.0f * ewaldradiussuper);
  if ((int64_t)a.tiles * batch > 0x7fffffffLL)
    return set_error(GTOMRLN_ERR_INVALID, "backproject: batch too large for one launch");

  const int choice = path_choice(GTOMRLN_OP_BACKPROJECT);
  const bool plain = !d_ivolume && mag.x == 1.f && mag.y == 0.f && mag.z == 0.f && mag.w == 1.f &&
                     a.ewalddiaminv == 0.f;
  // (the brick plans' integer square roots take radii below 4 096: seg_isqrt)
  const bool brick = ndp == 2 && vx == vy && vx == vz && vx >= 4 && a.rmax2 <= (1 << 24) &&
                     (d_volumeft || d_volumeweights) &&
                     (choice == GTOMRLN_PATH_BRICK || choice == GTOMRLN_PATH_SEGMENT ||
                      choice == GTOMRLN_PATH_SEGMENT_FP32 ||
                      (choice == GTOMRLN_PATH_AUTO && brick_path_pays(GTOMRLN_OP_BACKPROJECT, vx, batch)));
  const bool fixed_point = choice != GTOMRLN_PATH_SEGMENT_FP32;
  if (brick && plain)
    return backproject_brick(d_volumeft, d_volumeweights, d_projft, d_projweights, d_matrices, a, (int)rmax,
                             decentered, square, batch, stream, choice == GTOMRLN_PATH_BRICK ? 0 : 1, false,
                             nullptr, 1, fixed_point);
  // The general geometry (magnification, Ewald curvature, per-slice volumes)
  // takes the row-segment kernel for centred output when the magnification
  // is well conditioned; per-slice volumes need their count (from the host
  // array, else read back from the device, which waits for the stream and
  // is skipped under stream capture).
  if (brick && !decentered && choice != GTOMRLN_PATH_BRICK && mag_smin2(mag) > 1e-4 &&
      std::fabs(a.ewalddiaminv) < 1.f) {
    int nvol = 1;
    if (d_ivolume) {
      nvol = nvol_hint;
      if (nvol <= 0) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
          cudaGetLastError();
          cs = cudaStreamCaptureStatusActive;
        }
        int mx = -1;
        if (cs == cudaStreamCaptureStatusNone) {
          int st = device_max_index(d_ivolume, batch, stream, &mx);
          if (st) return st;
        }
        nvol = mx + 1;
      }
    }
    if (nvol >= 1 && nvol <= 4096)
      return backproject_brick(d_volumeft, d_volumeweights, d_projft, d_projweights, d_matrices, a, (int)rmax,
                               decentered, square, batch, stream, 1, true, d_ivolume, nvol, fixed_point);
  }

  launch_bp_direct_any(dim3((unsigned)(a.tiles * (int64_t)batch)), stream, (float2*)d_volumeft, d_volumeweights,
                       (const float2*)d_projft, d_projweights, d_matrices, d_ivolume, a, nullptr, nullptr, ndp,
                       decentered, square);
  GTOMRLN_LAUNCH_CHECK("backproject_direct_kernel");
  return GTOMRLN_OK;
}

}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_backproject(float* d_volumeft, float* d_volumeweights, int vx, int vy, int vz,
                        const float* d_projft, const float* d_projweights, int px, int py, int pz,
                        unsigned rmax, const float* d_matrices, const int* d_ivolume, float mag_x,
                        float mag_y, float mag_z, float mag_w, float ewaldradiussuper,
                        int outputdecentered, int squareinterpweights, unsigned batch,
                        void* stream) {
  clear_error();
  return backproject_launch(d_volumeft, d_volumeweights, vx, vy, vz, d_projft, d_projweights, px,
                            py, pz, rmax, d_matrices, d_ivolume,
                            make_float4(mag_x, mag_y, mag_z, mag_w), ewaldradiussuper,
                            outputdecentered, squareinterpweights, batch, (cudaStream_t)stream);
}

int gtomrln_backproject_angles(float* d_volumeft, float* d_volumeweights, int vx, int vy, int vz,
                               const float* d_projft, const float* d_projweights, int px, int py,
                               int pz, unsigned rmax, const float* h_angles, const int* h_ivolume,
                               float mag_x, float mag_y, float mag_z, float mag_w,
                               float ewaldradius, float supersample, int outputdecentered,
                               int squareinterpweights, unsigned batch, void* stream) {
  clear_error();
  cudaStream_t s = (cudaStream_t)stream;
  return with_device_matrices(h_angles, supersample, batch, s, [&](const float* d_m) -> int {
    int* d_iv = nullptr;
    if (h_ivolume && batch) {
      int st = pool_alloc((void**)&d_iv, sizeof(int) * (size_t)batch, s);
      if (st) return st;
      cudaError_t e =
          cudaMemcpyAsync(d_iv, h_ivolume, sizeof(int) * (size_t)batch, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) {
        pool_free(d_iv, s);
        return set_error(GTOMRLN_ERR_CUDA, "ivolume upload failed: %s", cudaGetErrorString(e));
      }
    }
    int hint = 0;
    if (h_ivolume && batch) hint = *std::max_element(h_ivolume, h_ivolume + batch) + 1;
    int st = backproject_launch(d_volumeft, d_volumeweights, vx, vy, vz, d_projft, d_projweights,
                                px, py, pz, rmax, d_m, d_iv, make_float4(mag_x, mag_y, mag_z, mag_w),
                                ewaldradius * supersample, outputdecentered, squareinterpweights,
                                batch, s, hint);
    int st2 = pool_free(d_iv, s);
    return st ? st : st2;
  });
}

// ---------------------------------------------------------------- shifted --
int gtomrln_backproject_shifted(float* d_volumeft, float* d_volumeweights, int vx, int vy, int vz,
                                const float* d_projft, const float* d_projweights, int px, int py,
                                int pz, unsigned rmax, const float* d_matrices,
                                const float* d_shifts, const float* d_globalweights,
                                unsigned batch, void* stream) {
  clear_error();
  int ndv = dimension_count(vx, vy, vz), ndp = dimension_count(px, py, pz);
  if (ndv < ndp || ndv != 3)
    return set_error(GTOMRLN_ERR_INVALID,
                     "backproject_shifted: volume must be 3D and have at least the projections' "
                     "dimensions (reference throws)");
  if (ndp != 2 && ndp != 3)
    return set_error(GTOMRLN_ERR_INVALID, "backproject_shifted: projections must be 2D or 3D");
  if (vx <= 0 || px <= 0) return set_error(GTOMRLN_ERR_INVALID, "backproject_shifted: non-positive dimension");
  if (batch == 0) return GTOMRLN_OK;
  if (!d_matrices || !d_shifts || !d_globalweights)
    return set_error(GTOMRLN_ERR_INVALID, "backproject_shifted: NULL matrices, shifts or weights");
  if (rmax > (unsigned)(px / 2)) rmax = px / 2;
  BpArgs a;
  a.n = px;
  a.dimft = px / 2 + 1;
  a.area = (int64_t)a.dimft * px;
  a.elements = ndp == 3 ? a.area * px : a.area;
  a.tiles = (int)((a.elements + kBpTile - 1) / kBpTile);
  a.rmax2 = (int)(rmax * rmax);
  a.P = vx;
  a.rowlen = vx / 2 + 1;
  a.nvox = (int64_t)a.rowlen * vx * vx;
  a.mag = make_float4(1.f, 0.f, 0.f, 1.f);
  a.ewalddiaminv = 0.f;
  if ((int64_t)a.tiles * batch > 0x7fffffffLL)
    return set_error(GTOMRLN_ERR_INVALID, "backproject_shifted: batch too large for one launch");
  const int choice = path_choice(GTOMRLN_OP_BACKPROJECT);
  if (ndp == 2 && vx == vy && vx == vz && vx >= 4 && a.rmax2 <= (1 << 24) && (d_volumeft || d_volumeweights) &&
      (choice == GTOMRLN_PATH_BRICK || choice == GTOMRLN_PATH_SEGMENT ||
       (choice == GTOMRLN_PATH_AUTO && brick_path_pays(GTOMRLN_OP_BACKPROJECT, vx, batch))))
    return backproject_shifted_brick(d_volumeft, d_volumeweights, d_projft, d_projweights, d_matrices, d_shifts,
                                     d_globalweights, a, (int)rmax, batch, (cudaStream_t)stream);
  dim3 grid((unsigned)(a.tiles * (int64_t)batch));
  if (ndp == 2)
    backproject_shifted_kernel<2><<<grid, kBpThreads, 0, (cudaStream_t)stream>>>(
        (float2*)d_volumeft, d_volumeweights, (const float2*)d_projft, d_projweights, d_matrices, d_shifts,
        d_globalweights, a, (int)rmax);
  else
    backproject_shifted_kernel<3><<<grid, kBpThreads, 0, (cudaStream_t)stream>>>(
        (float2*)d_volumeft, d_volumeweights, (const float2*)d_projft, d_projweights, d_matrices, d_shifts,
        d_globalweights, a, (int)rmax);
  GTOMRLN_LAUNCH_CHECK("backproject_shifted_kernel");
  return GTOMRLN_OK;
}

int gtomrln_backproject_shifted_angles(float* d_volumeft, float* d_volumeweights, int vx, int vy,
                                       int vz, const float* d_projft, const float* d_projweights,
                                       int px, int py, int pz, unsigned rmax, const float* h_angles,
                                       const float* h_shifts, const float* h_globalweights,
                                       float supersample, unsigned batch, void* stream) {
  clear_error();
  return with_device_shifted(h_angles, h_shifts, h_globalweights, supersample, px, batch,
                             (cudaStream_t)stream,
                             [&](const float* d_m, const float* d_s, const float* d_w) {
                               return gtomrln_backproject_shifted(d_volumeft, d_volumeweights, vx, vy, vz,
                                                                  d_projft, d_projweights, px, py, pz, rmax,
                                                                  d_m, d_s, d_w, batch, stream);
                             });
}

}  // extern "C"
