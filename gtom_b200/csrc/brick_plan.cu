// Binning plan for the brick-major kernels (see brick.cuh), built entirely
// on the device so that a call never synchronises with the host.
//
//   bin_slices_kernel   one CTA per slice: brick(s) of every pixel, a
//                       shared-memory histogram over bricks, the slice's bins
//                       and its pixel ids sorted by brick;
//   segment_pairs_kernel  (segment plan, instead of the above) one CTA per
//                       slice: the bricks its plane crosses, as bins
//                       without pixel lists;
//   pairs_scan_kernel   one CTA: per-brick bin offsets and work items, bricks
//                       in order of increasing distance from the origin so
//                       that the heaviest items start first;
//   pairs_fill_kernel   groups the bins by brick;
//   plan_items_kernel   writes the work items.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>

#include "brick.cuh"
#include "sample.cuh"
#include "segment.cuh"

namespace gtomrln {

constexpr int kBinThreads = 512;
constexpr int kMaxBinsPerSlice = 2048;  // bins reserved per slice on average

__device__ __forceinline__ bool in_pixel_set(const PixelSet& px, int u, int v) {
  int r2 = u * u + v * v;
  if (px.strict) return r2 < px.rmax2 && !(u == 0 && v < 0);
  return r2 <= px.rmax2;
}

// Brick indices along each axis spanned by the 2x2x2 voxel cube with lowest
// corner (x, y, z) (index 1 equals index 0 when the cube does not cross a
// brick face).
struct CubeBricks {
  int bx0, bx1, by0, by1, bz0, bz1;
};

__device__ __forceinline__ bool cube_bricks(const BrickGrid& g, int x, int y, int z, CubeBricks& c) {
  int dy = y - g.ylo, dz = z - g.zlo;
  if (x < 0 || dy < 0 || dz < 0) return false;
  const float inv = 1.f / (float)g.B;
  c.bx0 = div_brick(x, g.B, inv);
  c.bx1 = div_brick(x + 1, g.B, inv);
  c.by0 = div_brick(dy, g.B, inv);
  c.by1 = div_brick(dy + 1, g.B, inv);
  c.bz0 = div_brick(dz, g.B, inv);
  c.bz1 = div_brick(dz + 1, g.B, inv);
  return c.bx1 < g.nbx && c.by1 < g.nby && c.bz1 < g.nbz;
}

__device__ __forceinline__ bool cube_has(const CubeBricks& c, int bx, int by, int bz) {
  return (bx == c.bx0 || bx == c.bx1) && (by == c.by0 || by == c.by1) && (bz == c.bz0 || bz == c.bz1);
}

__device__ __forceinline__ bool cube_single(const CubeBricks& c) {
  return c.bx0 == c.bx1 && c.by0 == c.by1 && c.bz0 == c.bz1;
}

// f(b) for every brick of cube c, each once, skipping those of `skip`.
template <class F>
__device__ __forceinline__ void for_each_cube_brick(const BrickGrid& g, const CubeBricks& c,
                                                    const CubeBricks* skip, F&& f) {
#pragma unroll
  for (int iz = 0; iz < 2; iz++) {
    int bz = iz ? c.bz1 : c.bz0;
    if (iz && bz == c.bz0) continue;
#pragma unroll
    for (int iy = 0; iy < 2; iy++) {
      int by = iy ? c.by1 : c.by0;
      if (iy && by == c.by0) continue;
#pragma unroll
      for (int ix = 0; ix < 2; ix++) {
        int bx = ix ? c.bx1 : c.bx0;
        if (ix && bx == c.bx0) continue;
        if (skip && cube_has(*skip, bx, by, bz)) continue;
        f((bz * g.nby + by) * g.nbx + bx);
      }
    }
  }
}

// f(b, interior) for every brick pixel (u, v) of a slice with matrix m reads
// from (the projector: the brick of its base voxel) or adds to (the
// backprojector: the bricks of its target cube — for x0 >= 1 the cube at
// (x0, y0, z0), for x0 <= -2 the mirrored cube at (-x0-1, -y0-1, -z0-1), and
// near x = 0 both cubes with x in {0, 1}, which hold every direct, mirrored
// and second-plane target), each brick once.  interior: the pixel's whole
// single cube lies in that brick.  Returns false if a voxel falls outside
// the grid (the slice must then take the direct path).  A brick may receive
// a pixel none of whose targets it holds; the brick kernel adds only its own.
template <int OP, class F>
__device__ __forceinline__ bool pixel_bricks(const float* m, int u, int v, const BrickGrid& g, F&& f) {
  if (OP == GTOMRLN_OP_PROJECT) {
    ProjSample s = project_sample(m, u, v, 0);
    int b = brick_of(g, s.x0, s.y0, s.z0);
    if (b < 0) return false;
    f(b, true);
    return true;
  } else {
    BpSample s = backproject_sample(m, (float)u, (float)v, 0.f);
    CubeBricks c1, c2;
    if (s.x0 >= 1 || s.x0 <= -2) {
      bool ok = s.x0 >= 1 ? cube_bricks(g, s.x0, s.y0, s.z0, c1)
                          : cube_bricks(g, -s.x0 - 1, -s.y0 - 1, -s.z0 - 1, c1);
      if (!ok) return false;
      const bool single = cube_single(c1);
      for_each_cube_brick(g, c1, nullptr, [&](int b) { f(b, single); });
    } else {
      if (!cube_bricks(g, 0, s.y0, s.z0, c1) || !cube_bricks(g, 0, -s.y0 - 1, -s.z0 - 1, c2)) return false;
      for_each_cube_brick(g, c1, nullptr, [&](int b) { f(b, false); });
      for_each_cube_brick(g, c2, &c1, [&](int b) { f(b, false); });
    }
    return true;
  }
}

// Visits the slice's pixel set row by row (one warp per row, lanes along
// the row), so that no pixel id needs a division.
template <class F>
__device__ __forceinline__ void for_each_set_pixel(const PixelSet& px, F&& f) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int idy = warp; idy < px.n; idy += nw) {
    int v = idy <= px.n / 2 ? idy : idy - px.n;
    int rem = (px.strict ? px.rmax2 - 1 : px.rmax2) - v * v;
    if (rem < 0) continue;
    int umax = (int)sqrtf((float)rem);
    umax -= umax * umax > rem;
    umax += (umax + 1) * (umax + 1) <= rem;
    int u0 = (px.strict && v < 0) ? 1 : 0;
    for (int u = u0 + lane; u <= umax && u < px.dimft; u += 32) f(idy * px.dimft + u, u, v);
  }
}

template <int OP>
__global__ void __launch_bounds__(kBinThreads)
bin_slices_kernel(const float* __restrict__ mats, BrickGrid g, PixelSet px, float limit,
                  int* __restrict__ entries, int64_t entries_cap, PixelBin* __restrict__ bins,
                  int64_t bins_cap, unsigned long long* __restrict__ counters,
                  int* __restrict__ brick_pairs, int* __restrict__ fallback, int* __restrict__ nfallback,
                  int use_codes) {
  extern __shared__ int hist[];  // interior counts [nbricks], then boundary counts [nbricks]
  int* hist_b = hist + g.nbricks;
  // With use_codes, one 16-bit code per pixel id after the histograms: the
  // pixel's brick + 1 when it has exactly one brick and lies inside it
  // (every projector pixel, most backprojector pixels), else 0; the placing
  // pass then skips the sample evaluation for coded pixels.
  unsigned short* codes = reinterpret_cast<unsigned short*>(hist + 2 * g.nbricks);
  __shared__ int s_bad, s_sum[kBinThreads / 32], s_nz[kBinThreads / 32];
  __shared__ long long s_base_e, s_base_b;
  const int slice = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float m[9];
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)slice + k);
  if (!(plane_scale(m) * px.pmax < limit)) {  // uniform over the block
    if (tid == 0) fallback[atomicAdd(nfallback, 1)] = slice;
    return;
  }
  for (int b = tid; b < 2 * g.nbricks; b += kBinThreads) hist[b] = 0;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for_each_set_pixel(px, [&](int id, int u, int v) {
    int nb = 0, first = 0;
    bool first_in = false;
    bool ok = pixel_bricks<OP>(m, u, v, g, [&](int b, bool in) {
      atomicAdd(in ? &hist[b] : &hist_b[b], 1);
      if (nb++ == 0) {
        first = b;
        first_in = in;
      }
    });
    if (!ok) s_bad = 1;
    if (use_codes) codes[id] = (ok && nb == 1 && first_in) ? (unsigned short)(first + 1) : (unsigned short)0;
  });
  __syncthreads();
  if (s_bad) {
    if (tid == 0) fallback[atomicAdd(nfallback, 1)] = slice;
    return;
  }
  // Each thread owns a contiguous run of bricks: sum its counts and nonzero
  // bins, scan those over the block, then turn counts into offsets.
  const int per = (g.nbricks + kBinThreads - 1) / kBinThreads;
  const int b0 = min(tid * per, g.nbricks), b1 = min(b0 + per, g.nbricks);
  int sum = 0, nz = 0;
  for (int b = b0; b < b1; b++) {
    int c = hist[b] + hist_b[b];
    sum += c;
    nz += c > 0;
  }
  int isum = sum, inz = nz;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int a = __shfl_up_sync(0xffffffffu, isum, o), c = __shfl_up_sync(0xffffffffu, inz, o);
    if (lane >= o) {
      isum += a;
      inz += c;
    }
  }
  if (lane == 31) {
    s_sum[warp] = isum;
    s_nz[warp] = inz;
  }
  __syncthreads();
  int wsum = 0, wnz = 0, tsum = 0, tnz = 0;
  for (int w = 0; w < kBinThreads / 32; w++) {
    if (w < warp) {
      wsum += s_sum[w];
      wnz += s_nz[w];
    }
    tsum += s_sum[w];
    tnz += s_nz[w];
  }
  if (tid == 0) {
    s_base_e = (long long)atomicAdd(counters + 0, (unsigned long long)tsum);
    s_base_b = (long long)atomicAdd(counters + 1, (unsigned long long)tnz);
  }
  __syncthreads();
  if (s_base_e + tsum > entries_cap || s_base_b + tnz > bins_cap) {  // out of room: direct path
    for (long long k = s_base_b + tid; k < s_base_b + tnz && k < bins_cap; k += kBinThreads)
      bins[k].brick = -1;  // reserved but empty
    if (tid == 0) fallback[atomicAdd(nfallback, 1)] = slice;
    return;
  }
  int off = wsum + isum - sum, bi = wnz + inz - nz;
  for (int b = b0; b < b1; b++) {
    int ci = hist[b], cb = hist_b[b];
    hist[b] = off;  // next interior slot
    hist_b[b] = off + ci;  // next boundary slot
    if (ci + cb > 0) {
      bins[s_base_b + bi] = {slice, (int)(s_base_e + off), ci + cb, b, ci, 0, 0, 0};
      atomicAdd(brick_pairs + b, 1);
      bi++;
    }
    off += ci + cb;
  }
  __syncthreads();
  for_each_set_pixel(px, [&](int id, int u, int v) {
    const unsigned c = use_codes ? codes[id] : 0u;
    if (c) {
      entries[s_base_e + atomicAdd(&hist[c - 1], 1)] = id;
      return;
    }
    pixel_bricks<OP>(m, u, v, g, [&](int b, bool in) {
      entries[s_base_e + atomicAdd(in ? &hist[b] : &hist_b[b], 1)] = id;
    });
  });
}

// Segment plan: one CTA per slice lists the bricks whose box, widened by
// `below` voxels on the low side and by the segment margin, meets the
// slice's plane within the radius its samples reach.  Each becomes a bin
// without entries; the brick kernel finds the pixels by row segments
// (segment.cuh).  Positions of a slice lie on the plane through the origin
// spanned by the first two (magnified) matrix columns and within
// plane_scale * pmax of the origin, mirrored positions too, so the list
// covers every brick a pixel of the slice (or its mirror) can reach; with
// the Ewald curvature the samples leave the plane by at most its reach,
// which widens every box.  With per-slice volumes a pair's key is
// volume * nbricks + brick; a slice whose volume index is outside
// [0, nvol) takes the direct path.
constexpr int kPairThreads = 256;
__global__ void __launch_bounds__(kPairThreads)
segment_pairs_kernel(const float* __restrict__ mats, BrickGrid g, float pmax, float limit, float below,
                     PixelBin* __restrict__ bins, int64_t bins_cap, unsigned long long* __restrict__ counters,
                     int* __restrict__ brick_pairs, int* __restrict__ fallback, int* __restrict__ nfallback,
                     float2* __restrict__ zero_out, PixelSet zpx, SliceGeom gm) {
  extern __shared__ int hits[];  // brick ids of this slice, then a bitmap of the bricks
  __shared__ int s_n;
  __shared__ int s_wsum[kPairThreads / 32];
  __shared__ long long s_base;
  const int slice = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
  float m0[9], m[9];
#pragma unroll
  for (int k = 0; k < 9; k++) m0[k] = __ldg(mats + 9 * (int64_t)slice + k);
  effective_matrix(m0, gm, m);
  // Samples kept lie within R of the origin: |q| <= qmax in the plane of the
  // matrix's first two columns, plus the curvature's reach along the third.
  const float widen = curvature_reach(m0, gm, pmax);
  const float R = plane_scale(m0) * (gm.qmax < 0.f ? pmax : gm.qmax) + widen;
  const int vol = gm.ivolume ? __ldg(gm.ivolume + slice) : 0;
  if (!(R < limit) || vol < 0 || vol >= gm.nvol) {  // uniform over the block
    if (tid == 0) fallback[atomicAdd(nfallback, 1)] = slice;
    return;
  }
  if (zero_out) {
    // the projector's zeros outside rmax (Project.cu:111-115): in each row
    // the tail x > sqrt(rmax^2 - y^2), one warp per row (slices taking the
    // direct path write their own zeros)
    float2* out = zero_out + zpx.elements * slice;
    for (int idy = tid >> 5; idy < zpx.n; idy += kPairThreads / 32) {
      const int v = idy <= zpx.n / 2 ? idy : idy - zpx.n;
      const int rem = zpx.rmax2 - v * v;
      const int x0 = rem >= 0 ? seg_isqrt(rem) + 1 : 0;
      for (int x = x0 + lane; x < zpx.dimft; x += 32) out[(int64_t)idy * zpx.dimft + x] = make_float2(0.f, 0.f);
    }
  }
  if (tid == 0) s_n = 0;
  __syncthreads();
  const float n0 = m[1] * m[5] - m[2] * m[4], n1 = m[2] * m[3] - m[0] * m[5], n2 = m[0] * m[4] - m[1] * m[3];
  const float R2 = R * R * (1.f + 1e-5f) + 1e-3f;
  const float lo_pad = below + widen + kSegMargin, hi_pad = (float)g.B + widen + kSegMargin;
  // The exact test of brick b: its widened box meets the slice's plane and
  // the sphere of radius R.
  auto crosses = [&](int b) {
    const int3 o = brick_origin(g, b);
    const float lo0 = o.x - lo_pad, lo1 = o.y - lo_pad, lo2 = o.z - lo_pad;
    const float hi0 = o.x + hi_pad, hi1 = o.y + hi_pad, hi2 = o.z + hi_pad;
    const float c0 = 0.5f * (lo0 + hi0), c1 = 0.5f * (lo1 + hi1), c2 = 0.5f * (lo2 + hi2);
    const float h0 = 0.5f * (hi0 - lo0), h1 = 0.5f * (hi1 - lo1), h2 = 0.5f * (hi2 - lo2);
    const float dist = fabsf(n0 * c0 + n1 * c1 + n2 * c2);
    const float reach = fabsf(n0) * h0 + fabsf(n1) * h1 + fabsf(n2) * h2;
    const float eps = 1e-5f * (fabsf(n0) * (fabsf(c0) + h0) + fabsf(n1) * (fabsf(c1) + h1) +
                               fabsf(n2) * (fabsf(c2) + h2));
    const float d0 = fmaxf(0.f, fmaxf(lo0, -hi0)), d1 = fmaxf(0.f, fmaxf(lo1, -hi1)),
                d2 = fmaxf(0.f, fmaxf(lo2, -hi2));
    return dist <= reach + eps && d0 * d0 + d1 * d1 + d2 * d2 <= R2;
  };
  // Candidates: along the axis k where the normal is largest, a column of
  // bricks (fixed indices on the other two axes) meets the plane only where
  // the centre's k coordinate is within (reach + eps) / |n_k| of the plane's
  // over the column; that range, widened well beyond the float error of the
  // test, is searched with the exact test, so the hits are the ones testing
  // every brick finds (in another order).  A zero or non-finite normal tests
  // every brick.
  const float an0 = fabsf(n0), an1 = fabsf(n1), an2 = fabsf(n2);
  const int k = an0 >= an1 && an0 >= an2 ? 0 : (an1 >= an2 ? 1 : 2);
  const float ank = k == 0 ? an0 : (k == 1 ? an1 : an2);
  const bool columns = ank > 1e-30f && isfinite(n0) && isfinite(n1) && isfinite(n2) && isfinite(R2);
  if (columns) {
    // hits marked in a bitmap, then listed in brick order (pairs_fill_kernel's
    // per-brick atomics from consecutive bins then fall on neighbouring words)
    unsigned* bits = reinterpret_cast<unsigned*>(hits + g.nbricks);
    const int nwords = (g.nbricks + 31) / 32;
    for (int w = tid; w < nwords; w += kPairThreads) bits[w] = 0u;
    __syncthreads();
    const int nb[3] = {g.nbx, g.nby, g.nbz};
    const float base[3] = {0.f, (float)g.ylo, (float)g.zlo};
    const float nv[3] = {n0, n1, n2};
    const int i = k == 0 ? 1 : 0, j = k == 2 ? 1 : 2;  // the other two axes
    const float d = 0.5f * (hi_pad - lo_pad), h = 0.5f * (hi_pad + lo_pad);
    const float reach = (an0 + an1 + an2) * h;
    // |c| <= extent of the grid on every axis: a bound on the test's eps
    const float cmax = fmaxf(fmaxf((float)(g.nbx * g.B), fabsf(base[1])), fabsf(base[2])) +
                       (float)(g.nby > g.nbz ? g.nby : g.nbz) * (float)g.B + h;
    const float slack = reach + 1e-5f * (an0 + an1 + an2) * (cmax + h);
    const float invB = 1.f / (float)g.B;
    const int ncol = nb[i] * nb[j];
    for (int col = tid; col < ncol; col += kPairThreads) {
      const int a = col % nb[i], bj = col / nb[i];
      const float ci = base[i] + (float)(a * g.B) + d, cj = base[j] + (float)(bj * g.B) + d;
      const float sp = nv[i] * ci + nv[j] * cj;
      // centre k coordinate c with |n_k c + sp| <= slack
      const float mid = -sp / nv[k], half = slack / ank;
      const float margin = 1e-3f * (fabsf(mid) + half) + 0.01f * (float)g.B;
      float flo = (mid - half - margin - base[k] - d) * invB;
      float fhi = (mid + half + margin - base[k] - d) * invB;
      if (!(flo <= fhi)) continue;
      flo = fminf(fmaxf(flo, -1.f), (float)nb[k]);
      fhi = fminf(fmaxf(fhi, -1.f), (float)nb[k]);
      const int l0 = max(0, (int)floorf(flo)), l1 = min(nb[k] - 1, (int)ceilf(fhi));
      for (int l = l0; l <= l1; l++) {
        int idx[3];
        idx[k] = l;
        idx[i] = a;
        idx[j] = bj;
        const int b = idx[0] + g.nbx * (idx[1] + g.nby * idx[2]);
        if (crosses(b)) atomicOr(bits + (b >> 5), 1u << (b & 31));
      }
    }
    __syncthreads();
    // thread t lists the set bits of words [t W, (t+1) W) at its offset in a
    // block-wide scan of the words' counts
    const int W = (nwords + kPairThreads - 1) / kPairThreads;
    const int w0 = min(tid * W, nwords), w1 = min(w0 + W, nwords);
    int cnt = 0;
    for (int w = w0; w < w1; w++) cnt += __popc(bits[w]);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t2 = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t2;
    }
    if (lane == 31) s_wsum[tid >> 5] = incl;
    __syncthreads();
    int pos = incl - cnt;
    for (int k2 = 0; k2 < (tid >> 5); k2++) pos += s_wsum[k2];
    for (int w = w0; w < w1; w++) {
      unsigned m = bits[w];
      while (m) {
        hits[pos++] = 32 * w + __ffs(m) - 1;
        m &= m - 1u;
      }
    }
    if (tid == kPairThreads - 1) s_n = pos;
  } else {
    for (int base = 0; base < g.nbricks; base += kPairThreads) {
      const int b = base + tid;
      const bool hit = b < g.nbricks && crosses(b);
      const unsigned mask = __ballot_sync(0xffffffffu, hit);
      int wbase = 0;
      if (lane == 0 && mask) wbase = atomicAdd(&s_n, __popc(mask));
      wbase = __shfl_sync(0xffffffffu, wbase, 0);
      if (hit) hits[wbase + __popc(mask & ((1u << lane) - 1u))] = b;
    }
  }
  __syncthreads();
  const int nh = s_n;
  if (tid == 0) s_base = (long long)atomicAdd(counters + 1, (unsigned long long)nh);
  __syncthreads();
  if (s_base + nh > bins_cap) {  // out of room: direct path
    for (long long k = s_base + tid; k < s_base + nh && k < bins_cap; k += kPairThreads) bins[k].brick = -1;
    if (tid == 0) fallback[atomicAdd(nfallback, 1)] = slice;
    return;
  }
  // Each pair carries the row range of its two sides (the brick's box as the
  // brick kernels build it: widened by `below` on the low side, by the
  // curvature's reach and the margin on all), so that the kernels neither
  // recompute it per warp nor walk a side with no pixels.
  for (int k = tid; k < nh; k += kPairThreads) {
    const int local = hits[k];
    const int3 o = brick_origin(g, local);
    int rows[2];
#pragma unroll
    for (int side = 0; side < 2; side++) {
      const SegBox box = seg_box(m, side, o, g.B, below, widen);
      int vlo, vhi;
      rows[side] = seg_rows(box, zpx, vlo, vhi) ? seg_pack_rows(vlo, vhi) : kSegNoRows;
    }
    const int b = vol * g.nbricks + local;
    bins[s_base + k] = {slice, rows[0], rows[1], b, 0, 0, 0, 0};
    atomicAdd(brick_pairs + b, 1);
  }
}

// Single block.  Bricks are visited in `order` (increasing distance from the
// origin); writes bin-list offsets, per-brick item offsets and the item count.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads)
pairs_scan_kernel(const int* __restrict__ counts, const int* __restrict__ order, int nbricks, int nvol, int chunk,
                  int* __restrict__ offsets, int* __restrict__ item_off, int* __restrict__ cursor,
                  int* __restrict__ nitems) {
  __shared__ int s_c[kScanThreads], s_i[kScanThreads];
  __shared__ int carry_c, carry_i;
  if (threadIdx.x == 0) carry_c = carry_i = 0;
  __syncthreads();
  // keys volume * nbricks + brick, the volumes interleaved brick by brick so
  // that every volume's central bricks start first
  const int nkeys = nbricks * nvol;
  for (int base = 0; base < nkeys; base += kScanThreads) {
    int t = base + threadIdx.x;
    int b = t < nkeys ? (t % nvol) * nbricks + order[t / nvol] : -1;
    int c = b >= 0 ? counts[b] : 0;
    int ni = (c + chunk - 1) / chunk;
    s_c[threadIdx.x] = c;
    s_i[threadIdx.x] = ni;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {  // inclusive Hillis-Steele scan
      int vc = threadIdx.x >= o ? s_c[threadIdx.x - o] : 0;
      int vi = threadIdx.x >= o ? s_i[threadIdx.x - o] : 0;
      __syncthreads();
      s_c[threadIdx.x] += vc;
      s_i[threadIdx.x] += vi;
      __syncthreads();
    }
    if (b >= 0) {
      offsets[b] = carry_c + s_c[threadIdx.x] - c;
      item_off[b] = carry_i + s_i[threadIdx.x] - ni;
      cursor[b] = 0;
    }
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) {
      carry_c += s_c[threadIdx.x];
      carry_i += s_i[threadIdx.x];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *nitems = carry_i;
}

// Groups the bins by brick: pairs[offsets[b] ..] lists the bins of brick (or
// volume-brick key) b.
__global__ void pairs_fill_kernel(const PixelBin* __restrict__ bins,
                                  const unsigned long long* __restrict__ counters, int64_t bins_cap,
                                  const int* __restrict__ counts, const int* __restrict__ offsets,
                                  int* __restrict__ cursor, int* __restrict__ pairs) {
  int64_t nb = (int64_t)min(counters[1], (unsigned long long)bins_cap);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb;
       i += (int64_t)gridDim.x * blockDim.x) {
    int b = bins[i].brick;
    if (b < 0) continue;  // reserved by a slice that fell back
    int s = atomicAdd(cursor + b, 1);
    if (s < counts[b]) pairs[offsets[b] + s] = (int)i;
  }
}

__global__ void plan_items_kernel(const int* __restrict__ counts, const int* __restrict__ offsets,
                                  const int* __restrict__ item_off, int nbricks, int chunk,
                                  BrickItem* __restrict__ items) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbricks) return;
  int c = counts[b];
  if (!c) return;
  int nch = (c + chunk - 1) / chunk;
  for (int k = 0; k < nch; k++)
    items[item_off[b] + k] = {b, offsets[b] + k * chunk, min(chunk, c - k * chunk), nch == 1 ? 1 : 0};
}

// Brick visiting order per grid, cached per device and context.
static std::mutex g_order_mutex;
static std::map<std::tuple<int, unsigned long long, int, int, int, int, int>, int*> g_orders;

// Frees the orders of the current context on device dev and forgets those of
// earlier contexts there (gone with their context).
int release_brick_orders(int dev, unsigned long long ctx) {
  std::lock_guard<std::mutex> lock(g_order_mutex);
  for (auto it = g_orders.begin(); it != g_orders.end();) {
    if (std::get<0>(it->first) != dev) {
      ++it;
      continue;
    }
    if (std::get<1>(it->first) == ctx) cudaFree(it->second);
    it = g_orders.erase(it);
  }
  return GTOMRLN_OK;
}

static int brick_order(const BrickGrid& g, const int** out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  auto key = std::make_tuple(dev, ctx, g.V, g.B, g.nbx, g.nby, g.ylo);
  std::lock_guard<std::mutex> lock(g_order_mutex);
  auto it = g_orders.find(key);
  if (it != g_orders.end()) {
    *out = it->second;
    return GTOMRLN_OK;
  }
  std::vector<int> order(g.nbricks);
  std::vector<float> d2(g.nbricks);
  for (int b = 0; b < g.nbricks; b++) {
    int3 o = brick_origin(g, b);
    float cx = o.x + 0.5f * (g.B - 1), cy = o.y + 0.5f * (g.B - 1), cz = o.z + 0.5f * (g.B - 1);
    d2[b] = cx * cx + cy * cy + cz * cz;
  }
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d2[a] < d2[b]; });
  int* d = nullptr;
  GTOMRLN_CUDA_TRY(cudaMalloc(&d, sizeof(int) * order.size()));
  GTOMRLN_CUDA_TRY(cudaMemcpy(d, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
  g_orders[key] = d;
  *out = d;
  return GTOMRLN_OK;
}

int build_brick_plan(int op, const float* d_mats, int batch, const BrickGrid& g, const PixelSet& px,
                     float limit, int chunk, cudaStream_t stream, BrickPlan* plan, int segments,
                     void* zero_out, const SliceGeom& geom) {
  plan->g = g;
  plan->nvol = geom.nvol;
  plan->batch = batch;
  if (geom.nvol < 1 || (!segments && (geom.nvol != 1 || geom.curve != 0.f || geom.mag.x != 1.f ||
                                      geom.mag.y != 0.f || geom.mag.z != 0.f || geom.mag.w != 1.f)))
    return set_error(GTOMRLN_ERR_INVALID, "brick plan: the binning plan takes plain slices of one volume only");
  size_t hist_bytes = 2 * sizeof(int) * (size_t)g.nbricks;
  if (hist_bytes > 200 * 1024)
    return set_error(GTOMRLN_ERR_INVALID, "brick grid of %d bricks too fine for the binning plan", g.nbricks);
  // The per-pixel brick codes join the histograms when they fit (2 bytes per
  // pixel id of a slice: 66 KB at n = 256).
  const size_t code_bytes = ((size_t)px.elements * 2 + 3) & ~(size_t)3;
  const int use_codes = g.nbricks < 65535 && hist_bytes + code_bytes <= 200 * 1024 ? 1 : 0;
  // segment plan: the hit list and a bitmap of the bricks
  const size_t smem_bytes = segments ? sizeof(int) * ((size_t)g.nbricks + ((size_t)g.nbricks + 31) / 32)
                                     : hist_bytes + (use_codes ? code_bytes : 0);
  const int* d_order = nullptr;
  int st = brick_order(g, &d_order);
  if (st) return st;
  // Capacities: the projector bins each pixel once; the backprojector's
  // pixels land in ~1.2-1.5 bricks on average (8 at most), so twice the
  // pixel count is reserved.  A slice that does not fit takes the direct path.
  int64_t npix = 0;
  for (int idy = 0; idy < px.n; idy++) {
    int v = idy <= px.n / 2 ? idy : idy - px.n;
    for (int u = 0; u < px.dimft; u++) {
      int r2 = u * u + v * v;
      npix += px.strict ? (r2 < px.rmax2 && !(u == 0 && v < 0)) : (r2 <= px.rmax2);
    }
  }
  int64_t entries_cap =
      segments ? 1 : std::max<int64_t>(1, (int64_t)batch * npix * (op == GTOMRLN_OP_PROJECT ? 1 : 2));
  int per_slice = std::min(g.nbricks, kMaxBinsPerSlice);
  if (segments) {
    // A crossed brick's centre lies within h = sqrt(3)/2 * B' (B' the widened
    // edge) of the plane and within limit + h of the origin: about
    // pi (limit + h)^2 * 2h / B^3 lattice points per slice; half as much
    // again is reserved (the cap is an average over the batch).
    const double Bw = g.B + (op == GTOMRLN_OP_PROJECT ? 0.0 : 1.0) + 2.0 * kSegMargin;
    const double h = 0.8660254037844386 * Bw, R = (double)limit + h;
    const double est = 3.141592653589793 * R * R * 2.0 * h / ((double)g.B * g.B * g.B);
    per_slice = (int)std::min<double>(g.nbricks, 1.5 * est + 64.0);
  }
  int64_t bins_cap = std::max<int64_t>(1, (int64_t)batch * per_slice);
  if (entries_cap > 0x7fffffffLL || bins_cap > 0x7fffffffLL)
    return set_error(GTOMRLN_ERR_INVALID, "brick plan too large for one call; split the batch");
  const int64_t nkeys = (int64_t)g.nbricks * geom.nvol;  // work-item keys: volume * nbricks + brick
  if (nkeys > 0x7fffffffLL) return set_error(GTOMRLN_ERR_INVALID, "brick plan: too many volumes");
  int64_t cap_items = nkeys + bins_cap / chunk + 1;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t nb = (size_t)nkeys;
  size_t o_counts = 0;
  size_t o_offsets = o_counts + al(nb * 4);
  size_t o_itemoff = o_offsets + al(nb * 4);
  size_t o_cursor = o_itemoff + al(nb * 4);
  size_t o_misc = o_cursor + al(nb * 4);  // counters (2 x u64), work counter, nitems, nfallback
  size_t o_fallback = o_misc + 256;
  size_t o_items = o_fallback + al((size_t)std::max(batch, 1) * 4);
  size_t o_bins = o_items + al((size_t)cap_items * sizeof(BrickItem));
  size_t o_pairs = o_bins + al((size_t)bins_cap * sizeof(PixelBin));
  size_t o_entries = o_pairs + al((size_t)bins_cap * 4);
  size_t bytes = o_entries + al((size_t)entries_cap * 4);
  char* base = nullptr;
  st = scratch_alloc((void**)&base, bytes, stream);
  if (st) return st;
  plan->scratch = base;
  int* counts = (int*)(base + o_counts);
  int* offsets = (int*)(base + o_offsets);
  int* item_off = (int*)(base + o_itemoff);
  int* cursor = (int*)(base + o_cursor);
  unsigned long long* counters = (unsigned long long*)(base + o_misc);
  plan->counter = (int*)(base + o_misc + 16);
  plan->nitems = (int*)(base + o_misc + 20);
  plan->nfallback = (int*)(base + o_misc + 24);
  plan->fallback = (int*)(base + o_fallback);
  plan->items = (BrickItem*)(base + o_items);
  plan->bins = (PixelBin*)(base + o_bins);
  plan->pairs = (int*)(base + o_pairs);
  plan->entries = (int*)(base + o_entries);
  plan->max_items = (int)std::min<int64_t>(cap_items, 0x7fffffff);

  cudaError_t e = cudaMemsetAsync(counts, 0, nb * 4, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + o_misc, 0, 256, stream);
  if (e == cudaSuccess && batch > 0) {
    if (segments) {
      // The projector's samples reach the brick of their base voxel, the
      // backprojector's also the bricks of the voxel above it on each axis.
      const float below = op == GTOMRLN_OP_PROJECT ? 0.f : 1.f;
      cudaFuncSetAttribute(segment_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
      segment_pairs_kernel<<<batch, kPairThreads, smem_bytes, stream>>>(
          d_mats, g, px.pmax, limit, below, plan->bins, bins_cap, counters, counts, plan->fallback,
          plan->nfallback, (float2*)zero_out, px, geom);
    } else if (op == GTOMRLN_OP_PROJECT) {
      cudaFuncSetAttribute(bin_slices_kernel<GTOMRLN_OP_PROJECT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem_bytes);
      bin_slices_kernel<GTOMRLN_OP_PROJECT><<<batch, kBinThreads, smem_bytes, stream>>>(
          d_mats, g, px, limit, plan->entries, entries_cap, plan->bins, bins_cap, counters, counts,
          plan->fallback, plan->nfallback, use_codes);
    } else {
      cudaFuncSetAttribute(bin_slices_kernel<GTOMRLN_OP_BACKPROJECT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
      bin_slices_kernel<GTOMRLN_OP_BACKPROJECT><<<batch, kBinThreads, smem_bytes, stream>>>(
          d_mats, g, px, limit, plan->entries, entries_cap, plan->bins, bins_cap, counters, counts,
          plan->fallback, plan->nfallback, use_codes);
    }
    pairs_scan_kernel<<<1, kScanThreads, 0, stream>>>(counts, d_order, g.nbricks, geom.nvol, chunk, offsets,
                                                      item_off, cursor, plan->nitems);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    pairs_fill_kernel<<<sms * 4, 256, 0, stream>>>(plan->bins, counters, bins_cap, counts, offsets, cursor,
                                                   plan->pairs);
    plan_items_kernel<<<(int)((nkeys + 255) / 256), 256, 0, stream>>>(counts, offsets, item_off, (int)nkeys, chunk,
                                                                      plan->items);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    free_brick_plan(plan, stream);
    return set_error(GTOMRLN_ERR_CUDA, "brick plan failed: %s", cudaGetErrorString(e));
  }
  return GTOMRLN_OK;
}

int free_brick_plan(BrickPlan* plan, cudaStream_t stream) {
  int st = scratch_free(plan->scratch, stream);
  *plan = BrickPlan();
  return st;
}

}  // namespace gtomrln
