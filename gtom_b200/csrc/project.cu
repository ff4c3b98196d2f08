// Projector: trilinear central-slice gather from a decentred half-complex
// Fourier volume (RELION convention), the B200 replacement of
// Project3DArraytoNDKernel / Project3DtoNDKernel (src/Relion/Project.cu:89-272).
//
// Direct kernel: one thread per output element.  The block's slice matrix is
// read once into registers; the eight corner voxels are fetched through the
// read-only path so that consecutive slices of similar orientation hit L2.
// The per-sample arithmetic is the reference's, operation for operation, so
// the result is the same for the same inputs.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "brick.cuh"
#include "common.cuh"
#include "sample.cuh"
#include "segment.cuh"

namespace gtomrln {

constexpr int kProjThreads = 256;
constexpr int kProjPerThread = 4;
constexpr int kProjTile = kProjThreads * kProjPerThread;

struct ProjArgs {
  int n;          // dimsproj.x
  int dimft;      // n/2 + 1
  int64_t area;   // dimft * n
  int64_t elements;
  int tiles;      // tiles per slice
  int rmax2;
  int rmax;
  int P;          // dimsvolume.x
  int64_t nvox;   // (P/2+1) * P * P
};

struct ArrayFetch {
  const float2* __restrict__ vol;
  int P, rowlen;
  int64_t last;
  __device__ __forceinline__ float2 operator()(int x, int y, int z) const {
    // Flat index as in Project.cu:154-161; x == P/2+1 continues into the
    // next row like the reference, the one read past the end is clamped.
    int64_t i = ((int64_t)z * P + y) * rowlen + x;
    i = i < 0 ? 0 : (i > last ? last : i);
    return __ldg(vol + i);
  }
};

struct TexFetch {
  cudaTextureObject_t re, im;
  __device__ __forceinline__ float2 operator()(int x, int y, int z) const {
    // Project.cu:249-256: integer coordinates passed as floats.
    return make_float2(tex3D<float>(re, (float)x, (float)y, (float)z),
                       tex3D<float>(im, (float)x, (float)y, (float)z));
  }
};

// Value of an in-disk sample as stored: unchanged for d_rlnProject.
struct NoPost {
  template <int NDIMS>
  __device__ __forceinline__ float2 apply(int, int, int, int, float2 v) const { return v; }
};

// d_rlnProjectShifted (ProjectShifted.cu:214-220): the sample times
// exp(i phi), phi = -(x sx + y sy [+ z sz]) with the 2 pi / n-scaled shift of
// the slice, then times its global weight.  Phase and complex product with
// the contractions and fast sine/cosine of the reference's build.
struct ShiftPost {
  const float* __restrict__ shifts;   // 3 per slice
  const float* __restrict__ weights;  // 1 per slice
  template <int NDIMS>
  __device__ __forceinline__ float2 apply(int slice, int x, int y, int z, float2 v) const {
    float sx = __ldg(shifts + 3 * (int64_t)slice), sy = __ldg(shifts + 3 * (int64_t)slice + 1);
    float phase = fmaf((float)x, sx, (float)y * sy);
    if (NDIMS == 3) phase = fmaf((float)z, __ldg(shifts + 3 * (int64_t)slice + 2), phase);
    phase = -phase;
    float c = __cosf(phase), s = __sinf(phase);
    float w = __ldg(weights + slice);
    float re = fmaf(v.x, c, -(v.y * s)), im = fmaf(v.x, s, v.y * c);
    return make_float2(re * w, im * w);
  }
};

template <int NDIMS, class Fetch, class Post = NoPost>
__device__ __forceinline__ void project_direct_tile(const Fetch& fetch, float2* __restrict__ proj,
                                                    const float* __restrict__ mats, const ProjArgs& a,
                                                    int slice, int tile, const Post& post = Post()) {
  float m[9];
#pragma unroll
  for (int i = 0; i < 9; i++) m[i] = __ldg(mats + 9 * (int64_t)slice + i);
  float2* out = proj + a.elements * slice;
  const int half = a.n / 2;

#pragma unroll
  for (int k = 0; k < kProjPerThread; k++) {
    int64_t id = (int64_t)tile * kProjTile + k * kProjThreads + threadIdx.x;
    if (id >= a.elements) break;
    int idx, idy, idz;
    split_index(id, a.dimft, NDIMS == 3 ? a.area : a.elements, a.elements, idx, idy, idz);
    int x = idx;
    int y = idy <= half ? idy : idy - a.n;
    int z = idz <= half ? idz : idz - a.n;
    int r2 = NDIMS == 3 ? z * z + y * y + x * x : y * y + x * x;
    if (r2 > a.rmax2) {
      out[id] = make_float2(0.f, 0.f);
      continue;
    }
    float3 pos = mat_apply(m, (float)x, (float)y, (float)z);
    float sign = 1.f;
    if (pos.x < -1e-5f) {  // Friedel mate: only x >= 0 is stored
      pos.x = fabsf(pos.x);
      pos.y = -pos.y;
      pos.z = -pos.z;
      sign = -1.f;
    }
    float fx0 = floorf(pos.x + 1e-5f);
    int x0 = (int)fx0, x1 = x0 + 1;
    float fx = pos.x - fx0;
    float fy0 = floorf(pos.y);
    int y0 = (int)fy0, y1 = y0 + 1;
    if (y0 < 0) y0 += a.P;
    if (y1 < 0) y1 += a.P;
    float fy = pos.y - fy0;
    float fz0 = floorf(pos.z);
    int z0 = (int)fz0, z1 = z0 + 1;
    if (z0 < 0) z0 += a.P;
    if (z1 < 0) z1 += a.P;
    float fz = pos.z - fz0;

    float2 d000 = fetch(x0, y0, z0), d001 = fetch(x1, y0, z0);
    float2 d010 = fetch(x0, y1, z0), d011 = fetch(x1, y1, z0);
    float2 d100 = fetch(x0, y0, z1), d101 = fetch(x1, y0, z1);
    float2 d110 = fetch(x0, y1, z1), d111 = fetch(x1, y1, z1);

    float rx00 = lerpf(d000.x, d001.x, fx), ix00 = lerpf(d000.y, d001.y, fx);
    float rx01 = lerpf(d010.x, d011.x, fx), ix01 = lerpf(d010.y, d011.y, fx);
    float rx10 = lerpf(d100.x, d101.x, fx), ix10 = lerpf(d100.y, d101.y, fx);
    float rx11 = lerpf(d110.x, d111.x, fx), ix11 = lerpf(d110.y, d111.y, fx);
    float rxy0 = lerpf(rx00, rx01, fy), ixy0 = lerpf(ix00, ix01, fy);
    float rxy1 = lerpf(rx10, rx11, fy), ixy1 = lerpf(ix10, ix11, fy);
    float2 v = make_float2(lerpf(rxy0, rxy1, fz), lerpf(ixy0, ixy1, fz) * sign);
    out[id] = post.template apply<NDIMS>(slice, x, y, z, v);
  }
}

template <int NDIMS, class Fetch, class Post = NoPost>
__global__ void __launch_bounds__(kProjThreads)
project_direct_kernel(Fetch fetch, float2* __restrict__ proj, const float* __restrict__ mats,
                      ProjArgs a, Post post = Post()) {
  const int slice = blockIdx.x / a.tiles;
  project_direct_tile<NDIMS>(fetch, proj, mats, a, slice, blockIdx.x - slice * a.tiles, post);
}

// The direct kernel over the slices listed in list[0 .. *nlist), which the
// brick plan left to it; a persistent grid strides over (slice, tile).
template <class Post = NoPost>
__global__ void __launch_bounds__(kProjThreads)
project_listed_kernel(ArrayFetch fetch, float2* __restrict__ proj, const float* __restrict__ mats,
                      ProjArgs a, const int* __restrict__ list, const int* __restrict__ nlist,
                      Post post = Post()) {
  const int64_t total = (int64_t)(*nlist) * a.tiles;
  for (int64_t w = blockIdx.x; w < total; w += gridDim.x)
    project_direct_tile<2>(fetch, proj, mats, a, __ldg(list + w / a.tiles), (int)(w % a.tiles), post);
}

// ---------------------------------------------------------------------------
// Brick-major projector.  Each work item stages one brick of the volume
// (edge^3 voxels plus a one-voxel halo, in signed coordinates, wrapped into
// the decentred layout exactly as the reference's index arithmetic wraps
// them) in shared memory, then the warps take the item's bins (slice, pixel
// run) one at a time and evaluate those pixels — the plan put every in-disk
// pixel into the bin of the brick holding its interpolation base voxel
// (x0, y0, z0), so each is written exactly once, with the direct kernel's
// arithmetic on the same voxel values: the results are identical.  Pixels
// outside rmax are zeroed by project_zero_kernel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
project_brick_kernel(const float2* __restrict__ vol, float2* __restrict__ proj,
                     const float* __restrict__ mats, ProjArgs a, BrickGrid g,
                     const BrickItem* __restrict__ items, const int* __restrict__ nitems_ptr,
                     const int* __restrict__ pairs, const PixelBin* __restrict__ bins,
                     const int* __restrict__ entries, int* __restrict__ counter) {
  extern __shared__ float2 tile[];
  __shared__ int item_s, next_s;
  const int nitems = *nitems_ptr;
  const int B = g.B, T = g.B + 1;
  const int rowlen = a.P / 2 + 1;
  const int64_t last = a.nvox - 1;
  for (;;) {
    __syncthreads();  // previous item done with the tile
    if (threadIdx.x == 0) {
      item_s = atomicAdd(counter, 1);
      next_s = 0;
    }
    __syncthreads();
    const int w = item_s;
    if (w >= nitems) break;
    const BrickItem it = items[w];
    const int3 o = brick_origin(g, it.brick);
    for (int k = threadIdx.x; k < T * T * T; k += blockDim.x) {
      int tx = k % T, t2 = k / T, ty = t2 % T, tz = t2 / T;
      int x = o.x + tx, y = o.y + ty, z = o.z + tz;
      int ys = y < 0 ? y + a.P : y, zs = z < 0 ? z + a.P : z;
      int64_t i = ((int64_t)zs * a.P + ys) * rowlen + x;
      i = i < 0 ? 0 : (i > last ? last : i);
      tile[k] = __ldg(vol + i);
    }
    __syncthreads();
    for (;;) {  // warps take the item's bins one at a time
      int j = 0;
      if ((threadIdx.x & 31) == 0) j = atomicAdd(&next_s, 1);
      j = __shfl_sync(0xffffffffu, j, 0);
      if (j >= it.count) break;
      const PixelBin bn = bins[__ldg(pairs + it.offset + j)];
      float m[9];
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)bn.slice + k);
      float2* out = proj + a.elements * bn.slice;
      for (int k = threadIdx.x & 31; k < bn.count; k += 32) {
        const int id = __ldg(entries + bn.start + k);
        int u, v;
        pixel_uv(id, a.n, a.dimft, u, v);
        ProjSample s = project_sample(m, u, v, 0);
        int lx = s.x0 - o.x, ly = s.y0 - o.y, lz = s.z0 - o.z;
        if ((unsigned)lx >= (unsigned)B || (unsigned)ly >= (unsigned)B || (unsigned)lz >= (unsigned)B)
          continue;  // cannot happen: the plan used the same arithmetic
        const float2* c = tile + (lz * T + ly) * T + lx;
        out[id] = trilerp(s, c[0], c[1], c[T], c[T + 1], c[T * T], c[T * T + 1], c[T * T + T],
                          c[T * T + T + 1]);
      }
    }
  }
}

// Segment variant of the brick projector: the same staging and arithmetic,
// but a warp takes a (slice, brick) pair of the segment plan and finds the
// pixels itself, by row segments (segment.cuh), among those whose position
// (side 0) or mirrored position (side 1) falls in the brick.  A pixel is
// written by the pair whose brick holds its base voxel, on the side of its
// Friedel flip: exactly one pair, as in the binned variant.  Post turns the
// interpolated value into the stored one (identity, or the phase shift and
// weight of d_rlnProjectShifted), as in the direct kernel.
template <class Post = NoPost>
__global__ void __launch_bounds__(1024)
project_segment_kernel(const float2* __restrict__ vol, float2* __restrict__ proj,
                       const float* __restrict__ mats, ProjArgs a, BrickGrid g, PixelSet px,
                       const BrickItem* __restrict__ items, const int* __restrict__ nitems_ptr,
                       const int* __restrict__ pairs, const PixelBin* __restrict__ bins, int* __restrict__ counter, Post post = Post()) {
  extern __shared__ float2 tile[];
  __shared__ int item_s, next_s;
  const int nitems = *nitems_ptr;
  const int B = g.B, T = g.B + 1;
  const int rowlen = a.P / 2 + 1;
  const int64_t last = a.nvox - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (;;) {
    __syncthreads();  // previous item done with the tile
    if (threadIdx.x == 0) {
      item_s = atomicAdd(counter, 1);
      next_s = 0;
    }
    __syncthreads();
    const int w = item_s;
    if (w >= nitems) break;
    const BrickItem it = items[w];
    const int3 o = brick_origin(g, it.brick);
    // stage the brick and its halo, one warp per (y, z) row, lanes along x
    for (int r = warp; r < T * T; r += nwarps) {
      const int ty = r % T, tz = r / T;
      const int y = o.y + ty, z = o.z + tz;
      const int ys = y < 0 ? y + a.P : y, zs = z < 0 ? z + a.P : z;
      const int64_t row = ((int64_t)zs * a.P + ys) * rowlen + o.x;
      for (int tx = lane; tx < T; tx += 32) {
        int64_t i = row + tx;
        i = i < 0 ? 0 : (i > last ? last : i);
        tile[r * T + tx] = __ldg(vol + i);
      }
    }
    __syncthreads();
    // warps take the item's pairs one at a time, the next one's slice
    // fetched before the current one is processed
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
      float2* out = proj + a.elements * slice;
#pragma unroll 1
      for (int side = 0; side < 2; side++) {
        int vlo, vhi;
        seg_unpack_rows(side ? pr.z : pr.y, vlo, vhi);
        if (vlo > vhi) continue;  // no pixel of this side
        const SegBox box = seg_box(m, side, o, B, 0.f);
        seg_for_each_pixel_rows(box, px, vlo, vhi, [&](int u, int v, bool valid) {
          if (!valid) return;
          ProjSample s = project_sample(m, u, v, 0);
          if ((s.sign < 0.f) != (side == 1)) return;  // the other side's pixel
          int lx = s.x0 - o.x, ly = s.y0 - o.y, lz = s.z0 - o.z;
          if ((unsigned)lx >= (unsigned)B || (unsigned)ly >= (unsigned)B || (unsigned)lz >= (unsigned)B)
            return;  // another brick's pixel
          const float2* c = tile + (lz * T + ly) * T + lx;
          const int idy = v < 0 ? v + a.n : v;
          const float2 val = trilerp(s, c[0], c[1], c[T], c[T + 1], c[T * T], c[T * T + 1], c[T * T + T],
                                     c[T * T + T + 1]);
          out[(int64_t)idy * a.dimft + u] = post.template apply<2>(slice, u, v, 0, val);
        });
      }
      j = jn;
      pr = nx;
    }
  }
}

// Zeroes the elements outside rmax (Project.cu:111-115) for the brick path.
// In each row they form the tail x > sqrt(rmax^2 - y^2); one warp writes
// one row's tail, coalesced.
__global__ void project_zero_kernel(float2* __restrict__ proj, ProjArgs a, int64_t rows) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
    int idy = (int)(r % a.n);
    int y = idy <= a.n / 2 ? idy : idy - a.n;
    int rem = a.rmax2 - y * y;
    int x0 = 0;
    if (rem >= 0) {
      x0 = (int)sqrtf((float)rem);
      while (x0 * x0 > rem) x0--;
      while ((x0 + 1) * (x0 + 1) <= rem) x0++;
      x0++;  // first x with x^2 + y^2 > rmax^2
    }
    float2* row = proj + r * a.dimft;
    for (int x = x0 + lane; x < a.dimft; x += 32) row[x] = make_float2(0.f, 0.f);
  }
}


// The brick path: plan, zero fill outside rmax, brick kernel, and the direct
// kernel for any slice the plan could not take.  Nothing synchronises.  A
// Post other than NoPost (the shifted projector) takes the segment variant.
template <class Post = NoPost>
static int project_brick(const float* d_volumeft, float* d_proj, const float* d_mats, const ProjArgs& a,
                         unsigned batch, cudaStream_t stream, int segments, Post post = Post()) {
  if (!std::is_same<Post, NoPost>::value) segments = 1;
  const int P = a.P;
  const BrickTuning tune = brick_tuning(GTOMRLN_OP_PROJECT);
  // While every sample radius stays below P/2 + 0.99, the base voxels lie in
  // x [0, P/2] and y, z [-P/2 - 1, P/2].
  BrickGrid g = make_brick_grid(P, tune.edge, P / 2, -(P / 2) - 1, P / 2);
  size_t smem = sizeof(float2) * (size_t)(tune.edge + 1) * (tune.edge + 1) * (tune.edge + 1);
  auto kern = project_segment_kernel<Post>;
  cudaError_t e = segments ? cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                           : cudaFuncSetAttribute(project_brick_kernel,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return set_error(GTOMRLN_ERR_CUDA, "brick projector: %zu B of shared memory refused: %s", smem,
                     cudaGetErrorString(e));
  int dev = 0, sms = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (segments)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, tune.threads, smem);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, project_brick_kernel, tune.threads, smem);
  PixelSet px;
  px.n = a.n;
  px.dimft = a.dimft;
  px.elements = a.elements;
  px.rmax2 = a.rmax2;
  px.strict = 0;
  px.pmax = (float)a.rmax;
  BrickPlan plan;
  // the segment plan writes the zeros outside rmax of the slices it plans
  // (the direct kernel those of the slices it leaves over)
  int st = build_brick_plan(GTOMRLN_OP_PROJECT, d_mats, (int)batch, g, px, (float)(P / 2) + 0.99f, tune.chunk,
                            stream, &plan, segments, segments ? d_proj : nullptr);
  if (st) return st;
  if (!segments) {
    int64_t rows = (int64_t)a.n * batch;  // 2D slices: n rows of dimft elements each
    project_zero_kernel<<<sms * 8, 256, 0, stream>>>((float2*)d_proj, a, rows);
  }
  if (segments)
    kern<<<sms * std::max(occ, 1), tune.threads, smem, stream>>>(
        (const float2*)d_volumeft, (float2*)d_proj, d_mats, a, g, px, plan.items, plan.nitems, plan.pairs,
        plan.bins, plan.counter, post);
  else
    project_brick_kernel<<<sms * std::max(occ, 1), tune.threads, smem, stream>>>(
        (const float2*)d_volumeft, (float2*)d_proj, d_mats, a, g, plan.items, plan.nitems, plan.pairs, plan.bins,
        plan.entries, plan.counter);
  ArrayFetch f{(const float2*)d_volumeft, a.P, a.P / 2 + 1, a.nvox - 1};
  project_listed_kernel<Post><<<sms * 4, kProjThreads, 0, stream>>>(f, (float2*)d_proj, d_mats, a, plan.fallback,
                                                                     plan.nfallback, post);
  e = cudaGetLastError();
  free_brick_plan(&plan, stream);
  if (e != cudaSuccess)
    return set_error(GTOMRLN_ERR_CUDA, "launch of the brick projector failed: %s", cudaGetErrorString(e));
  return GTOMRLN_OK;
}

// Validates dimensions the way Project.cu:27-32 does and fills ProjArgs.
static int project_setup(int vx, int vy, int vz, int px, int py, int pz, unsigned rmax,
                         unsigned batch, ProjArgs* a, int* ndims_proj) {
  int ndv = dimension_count(vx, vy, vz), ndp = dimension_count(px, py, pz);
  if (ndv < ndp)
    return set_error(GTOMRLN_ERR_INVALID,
                     "project: volume has %d dimensions, projections %d (reference throws)", ndv,
                     ndp);
  if (ndp != 2 && ndp != 3)
    return set_error(GTOMRLN_ERR_INVALID, "project: projections must be 2D or 3D (got %dD)", ndp);
  if (vx <= 0 || px <= 0)
    return set_error(GTOMRLN_ERR_INVALID, "project: non-positive dimension");
  if (rmax > (unsigned)(px / 2)) rmax = px / 2;
  a->n = px;
  a->dimft = px / 2 + 1;
  a->area = (int64_t)a->dimft * px;
  a->elements = ndp == 3 ? a->area * px : a->area;
  a->tiles = (int)((a->elements + kProjTile - 1) / kProjTile);
  a->rmax2 = (int)(rmax * rmax);
  a->rmax = (int)rmax;
  a->P = vx;
  a->nvox = (int64_t)(vx / 2 + 1) * vx * vx;
  *ndims_proj = ndp;
  if ((int64_t)a->tiles * batch > 0x7fffffffLL)
    return set_error(GTOMRLN_ERR_INVALID, "project: batch too large for one launch");
  return GTOMRLN_OK;
}

template <class Fetch, class Post = NoPost>
static int launch_project(Fetch f, int ndp, float* d_proj, const float* d_mats, const ProjArgs& a,
                          unsigned batch, cudaStream_t stream, Post post = Post()) {
  if (batch == 0) return GTOMRLN_OK;
  dim3 grid((unsigned)(a.tiles * (int64_t)batch));
  if (ndp == 2)
    project_direct_kernel<2, Fetch, Post><<<grid, kProjThreads, 0, stream>>>(f, (float2*)d_proj, d_mats, a, post);
  else
    project_direct_kernel<3, Fetch, Post><<<grid, kProjThreads, 0, stream>>>(f, (float2*)d_proj, d_mats, a, post);
  GTOMRLN_LAUNCH_CHECK("project_direct_kernel");
  return GTOMRLN_OK;
}

// ---------------------------------------------------------------------------
// Projection from host angles without any device allocation.
//
// The h_angles overload has to place the slices' rotation matrices in device
// memory; gtomrln_project_angles takes that scratch from the library's
// memory pool.  gtomrln_project_angles_noalloc keeps it instead in the
// fixed array below, which is part of the library image: every device that
// loads the library holds these kNoAllocMaxBatch * 36 bytes until the
// process exits, and no call allocates anything.
// ---------------------------------------------------------------------------
constexpr unsigned kNoAllocMaxBatch = 4096;
static __device__ __align__(256) float g_noalloc_matrices[kNoAllocMaxBatch * 9];

// In host code g_noalloc_matrices is only a host-side stand-in; the device
// address comes from cudaGetSymbolAddress with the calling device current.
// It is looked up on every call rather than cached: the lookup is cheap once
// the module is loaded, and a cached address would go stale if the caller
// reset the device (cudaDeviceReset) and the module were loaded again
// elsewhere.
static int noalloc_matrices(float** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_matrices);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(GTOMRLN_ERR_CUDA, "cudaGetSymbolAddress of the fixed matrix array failed: %s",
                     cudaGetErrorString(e));
  }
  *out = (float*)p;
  return GTOMRLN_OK;
}

}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_project_angles_noalloc(const float* d_volumeft, int vx, int vy, int vz, float* d_proj,
                                   int px, int py, int pz, const float* h_angles, float supersample,
                                   unsigned batch, void* stream) {
  clear_error();
  if (batch > kNoAllocMaxBatch)
    return set_error(GTOMRLN_ERR_INVALID,
                     "project_angles_noalloc: batch %u exceeds the fixed capacity of %u slices; "
                     "split the batch",
                     batch, kNoAllocMaxBatch);
  ProjArgs a;
  int ndp;
  int st = project_setup(vx, vy, vz, px, py, pz, (unsigned)(px / 2), batch, &a, &ndp);
  if (st) return st;
  if (batch == 0) return GTOMRLN_OK;
  if (!d_volumeft || !d_proj || !h_angles)
    return set_error(GTOMRLN_ERR_INVALID, "project_angles_noalloc: NULL pointer");
  float* d_mats = nullptr;
  st = noalloc_matrices(&d_mats);
  if (st) return st;
  // Host side without allocation: the matrices are built in a fixed
  // per-thread buffer and carried to the array as kernel parameters (at most
  // 4096 * 9 floats, five launches), so the upload holds no reference to
  // host memory after this call returns and no copy engine is involved.
  static thread_local float h_mats[kNoAllocMaxBatch * 9];
  matrices_from_angles(h_angles, supersample, batch, h_mats);
  cudaStream_t s = (cudaStream_t)stream;
  // Every matrix the kernel reads is rewritten here, so nothing left from an
  // earlier call needs clearing.  The upload is ordered on `s` after earlier
  // work on `s`; calls on different streams that overlap on the GPU race for
  // the shared array.  The projection always takes the direct kernel: the
  // brick kernels need plan scratch, which this entry point does not allocate.
  st = upload_via_params(d_mats, h_mats, 9 * (size_t)batch, s);
  if (st) return st;
  ArrayFetch f{(const float2*)d_volumeft, a.P, a.P / 2 + 1, a.nvox - 1};
  return launch_project(f, ndp, d_proj, d_mats, a, batch, s);
}

int gtomrln_project(const float* d_volumeft, int vx, int vy, int vz, float* d_proj, int px, int py,
                    int pz, unsigned rmax, const float* d_matrices, unsigned batch, void* stream) {
  clear_error();
  ProjArgs a;
  int ndp;
  int st = project_setup(vx, vy, vz, px, py, pz, rmax, batch, &a, &ndp);
  if (st) return st;
  if (batch && (!d_volumeft || !d_proj || !d_matrices))
    return set_error(GTOMRLN_ERR_INVALID, "project: NULL device pointer");
  const int choice = path_choice(GTOMRLN_OP_PROJECT);
  // the brick plans' integer square roots take radii below 4 096 (seg_isqrt)
  if (ndp == 2 && vx == vy && vx == vz && vx >= 4 && a.rmax2 <= (1 << 24) &&
      (choice == GTOMRLN_PATH_BRICK || choice == GTOMRLN_PATH_SEGMENT ||
       (choice == GTOMRLN_PATH_AUTO && brick_path_pays(GTOMRLN_OP_PROJECT, vx, batch))))
    return project_brick(d_volumeft, d_proj, d_matrices, a, batch, (cudaStream_t)stream,
                         choice == GTOMRLN_PATH_BRICK ? 0 : 1);
  ArrayFetch f{(const float2*)d_volumeft, a.P, a.P / 2 + 1, a.nvox - 1};
  return launch_project(f, ndp, d_proj, d_matrices, a, batch, (cudaStream_t)stream);
}

int gtomrln_project_angles(const float* d_volumeft, int vx, int vy, int vz, float* d_proj, int px,
                           int py, int pz, const float* h_angles, float supersample, unsigned batch,
                           void* stream) {
  clear_error();
  return with_device_matrices(h_angles, supersample, batch, (cudaStream_t)stream,
                              [&](const float* d_m) {
                                return gtomrln_project(d_volumeft, vx, vy, vz, d_proj, px, py, pz,
                                                       (unsigned)(px / 2), d_m, batch, stream);
                              });
}

int gtomrln_project_tex(unsigned long long t_re, unsigned long long t_im, int vx, int vy, int vz,
                        float* d_proj, int px, int py, int pz, unsigned rmax,
                        const float* d_matrices, unsigned batch, void* stream) {
  clear_error();
  ProjArgs a;
  int ndp;
  int st = project_setup(vx, vy, vz, px, py, pz, rmax, batch, &a, &ndp);
  if (st) return st;
  if (batch && (!d_proj || !d_matrices))
    return set_error(GTOMRLN_ERR_INVALID, "project_tex: NULL device pointer");
  TexFetch f{(cudaTextureObject_t)t_re, (cudaTextureObject_t)t_im};
  return launch_project(f, ndp, d_proj, d_matrices, a, batch, (cudaStream_t)stream);
}

int gtomrln_project_tex_angles(unsigned long long t_re, unsigned long long t_im, int vx, int vy,
                               int vz, float* d_proj, int px, int py, int pz,
                               const float* h_angles, float supersample, unsigned batch,
                               void* stream) {
  clear_error();
  return with_device_matrices(h_angles, supersample, batch, (cudaStream_t)stream,
                              [&](const float* d_m) {
                                return gtomrln_project_tex(t_re, t_im, vx, vy, vz, d_proj, px, py,
                                                           pz, (unsigned)(px / 2), d_m, batch,
                                                           stream);
                              });
}

// ---------------------------------------------------------------- shifted --
int gtomrln_project_shifted(const float* d_volumeft, int vx, int vy, int vz, float* d_proj, int px,
                            int py, int pz, unsigned rmax, const float* d_matrices,
                            const float* d_shifts, const float* d_globalweights, unsigned batch,
                            void* stream) {
  clear_error();
  ProjArgs a;
  int ndp;
  int st = project_setup(vx, vy, vz, px, py, pz, rmax, batch, &a, &ndp);
  if (st) return st;
  if (batch && (!d_volumeft || !d_proj || !d_matrices || !d_shifts || !d_globalweights))
    return set_error(GTOMRLN_ERR_INVALID, "project_shifted: NULL device pointer");
  const int choice = path_choice(GTOMRLN_OP_PROJECT);
  // the brick plans' integer square roots take radii below 4 096 (seg_isqrt)
  if (ndp == 2 && vx == vy && vx == vz && vx >= 4 && a.rmax2 <= (1 << 24) &&
      (choice == GTOMRLN_PATH_BRICK || choice == GTOMRLN_PATH_SEGMENT ||
       (choice == GTOMRLN_PATH_AUTO && brick_path_pays(GTOMRLN_OP_PROJECT, vx, batch))))
    return project_brick(d_volumeft, d_proj, d_matrices, a, batch, (cudaStream_t)stream, 1,
                         ShiftPost{d_shifts, d_globalweights});
  ArrayFetch f{(const float2*)d_volumeft, a.P, a.P / 2 + 1, a.nvox - 1};
  return launch_project(f, ndp, d_proj, d_matrices, a, batch, (cudaStream_t)stream,
                        ShiftPost{d_shifts, d_globalweights});
}

int gtomrln_project_shifted_angles(const float* d_volumeft, int vx, int vy, int vz, float* d_proj,
                                   int px, int py, int pz, const float* h_angles,
                                   const float* h_shifts, const float* h_globalweights,
                                   float supersample, unsigned batch, void* stream) {
  clear_error();
  return with_device_shifted(h_angles, h_shifts, h_globalweights, supersample, px, batch,
                             (cudaStream_t)stream,
                             [&](const float* d_m, const float* d_s, const float* d_w) {
                               return gtomrln_project_shifted(d_volumeft, vx, vy, vz, d_proj, px, py, pz,
                                                              (unsigned)(px / 2), d_m, d_s, d_w, batch,
                                                              stream);
                             });
}

int gtomrln_project_shifted_tex(unsigned long long t_re, unsigned long long t_im, int vx, int vy,
                                int vz, float* d_proj, int px, int py, int pz, unsigned rmax,
                                const float* d_matrices, const float* d_shifts,
                                const float* d_globalweights, unsigned batch, void* stream) {
  clear_error();
  ProjArgs a;
  int ndp;
  int st = project_setup(vx, vy, vz, px, py, pz, rmax, batch, &a, &ndp);
  if (st) return st;
  if (batch && (!d_proj || !d_matrices || !d_shifts || !d_globalweights))
    return set_error(GTOMRLN_ERR_INVALID, "project_shifted_tex: NULL device pointer");
  TexFetch f{(cudaTextureObject_t)t_re, (cudaTextureObject_t)t_im};
  return launch_project(f, ndp, d_proj, d_matrices, a, batch, (cudaStream_t)stream,
                        ShiftPost{d_shifts, d_globalweights});
}

int gtomrln_project_shifted_tex_angles(unsigned long long t_re, unsigned long long t_im, int vx,
                                       int vy, int vz, float* d_proj, int px, int py, int pz,
                                       const float* h_angles, const float* h_shifts,
                                       const float* h_globalweights, float supersample,
                                       unsigned batch, void* stream) {
  clear_error();
  return with_device_shifted(h_angles, h_shifts, h_globalweights, supersample, px, batch,
                             (cudaStream_t)stream,
                             [&](const float* d_m, const float* d_s, const float* d_w) {
                               return gtomrln_project_shifted_tex(t_re, t_im, vx, vy, vz, d_proj, px, py,
                                                                  pz, (unsigned)(px / 2), d_m, d_s, d_w,
                                                                  batch, stream);
                             });
}

}  // extern "C"
