// Plan construction for the brick-major kernels, entirely on the device (no
// host synchronisation, so a call can be captured in a CUDA graph):
//
//  1. bin_count: one warp per slice rasterises the slice's central plane
//     over the brick grid (columns along the plane normal's dominant axis)
//     and counts, per brick, the slices that cross it.  Slices whose samples
//     could leave the region the brick kernels handle (larger radius than
//     `limit`) go to a fallback list for the direct kernels instead.
//  2. plan_scan: one block turns the counts into list offsets and work
//     items (at most `chunk` slices each), bricks in order of increasing
//     distance from the origin so that the heaviest items start first.
//  3. bin_fill: the same rasterisation writes each slice into its bricks'
//     lists.
//  4. plan_items: one thread per brick writes its items.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>

#include "brick.cuh"

namespace gtomrln {

constexpr int kBinWarps = 8;  // warps (slices) per block of the binning kernels

__device__ __forceinline__ bool box_within_disk(float3 qlo, float3 qhi, float rdisk) {
  float px = fminf(fmaxf(0.f, qlo.x), qhi.x), py = fminf(fmaxf(0.f, qlo.y), qhi.y),
        pz = fminf(fmaxf(0.f, qlo.z), qhi.z);
  return px * px + py * py + pz * pz <= rdisk * rdisk;
}

// Calls hit(b) for every brick b whose dilated box the slice's plane
// crosses within its disk (the same test as plane_hits_box).  Warp-wide:
// the lanes split the columns.
template <class Hit>
__device__ __forceinline__ void for_each_crossed_brick(const float* m, const BrickGrid& g, float rdisk,
                                                       Hit&& hit) {
  const int lane = threadIdx.x & 31;
  float3 c0 = make_float3(m[0], m[1], m[2]), c1 = make_float3(m[3], m[4], m[5]);
  float n[3] = {c0.y * c1.z - c0.z * c1.y, c0.z * c1.x - c0.x * c1.z, c0.x * c1.y - c0.y * c1.x};
  float an[3] = {fabsf(n[0]), fabsf(n[1]), fabsf(n[2])};
  int k = an[0] >= an[1] ? (an[0] >= an[2] ? 0 : 2) : (an[1] >= an[2] ? 1 : 2);  // dominant axis
  int i = k == 0 ? 1 : 0, j = k == 2 ? 1 : 2;
  const int nb[3] = {g.nbx, g.nby, g.nbz};
  const int lo0[3] = {0, g.ylo, g.zlo};
  const float guard = 1.0f + 1e-2f;
  // Covers plane_hits_box's own tolerance (1e-3 |n| (1 + |c|_1) along n,
  // at most sqrt(3) times that along the dominant axis).
  const float tol = 4e-3f;
  int ncols = nb[i] * nb[j];
  for (int col = lane; col < ncols; col += 32) {
    int bi = col % nb[i], bj = col / nb[i];
    float ilo = lo0[i] + bi * g.B - guard, ihi = lo0[i] + bi * g.B + g.B - 1 + guard;
    float jlo = lo0[j] + bj * g.B - guard, jhi = lo0[j] + bj * g.B + g.B - 1 + guard;
    // plane: n_k x_k = -(n_i x_i + n_j x_j); its x_k range over the column's rectangle
    float a0 = n[i] * ilo, a1 = n[i] * ihi, b0 = n[j] * jlo, b1 = n[j] * jhi;
    float smin = fminf(a0, a1) + fminf(b0, b1), smax = fmaxf(a0, a1) + fmaxf(b0, b1);
    float kmin = fminf(-smin / n[k], -smax / n[k]), kmax = fmaxf(-smin / n[k], -smax / n[k]);
    float pad = guard + tol * (1.f + fabsf(kmin) + fabsf(kmax) + fmaxf(fabsf(ilo), fabsf(ihi)) +
                               fmaxf(fabsf(jlo), fabsf(jhi)));
    int b_lo = (int)floorf((kmin - pad - lo0[k]) / g.B);
    int b_hi = (int)floorf((kmax + pad - lo0[k]) / g.B);
    b_lo = max(b_lo, 0);
    b_hi = min(b_hi, nb[k] - 1);
    for (int bk = b_lo; bk <= b_hi; bk++) {
      int idx[3];
      idx[i] = bi;
      idx[j] = bj;
      idx[k] = bk;
      int b = (idx[2] * g.nby + idx[1]) * g.nbx + idx[0];
      float3 qlo, qhi;
      brick_box(g, b, qlo, qhi);
      if (box_within_disk(qlo, qhi, rdisk) && plane_hits_box(m, qlo, qhi, rdisk)) hit(b);
    }
  }
}

__global__ void __launch_bounds__(kBinWarps * 32)
bin_count_kernel(const float* __restrict__ mats, int batch, BrickGrid g, float pmax, float limit,
                 int* __restrict__ counts, int* __restrict__ fallback, int* __restrict__ nfallback) {
  const int slice = blockIdx.x * kBinWarps + (threadIdx.x >> 5);
  if (slice >= batch) return;
  float m[9];
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)slice + k);
  float r = plane_scale(m) * pmax;
  if (!(r < limit)) {
    if ((threadIdx.x & 31) == 0) fallback[atomicAdd(nfallback, 1)] = slice;
    return;
  }
  for_each_crossed_brick(m, g, r + 1e-2f, [&](int b) { atomicAdd(counts + b, 1); });
}

__global__ void __launch_bounds__(kBinWarps * 32)
bin_fill_kernel(const float* __restrict__ mats, int batch, BrickGrid g, float pmax, float limit,
                const int* __restrict__ offsets, const int* __restrict__ counts,
                int* __restrict__ cursor, int* __restrict__ lists) {
  const int slice = blockIdx.x * kBinWarps + (threadIdx.x >> 5);
  if (slice >= batch) return;
  float m[9];
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)slice + k);
  float r = plane_scale(m) * pmax;
  if (!(r < limit)) return;
  for_each_crossed_brick(m, g, r + 1e-2f, [&](int b) {
    int s = atomicAdd(cursor + b, 1);
    if (s < counts[b]) lists[offsets[b] + s] = slice;  // never past the brick's share
  });
}

// Single block.  Bricks are visited in `order` (increasing distance from
// the origin); writes list offsets, per-brick item offsets and the item count.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads)
plan_scan_kernel(const int* __restrict__ counts, const int* __restrict__ order, int nbricks, int chunk,
                 int* __restrict__ offsets, int* __restrict__ item_off, int* __restrict__ cursor,
                 int* __restrict__ nitems) {
  __shared__ int s_c[kScanThreads], s_i[kScanThreads];
  __shared__ int carry_c, carry_i;
  if (threadIdx.x == 0) carry_c = carry_i = 0;
  __syncthreads();
  for (int base = 0; base < nbricks; base += kScanThreads) {
    int t = base + threadIdx.x;
    int b = t < nbricks ? order[t] : -1;
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

// Brick visiting order per grid, cached on each device.
static std::mutex g_order_mutex;
static std::map<std::tuple<int, int, int, int, int, int>, int*> g_orders;

static int brick_order(const BrickGrid& g, const int** out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  auto key = std::make_tuple(dev, g.V, g.B, g.nbx, g.nby, g.ylo);
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

int build_brick_plan(const float* d_mats, int batch, const BrickGrid& g, float pmax, float limit,
                     int chunk, cudaStream_t stream, BrickPlan* plan) {
  plan->g = g;
  plan->batch = batch;
  const int* d_order = nullptr;
  int st = brick_order(g, &d_order);
  if (st) return st;
  // Upper bound of the bricks one plane can cross: per column along the
  // dominant axis of its normal the plane spans at most 3 (B + 2.02) voxels
  // (the other two slopes are <= 1), i.e. at most 5 bricks.
  int64_t cols = std::max({(int64_t)g.nby * g.nbz, (int64_t)g.nbx * g.nbz, (int64_t)g.nbx * g.nby});
  int64_t cap_lists = std::max<int64_t>(1, (int64_t)batch * cols * 5);
  int64_t cap_items = (int64_t)g.nbricks + cap_lists / chunk + 1;
  if (cap_lists > 0x7fffffffLL)
    return set_error(GTOMRLN_ERR_INVALID, "brick plan too large for one call; split the batch");
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t nb = (size_t)g.nbricks;
  size_t off_counts = 0;
  size_t off_offsets = off_counts + al(nb * 4);
  size_t off_itemoff = off_offsets + al(nb * 4);
  size_t off_cursor = off_itemoff + al(nb * 4);
  size_t off_misc = off_cursor + al(nb * 4);                // counter, nitems, nfallback
  size_t off_fallback = off_misc + 256;
  size_t off_items = off_fallback + al((size_t)std::max(batch, 1) * 4);
  size_t off_lists = off_items + al((size_t)cap_items * sizeof(BrickItem));
  size_t bytes = off_lists + al((size_t)cap_lists * 4);
  char* base = nullptr;
  st = pool_alloc((void**)&base, bytes, stream);
  if (st) return st;
  plan->scratch = base;
  int* counts = (int*)(base + off_counts);
  int* offsets = (int*)(base + off_offsets);
  int* item_off = (int*)(base + off_itemoff);
  int* cursor = (int*)(base + off_cursor);
  plan->counter = (int*)(base + off_misc);
  plan->nitems = (int*)(base + off_misc) + 1;
  plan->nfallback = (int*)(base + off_misc) + 2;
  plan->fallback = (int*)(base + off_fallback);
  plan->items = (BrickItem*)(base + off_items);
  plan->lists = (int*)(base + off_lists);
  plan->max_items = (int)std::min<int64_t>(cap_items, 0x7fffffff);

  cudaError_t e = cudaMemsetAsync(counts, 0, nb * 4, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + off_misc, 0, 256, stream);
  if (e == cudaSuccess && batch > 0) {
    int blocks = (batch + kBinWarps - 1) / kBinWarps;
    bin_count_kernel<<<blocks, kBinWarps * 32, 0, stream>>>(d_mats, batch, g, pmax, limit, counts,
                                                            plan->fallback, plan->nfallback);
    plan_scan_kernel<<<1, kScanThreads, 0, stream>>>(counts, d_order, g.nbricks, chunk, offsets, item_off,
                                                     cursor, plan->nitems);
    bin_fill_kernel<<<blocks, kBinWarps * 32, 0, stream>>>(d_mats, batch, g, pmax, limit, offsets, counts,
                                                           cursor, plan->lists);
    plan_items_kernel<<<(g.nbricks + 255) / 256, 256, 0, stream>>>(counts, offsets, item_off, g.nbricks,
                                                                   chunk, plan->items);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    free_brick_plan(plan, stream);
    return set_error(GTOMRLN_ERR_CUDA, "brick plan failed: %s", cudaGetErrorString(e));
  }
  return GTOMRLN_OK;
}

int free_brick_plan(BrickPlan* plan, cudaStream_t stream) {
  int st = pool_free(plan->scratch, stream);
  *plan = BrickPlan();
  return st;
}

}  // namespace gtomrln
