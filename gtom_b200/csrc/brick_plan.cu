// Plan construction for the brick-major kernels: which slices cross which
// brick, cut into balanced work items.
#include <algorithm>
#include <cstring>

#include "brick.cuh"

namespace gtomrln {

constexpr int kPlanThreads = 256;

__device__ __forceinline__ bool box_outside_disk(float3 qlo, float3 qhi, float rdisk) {
  float px = fminf(fmaxf(0.f, qlo.x), qhi.x), py = fminf(fmaxf(0.f, qlo.y), qhi.y),
        pz = fminf(fmaxf(0.f, qlo.z), qhi.z);
  return px * px + py * py + pz * pz > rdisk * rdisk;
}

// Counts the slices crossing each brick.  Block 0 also records the largest
// sample radius of the batch so that the host can check the geometry.
__global__ void __launch_bounds__(kPlanThreads)
brick_count_kernel(const float* __restrict__ mats, int batch, BrickGrid g, float pmax, float rbound,
                   int* __restrict__ counts, unsigned* __restrict__ max_radius) {
  const int b = blockIdx.x;
  float3 qlo, qhi;
  brick_box(g, b, qlo, qhi);
  __shared__ int total;
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  if (b == 0) {
    float r = 0.f;
    for (int i = threadIdx.x; i < batch; i += kPlanThreads)
      r = fmaxf(r, plane_scale(mats + 9 * (int64_t)i) * pmax);
    for (int o = 16; o > 0; o >>= 1) r = fmaxf(r, __shfl_down_sync(0xffffffffu, r, o));
    if ((threadIdx.x & 31) == 0) atomicMax(max_radius, __float_as_uint(r));  // r >= 0
  }
  if (!box_outside_disk(qlo, qhi, rbound)) {
    int c = 0;
    for (int i = threadIdx.x; i < batch; i += kPlanThreads) {
      float m[9];
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)i + k);
      c += plane_hits_box(m, qlo, qhi, plane_scale(m) * pmax + 1e-2f);
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&total, c);
  }
  __syncthreads();
  if (threadIdx.x == 0) counts[b] = total;
}

// Writes each brick's crossing slices, in ascending order, at its offset.
// Uses the same test as the count kernel, so the counts match.
__global__ void __launch_bounds__(kPlanThreads)
brick_fill_kernel(const float* __restrict__ mats, int batch, BrickGrid g, float pmax,
                  const int* __restrict__ offsets, const int* __restrict__ counts,
                  int* __restrict__ lists) {
  const int b = blockIdx.x;
  if (counts[b] == 0) return;
  float3 qlo, qhi;
  brick_box(g, b, qlo, qhi);
  __shared__ int warp_tot[kPlanThreads / 32];
  __shared__ int base;
  if (threadIdx.x == 0) base = offsets[b];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = 0; i0 < batch; i0 += kPlanThreads) {
    int i = i0 + threadIdx.x;
    bool hit = false;
    if (i < batch) {
      float m[9];
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)i + k);
      hit = plane_hits_box(m, qlo, qhi, plane_scale(m) * pmax + 1e-2f);
    }
    unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    int before = 0, all = 0;
    for (int w = 0; w < kPlanThreads / 32; w++) {
      if (w < warp) before += warp_tot[w];
      all += warp_tot[w];
    }
    int slot = base + before + __popc(bal & ((1u << lane) - 1));
    if (hit && slot < offsets[b] + counts[b]) lists[slot] = i;  // never past the brick's share
    __syncthreads();
    if (threadIdx.x == 0) base += all;
    __syncthreads();
  }
}

int build_brick_plan(const float* d_mats, int batch, const BrickGrid& g, float pmax, float limit,
                     int chunk, cudaStream_t stream, BrickPlan* plan, bool* fits) {
  plan->g = g;
  *fits = false;
  int* d_counts = nullptr;
  int st = pool_alloc((void**)&d_counts, sizeof(int) * ((size_t)g.nbricks + 1), stream);
  if (st) return st;
  unsigned* d_maxr = (unsigned*)(d_counts + g.nbricks);
  std::vector<int> counts(g.nbricks + 1);
  cudaError_t e = cudaMemsetAsync(d_maxr, 0, sizeof(unsigned), stream);
  if (e == cudaSuccess) {
    brick_count_kernel<<<g.nbricks, kPlanThreads, 0, stream>>>(d_mats, batch, g, pmax, limit + 2.f,
                                                               d_counts, d_maxr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(counts.data(), d_counts, sizeof(int) * counts.size(), cudaMemcpyDeviceToHost,
                        stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    pool_free(d_counts, stream);
    return set_error(GTOMRLN_ERR_CUDA, "brick count failed: %s", cudaGetErrorString(e));
  }
  float maxr;
  memcpy(&maxr, &counts[g.nbricks], sizeof(float));
  if (!(maxr < limit)) {  // some sample may need the direct path's clamps
    pool_free(d_counts, stream);
    return GTOMRLN_OK;
  }
  *fits = true;

  std::vector<int> offsets(g.nbricks);
  std::vector<BrickItem> items;
  int64_t total = 0;
  for (int b = 0; b < g.nbricks; b++) {
    offsets[b] = (int)total;
    int c = counts[b];
    if (!c) continue;
    int nch = (c + chunk - 1) / chunk;
    for (int k = 0; k < nch; k++)
      items.push_back({b, (int)total + k * chunk, std::min(chunk, c - k * chunk), nch == 1 ? 1 : 0});
    total += c;
  }
  if (total > 0x7fffffffLL) {
    pool_free(d_counts, stream);
    return set_error(GTOMRLN_ERR_INVALID, "brick plan too large; split the batch");
  }
  // Largest items first, so that the longest ones do not start last.
  std::stable_sort(items.begin(), items.end(),
                   [](const BrickItem& a, const BrickItem& b) { return a.count > b.count; });
  size_t bytes_items = sizeof(BrickItem) * std::max<size_t>(1, items.size());
  size_t bytes_lists = sizeof(int) * std::max<int64_t>(1, total);
  size_t bytes_off = sizeof(int) * (size_t)g.nbricks;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t bytes = al(bytes_items) + al(bytes_lists) + al(bytes_off) + 256;
  char* base = nullptr;
  st = pool_alloc((void**)&base, bytes, stream);
  if (st) {
    pool_free(d_counts, stream);
    return st;
  }
  plan->scratch = base;
  plan->items = (BrickItem*)base;
  plan->lists = (int*)(base + al(bytes_items));
  int* d_off = (int*)(base + al(bytes_items) + al(bytes_lists));
  plan->counter = (int*)(base + al(bytes_items) + al(bytes_lists) + al(bytes_off));
  plan->nitems = (int)items.size();
  e = cudaSuccess;
  if (!items.empty())
    e = cudaMemcpyAsync(plan->items, items.data(), sizeof(BrickItem) * items.size(),
                        cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_off, offsets.data(), bytes_off, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(plan->counter, 0, sizeof(int), stream);
  if (e == cudaSuccess && total > 0) {
    brick_fill_kernel<<<g.nbricks, kPlanThreads, 0, stream>>>(d_mats, batch, g, pmax, d_off,
                                                              d_counts, plan->lists);
    e = cudaGetLastError();
  }
  // The host vectors must outlive the copies that read them.
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  pool_free(d_counts, stream);
  if (e != cudaSuccess) {
    free_brick_plan(plan, stream);
    return set_error(GTOMRLN_ERR_CUDA, "brick plan failed: %s", cudaGetErrorString(e));
  }
  return GTOMRLN_OK;
}

int free_brick_plan(BrickPlan* plan, cudaStream_t stream) {
  int st = pool_free(plan->scratch, stream);
  plan->scratch = nullptr;
  plan->items = nullptr;
  plan->lists = nullptr;
  plan->counter = nullptr;
  plan->nitems = 0;
  return st;
}

}  // namespace gtomrln
