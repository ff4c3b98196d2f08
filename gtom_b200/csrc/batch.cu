// Batched reconstruction of many volumes of uneven box size (sub-tomograms,
// half-maps, classes): every slice of every volume inserted by ONE
// persistent launch, then the gridding correction of each size class as
// stacks (batch.cuh), the whole sequence captured once in a CUDA graph and
// replayed.  Per volume the result equals d_rlnBackproject (matrix overload,
// rmax = box / 2, centred accumulators of P + 1, P = box * pad) followed by
// d_ReconstructGridding with a fixed iteration count
// (src/Relion/Backproject.cu:48-124, src/Reconstruction/RecFourier.cu:98-241);
// the reference batches only volumes of one size, through d_ivolume.
//
// Insertion: work items are runs of consecutive slices of one volume,
// largest boxes first; persistent CTAs take items from an atomic counter.
// Per slice the CTA's threads stride over its elements and add the
// reference's eight binary16-weighted targets per sample (sample.cuh) to
// the volume's accumulators with vector L2 reductions.  The launch shape
// (threads per CTA, slices per item, CTAs per SM) is a tuning parameter
// (gtomrln_batch_set_tuning; gtom_b200.batch.autotune picks it).
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "sample.cuh"

namespace gtomrln {

struct BatchVolume {
  float2* acc_ft;        // centred (D/2+1) x D x D accumulators, inside the class stack
  float* acc_w;
  const float2* projft;  // nslices x (n/2+1) x n slices (NULL: value 1)
  const float* projw;    // NULL: weight 1
  const float* mats;     // nslices x 9
  int n, D, rmax2;
};

struct BatchWork {
  int vol, slice0, nslices;
};

// place<false> of backproject.cu: centred storage of signed (x, y, z) with
// the reference's unsigned clamps.
__device__ __forceinline__ int64_t batch_place(int x, int y, int z, int D, int rowlen) {
  y += D / 2;
  z += D / 2;
  unsigned half = (unsigned)(D / 2), last = (unsigned)(D - 1);
  x = (unsigned)x > half ? (int)half : x;
  y = (unsigned)y > last ? (int)last : y;
  z = (unsigned)z > last ? (int)last : z;
  return ((int64_t)z * D + y) * rowlen + x;
}

__global__ void batch_insert_kernel(const BatchVolume* __restrict__ vols,
                                    const BatchWork* __restrict__ work, int nwork,
                                    int* __restrict__ counter) {
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();  // all threads have the item before thread 0 takes the next
    if (item >= nwork) break;
    const BatchWork w = work[item];
    const BatchVolume v = vols[w.vol];
    const int half = v.n / 2, dimft = v.n / 2 + 1;
    const int64_t elements = (int64_t)dimft * v.n;
    const int rowlen = v.D / 2 + 1;
    for (int s = 0; s < w.nslices; s++) {
      const int slice = w.slice0 + s;
      float m[9];
#pragma unroll
      for (int i = 0; i < 9; i++) m[i] = __ldg(v.mats + 9 * (int64_t)slice + i);
      for (int64_t id = threadIdx.x; id < elements; id += blockDim.x) {
        int x = (int)(id % dimft);
        int idy = (int)(id / dimft);
        int y = idy <= half ? idy : idy - v.n;
        if (x == 0 && y < 0) continue;
        if (x * x + y * y >= v.rmax2) continue;
        BpSample smp = backproject_sample(m, (float)x, (float)y, 0.f);
        float2 val = v.projft ? __ldg(v.projft + elements * slice + id) : make_float2(1.f, 0.f);
        float pw = v.projw ? __ldg(v.projw + elements * slice + id) : 1.f;
        for_each_target(smp.x0, smp.y0, smp.z0, [&](int i, int tx, int ty, int tz, bool conj) {
          float iw = smp.w[i];
          int64_t o = batch_place(tx, ty, tz, v.D, rowlen);
          red_add2((float*)(v.acc_ft + o), iw * val.x, iw * (conj ? -val.y : val.y));
          red_add(v.acc_w + o, iw * pw);
        });
      }
    }
  }
}

struct BatchClass {
  int box = 0;
  std::vector<int> members;  // subvolume indices, in stack order
  float2* acc_ft = nullptr;  // stacks of centred accumulators
  float* acc_w = nullptr;
  float** outs = nullptr;    // device array: members' output maps
  GridBatch grid;
};

struct BatchHandle {
  int device = 0;
  int pad = 2, iterations = 10;
  int threads = 256, slices_per_item = 4, blocks_per_sm = 4;
  std::vector<gtomrln_subvolume_t> items;
  std::vector<BatchClass> classes;
  BatchVolume* d_vols = nullptr;
  BatchWork* d_work = nullptr;
  int nwork = 0;
  int* d_counter = nullptr;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static void destroy_graph(BatchHandle* h) {
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->exec = nullptr;
  h->graph = nullptr;
}

static void destroy_handle(BatchHandle* h) {
  destroy_graph(h);
  for (auto& c : h->classes) {
    cudaFree(c.acc_ft);
    cudaFree(c.acc_w);
    cudaFree(c.outs);
    gridding_batch_free(&c.grid);
  }
  cudaFree(h->d_vols);
  cudaFree(h->d_work);
  cudaFree(h->d_counter);
  if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
  delete h;
}

// Work items of `slices_per_item` slices, largest boxes first.
static int build_work(BatchHandle* h) {
  std::vector<int> order(h->items.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return h->items[a].box > h->items[b].box; });
  std::vector<BatchWork> work;
  for (int v : order)
    for (int s = 0; s < h->items[v].nslices; s += h->slices_per_item)
      work.push_back({v, s, std::min(h->slices_per_item, h->items[v].nslices - s)});
  cudaFree(h->d_work);
  h->d_work = nullptr;
  h->nwork = (int)work.size();
  if (work.empty()) return GTOMRLN_OK;
  GTOMRLN_CUDA_TRY(cudaMalloc(&h->d_work, work.size() * sizeof(BatchWork)));
  GTOMRLN_CUDA_TRY(cudaMemcpy(h->d_work, work.data(), work.size() * sizeof(BatchWork), cudaMemcpyHostToDevice));
  return GTOMRLN_OK;
}

// Enqueues one whole run on stream.
static int enqueue(BatchHandle* h, cudaStream_t stream) {
  for (auto& c : h->classes) {
    size_t n = (size_t)c.members.size() * c.grid.wstride;
    GTOMRLN_CUDA_TRY(cudaMemsetAsync(c.acc_ft, 0, n * sizeof(float2), stream));
    GTOMRLN_CUDA_TRY(cudaMemsetAsync(c.acc_w, 0, n * sizeof(float), stream));
  }
  GTOMRLN_CUDA_TRY(cudaMemsetAsync(h->d_counter, 0, sizeof(int), stream));
  if (h->nwork > 0) {
    int sms = 0;
    GTOMRLN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    int blocks = std::min(h->nwork, sms * h->blocks_per_sm);
    batch_insert_kernel<<<blocks, h->threads, 0, stream>>>(h->d_vols, h->d_work, h->nwork, h->d_counter);
    GTOMRLN_LAUNCH_CHECK("batch_insert_kernel");
  }
  for (auto& c : h->classes) {
    int st = gridding_batch_run(c.grid, c.acc_ft, c.acc_w, c.outs, h->iterations, stream);
    if (st) return st;
  }
  return GTOMRLN_OK;
}

static int create(const gtomrln_subvolume_t* items, int count, int pad, int iterations,
                  BatchHandle** out) {
  if (count <= 0 || !items || pad <= 0 || iterations < 0)
    return set_error(GTOMRLN_ERR_INVALID, "batch_create: bad arguments");
  for (int i = 0; i < count; i++) {
    const auto& it = items[i];
    if (it.box < 4 || (it.box & 1) || it.nslices < 0 || !it.d_out || (it.nslices > 0 && !it.d_matrices))
      return set_error(GTOMRLN_ERR_INVALID, "batch_create: subvolume %d: bad box, slices or pointers", i);
  }
  BatchHandle* h = new BatchHandle();
  h->pad = pad;
  h->iterations = iterations;
  h->items.assign(items, items + count);
  int st = GTOMRLN_OK;
  auto fail = [&](int s) {
    destroy_handle(h);
    return s;
  };
  if (cudaGetDevice(&h->device) != cudaSuccess) return fail(set_error(GTOMRLN_ERR_CUDA, "cudaGetDevice failed"));
  std::vector<int> boxes;
  for (auto& it : h->items) boxes.push_back(it.box);
  std::sort(boxes.begin(), boxes.end());
  boxes.erase(std::unique(boxes.begin(), boxes.end()), boxes.end());
  std::vector<BatchVolume> vols(count);
  for (int box : boxes) {
    BatchClass c;
    c.box = box;
    for (int i = 0; i < count; i++)
      if (h->items[i].box == box) c.members.push_back(i);
    h->classes.push_back(c);
    BatchClass& cc = h->classes.back();
    st = gridding_batch_prepare(&cc.grid, (int)cc.members.size(), box, pad, 1.9, 0, 15.0);
    if (st) return fail(st);
    size_t n = (size_t)cc.members.size() * cc.grid.wstride;
    if (cudaMalloc(&cc.acc_ft, n * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&cc.acc_w, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&cc.outs, cc.members.size() * sizeof(float*)) != cudaSuccess)
      return fail(set_error(GTOMRLN_ERR_ALLOC, "batch_create: out of device memory for box %d", box));
    std::vector<float*> outs;
    for (size_t k = 0; k < cc.members.size(); k++) {
      int i = cc.members[k];
      const auto& it = h->items[i];
      BatchVolume& v = vols[i];
      v.acc_ft = cc.acc_ft + k * cc.grid.wstride;
      v.acc_w = cc.acc_w + k * cc.grid.wstride;
      v.projft = (const float2*)it.d_projft;
      v.projw = it.d_projweights;
      v.mats = it.d_matrices;
      v.n = box;
      v.D = cc.grid.D;
      v.rmax2 = (box / 2) * (box / 2);
      outs.push_back(it.d_out);
    }
    if (cudaMemcpy(cc.outs, outs.data(), outs.size() * sizeof(float*), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(set_error(GTOMRLN_ERR_CUDA, "batch_create: copy of the output table failed"));
  }
  if (cudaMalloc(&h->d_vols, count * sizeof(BatchVolume)) != cudaSuccess ||
      cudaMalloc(&h->d_counter, sizeof(int)) != cudaSuccess)
    return fail(set_error(GTOMRLN_ERR_ALLOC, "batch_create: out of device memory"));
  if (cudaMemcpy(h->d_vols, vols.data(), count * sizeof(BatchVolume), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(set_error(GTOMRLN_ERR_CUDA, "batch_create: copy of the volume table failed"));
  st = build_work(h);
  if (st) return fail(st);
  if (cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(GTOMRLN_ERR_CUDA, "batch_create: stream creation failed"));
  *out = h;
  return GTOMRLN_OK;
}

}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_batch_create(const gtomrln_subvolume_t* items, int count, int paddingfactor,
                         int iterations, void** handle) {
  clear_error();
  if (!handle) return set_error(GTOMRLN_ERR_INVALID, "batch_create: NULL handle");
  *handle = nullptr;
  BatchHandle* h = nullptr;
  int st = create(items, count, paddingfactor, iterations, &h);
  if (st) return st;
  *handle = h;
  return GTOMRLN_OK;
}

int gtomrln_batch_set_tuning(void* handle, int threads, int slices_per_item, int blocks_per_sm) {
  clear_error();
  BatchHandle* h = (BatchHandle*)handle;
  if (!h) return set_error(GTOMRLN_ERR_INVALID, "batch_set_tuning: NULL handle");
  if ((threads && (threads < 32 || threads > 1024 || threads % 32)) || slices_per_item < 0 ||
      blocks_per_sm < 0 || blocks_per_sm > 32)
    return set_error(GTOMRLN_ERR_INVALID, "batch_set_tuning: threads %d, slices %d, blocks/SM %d out of range",
                     threads, slices_per_item, blocks_per_sm);
  if (threads) h->threads = threads;
  if (blocks_per_sm) h->blocks_per_sm = blocks_per_sm;
  if (slices_per_item && slices_per_item != h->slices_per_item) {
    h->slices_per_item = slices_per_item;
    int st = build_work(h);
    if (st) return st;
  }
  destroy_graph(h);  // the captured launch shape is stale
  return GTOMRLN_OK;
}

int gtomrln_batch_run(void* handle, int use_graph, void* stream) {
  clear_error();
  BatchHandle* h = (BatchHandle*)handle;
  if (!h) return set_error(GTOMRLN_ERR_INVALID, "batch_run: NULL handle");
  int dev = -1;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  if (dev != h->device)
    return set_error(GTOMRLN_ERR_INVALID, "batch_run: handle made on device %d, current device %d", h->device, dev);
  if (!use_graph) return enqueue(h, (cudaStream_t)stream);
  if (!h->exec) {
    GTOMRLN_CUDA_TRY(cudaStreamBeginCapture(h->capture_stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue(h, h->capture_stream);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->capture_stream, &graph);
    if (st) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess)
      return set_error(GTOMRLN_ERR_CUDA, "batch_run: capture failed: %s", cudaGetErrorString(e));
    h->graph = graph;
    e = cudaGraphInstantiate(&h->exec, h->graph, 0);
    if (e != cudaSuccess) {
      destroy_graph(h);
      return set_error(GTOMRLN_ERR_CUDA, "batch_run: graph instantiation failed: %s", cudaGetErrorString(e));
    }
  }
  GTOMRLN_CUDA_TRY(cudaGraphLaunch(h->exec, (cudaStream_t)stream));
  return GTOMRLN_OK;
}

int gtomrln_batch_destroy(void* handle) {
  clear_error();
  if (handle) destroy_handle((BatchHandle*)handle);
  return GTOMRLN_OK;
}

}  // extern "C"
