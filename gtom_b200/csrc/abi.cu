// Library-wide pieces of the C ABI: error state, version, the device memory
// pool for per-call scratch, and the host matrix builder.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdarg>
#include <deque>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace gtomrln {

static thread_local std::string g_last_error;

int set_error(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

void clear_error() { g_last_error.clear(); }

// Single-precision ZYZ Euler matrix in the order src/Helpers/Euler.cu:39-68
// evaluates it, transposed and scaled (Project.cu:16).  For s = 1 or a power
// of two the scale is exact.
void matrices_from_angles(const float* angles, float s, unsigned batch, float* out) {
  for (unsigned b = 0; b < batch; b++) {
    float alpha = angles[3 * b], beta = angles[3 * b + 1], gamma = angles[3 * b + 2];
    float ca = std::cos(alpha), cb = std::cos(beta), cg = std::cos(gamma);
    float sa = std::sin(alpha), sb = std::sin(beta), sg = std::sin(gamma);
    float cc = cb * ca, cs = cb * sa, sc = sb * ca, ss = sb * sa;
    // E as a math matrix, row-major E[r][c] (glm column c = (E[0][c], E[1][c], E[2][c])).
    float E[3][3];
    E[0][0] = cg * cc - sg * sa;  E[1][0] = -sg * cc - cg * sa;  E[2][0] = sc;
    E[0][1] = cg * cs + sg * ca;  E[1][1] = -sg * cs + cg * ca;  E[2][1] = ss;
    E[0][2] = -cg * sb;           E[1][2] = sg * sb;             E[2][2] = cb;
    // M = E^T * s; column-major M[c*3 + r] = M(r, c) = E(c, r) * s.
    float* o = out + 9 * (size_t)b;
    for (int c = 0; c < 3; c++)
      for (int r = 0; r < 3; r++) o[c * 3 + r] = E[c][r] * s;
  }
}

// The context id through the driver's cuCtxGetCurrent / cuCtxGetId, looked
// up once through the runtime (no link against the driver library).
namespace {
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
std::once_flag g_ctx_once;
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
}  // namespace

unsigned long long context_id() {
  std::call_once(g_ctx_once, [] {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&g_ctx_current, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      g_ctx_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&g_ctx_id, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      g_ctx_id = nullptr;
    cudaGetLastError();
  });
  if (!g_ctx_current || !g_ctx_id) return 0;
  void* ctx = nullptr;
  if (g_ctx_current(&ctx) != 0 || !ctx) {
    // no context current yet (or it was destroyed): the runtime creates the
    // device's primary context and makes it current
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    if (g_ctx_current(&ctx) != 0 || !ctx) return 0;
  }
  unsigned long long id = 0;
  return g_ctx_id(ctx, &id) == 0 ? id : 0;
}

// One pool per device and context.  Freed scratch stays mapped in the pool
// (no release threshold) so that repeated calls reuse it instead of
// remapping gigabytes each time; gtomrln_release_caches() returns it to the
// device and destroys the pool.
namespace {
struct PoolEntry {
  int dev;
  unsigned long long ctx;
  cudaMemPool_t pool;
};
std::mutex g_pool_mutex;
std::vector<PoolEntry> g_pools;
}  // namespace

static int get_pool(cudaMemPool_t* out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  for (size_t i = 0; i < g_pools.size(); i++) {
    if (g_pools[i].dev != dev) continue;
    if (g_pools[i].ctx == ctx) {
      *out = g_pools[i].pool;
      return GTOMRLN_OK;
    }
    // made in a context that no longer exists: its memory went with it
    g_pools.erase(g_pools.begin() + i);
    break;
  }
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool;
  GTOMRLN_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
  uint64_t threshold = UINT64_MAX;
  GTOMRLN_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  g_pools.push_back({dev, ctx, pool});
  *out = pool;
  return GTOMRLN_OK;
}

int pool_alloc(void** ptr, size_t bytes, cudaStream_t stream) {
  cudaMemPool_t pool;
  int st = get_pool(&pool);
  if (st) return st;
  if (bytes == 0) bytes = 256;
  cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, pool, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(GTOMRLN_ERR_ALLOC, "device allocation of %zu bytes failed: %s", bytes,
                     cudaGetErrorString(e));
  }
  return GTOMRLN_OK;
}

int pool_free(void* ptr, cudaStream_t stream) {
  if (!ptr) return GTOMRLN_OK;
  GTOMRLN_CUDA_TRY(cudaFreeAsync(ptr, stream));
  return GTOMRLN_OK;
}

// Per-(device, stream) scratch that outlives a call: the brick plans take it
// instead of a pool allocation, so that repeated calls allocate nothing.  A
// pool allocation that has to map new memory blocks the host for
// milliseconds (observed 5-45 ms for ~700 MB after a device synchronisation
// had regrouped the pool's free blocks), while the device drains the queue
// and idles.  A slot grows (by 1/8 plus rounding to 64 MB) and never shrinks
// until gtomrln_release_caches().  Calls on the same stream reuse it in
// stream order; an event recorded at release and waited for at the next
// acquisition covers a stream handle that was destroyed and handed out
// again.  Under stream capture, or while the slot is held by another host
// thread, a plain pool allocation is used.
namespace {
struct ScratchSlot {
  int dev;
  unsigned long long ctx;
  cudaStream_t stream;
  void* ptr;
  size_t bytes;
  bool busy;
  cudaEvent_t done;
};
std::mutex g_scratch_mutex;
std::vector<ScratchSlot> g_scratch;
}  // namespace

int scratch_alloc(void** ptr, size_t bytes, cudaStream_t stream) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    cs = cudaStreamCaptureStatusActive;
  }
  if (cs != cudaStreamCaptureStatusNone) return pool_alloc(ptr, bytes, stream);
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  // slots of this device made in an earlier context are gone with it
  g_scratch.erase(std::remove_if(g_scratch.begin(), g_scratch.end(),
                                 [&](const ScratchSlot& s) { return s.dev == dev && s.ctx != ctx; }),
                  g_scratch.end());
  ScratchSlot* slot = nullptr;
  for (auto& s : g_scratch)
    if (s.dev == dev && s.stream == stream) slot = &s;
  if (!slot) {
    cudaEvent_t ev;
    GTOMRLN_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    g_scratch.push_back({dev, ctx, stream, nullptr, 0, false, ev});
    slot = &g_scratch.back();
  }
  if (slot->busy) return pool_alloc(ptr, bytes, stream);
  GTOMRLN_CUDA_TRY(cudaStreamWaitEvent(stream, slot->done, 0));
  if (slot->bytes < bytes) {
    if (slot->ptr) {
      int st = pool_free(slot->ptr, stream);
      slot->ptr = nullptr;
      slot->bytes = 0;
      if (st) return st;
    }
    const size_t grain = (size_t)64 << 20;
    const size_t want = (bytes + bytes / 8 + grain - 1) / grain * grain;
    int st = pool_alloc(&slot->ptr, want, stream);
    if (st) return st;
    slot->bytes = want;
  }
  slot->busy = true;
  *ptr = slot->ptr;
  return GTOMRLN_OK;
}

int scratch_free(void* ptr, cudaStream_t stream) {
  if (!ptr) return GTOMRLN_OK;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    for (auto& s : g_scratch)
      if (s.busy && s.ptr == ptr) {
        s.busy = false;
        GTOMRLN_CUDA_TRY(cudaEventRecord(s.done, stream));
        return GTOMRLN_OK;
      }
  }
  return pool_free(ptr, stream);
}

// Pinned host staging for the uploads of the h_angles overloads.  A
// cudaMemcpyAsync from pageable memory is staged by the driver before it
// returns, behind every transfer already queued on the copy engine, so a
// caller that overlaps its own gigabyte copies with compute would stall in
// each call.  From a pinned slot the copy is truly asynchronous; a slot is
// reused once the event recorded after its copy has completed (eight slots
// per device in turn, so the wait is normally over before it starts).  When
// every slot is held by another host thread the caller falls back to its
// pageable copy.
namespace {
constexpr int kStageSlots = 8;
struct StageSlot {
  int dev;
  unsigned long long ctx;
  void* ptr;
  size_t cap;
  cudaEvent_t done;
  bool busy;
};
std::mutex g_stage_mutex;
std::deque<StageSlot> g_stage;  // stable references under push_back
unsigned g_stage_turn = 0;
}  // namespace

int stage_acquire(size_t bytes, void** ptr, int* slot) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  StageSlot* s = nullptr;
  int idx = -1;
  {
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    std::vector<int> mine;
    for (int i = 0; i < (int)g_stage.size(); i++) {
      StageSlot& t = g_stage[i];
      if (t.dev != dev) continue;
      if (t.ctx != ctx) {
        // made in a context that no longer exists (its pinned memory and
        // event went with it): retire the slot for good
        t.dev = -1;
        t.ptr = nullptr;
        t.cap = 0;
        continue;
      }
      mine.push_back(i);
    }
    if (mine.empty()) {
      for (int k = 0; k < kStageSlots; k++) {
        cudaEvent_t ev;
        GTOMRLN_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        g_stage.push_back({dev, ctx, nullptr, 0, ev, false});
        mine.push_back((int)g_stage.size() - 1);
      }
    }
    for (int t = 0; t < (int)mine.size() && !s; t++) {
      const int i = mine[(g_stage_turn + t) % mine.size()];
      if (!g_stage[i].busy) {
        s = &g_stage[i];
        idx = i;
      }
    }
    if (!s) return GTOMRLN_ERR_ALLOC;  // all held: the caller copies from pageable memory
    g_stage_turn++;
    s->busy = true;
  }
  cudaError_t e = cudaEventSynchronize(s->done);  // this slot's previous copy has read it
  if (e == cudaSuccess && s->cap < bytes) {
    if (s->ptr) cudaFreeHost(s->ptr);
    s->ptr = nullptr;
    s->cap = 0;
    const size_t want = std::max<size_t>(bytes, (size_t)64 << 10);
    e = cudaHostAlloc(&s->ptr, want, cudaHostAllocDefault);
    if (e == cudaSuccess) s->cap = want;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    s->busy = false;
    return GTOMRLN_ERR_ALLOC;
  }
  *ptr = s->ptr;
  *slot = idx;
  return GTOMRLN_OK;
}

int stage_release(int slot, cudaStream_t stream) {
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  StageSlot& s = g_stage[slot];
  cudaError_t e = cudaEventRecord(s.done, stream);
  s.busy = false;
  if (e != cudaSuccess) return set_error(GTOMRLN_ERR_CUDA, "staging event: %s", cudaGetErrorString(e));
  return GTOMRLN_OK;
}

// Host floats to device memory through kernel parameters: each launch carries
// up to kParamFloats floats by value (30 KB of the 32 764-byte parameter
// space), so the upload never enters a copy engine's queue.  A stream-ordered
// cudaMemcpyAsync of the same few kilobytes waits behind every transfer the
// caller has queued in that direction (measured: 3 ms per call behind an
// 800 MB copy of the next batch), stalling the compute that needs it.
namespace {
constexpr int kParamFloats = 7680;
struct ParamChunk {
  float v[kParamFloats];
};
__global__ void param_copy_kernel(const ParamChunk c, float* __restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = c.v[i];
}
}  // namespace

size_t param_upload_limit() { return (size_t)64 * kParamFloats; }

int upload_via_params(float* dst, const float* src, size_t count, cudaStream_t stream) {
  ParamChunk c;
  for (size_t off = 0; off < count; off += kParamFloats) {
    const int n = (int)std::min<size_t>(kParamFloats, count - off);
    std::copy(src + off, src + off + n, c.v);
    param_copy_kernel<<<(n + 255) / 256, 256, 0, stream>>>(c, dst + off, n);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(GTOMRLN_ERR_CUDA, "parameter upload failed: %s", cudaGetErrorString(e));
  return GTOMRLN_OK;
}

// Frees the idle staging slots' pinned memory of the current context on
// device dev (after a device synchronisation); the slots and their events
// stay.
static void release_stage(int dev, unsigned long long ctx) {
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  for (auto& s : g_stage)
    if (s.dev == dev && s.ctx == ctx && !s.busy && s.ptr) {
      cudaFreeHost(s.ptr);
      s.ptr = nullptr;
      s.cap = 0;
    }
}

// Frees the idle scratch slots of the current context on device dev (after
// a device synchronisation) and forgets those of earlier contexts.
static int release_scratch(int dev, unsigned long long ctx) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  std::vector<ScratchSlot> keep;
  for (auto& s : g_scratch) {
    if (s.dev != dev || (s.ctx == ctx && s.busy)) {
      keep.push_back(s);
      continue;
    }
    if (s.ctx != ctx) continue;  // gone with its context
    if (s.ptr) {
      GTOMRLN_CUDA_TRY(cudaFreeAsync(s.ptr, 0));
      GTOMRLN_CUDA_TRY(cudaStreamSynchronize(0));
    }
    GTOMRLN_CUDA_TRY(cudaEventDestroy(s.done));
  }
  g_scratch.swap(keep);
  return GTOMRLN_OK;
}

// Trims and destroys the memory pool of the current context on device dev,
// and forgets pools of earlier contexts there.
static int release_pool(int dev, unsigned long long ctx) {
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  std::vector<PoolEntry> keep;
  int st = GTOMRLN_OK;
  for (auto& p : g_pools) {
    if (p.dev != dev) {
      keep.push_back(p);
      continue;
    }
    if (p.ctx != ctx) continue;
    cudaError_t e = cudaMemPoolTrimTo(p.pool, 0);
    if (e == cudaSuccess) e = cudaMemPoolDestroy(p.pool);
    if (e != cudaSuccess && !st) st = set_error(GTOMRLN_ERR_CUDA, "memory pool release: %s", cudaGetErrorString(e));
  }
  g_pools.swap(keep);
  return st;
}

int release_gridding_caches(int dev, unsigned long long ctx);  // gridding.cu
int release_ctf_plans(int dev, unsigned long long ctx);        // ctf.cu
int release_brick_orders(int dev, unsigned long long ctx);     // brick_plan.cu
int release_gridfft_tables(int dev, unsigned long long ctx);   // gridfft.cu
int release_gridsym_caches(int dev, unsigned long long ctx);   // gridsym.cu

static std::atomic<int> g_path[3] = {{GTOMRLN_PATH_AUTO}, {GTOMRLN_PATH_AUTO}, {GTOMRLN_PATH_AUTO}};

int path_choice(int op) { return (op >= 0 && op <= 2) ? g_path[op].load() : GTOMRLN_PATH_AUTO; }

// Crossovers measured at padding 2 (direct vs row-segment, ms):
// backprojector  n = 128: 1 000 slices 0.48 vs 0.76, 3 000: 1.40 vs 1.97,
//                10 000: 4.56 vs 3.23; n = 192: 300 slices 0.64 vs 0.52;
//                n = 96, 10 000: 2.65 vs 2.97;
// projector      n = 192: 3 000 slices 0.86 vs 1.05, 10 000: 2.99 vs 2.08;
//                n = 256: 300 slices 0.26 vs 0.50, 1 000: 0.83 vs 0.72.
bool brick_path_pays(int op, int V, unsigned batch) {
  if (op == GTOMRLN_OP_BACKPROJECT) return (V >= 384 && batch >= 300) || (V >= 256 && batch >= 6000);
  return (V >= 512 && batch >= 1000) || (V >= 384 && batch >= 6000);
}

// Defaults measured on the B200 at 256^3 (padding 2) with 10,000-slice
// batches (row-segment variants; the largest bricks whose shared memory fits
// a CTA win); the autotuner (gtom_b200/autotune.py) can replace them.
static const BrickTuning kDefaultTuning[2] = {{29, 1024, 4096}, {26, 1024, 4096}};
static std::mutex g_tuning_mutex;
static BrickTuning g_tuning[2] = {kDefaultTuning[0], kDefaultTuning[1]};

BrickTuning brick_tuning(int op) {
  std::lock_guard<std::mutex> lock(g_tuning_mutex);
  return g_tuning[op == 1 ? 1 : 0];
}

}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_version(void) { return 100; }

const char* gtomrln_last_error(void) { return g_last_error.c_str(); }

int gtomrln_release_caches(void) {
  clear_error();
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  GTOMRLN_CUDA_TRY(cudaDeviceSynchronize());
  int st = release_gridding_caches(dev, ctx);
  if (!st) st = release_ctf_plans(dev, ctx);
  if (!st) st = release_brick_orders(dev, ctx);
  if (!st) st = release_gridfft_tables(dev, ctx);
  if (!st) st = release_gridsym_caches(dev, ctx);
  if (!st) st = release_scratch(dev, ctx);
  if (st) return st;
  release_stage(dev, ctx);
  return release_pool(dev, ctx);
}

int gtomrln_set_path(int op, int path) {
  clear_error();
  const bool grid = op == GTOMRLN_OP_GRIDDING;
  if ((op != GTOMRLN_OP_PROJECT && op != GTOMRLN_OP_BACKPROJECT && !grid) || path < GTOMRLN_PATH_AUTO ||
      (!grid && path > GTOMRLN_PATH_SEGMENT &&
       !(op == GTOMRLN_OP_BACKPROJECT && path == GTOMRLN_PATH_SEGMENT_FP32)) ||
      (grid && path != GTOMRLN_PATH_AUTO && path != GTOMRLN_PATH_DIRECT && path != GTOMRLN_PATH_FUSED &&
       path != GTOMRLN_PATH_SYMMETRIC))
    return set_error(GTOMRLN_ERR_INVALID, "set_path: unknown op %d or path %d", op, path);
  g_path[op].store(path);
  return GTOMRLN_OK;
}

int gtomrln_set_brick_tuning(int op, int edge, int threads, int chunk) {
  clear_error();
  if (op != GTOMRLN_OP_PROJECT && op != GTOMRLN_OP_BACKPROJECT)
    return set_error(GTOMRLN_ERR_INVALID, "set_brick_tuning: unknown op %d", op);
  BrickTuning t = kDefaultTuning[op];
  if (edge) t.edge = edge;
  if (threads) t.threads = threads;
  if (chunk) t.chunk = chunk;
  // Shared memory per CTA: the projector stages (edge+1)^3 complex voxels,
  // the backprojector keeps 3 * edge * (edge+1)^2 floats; both <= 227 KB.
  size_t smem = op == GTOMRLN_OP_PROJECT ? 8 * (size_t)(t.edge + 1) * (t.edge + 1) * (t.edge + 1)
                                         : 12 * (size_t)t.edge * (t.edge + 1) * (t.edge + 1);
  if (t.edge < 4 || t.edge > 64 || smem > 227 * 1024 || t.threads < 64 || t.threads > 1024 ||
      t.threads % 32 || t.chunk < 1)
    return set_error(GTOMRLN_ERR_INVALID, "set_brick_tuning: edge %d, threads %d, chunk %d out of range",
                     t.edge, t.threads, t.chunk);
  std::lock_guard<std::mutex> lock(g_tuning_mutex);
  g_tuning[op] = t;
  return GTOMRLN_OK;
}

int gtomrln_matrices_from_angles(const float* h_angles, float supersample, unsigned batch,
                                 float* h_matrices) {
  clear_error();
  if (batch && (!h_angles || !h_matrices))
    return set_error(GTOMRLN_ERR_INVALID, "matrices_from_angles: NULL array");
  matrices_from_angles(h_angles, supersample, batch, h_matrices);
  return GTOMRLN_OK;
}

}  // extern "C"
