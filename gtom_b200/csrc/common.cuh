// Shared helpers of the gtomrln library: status handling, the slice
// geometry, binary16 weight rounding and vector reductions.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/gtomrln.h"

namespace gtomrln {

// ---------------------------------------------------------------- errors --
// Records msg as the calling thread's last error and returns status.
int set_error(int status, const char* fmt, ...);
void clear_error();

#define GTOMRLN_CUDA_TRY(expr)                                                    \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess)                                                        \
      return ::gtomrln::set_error(GTOMRLN_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, \
                                  cudaGetErrorString(_e), __FILE__, __LINE__);    \
  } while (0)

#define GTOMRLN_LAUNCH_CHECK(what)                                                 \
  do {                                                                             \
    cudaError_t _e = cudaGetLastError();                                           \
    if (_e != cudaSuccess)                                                         \
      return ::gtomrln::set_error(GTOMRLN_ERR_CUDA, "launch of %s failed: %s", what, \
                                  cudaGetErrorString(_e));                         \
  } while (0)

// Number of dimensions the reference assigns to an int3
// (include/Prerequisites.cuh:219, DimensionCount).
inline int dimension_count(int x, int y, int z) {
  auto mx = [](int a, int b) { return a > b ? a : b; };
  return 3 - mx(2 - mx(z, 1), 0) - mx(2 - mx(y, 1), 0) - mx(2 - mx(x, 1), 0);
}

// Host matrices exactly as Project.cu:14-16 builds them (single precision).
void matrices_from_angles(const float* angles, float supersample, unsigned batch, float* out);

// Implementation chosen for op (GTOMRLN_OP_*) by gtomrln_set_path.
int path_choice(int op);

// Whether GTOMRLN_PATH_AUTO takes the brick-major (row-segment) kernels for
// op on a cubic volume of edge V and a batch of 2D slices: they win once the
// volume no longer fits in L2 and the batch amortises their plan, while the
// direct kernels, whose gathers and reductions then stay in L2, win on
// smaller volumes.  Thresholds from a B200 sweep of boxes 32-256 (V = 2n
// or 2n + 1) and batches 100-10 000 (abi.cu).
bool brick_path_pays(int op, int V, unsigned batch);

// Launch shape of the brick kernels for op: brick edge in voxels, threads
// per CTA, and the most slices one work item takes (gtomrln_set_brick_tuning).
struct BrickTuning {
  int edge, threads, chunk;
};
BrickTuning brick_tuning(int op);

// Unique id of the calling thread's current CUDA context (the device's
// primary context, made current if no context is), 0 if it cannot be
// determined.  The library's per-device caches (memory pool, scratch and
// staging slots, FFT plans, tables) are keyed on it, so that nothing made in
// a context that the caller has since destroyed (cudaDeviceReset) is used
// again: a new context never shares an id with an earlier one.
unsigned long long context_id();

// Stream-ordered device scratch from the library's memory pool.
int pool_alloc(void** ptr, size_t bytes, cudaStream_t stream);
int pool_free(void* ptr, cudaStream_t stream);
// Scratch cached per (device, stream) across calls (abi.cu); the pointer is
// valid until the matching scratch_free, in stream order.
int scratch_alloc(void** ptr, size_t bytes, cudaStream_t stream);
int scratch_free(void* ptr, cudaStream_t stream);
// Pinned host staging slot for an upload (abi.cu): write the data into *ptr,
// issue the cudaMemcpyAsync, then stage_release(slot, stream).  A non-zero
// return means no slot is free: copy from pageable memory instead.
int stage_acquire(size_t bytes, void** ptr, int* slot);
int stage_release(int slot, cudaStream_t stream);
// Copies count host floats to dst in stream order through kernel parameters
// (no copy engine; abi.cu); for count <= param_upload_limit().
int upload_via_params(float* dst, const float* src, size_t count, cudaStream_t stream);
size_t param_upload_limit();

// Uploads count host floats built by fill(float* host) to dst on stream: by
// kernel parameters when small enough, else from a pinned staging slot,
// else from pageable memory.
template <class Fill>
inline cudaError_t upload_host_floats(float* dst, size_t count, cudaStream_t stream, Fill fill) {
  if (count <= param_upload_limit()) {
    std::vector<float> h(count);
    fill(h.data());
    return upload_via_params(dst, h.data(), count, stream) == GTOMRLN_OK ? cudaSuccess : cudaErrorUnknown;
  }
  void* hp = nullptr;
  int slot = -1;
  if (stage_acquire(count * sizeof(float), &hp, &slot) == GTOMRLN_OK) {
    fill((float*)hp);
    cudaError_t e = cudaMemcpyAsync(dst, hp, count * sizeof(float), cudaMemcpyHostToDevice, stream);
    if (stage_release(slot, stream) && e == cudaSuccess) e = cudaErrorUnknown;
    return e;
  }
  std::vector<float> h(count);  // cudaMemcpyAsync stages pageable memory before returning
  fill(h.data());
  return cudaMemcpyAsync(dst, h.data(), count * sizeof(float), cudaMemcpyHostToDevice, stream);
}

// ---------------------------------------------------------------- device --
struct Mat3 {
  float m[9];  // column-major, as glm::mat3
};

// glm's mat3 * vec3 (m[0][0]*v.x + m[1][0]*v.y + m[2][0]*v.z per row),
// contracted the way the compiler contracts that sum in the reference: the
// left product is fused with the rounded middle one, then the right product
// is fused onto that.  Keeping the same roundings matters because the
// backprojector rounds its weights to binary16, which turns a one-ulp
// difference in a position into a 2^-11 difference in a weight.
__device__ __forceinline__ float3 mat_apply(const float* m, float x, float y, float z) {
  float3 r;
  r.x = fmaf(m[6], z, fmaf(m[0], x, m[3] * y));
  r.y = fmaf(m[7], z, fmaf(m[1], x, m[4] * y));
  r.z = fmaf(m[8], z, fmaf(m[2], x, m[5] * y));
  return r;
}

// lerp of cutil_math_bugfixes.cuh:212: fma(b - a, t, a).
__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(b - a, t, a); }

// lerpf on both components of a complex pair at once: one packed
// subtraction and one packed FMA (sub.rn / fma.rn per lane, so each
// component equals lerpf's bit for bit) in two issue slots instead of four.
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float t) {
  unsigned long long av, bv, tv, d, r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(av) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(bv) : "f"(b.x), "f"(b.y));
  asm("mov.b64 %0, {%1, %1};" : "=l"(tv) : "f"(t));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(bv), "l"(av));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(d), "l"(tv), "l"(av));
  float2 out;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(out.x), "=f"(out.y) : "l"(r));
  return out;
}

__device__ __forceinline__ float half_round(float v) { return __half2float(__float2half_rn(v)); }

// Fire-and-forget FP32 reductions in L2 (no return value).
// Splits a flat index into (x, row, plane) of rows of `row` elements and
// planes of `plane` elements: 32-bit divisions when the index space stays
// below 2^31 (every slice, volume and P grid in practice), 64-bit otherwise.
__device__ __forceinline__ void split_index(int64_t id, int row, int64_t plane, int64_t total, int& x, int& y,
                                            int& z) {
  if (total < 0x7fffffffLL) {
    const int i = (int)id, pl = (int)plane;
    const int r = i % pl;
    x = r % row;
    y = r / row;
    z = i / pl;
  } else {
    const int64_t r = id % plane;
    x = (int)(r % row);
    y = (int)(r / row);
    z = (int)(id / plane);
  }
}

__device__ __forceinline__ void red_add(float* p, float a) {
  asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(p), "f"(a) : "memory");
}
__device__ __forceinline__ void red_add2(float* p, float a, float b) {
  asm volatile("red.relaxed.gpu.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b)
               : "memory");
}
__device__ __forceinline__ void red_add4(float* p, float a, float b, float c, float d) {
  asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a),
               "f"(b), "f"(c), "f"(d)
               : "memory");
}

// Copies host-built matrices to stream-ordered scratch, runs fn, frees.
template <class Fn>
inline int with_device_matrices(const float* h_angles, float supersample, unsigned batch,
                                cudaStream_t stream, Fn fn) {
  if (batch == 0) return fn((const float*)nullptr);
  if (!h_angles) return set_error(GTOMRLN_ERR_INVALID, "h_angles is NULL");
  const size_t count = 9 * (size_t)batch;
  void* d = nullptr;
  int st = pool_alloc(&d, count * sizeof(float), stream);
  if (st) return st;
  cudaError_t e = upload_host_floats((float*)d, count, stream,
                                     [&](float* h) { matrices_from_angles(h_angles, supersample, batch, h); });
  if (e != cudaSuccess) {
    pool_free(d, stream);
    return set_error(GTOMRLN_ERR_CUDA, "matrix upload failed: %s", cudaGetErrorString(e));
  }
  st = fn((const float*)d);
  int st2 = pool_free(d, stream);
  if (!st) st = st2;
  return st;
}

// The h_angles overloads of the shifted projector / backprojector
// (ProjectShifted.cu:32-56, BackprojectShifted.cu:11-35): matrices as above,
// shifts scaled to radians per pixel, shift * 2 pi / n in float, and the
// global weights, uploaded together; fn(d_matrices, d_shifts, d_weights).
template <class Fn>
inline int with_device_shifted(const float* h_angles, const float* h_shifts, const float* h_weights,
                               float supersample, int n, unsigned batch, cudaStream_t stream, Fn fn) {
  if (batch == 0) return fn((const float*)nullptr, (const float*)nullptr, (const float*)nullptr);
  if (!h_angles || !h_shifts || !h_weights)
    return set_error(GTOMRLN_ERR_INVALID, "h_angles, h_shifts or h_globalweights is NULL");
  const size_t count = 13 * (size_t)batch;
  void* d = nullptr;
  int st = pool_alloc(&d, count * sizeof(float), stream);
  if (st) return st;
  cudaError_t e = upload_host_floats((float*)d, count, stream, [&](float* hm) {
    matrices_from_angles(h_angles, supersample, batch, hm);
    float* sh = hm + 9 * (size_t)batch;
    const float two_pi = 6.28318530717958647692f;
    for (unsigned i = 0; i < 3 * batch; i++) sh[i] = h_shifts[i] * two_pi / (float)n;
    for (unsigned i = 0; i < batch; i++) sh[3 * batch + i] = h_weights[i];
  });
  if (e != cudaSuccess) {
    pool_free(d, stream);
    return set_error(GTOMRLN_ERR_CUDA, "upload of matrices and shifts failed: %s", cudaGetErrorString(e));
  }
  const float* dm = (const float*)d;
  st = fn(dm, dm + 9 * (size_t)batch, dm + 12 * (size_t)batch);
  int st2 = pool_free(d, stream);
  if (!st) st = st2;
  return st;
}

}  // namespace gtomrln
