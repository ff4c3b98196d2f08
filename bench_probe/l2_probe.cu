// Roofline denominators that the driver's peak file does not hold, measured
// on the device the benchmark runs on:
//   * L2 FP32 reduction rate: fire-and-forget red.global.add to random
//     addresses of an L2-resident buffer (scalar, .v2 and .v4 forms),
//   * L2 -> SM gather bandwidth: random 8-byte loads from an L2-resident
//     buffer, the access pattern of the projector's corner fetches,
//   * shared-memory update rates (FP32 / int32 / int64 atomics, plain
//     read-add-write) and the CUDA cores' FP32 FMA rate.
// Bench-only: bench.py builds it into bench_probe/libbench_probe.so; the
// product library (gtom_b200/) neither contains nor loads it.
#include <cuda_runtime.h>
#include <cstdint>

namespace {

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

template <int VEC>
__global__ void red_probe_kernel(float* __restrict__ buf, uint32_t mask_vec, int iters) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t h = hash32(t * 2654435761U + 12345U);
  for (int i = 0; i < iters; i++) {
    h = hash32(h + (uint32_t)i);
    float* p = buf + (size_t)(h & mask_vec) * VEC;
    if (VEC == 1)
      asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(p), "f"(1.0f) : "memory");
    else if (VEC == 2)
      asm volatile("red.relaxed.gpu.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(1.0f), "f"(1.0f)
                   : "memory");
    else
      asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(1.0f),
                   "f"(1.0f), "f"(1.0f), "f"(1.0f)
                   : "memory");
  }
}

__global__ void gather_probe_kernel(const float2* __restrict__ buf, uint32_t mask, int iters,
                                    float* __restrict__ sink) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t h = hash32(t * 2654435761U + 777U);
  float acc = 0.f;
  for (int i = 0; i < iters; i += 8) {
    float2 v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      h = hash32(h + (uint32_t)(i + k));
      v[k] = __ldg(buf + (h & mask));
    }
#pragma unroll
    for (int k = 0; k < 8; k++) acc += v[k].x + v[k].y;
  }
  if (acc == 123.456f) sink[t] = acc;  // keeps the loads alive
}

// Shared-memory update rate: every thread adds to pseudo-random words of a
// 12K-word (48 KB) array.  mode 0: FP32 atomicAdd, 1: int32 atomicAdd,
// 2: plain FP32 read-add-write (no atomicity), 3: int64 atomicAdd,
// 4: FP32 red.shared.add (no returned value).
template <int MODE>
__global__ void smem_probe_kernel(float* __restrict__ sink, int iters) {
  __shared__ float s[12288];
  for (int i = threadIdx.x; i < 12288; i += blockDim.x) s[i] = 0.f;
  __syncthreads();
  uint32_t h = hash32(blockIdx.x * blockDim.x + threadIdx.x);
  for (int i = 0; i < iters; i++) {
    h = h * 1664525u + 1013904223u;
    uint32_t k = (h >> 8) % (MODE == 3 ? 6144u : 12288u);
    if (MODE == 0) atomicAdd(s + k, 1.0f);
    if (MODE == 1) atomicAdd((int*)s + k, 1);
    if (MODE == 2) s[k] += 1.0f;
    if (MODE == 3) atomicAdd((unsigned long long*)s + k, 1ull);
    if (MODE == 4) {  // explicit reduction (no returned value)
      const unsigned a = (unsigned)__cvta_generic_to_shared(s + k);
      asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a), "f"(1.0f) : "memory");
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) sink[blockIdx.x] = s[blockIdx.x % 12288];
}

// FP32 FMA rate of the CUDA cores: eight independent chains per thread
// (enough to cover the FMA latency at full occupancy).
__global__ void fma_probe_kernel(float* __restrict__ sink, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = fmaf(x[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == 123.456f) sink[blockIdx.x] = s;  // keeps the chains alive
}

// The packed form: eight independent chains of fma.rn.f32x2 (two FMAs per
// instruction) per thread.
__global__ void fma2_probe_kernel(float* __restrict__ sink, int iters, float a, float b) {
  unsigned long long x[8];
  const float2 av = make_float2(a, a), bv = make_float2(b, b);
  const unsigned long long A = *reinterpret_cast<const unsigned long long*>(&av);
  const unsigned long long Bv = *reinterpret_cast<const unsigned long long*>(&bv);
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const float2 v = make_float2((float)(threadIdx.x + k) * 1e-3f, (float)k);
    x[k] = *reinterpret_cast<const unsigned long long*>(&v);
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[k]) : "l"(A), "l"(Bv));
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const float2 v = *reinterpret_cast<const float2*>(&x[k]);
    s += v.x + v.y;
  }
  if (s == 123.456f) sink[blockIdx.x] = s;
}

}  // namespace

extern "C" {

__attribute__((visibility("default")))
// Returns FP32 FLOP/s of packed f32x2 fused multiply-adds (4 per instruction).
double gtomrln_probe_fp32x2_fma(int blocks, int threads, int iters) {
  float* sink = nullptr;
  if (cudaMalloc(&sink, (size_t)blocks * sizeof(float)) != cudaSuccess) return -1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  fma2_probe_kernel<<<blocks, threads>>>(sink, iters, 0.999f, 1e-3f);
  cudaEventRecord(a);
  fma2_probe_kernel<<<blocks, threads>>>(sink, iters, 0.999f, 1e-3f);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return -(double)e;
  return 4.0 * 8.0 * (double)blocks * threads * iters / (ms * 1e-3);
}

__attribute__((visibility("default")))
// Returns FP32 FLOP/s of fused multiply-adds (2 per FMA) over the whole device.
double gtomrln_probe_fp32_fma(int blocks, int threads, int iters) {
  float* sink = nullptr;
  if (cudaMalloc(&sink, (size_t)blocks * sizeof(float)) != cudaSuccess) return -1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  fma_probe_kernel<<<blocks, threads>>>(sink, iters, 0.999f, 1e-3f);
  cudaEventRecord(a);
  fma_probe_kernel<<<blocks, threads>>>(sink, iters, 0.999f, 1e-3f);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return -(double)e;
  return 2.0 * 8.0 * (double)blocks * threads * iters / (ms * 1e-3);
}

__attribute__((visibility("default")))
// Returns shared-memory updates per second over the whole device.
double gtomrln_probe_smem_update(int mode, int blocks, int threads, int iters) {
  float* sink = nullptr;
  if (cudaMalloc(&sink, (size_t)blocks * sizeof(float)) != cudaSuccess) return -1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  auto launch = [&]() {
    if (mode == 0) smem_probe_kernel<0><<<blocks, threads>>>(sink, iters);
    else if (mode == 1) smem_probe_kernel<1><<<blocks, threads>>>(sink, iters);
    else if (mode == 2) smem_probe_kernel<2><<<blocks, threads>>>(sink, iters);
    else if (mode == 3) smem_probe_kernel<3><<<blocks, threads>>>(sink, iters);
    else smem_probe_kernel<4><<<blocks, threads>>>(sink, iters);
  };
  launch();
  cudaEventRecord(a);
  launch();
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return -(double)e;
  return (double)blocks * threads * iters / (ms * 1e-3);
}

__attribute__((visibility("default")))
// Returns FP32 additions per second (vec * reductions), or a negative CUDA error.
double gtomrln_probe_l2_red(int vec, int log2_bytes, int blocks, int threads, int iters) {
  size_t bytes = (size_t)1 << log2_bytes;
  float* buf = nullptr;
  if (cudaMalloc(&buf, bytes) != cudaSuccess) return -1;
  cudaMemset(buf, 0, bytes);
  uint32_t nvec = (uint32_t)(bytes / (4 * vec));
  uint32_t mask = nvec - 1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  auto launch = [&]() {
    if (vec == 1) red_probe_kernel<1><<<blocks, threads>>>(buf, mask, iters);
    else if (vec == 2) red_probe_kernel<2><<<blocks, threads>>>(buf, mask, iters);
    else red_probe_kernel<4><<<blocks, threads>>>(buf, mask, iters);
  };
  launch();  // warm-up
  cudaEventRecord(a);
  launch();
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(buf);
  if (e != cudaSuccess) return -(double)e;
  return (double)blocks * threads * iters * vec / (ms * 1e-3);
}

__attribute__((visibility("default")))
// Returns bytes per second of random 8-byte gathers from a buffer of 2^log2_bytes.
double gtomrln_probe_l2_gather(int log2_bytes, int blocks, int threads, int iters) {
  size_t bytes = (size_t)1 << log2_bytes;
  float2* buf = nullptr;
  float* sink = nullptr;
  if (cudaMalloc(&buf, bytes) != cudaSuccess) return -1;
  if (cudaMalloc(&sink, (size_t)blocks * threads * sizeof(float)) != cudaSuccess) {
    cudaFree(buf);
    return -1;
  }
  cudaMemset(buf, 0, bytes);
  uint32_t mask = (uint32_t)(bytes / 8) - 1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  gather_probe_kernel<<<blocks, threads>>>(buf, mask, iters, sink);
  cudaEventRecord(a);
  gather_probe_kernel<<<blocks, threads>>>(buf, mask, iters, sink);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(buf);
  cudaFree(sink);
  if (e != cudaSuccess) return -(double)e;
  return (double)blocks * threads * iters * 8.0 / (ms * 1e-3);
}

}  // extern "C"
