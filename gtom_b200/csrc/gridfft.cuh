// Pieces of the gridding reconstructor shared by its cuFFT path
// (gridding.cu) and its fused FFT path (gridfft.cu): the P-grid geometry,
// the blob lookup, and the per-voxel weight updates.
#pragma once

#include "common.cuh"

namespace gtomrln {

constexpr int kBlobSamples = 10000;

struct GridGeom {
  int P;         // padded working grid
  int rowlen;    // P/2 + 1
  int64_t nc;    // rowlen * P * P complex elements
  int64_t nr;    // P^3 real elements
};

// The reference's gridding is compiled with fast math (-use_fast_math,
// CMakeLists.txt:36): its FP32 square root is the approximate one and its
// FP32 division the full-range approximate one, both flushing denormals.
// The gridding kernels here use the same instructions for the reference's
// blob radius and weight update.
__device__ __forceinline__ float grid_sqrt(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float grid_div(float a, float b) {
  float r;
  asm("div.full.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// PrecomputeBlobKernel's table index (RecFourier.cu:243-262) at real-space
// voxel (x, y, z) of the P grid, the radius evaluated as the reference's
// build does: sqrt(xp^2 + yp^2 + zp^2) / P / funcsampling with its fast-math
// square root and divisions (the squares are integers below 2^24, exact in
// FP32 however they are summed).
__device__ __forceinline__ int grid_blob_index_sq(float r2, float P, float funcsampling) {
  const int ti = (int)grid_div(grid_div(grid_sqrt(r2), P), funcsampling);
  return ti < kBlobSamples - 1 ? ti : kBlobSamples - 1;
}
__device__ __forceinline__ int grid_blob_index(int P, int x, int y, int z, float funcsampling) {
  const int zp = z < P / 2 ? z : z - P;
  const int yp = y < P / 2 ? y : y - P;
  const float xp = (float)(x < P / 2 ? x : x - P);
  return grid_blob_index_sq(xp * xp + (float)(yp * yp) + (float)(zp * zp), (float)P, funcsampling);
}

// The table value there, read from global memory.  Lanes at consecutive x
// read entries ~20000/P apart, one cache line each: kernels that stream
// many voxels stage the table in shared memory and use grid_blob_index.
__device__ __forceinline__ float grid_blob_at(const float* __restrict__ table, int P, int x, int y, int z,
                                              float funcsampling) {
  return __ldg(table + grid_blob_index(P, x, y, z, funcsampling));
}

// Iteration2Kernel (RecFourier.cu:293-308) for one voxel: the new
// Fnewweight from the real part c of the convolved spectrum (the division
// as the reference's fast-math build does it).
__device__ __forceinline__ float grid_update_value(float c, float old) {
  const float w = fmaxf(1e-4f, c);
  return fminf(1e20f, grid_div(old, w));
}

// The same update applied at the extrapolated point v (momentum in the
// logarithm of the weights): nw = min(1e20, v / max(1e-4, c)) and the next
// extrapolation ext = min(1e20, nw (nw / old)^beta).  The extrapolation is a
// heuristic of this library (its fixed points are the plain update's), so
// its power runs on the fast intrinsics (__fdividef, __powf: relative error
// ~1e-6 on ratios near 1); the update itself keeps the reference's division.
__device__ __forceinline__ void grid_update_momentum_value(float c, float old, float v, float beta, float& nw,
                                                           float& ext) {
  const float w = fmaxf(1e-4f, c);
  nw = fminf(1e20f, grid_div(v, w));
  ext = nw;
  if (old > 0.f && nw > 0.f) ext = fminf(1e20f, nw * __powf(__fdividef(nw, old), beta));
}

// Adds the block's (d2, o2) to change[0..1] (one atomic pair per block).
__device__ __forceinline__ void grid_change_reduce(double d2, double o2, double* change) {
  for (int off = 16; off > 0; off >>= 1) {
    d2 += __shfl_down_sync(0xffffffffu, d2, off);
    o2 += __shfl_down_sync(0xffffffffu, o2, off);
  }
  __shared__ double s[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s[0][warp] = d2;
    s[1][warp] = o2;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    d2 = lane < nw ? s[0][lane] : 0;
    o2 = lane < nw ? s[1][lane] : 0;
    for (int off = 16; off > 0; off >>= 1) {
      d2 += __shfl_down_sync(0xffffffffu, d2, off);
      o2 += __shfl_down_sync(0xffffffffu, o2, off);
    }
    if (lane == 0) {
      atomicAdd(change, d2);
      atomicAdd(change + 1, o2);
    }
  }
}

// ------------------------------------------------------- fused FFT path --
// For power-of-two grids P in [64, 512] the iteration's two 3D transforms,
// the blob multiply and the weight update run as two kernels of gridfft.cu
// (see there).  `data` is the complex working spectrum (nc per volume).

// Whether the fused path can run `count` volumes of grid P on this device.
bool gridfft_available(int P, int count);
// data <- inverse transform along z of data (before the first iteration).
int gridfft_first(float2* data, const GridGeom& g, int count, cudaStream_t stream);
// One iteration: the rest of the inverse transform, the blob multiply
// (with the in-loop 1/P^3), the forward transform and the update of Fnw
// (and V with momentum beta > 0; change accumulates the convergence sums
// when non-null); with write_next, data <- the inverse transform along z of
// Fw * Fnw (Fw * V) for the next iteration.
int gridfft_iteration(float2* data, const GridGeom& g, int count, const float* table, const float* Fw,
                      float* Fnw, float* V, float beta, bool write_next, double* change, cudaStream_t stream);

// Twiddle table e(-2 pi i m / N), m < N, on the current device (built once
// per device, context and N in double precision; freed by the library's
// cache release).
int fft_twiddles(int N, const float2** out);

// ------------------------------------------- symmetric-spectrum path --
// The iteration on the Hermitian half along z of the real spectrum
// (gridsym.cu): four passes over a (P/2+1) x P x (P/2+1) complex work array
// W (which fits in the cuFFT path's spectrum buffer).  Power-of-two grids
// P = 64 .. 512.

bool gridsym_available(int P);
// Launch attributes and twiddle table of grid P on the current device, made
// ahead of a stream capture (later calls only look them up).
int gridsym_prepare(int P);
// W <- transform along z of S = Fw * Fnw (Fw * V when V is non-null), the
// start of the loop.
int gridsym_first(float2* W, const GridGeom& g, int count, const float* Fw, float* Fnw, float* V,
                  cudaStream_t stream);
// One iteration: transforms along y, x (with the blob) and y, then along
// z with the update of Fnw (and V with momentum beta > 0); change (one
// volume) accumulates the convergence sums when non-null, and with ref also
// the distance to the reference weights ref; with write_next, W <- the
// transform along z of the next iteration's Fw * Fnw (Fw * V).
int gridsym_iteration(float2* W, const GridGeom& g, int count, const float* table, const float* Fw, float* Fnw,
                      float* V, float beta, bool write_next, double* change, const float* ref,
                      cudaStream_t stream);

}  // namespace gtomrln
