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

// One element (x, y, z) of the final spectrum, before its inverse
// transform: DecenterKernel<tcomplex> of the centred input data
// (RecFourier.cu:175-179: the masked sample of the old (oldx, oldy, oldz)
// box), times Fnewweight (RecFourier.cu:206) or divided by
// max(|Fweight|, 1e-4) when no iteration ran (RecFourier.cu:200-202), then
// d_Shift by P/2 in every axis (RecFourier.cu:213-214), the factor
// (-1)^(x+y+z).  In two steps, so that callers can issue their loads
// first: grid_final_source gives the element's index in the input box (-1:
// outside it, the value 0), grid_final_apply the value from the sample v
// and the weight w (Fw[i] when divide, else Fnw[i]; i: the element's index
// on the P grid, rows of P/2 + 1).
__device__ __forceinline__ int64_t grid_final_source(int oldx, int oldy, int oldz, int P, int x, int y, int z) {
  const int zp = z < P / 2 + 1 ? z : z - P;
  const int yp = y < P / 2 + 1 ? y : y - P;
  const int zi = zp + oldz / 2, yi = yp + oldy / 2;
  if (zi >= 0 && zi < oldz && yi >= 0 && yi < oldy && x < oldx / 2 + 1)
    return ((int64_t)zi * oldy + yi) * (oldx / 2 + 1) + x;
  return -1;
}
__device__ __forceinline__ float2 grid_final_apply(float2 v, float w, int P, int x, int y, int z, bool divide) {
  const int zp = z < P / 2 + 1 ? z : z - P;
  const int yp = y < P / 2 + 1 ? y : y - P;
  const float r = (float)(zp * zp) + (float)(yp * yp);
  const float rr = r + (float)(x * x);
  const float mask = rr < (float)(P * P / 4) ? 1.f : 0.f;
  v.x *= mask;
  v.y *= mask;
  if (divide) {
    const float inv = 1.0f / fmaxf(fabsf(w), 1e-4f);  // Arithmetics.cu:310-311
    v.x *= inv;
    v.y *= inv;
  } else {
    v.x *= w;
    v.y *= w;
  }
  if ((x + y + z) & 1) {
    v.x = -v.x;
    v.y = -v.y;
  }
  return v;
}
__device__ __forceinline__ float2 grid_final_value(const float2* __restrict__ data, int oldx, int oldy, int oldz,
                                                   const float* __restrict__ Fw, const float* __restrict__ Fnw,
                                                   int P, int x, int y, int z, int64_t i, bool divide) {
  const int64_t src = grid_final_source(oldx, oldy, oldz, P, x, y, z);
  const float2 v = src >= 0 ? __ldg(data + src) : make_float2(0.f, 0.f);
  return grid_final_apply(v, divide ? Fw[i] : Fnw[i], P, x, y, z, divide);
}

// The map value at (x, y, z) of the ori^3 output from the real grid's value
// v at its centred position: CorrectGriddingKernel's division by sinc^2(r/P)
// (RecFourier.cu:310-332) and the final scale (RecFourier.cu:237).
__device__ __forceinline__ float grid_crop_value(float v, int x, int y, int z, int ori, int P, float scale) {
  const int yy = (y - ori / 2) * (y - ori / 2);
  const int zz = (z - ori / 2) * (z - ori / 2);
  const float xx = (float)(x - ori / 2);
  const float r = sqrtf(xx * xx + (float)yy + (float)zz) / (float)P;
  if (r > 0) {
    const float s = fabsf(r) <= 1e-4f ? 1.f : sinpif(r) / (r * 3.14159265358979f);
    v /= s * s;
  }
  return v * scale;
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
// The final map: the corrected data's inverse transform (decentred and
// centred per element from the caller's centred data of box (oldx, oldy,
// oldz), volumes wstride apart; times Fnw, or divided by max(|Fw|, 1e-4)
// when divide), cropped to the central ori^3 and gridding-corrected, times
// scale, into out (or outs[volume]).  T needs (P/2+1) P ori complex
// elements per volume (it fits in the loop's W buffer).  The x = 0 and
// x = P/2 terms of each transformed row are taken as real: a spectrum whose
// x = 0 plane is not Hermitian is transformed by its Hermitian part.
int gridsym_final(float2* T, const GridGeom& g, int count, const float2* data, int oldx, int oldy, int oldz,
                  int64_t wstride, const float* Fw, const float* Fnw, bool divide, int ori, float scale, float* out,
                  float* const* outs, cudaStream_t stream);

}  // namespace gtomrln
