// Per-voxel MLP that predicts the gridding correction (the converged
// Fnewweight of the iterative gridding) from the local sampling weights.
//
// Input (28): the log of the 27 sampling weights of the 3x3x3 neighbourhood
// on the padded half-Fourier grid, divided by the distribution's weight
// scale s (the mean of the non-zero weights inside the gridding sphere),
//   f_k = log(Fw[neighbour k] / s + 1e-6),  k = (dz+1)*9 + (dy+1)*3 + (dx+1),
// and the normalised radius |(x, y, z)| / (P/2).  The neighbour at x = -1 of
// a voxel on the x = 0 plane is the Hermitian mate (1, -y, -z) of the
// half-volume, y and z wrap periodically.  Each input is standardised by a
// fixed affine map stored with the parameters (shift, scale).
// Network: 28 -> 64 (ReLU) -> 64 (ReLU) -> 1, FP32, no tensor cores.
// Output: log(Fnewweight * s); the predicted start is exp(out) / s.
//
// Parameter block (floats, one contiguous array):
//   [0, 28)       input shift       (not trained)
//   [28, 56)      input scale       (not trained)
//   [56, 1848)    W1, 64 rows of 28 (row j feeds hidden unit j)
//   [1848, 1912)  b1
//   [1912, 6008)  W2, 64 rows of 64
//   [6008, 6072)  b2
//   [6072, 6136)  W3
//   [6136]        b3
// Gradients and the Adam moments use the same indexing.
#pragma once

#include <cstdint>

namespace gtomrln {

constexpr int kMlpIn = 28;
constexpr int kMlpHidden = 64;
constexpr int kMlpOffShift = 0;
constexpr int kMlpOffScale = kMlpIn;
constexpr int kMlpOffW1 = 2 * kMlpIn;
constexpr int kMlpOffB1 = kMlpOffW1 + kMlpHidden * kMlpIn;
constexpr int kMlpOffW2 = kMlpOffB1 + kMlpHidden;
constexpr int kMlpOffB2 = kMlpOffW2 + kMlpHidden * kMlpHidden;
constexpr int kMlpOffW3 = kMlpOffB2 + kMlpHidden;
constexpr int kMlpOffB3 = kMlpOffW3 + kMlpHidden;
constexpr int kMlpParams = kMlpOffB3 + 1;
constexpr float kMlpWeightFloor = 1e-6f;
static_assert(kMlpOffW1 % 4 == 0 && kMlpOffW2 % 4 == 0 && kMlpIn % 4 == 0, "float4 rows");

// Index of the stored half-volume element for the neighbour (x+dx, y+dy,
// z+dz) of voxel (x, y, z) on the decentred (P/2+1) x P x P grid.
__device__ __forceinline__ int64_t mlp_neighbour_index(int P, int x, int y, int z, int dx, int dy,
                                                       int dz) {
  int xx = x + dx, yy = y + dy, zz = z + dz;
  if (xx < 0) {  // Hermitian mate across the x = 0 plane
    xx = -xx;
    yy = -yy;
    zz = -zz;
  }
  yy = yy < 0 ? yy + P : (yy >= P ? yy - P : yy);
  zz = zz < 0 ? zz + P : (zz >= P ? zz - P : zz);
  xx = xx > P / 2 ? P / 2 : xx;
  return ((int64_t)zz * P + yy) * (P / 2 + 1) + xx;
}

// Raw (unstandardised) features of voxel (x, y, z).
__device__ __forceinline__ void mlp_voxel_features(const float* __restrict__ fw, int P,
                                                   float inv_scale, int x, int y, int z,
                                                   float* f) {
  int k = 0;
#pragma unroll
  for (int dz = -1; dz <= 1; dz++)
#pragma unroll
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll
      for (int dx = -1; dx <= 1; dx++) {
        float w = __ldg(fw + mlp_neighbour_index(P, x, y, z, dx, dy, dz));
        f[k++] = logf(w * inv_scale + kMlpWeightFloor);
      }
  int yp = y < P / 2 + 1 ? y : y - P;
  int zp = z < P / 2 + 1 ? z : z - P;
  f[27] = sqrtf((float)(x * x + yp * yp + zp * zp)) / (float)(P / 2);
}

// Standardises raw features f into xin.
__device__ __forceinline__ void mlp_standardise(const float* __restrict__ p, const float* f,
                                                float* xin) {
#pragma unroll
  for (int i = 0; i < kMlpIn; i++) xin[i] = (f[i] - p[kMlpOffShift + i]) * p[kMlpOffScale + i];
}

// First layer: h1 = relu(W1 xin + b1), four hidden units at a time so that
// four accumulation chains are in flight.  p: the parameter block (shared
// memory in the kernels).
__device__ __forceinline__ void mlp_layer1(const float* __restrict__ p, const float* xin,
                                           float* h1) {
#pragma unroll
  for (int j = 0; j < kMlpHidden; j += 4) {
    const float4* w = reinterpret_cast<const float4*>(p + kMlpOffW1 + j * kMlpIn);
    float a0 = p[kMlpOffB1 + j], a1 = p[kMlpOffB1 + j + 1];
    float a2 = p[kMlpOffB1 + j + 2], a3 = p[kMlpOffB1 + j + 3];
#pragma unroll
    for (int i = 0; i < kMlpIn / 4; i++) {
      float4 q0 = w[i], q1 = w[i + kMlpIn / 4], q2 = w[i + 2 * (kMlpIn / 4)], q3 = w[i + 3 * (kMlpIn / 4)];
      float x0 = xin[4 * i], x1 = xin[4 * i + 1], x2 = xin[4 * i + 2], x3 = xin[4 * i + 3];
      a0 = fmaf(q0.x, x0, a0); a0 = fmaf(q0.y, x1, a0); a0 = fmaf(q0.z, x2, a0); a0 = fmaf(q0.w, x3, a0);
      a1 = fmaf(q1.x, x0, a1); a1 = fmaf(q1.y, x1, a1); a1 = fmaf(q1.z, x2, a1); a1 = fmaf(q1.w, x3, a1);
      a2 = fmaf(q2.x, x0, a2); a2 = fmaf(q2.y, x1, a2); a2 = fmaf(q2.z, x2, a2); a2 = fmaf(q2.w, x3, a2);
      a3 = fmaf(q3.x, x0, a3); a3 = fmaf(q3.y, x1, a3); a3 = fmaf(q3.z, x2, a3); a3 = fmaf(q3.w, x3, a3);
    }
    h1[j] = fmaxf(a0, 0.f);
    h1[j + 1] = fmaxf(a1, 0.f);
    h1[j + 2] = fmaxf(a2, 0.f);
    h1[j + 3] = fmaxf(a3, 0.f);
  }
}

// Pre-activation of second-layer unit j: b2[j] + W2[j] . h1.
__device__ __forceinline__ float mlp_layer2_unit(const float* __restrict__ p, const float* h1,
                                                 int j) {
  const float4* w = reinterpret_cast<const float4*>(p + kMlpOffW2 + j * kMlpHidden);
  float a0 = p[kMlpOffB2 + j], a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
  for (int k = 0; k < kMlpHidden / 4; k++) {
    float4 q = w[k];
    a0 = fmaf(q.x, h1[4 * k], a0);
    a1 = fmaf(q.y, h1[4 * k + 1], a1);
    a2 = fmaf(q.z, h1[4 * k + 2], a2);
    a3 = fmaf(q.w, h1[4 * k + 3], a3);
  }
  return (a0 + a1) + (a2 + a3);
}

// Network output for raw features f.
__device__ __forceinline__ float mlp_forward(const float* __restrict__ p, const float* f) {
  float xin[kMlpIn];
  mlp_standardise(p, f, xin);
  float h1[kMlpHidden];
  mlp_layer1(p, xin, h1);
  float out = p[kMlpOffB3];
#pragma unroll 1
  for (int j = 0; j < kMlpHidden; j++)
    out = fmaf(p[kMlpOffW3 + j], fmaxf(mlp_layer2_unit(p, h1, j), 0.f), out);
  return out;
}

// Host launcher (mlp.cu): writes the predicted gridding start for every
// voxel of the decentred half grid of P: 0 outside the sphere r^2 < maskr2,
// 1 where Fw = 0 inside it (the cold value), exp(out) / s elsewhere, with
// the x = 0 plane made Hermitian-symmetric (both mates get the geometric
// mean of their two starts, exp(mean of the outputs) / s).  s is read on
// the device from scale_sums = {sum of Fw, count} over the sphere's
// non-zero weights (mlp_weight_scale).  Also writes convft = Fw * start as
// the first iteration's input spectrum.
int mlp_predict_start(const float* d_params, const float* Fw, int P, int maskr2,
                      const double* scale_sums, float* Fnw, float2* convft, cudaStream_t stream);

// Accumulates {sum of Fw, count of Fw > 0} over r^2 < maskr2 into sums[2]
// (the caller zeroes them).
int mlp_weight_scale(const float* Fw, int P, int maskr2, double* sums, cudaStream_t stream);

}  // namespace gtomrln
