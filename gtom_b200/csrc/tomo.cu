// Tomographic gather-insertion: the B200 replacement of gtom::d_BackprojectTomo
// (include/Relion.cuh:13-14, src/Relion/BackprojectTomo.cu:11-153).
//
// Every voxel of the half-complex volume inside rmax gathers from every
// slice whose plane passes within 5 voxels of it, with a Lanczos-5
// (windowed sinc) weight per axis of the distance between the voxel and
// each pixel's rotated position (Friedel-mirrored with conjugation when its
// x is negative); the voxel becomes sum(w * value) / sum(w * weight), scaled
// by the total kernel weight clamped to [-1, 1], and is written only where
// that total exceeds 1e-3 in magnitude.  The reference tests every pixel of
// every slice for every voxel (voxels x slices x pixels); here a voxel only
// visits the pixels of a window around its position in the slice's frame
// (and around the mirrored position), the only ones whose distance can pass
// the reference's per-axis test, and applies that same test and arithmetic
// to them.  One thread per voxel; the sums differ from the reference's only
// in the order of the additions.
#include <cmath>

#include "common.cuh"

namespace gtomrln {

namespace {

constexpr float kTomoReach = 5.f;   // the reference's per-axis window and plane distance
constexpr float kTomoReachDiag = 8.6602540378f;  // 5 * sqrt(3): reach along any direction

// The reference is built with fast math (-use_fast_math; FastMath in its
// Release configuration): its sine is the fast sine and its FP32 division the
// full-range approximate one, div.full.f32, used here as well.
__device__ __forceinline__ float fast_div(float a, float b) {
  float r;
  asm("div.full.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

__device__ __forceinline__ float tomo_sinc(float x) {  // DeviceFunctions.cuh:11-17
  if (fabsf(x) <= 1e-4f) return 1.f;
  const float pi = 3.14159265358979323846f;
  return fast_div(__sinf(x * pi), x * pi);
}

// glm mat3 * vec3 and transpose(mat3) * vec3, column-major m[c*3 + r].
__device__ __forceinline__ float3 tomo_apply(const float* m, float x, float y, float z) {
  return mat_apply(m, x, y, z);
}
__device__ __forceinline__ float3 tomo_apply_t(const float* m, float x, float y, float z) {
  return make_float3(fmaf(m[2], z, fmaf(m[0], x, m[1] * y)), fmaf(m[5], z, fmaf(m[3], x, m[4] * y)),
                     fmaf(m[8], z, fmaf(m[6], x, m[7] * y)));
}

__global__ void tomo_kernel(float2* __restrict__ vol, int vx, int vy, int vz, const float2* __restrict__ proj,
                            const float* __restrict__ projw, int n, const float* __restrict__ mats, int batch,
                            float rmax) {
  const int rowlen = vx / 2 + 1;
  const int64_t nvox = (int64_t)rowlen * vy * vz;
  const int dimft = n / 2 + 1;
  const int64_t elements = (int64_t)dimft * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i % rowlen);
    const int iy = (int)((i / rowlen) % vy), iz = (int)(i / ((int64_t)rowlen * vy));
    const float px = (float)ix;
    const float py = (float)(iy < vx / 2 ? iy : iy - vx);
    const float pz = (float)(iz < vx / 2 ? iz : iz - vx);
    if (sqrtf(fmaf(px, px, fmaf(py, py, pz * pz))) >= rmax) continue;
    float vre = 0.f, vim = 0.f, wsum = 0.f, ssum = 0.f;
    for (int b = 0; b < batch; b++) {
      float m[9];
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = __ldg(mats + 9 * (int64_t)b + k);
      const float3 local = tomo_apply_t(m, px, py, pz);  // the voxel in the slice's frame (times s^2)
      if (fabsf(local.z) > kTomoReach) continue;
      // M = s R: a pixel within reach lies within 5 sqrt(3) / s of R^T v / s = local / s^2
      const float s2 = fmaf(m[0], m[0], fmaf(m[1], m[1], m[2] * m[2]));
      const float inv_s2 = 1.f / s2;
      const int reach = (int)ceilf(kTomoReachDiag * rsqrtf(s2)) + 1;
      // pixels near the voxel's position (direct) and near its mirror
      // (pixels whose position has x < 0 are flipped onto the voxel)
#pragma unroll 1
      for (int side = 0; side < 2; side++) {
        const float cx = (side ? -local.x : local.x) * inv_s2, cy = (side ? -local.y : local.y) * inv_s2;
        const int x0 = max(0, (int)floorf(cx) - reach), x1 = min(n / 2, (int)ceilf(cx) + reach);
        const int y0 = max(-n / 2 + 1, (int)floorf(cy) - reach), y1 = min(n / 2, (int)ceilf(cy) + reach);
        for (int y = y0; y <= y1; y++) {
          const int idy = y < 0 ? y + n : y;
          for (int x = x0; x <= x1; x++) {
            float3 pos = tomo_apply(m, (float)x, (float)y, 0.f);
            const bool neg = pos.x < 0.f;
            if (neg != (side == 1)) continue;  // each pixel counted on its own side only
            if (neg) {
              pos.x = -pos.x;
              pos.y = -pos.y;
              pos.z = -pos.z;
            }
            const float dx = px - pos.x, dy = py - pos.y, dz = pz - pos.z;
            if (fabsf(dx) > kTomoReach || fabsf(dy) > kTomoReach || fabsf(dz) > kTomoReach) continue;
            const float sample = tomo_sinc(dx) * tomo_sinc(fast_div(dx, kTomoReach)) *
                                 (tomo_sinc(dy) * tomo_sinc(fast_div(dy, kTomoReach))) *
                                 (tomo_sinc(dz) * tomo_sinc(fast_div(dz, kTomoReach)));
            const int64_t id = (int64_t)idy * dimft + x;
            ssum += sample;
            wsum += sample * __ldg(projw + elements * b + id);
            float2 v = __ldg(proj + elements * b + id);
            vre = fmaf(sample, v.x, vre);
            vim = fmaf(sample, neg ? -v.y : v.y, vim);
          }
        }
      }
    }
    if (fabsf(ssum) > 1e-3f) {
      const float scale = fminf(1.f, fmaxf(-1.f, ssum));
      vol[i] = make_float2(vre / wsum * scale, vim / wsum * scale);
    }
  }
}

}  // namespace
}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_backproject_tomo(float* d_volumeft, int vx, int vy, int vz, const float* d_projft,
                             const float* d_projweights, int px, int py, int pz, unsigned rmax,
                             const float* d_matrices, unsigned batch, void* stream) {
  clear_error();
  if (dimension_count(vx, vy, vz) < dimension_count(px, py, pz))
    return set_error(GTOMRLN_ERR_INVALID, "backproject_tomo: volume has fewer dimensions than the slices (reference throws)");
  if (vx <= 0 || vy != vx || vz != vx || px <= 0)
    return set_error(GTOMRLN_ERR_INVALID, "backproject_tomo: the volume must be cubic (the reference indexes it so)");
  if (batch == 0) return GTOMRLN_OK;
  if (!d_volumeft || !d_projft || !d_projweights || !d_matrices)
    return set_error(GTOMRLN_ERR_INVALID, "backproject_tomo: NULL pointer");
  if (rmax > (unsigned)(vx / 2)) rmax = vx / 2;
  int64_t nvox = (int64_t)(vx / 2 + 1) * vy * vz;
  unsigned blocks = (unsigned)std::min<int64_t>((nvox + 127) / 128, 148 * 64);
  tomo_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>((float2*)d_volumeft, vx, vy, vz, (const float2*)d_projft,
                                                        d_projweights, px, d_matrices, (int)batch, (float)rmax);
  GTOMRLN_LAUNCH_CHECK("tomo_kernel");
  return GTOMRLN_OK;
}

int gtomrln_backproject_tomo_angles(float* d_volumeft, int vx, int vy, int vz, const float* d_projft,
                                    const float* d_projweights, int px, int py, int pz, unsigned rmax,
                                    const float* h_angles, unsigned batch, void* stream) {
  clear_error();
  return with_device_matrices(h_angles, 1.0f, batch, (cudaStream_t)stream, [&](const float* d_m) {
    return gtomrln_backproject_tomo(d_volumeft, vx, vy, vz, d_projft, d_projweights, px, py, pz, rmax, d_m, batch,
                                    stream);
  });
}

}  // extern "C"
