// Per-sample arithmetic of the projector and backprojector, shared by the
// direct kernels, the brick kernels and the brick plan so that all of them
// see bit-identical positions, base voxels and weights.
#pragma once

#include "common.cuh"

namespace gtomrln {

// Projector (src/Relion/Project.cu:118-152): sample position M (x, y, z),
// Friedel flip when pos.x < -1e-5, base voxel (signed, before wrapping) and
// the interpolation fractions.
struct ProjSample {
  int x0, y0, z0;
  float fx, fy, fz, sign;
};

__device__ __forceinline__ ProjSample project_sample(const float* m, int x, int y, int z) {
  float3 pos = mat_apply(m, (float)x, (float)y, (float)z);
  ProjSample s;
  s.sign = 1.f;
  if (pos.x < -1e-5f) {
    pos.x = fabsf(pos.x);
    pos.y = -pos.y;
    pos.z = -pos.z;
    s.sign = -1.f;
  }
  float fx0 = floorf(pos.x + 1e-5f), fy0 = floorf(pos.y), fz0 = floorf(pos.z);
  s.x0 = (int)fx0;
  s.y0 = (int)fy0;
  s.z0 = (int)fz0;
  s.fx = pos.x - fx0;
  s.fy = pos.y - fy0;
  s.fz = pos.z - fz0;
  return s;
}

// Trilinear interpolation of the eight corner values (cutil lerp order:
// x, then y, then z; Project.cu:163-173).
__device__ __forceinline__ float2 trilerp(const ProjSample& s, float2 d000, float2 d001, float2 d010,
                                          float2 d011, float2 d100, float2 d101, float2 d110,
                                          float2 d111) {
  // each lerp2 is lerpf on the real and the imaginary part
  const float2 x00 = lerp2(d000, d001, s.fx), x01 = lerp2(d010, d011, s.fx);
  const float2 x10 = lerp2(d100, d101, s.fx), x11 = lerp2(d110, d111, s.fx);
  const float2 xy0 = lerp2(x00, x01, s.fy), xy1 = lerp2(x10, x11, s.fy);
  const float2 v = lerp2(xy0, xy1, s.fz);
  return make_float2(v.x, v.y * s.sign);
}

// Backprojector (src/Relion/Backproject.cu:194-238): base neighbour of the
// rotated (magnified, curved) position q and the eight binary16-rounded
// trilinear weights, in the reference's neighbour order
// (x0,y0,z0) (x1,y0,z0) (x0,y1,z0) (x1,y1,z0) (x0,y0,z1) ... (x1,y1,z1).
struct BpSample {
  int x0, y0, z0;
  float w[8];
};

__device__ __forceinline__ BpSample backproject_sample(const float* m, float qx, float qy, float qz) {
  float3 pos = mat_apply(m, qx, qy, qz);
  BpSample s;
  s.x0 = (short)floorf(pos.x + 1e-5f);
  s.y0 = (short)floorf(pos.y);
  s.z0 = (short)floorf(pos.z);
  float fx = pos.x - (float)s.x0, fy = pos.y - (float)s.y0, fz = pos.z - (float)s.z0;
  float c0 = 1.f - fz, c1 = fz;
  float c00 = half_round((1.f - fy) * c0), c10 = half_round(fy * c0);
  float c01 = half_round((1.f - fy) * c1), c11 = half_round(fy * c1);
  s.w[0] = half_round((1.f - fx) * c00); s.w[1] = half_round(fx * c00);
  s.w[2] = half_round((1.f - fx) * c10); s.w[3] = half_round(fx * c10);
  s.w[4] = half_round((1.f - fx) * c01); s.w[5] = half_round(fx * c01);
  s.w[6] = half_round((1.f - fx) * c11); s.w[7] = half_round(fx * c11);
  return s;
}

// Visits the targets of a backprojector sample in the reference's order:
// for each neighbour i, its own target (mirrored to -n with conjugation when
// n.x < 0; Backproject.cu:253-259), then, if n.x == 0 and (n.y, n.z) != 0,
// the second insertion at (0, -n.y, -n.z), conjugated (Backproject.cu:289-319).
// visit(i, x, y, z, conj) gets signed coordinates (before decentring).
template <class Visit>
__device__ __forceinline__ void for_each_target(int x0, int y0, int z0, Visit&& visit) {
#pragma unroll
  for (int i = 0; i < 8; i++) {
    int nx = x0 + (i & 1), ny = y0 + ((i >> 1) & 1), nz = z0 + ((i >> 2) & 1);
    if (nx < 0)
      visit(i, -nx, -ny, -nz, true);
    else
      visit(i, nx, ny, nz, false);
    if (nx == 0 && (ny != 0 || nz != 0)) visit(i, 0, -ny, -nz, true);
  }
}

}  // namespace gtomrln
