// Kernels of the learned gridding warm start: the per-voxel MLP's inference
// over a padded half grid, its training step (forward, backward and the
// gradient reduction in one kernel) and Adam.  The network, its inputs and
// the parameter layout are described in mlp.cuh.  The reference has no such
// component; it runs its gridding iterations from the sphere-mask start
// (src/Reconstruction/RecFourier.cu:149-150).
#include <cmath>

#include "common.cuh"
#include "mlp.cuh"

namespace gtomrln {

namespace {

constexpr int kInferThreads = 256;
constexpr int kTrainThreads = 128;  // samples per training block
constexpr int kRow = 68;            // padded row of the per-sample 64-wide activations
constexpr int kParamsPadded = (kMlpParams + 3) / 4 * 4;

__device__ __forceinline__ void load_params(const float* __restrict__ g, float* s) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) s[i] = __ldg(g + i);
}

// Decodes a half-grid element index into (x, y, z).
__device__ __forceinline__ void voxel_xyz(int64_t i, int P, int* x, int* y, int* z) {
  int rowlen = P / 2 + 1;
  *x = (int)(i % rowlen);
  int64_t t = i / rowlen;
  *y = (int)(t % P);
  *z = (int)(t / P);
}

__device__ __forceinline__ int signed_coord(int v, int P) { return v < P / 2 + 1 ? v : v - P; }

// ------------------------------------------------------------- inference --
// Predicted start over a half grid.  A block scans chunks of kChunk
// consecutive voxels: voxels outside the sphere or without weight get the
// cold value at once; the others are compacted into a list and evaluated
// in tiles of kTileV voxels as two small matrix products in shared memory,
//   H1 = relu(X W1^T + b1)   (kTileV x 28) . (28 x 64)
//   out = b3 + relu(H1 W2^T + b2) . W3
// each thread holding an 8-voxel x 4-unit register tile, so that three
// shared-memory loads feed 32 FMAs.  Inputs and activations are stored
// transposed (feature-major) for float4 loads along the voxels.
constexpr int kTileV = 128;
constexpr int kChunk = 1024;
constexpr int kStartThreads = 256;  // two threads per tile voxel for the features
constexpr int kH1Row = kTileV + 4;  // padded: the 16 rows a warp stores hit distinct banks

struct StartShared {
  float xt[kMlpIn][kTileV];
  float h1t[kMlpHidden][kH1Row];
  float w1t[kMlpIn][kMlpHidden];
  float w2t[kMlpHidden][kMlpHidden];
  float b1[kMlpHidden], b2[kMlpHidden], w3[kMlpHidden];
  float shift[kMlpIn], scale[kMlpIn];
  unsigned short list[kChunk];
  int count;
};

// Feature k (0..26) of voxel (x, y, z), standardised.
__device__ __forceinline__ float start_feature(const StartShared& S, const float* __restrict__ Fw,
                                               int P, float inv_s, int x, int y, int z, int k) {
  int dz = k / 9 - 1, dy = (k / 3) % 3 - 1, dx = k % 3 - 1;
  float w = __ldg(Fw + mlp_neighbour_index(P, x, y, z, dx, dy, dz));
  return (logf(w * inv_s + kMlpWeightFloor) - S.shift[k]) * S.scale[k];
}

__global__ void __launch_bounds__(kStartThreads) mlp_start_kernel(
    const float* __restrict__ params, const float* __restrict__ Fw, int P, int maskr2,
    const double* __restrict__ scale_sums, float* __restrict__ Fnw, float2* __restrict__ convft) {
  extern __shared__ __align__(16) unsigned char start_raw[];
  StartShared& S = *reinterpret_cast<StartShared*>(start_raw);
  const int t = threadIdx.x;
  for (int i = t; i < kMlpIn * kMlpHidden; i += kStartThreads)
    S.w1t[i / kMlpHidden][i % kMlpHidden] = __ldg(params + kMlpOffW1 + (i % kMlpHidden) * kMlpIn + i / kMlpHidden);
  for (int i = t; i < kMlpHidden * kMlpHidden; i += kStartThreads)
    S.w2t[i / kMlpHidden][i % kMlpHidden] =
        __ldg(params + kMlpOffW2 + (i % kMlpHidden) * kMlpHidden + i / kMlpHidden);
  if (t < kMlpHidden) {
    S.b1[t] = __ldg(params + kMlpOffB1 + t);
    S.b2[t] = __ldg(params + kMlpOffB2 + t);
    S.w3[t] = __ldg(params + kMlpOffW3 + t);
  }
  if (t < kMlpIn) {
    S.shift[t] = __ldg(params + kMlpOffShift + t);
    S.scale[t] = __ldg(params + kMlpOffScale + t);
  }
  const float b3 = __ldg(params + kMlpOffB3);
  const double sum = scale_sums[0], cnt = scale_sums[1];
  const float inv_s = sum > 0 ? (float)(cnt / sum) : 1.f;
  const int rowlen = P / 2 + 1;
  const int64_t nc = (int64_t)rowlen * P * P;
  const int64_t nchunks = (nc + kChunk - 1) / kChunk;
  const int lane = t & 31;
  const int tj = t & 15, tv = t >> 4;  // register tile: units 4 tj .. +3, voxels 8 tv .. +7
  const int j0 = tj * 4, v0 = tv * 8;

  for (int64_t chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    const int64_t base = chunk * kChunk;
    if (t == 0) S.count = 0;
    __syncthreads();
#pragma unroll 1
    for (int q = 0; q < kChunk / kStartThreads; q++) {
      const int local = q * kStartThreads + t;
      const int64_t i = base + local;
      bool elig = false;
      if (i < nc) {
        int x = (int)(i % rowlen);
        int64_t r = i / rowlen;
        int y = (int)(r % P), z = (int)(r / P);
        int yp = y < P / 2 + 1 ? y : y - P, zp = z < P / 2 + 1 ? z : z - P;
        bool inside = x * x + yp * yp + zp * zp < maskr2;
        float fw = Fw[i];
        elig = inside && fw > 0.f;
        if (!elig) {
          float nw = inside ? 1.f : 0.f;
          Fnw[i] = nw;
          if (convft) convft[i] = make_float2(fw * nw, 0.f);
        }
      }
      unsigned m = __ballot_sync(0xffffffffu, elig);
      if (m) {
        int leader = __ffs(m) - 1, first = 0;
        if (lane == leader) first = atomicAdd(&S.count, __popc(m));
        first = __shfl_sync(0xffffffffu, first, leader);
        if (elig) S.list[first + __popc(m & ((1u << lane) - 1))] = (unsigned short)local;
      }
    }
    __syncthreads();
    const int n = S.count;
#pragma unroll 1
    for (int t0 = 0; t0 < n; t0 += kTileV) {
      {  // features: thread pairs split the 27 neighbours (+ radius)
        const int v = t & (kTileV - 1), half = t >> 7;
        const int k0 = half ? 14 : 0, k1 = half ? 27 : 14;
        if (t0 + v < n) {
          int64_t i = base + S.list[t0 + v];
          int x = (int)(i % rowlen);
          int64_t r = i / rowlen;
          int y = (int)(r % P), z = (int)(r / P);
          for (int k = k0; k < k1; k++) S.xt[k][v] = start_feature(S, Fw, P, inv_s, x, y, z, k);
          if (half) {
            int yp = y < P / 2 + 1 ? y : y - P, zp = z < P / 2 + 1 ? z : z - P;
            float rad = sqrtf((float)(x * x + yp * yp + zp * zp)) / (float)(P / 2);
            S.xt[27][v] = (rad - S.shift[27]) * S.scale[27];
          }
        } else {
          for (int k = k0; k < k1; k++) S.xt[k][v] = 0.f;
          if (half) S.xt[27][v] = 0.f;
        }
      }
      __syncthreads();
      float acc[4][8];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = S.b1[j0 + a];
#pragma unroll 4
      for (int k = 0; k < kMlpIn; k++) {
        float4 xa = *reinterpret_cast<const float4*>(&S.xt[k][v0]);
        float4 xb = *reinterpret_cast<const float4*>(&S.xt[k][v0 + 4]);
        float4 w = *reinterpret_cast<const float4*>(&S.w1t[k][j0]);
        float xv[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
        float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 8; b++) acc[a][b] = fmaf(wv[a], xv[b], acc[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 4; a++) {
        *reinterpret_cast<float4*>(&S.h1t[j0 + a][v0]) =
            make_float4(fmaxf(acc[a][0], 0.f), fmaxf(acc[a][1], 0.f), fmaxf(acc[a][2], 0.f), fmaxf(acc[a][3], 0.f));
        *reinterpret_cast<float4*>(&S.h1t[j0 + a][v0 + 4]) =
            make_float4(fmaxf(acc[a][4], 0.f), fmaxf(acc[a][5], 0.f), fmaxf(acc[a][6], 0.f), fmaxf(acc[a][7], 0.f));
      }
      __syncthreads();
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = S.b2[j0 + a];
#pragma unroll 4
      for (int k = 0; k < kMlpHidden; k++) {
        float4 ha = *reinterpret_cast<const float4*>(&S.h1t[k][v0]);
        float4 hb = *reinterpret_cast<const float4*>(&S.h1t[k][v0 + 4]);
        float4 w = *reinterpret_cast<const float4*>(&S.w2t[k][j0]);
        float hv[8] = {ha.x, ha.y, ha.z, ha.w, hb.x, hb.y, hb.z, hb.w};
        float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 8; b++) acc[a][b] = fmaf(wv[a], hv[b], acc[a][b]);
      }
      float o[8];
#pragma unroll
      for (int b = 0; b < 8; b++) {
        o[b] = 0.f;
#pragma unroll
        for (int a = 0; a < 4; a++) o[b] = fmaf(S.w3[j0 + a], fmaxf(acc[a][b], 0.f), o[b]);
#pragma unroll
        for (int off = 1; off < 16; off <<= 1) o[b] += __shfl_xor_sync(0xffffffffu, o[b], off);
      }
      if (tj == 0) {
#pragma unroll
        for (int b = 0; b < 8; b++) {
          int e = t0 + v0 + b;
          if (e < n) {
            int64_t i = base + S.list[e];
            float nw = fminf(1e20f, expf(o[b] + b3) * inv_s);
            Fnw[i] = nw;
            if (convft) convft[i] = make_float2(Fw[i] * nw, 0.f);
          }
        }
      }
      __syncthreads();
    }
  }
}

// The two Hermitian mates (0, y, z) and (0, -y, -z) of the x = 0 plane are
// one Fourier component: both get the geometric mean of their starts, i.e.
// exp(mean of the two outputs) / s.  One thread per canonical mate.
__global__ void mlp_start_mates_kernel(const float* __restrict__ Fw, int P, int maskr2,
                                       float* __restrict__ Fnw, float2* __restrict__ convft) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= P * P) return;
  int y = idx % P, z = idx / P;
  int yp = y < P / 2 + 1 ? y : y - P, zp = z < P / 2 + 1 ? z : z - P;
  if (!(zp > 0 || (zp == 0 && yp > 0))) return;
  if (yp * yp + zp * zp >= maskr2) return;
  const int rowlen = P / 2 + 1;
  int my = y == 0 ? 0 : P - y, mz = z == 0 ? 0 : P - z;
  int64_t a = ((int64_t)z * P + y) * rowlen, b = ((int64_t)mz * P + my) * rowlen;
  if (a == b) return;
  float fa = Fw[a], fb = Fw[b];
  if (!(fa > 0.f && fb > 0.f)) return;
  float m = sqrtf(Fnw[a]) * sqrtf(Fnw[b]);
  Fnw[a] = m;
  Fnw[b] = m;
  if (convft) {
    convft[a] = make_float2(fa * m, 0.f);
    convft[b] = make_float2(fb * m, 0.f);
  }
}

__global__ void mlp_scale_kernel(const float* __restrict__ Fw, int P, int maskr2,
                                 double* __restrict__ sums) {
  const int64_t nc = (int64_t)(P / 2 + 1) * P * P;
  double s = 0, c = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    voxel_xyz(i, P, &x, &y, &z);
    int yp = signed_coord(y, P), zp = signed_coord(z, P);
    float w = Fw[i];
    if (w > 0.f && x * x + yp * yp + zp * zp < maskr2) {
      s += w;
      c += 1;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, off);
    c += __shfl_down_sync(0xffffffffu, c, off);
  }
  __shared__ double red[2][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = s;
    red[1][warp] = c;
  }
  __syncthreads();
  if (warp == 0) {
    int nwarps = blockDim.x >> 5;
    s = lane < nwarps ? red[0][lane] : 0;
    c = lane < nwarps ? red[1][lane] : 0;
    for (int off = 16; off > 0; off >>= 1) {
      s += __shfl_down_sync(0xffffffffu, s, off);
      c += __shfl_down_sync(0xffffffffu, c, off);
    }
    if (lane == 0) {
      atomicAdd(sums, s);
      atomicAdd(sums + 1, c);
    }
  }
}

// Network outputs for a matrix of raw features (n x 28).
__global__ void __launch_bounds__(kInferThreads) mlp_forward_kernel(
    const float* __restrict__ params, const float* __restrict__ feats, int n,
    float* __restrict__ out) {
  __shared__ __align__(16) float sp[kParamsPadded];
  load_params(params, sp);
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float f[kMlpIn];
#pragma unroll
  for (int k = 0; k < kMlpIn; k++) f[k] = feats[(int64_t)i * kMlpIn + k];
  out[i] = mlp_forward(sp, f);
}

// Raw features of sample voxels of a stack of half grids of P: sample s is
// element index[s] of the stack (volume index[s] / nc), whose weight scale
// is 1 / inv_scale[volume].
__global__ void mlp_features_kernel(const float* __restrict__ fw, int P,
                                    const float* __restrict__ inv_scale,
                                    const long long* __restrict__ index, int n,
                                    float* __restrict__ feats) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int64_t nc = (int64_t)(P / 2 + 1) * P * P;
  int64_t e = index[s];
  int64_t vol = e / nc;
  int x, y, z;
  voxel_xyz(e - vol * nc, P, &x, &y, &z);
  float f[kMlpIn];
  mlp_voxel_features(fw + vol * nc, P, inv_scale[vol], x, y, z, f);
#pragma unroll
  for (int k = 0; k < kMlpIn; k++) feats[(int64_t)s * kMlpIn + k] = f[k];
}

// -------------------------------------------------------------- training --
// One block = up to 128 samples, one per thread.  Loss
//   L = loss_scale * sum_s w_s (out_s - t_s)^2
// accumulated into *loss; dL/dparams accumulated into grad (same indexing
// as the parameters; the input standardisation is not trained).
//
// Phase 1 (thread s): forward pass, keeping the standardised input X, the
// first-layer activations H1 and the second-layer activations H2 in shared
// memory, dout = dL/dout, and G1 = dL/d(first-layer pre-activation)
//   G1[k] = dout * [H1[k] > 0] * sum_j W3[j] [H2[j] > 0] W2[j][k],
// whose sum over j (u below) is accumulated while layer 2 is evaluated.
// Phase 2 (thread t): gradient entries, each a sum over the block's samples:
//   dW2[j][k] = W3[j] sum_s dout_s [H2_s[j] > 0] H1_s[k]   (4x4 tiles)
//   db2[j]    = W3[j] sum_s dout_s [H2_s[j] > 0]
//   dW3[j]    = sum_s dout_s H2_s[j],   db3 = sum_s dout_s
//   dW1[j][i] = sum_s G1_s[j] X_s[i]                        (4x4 tiles)
//   db1[j]    = sum_s G1_s[j]
// then one red.add per entry and block.
struct TrainShared {
  float p[kParamsPadded];
  float x[kTrainThreads][kMlpIn];
  float h1[kTrainThreads][kRow];
  float h2[kTrainThreads][kRow];
  float g1[kTrainThreads][kRow];
  float dout[kTrainThreads];
  float loss[kTrainThreads / 32];
};

struct MatrixSource {  // features given as a matrix
  const float* feats;
  const float* targets;
  const float* weights;
  __device__ void load(int s, float* f, float* t, float* w) const {
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) f[k] = feats[(int64_t)s * kMlpIn + k];
    *t = targets[s];
    *w = weights[s];
  }
};

struct VolumeSource {  // features gathered from a stack of half grids
  const float* fw;
  const float* target;
  const float* weight;
  const float* inv_scale;
  const long long* index;
  int P;
  __device__ void load(int s, float* f, float* t, float* w) const {
    const int64_t nc = (int64_t)(P / 2 + 1) * P * P;
    int64_t e = index[s];
    int64_t vol = e / nc;
    int x, y, z;
    voxel_xyz(e - vol * nc, P, &x, &y, &z);
    mlp_voxel_features(fw + vol * nc, P, inv_scale[vol], x, y, z, f);
    *t = target[e];
    *w = weight[e];
  }
};

template <class Src>
__global__ void __launch_bounds__(kTrainThreads) mlp_train_kernel(const float* __restrict__ params,
                                                                  Src src, int n, float loss_scale,
                                                                  float* __restrict__ grad,
                                                                  float* __restrict__ loss) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainShared& S = *reinterpret_cast<TrainShared*>(smem_raw);
  load_params(params, S.p);
  __syncthreads();
  const float* p = S.p;
  const int t = threadIdx.x;
  const int s = blockIdx.x * kTrainThreads + t;

  // ---- phase 1
  float dout = 0.f, l = 0.f;
  {
    float f[kMlpIn], target = 0.f, w = 0.f;
    const bool valid = s < n;
    if (valid) {
      src.load(s, f, &target, &w);
    } else {
#pragma unroll
      for (int k = 0; k < kMlpIn; k++) f[k] = 0.f;
    }
    float xin[kMlpIn];
    mlp_standardise(p, f, xin);
#pragma unroll
    for (int i = 0; i < kMlpIn; i += 4)
      *reinterpret_cast<float4*>(&S.x[t][i]) = make_float4(xin[i], xin[i + 1], xin[i + 2], xin[i + 3]);
    float h1[kMlpHidden];
    mlp_layer1(p, xin, h1);
#pragma unroll
    for (int k = 0; k < kMlpHidden; k += 4)
      *reinterpret_cast<float4*>(&S.h1[t][k]) = make_float4(h1[k], h1[k + 1], h1[k + 2], h1[k + 3]);
    float u[kMlpHidden];
#pragma unroll
    for (int k = 0; k < kMlpHidden; k++) u[k] = 0.f;
    float out = p[kMlpOffB3];
#pragma unroll 1
    for (int j = 0; j < kMlpHidden; j++) {
      float a = mlp_layer2_unit(p, h1, j);
      float h2 = fmaxf(a, 0.f);
      S.h2[t][j] = h2;
      float w3 = p[kMlpOffW3 + j];
      out = fmaf(w3, h2, out);
      float m = a > 0.f ? w3 : 0.f;
      const float4* w2 = reinterpret_cast<const float4*>(p + kMlpOffW2 + j * kMlpHidden);
#pragma unroll
      for (int k = 0; k < kMlpHidden / 4; k++) {
        float4 q = w2[k];
        u[4 * k] = fmaf(m, q.x, u[4 * k]);
        u[4 * k + 1] = fmaf(m, q.y, u[4 * k + 1]);
        u[4 * k + 2] = fmaf(m, q.z, u[4 * k + 2]);
        u[4 * k + 3] = fmaf(m, q.w, u[4 * k + 3]);
      }
    }
    if (valid) {
      float d = out - target;
      l = loss_scale * w * d * d;
      dout = 2.f * loss_scale * w * d;
    }
    S.dout[t] = dout;
#pragma unroll
    for (int k = 0; k < kMlpHidden; k += 4)
      *reinterpret_cast<float4*>(&S.g1[t][k]) =
          make_float4(h1[k] > 0.f ? dout * u[k] : 0.f, h1[k + 1] > 0.f ? dout * u[k + 1] : 0.f,
                      h1[k + 2] > 0.f ? dout * u[k + 2] : 0.f, h1[k + 3] > 0.f ? dout * u[k + 3] : 0.f);
  }
  for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
  if ((t & 31) == 0) S.loss[t >> 5] = l;
  __syncthreads();
  if (t == 0) {
    float b = 0.f;
    for (int w = 0; w < kTrainThreads / 32; w++) b += S.loss[w];
    atomicAdd(loss, b);
  }
  const int rows = min(kTrainThreads, n - (int)blockIdx.x * kTrainThreads);

  // ---- phase 2: dW2 (256 tiles of 4x4, two per thread) and dW1 (112 tiles)
#pragma unroll 1
  for (int tile = t; tile < 256; tile += kTrainThreads) {
    int j0 = (tile >> 4) * 4, k0 = (tile & 15) * 4;
    float acc[4][4] = {};
    for (int r = 0; r < rows; r++) {
      float d = S.dout[r];
      float4 h2 = *reinterpret_cast<const float4*>(&S.h2[r][j0]);
      float4 hh = *reinterpret_cast<const float4*>(&S.h1[r][k0]);
      float g[4] = {h2.x > 0.f ? d : 0.f, h2.y > 0.f ? d : 0.f, h2.z > 0.f ? d : 0.f,
                    h2.w > 0.f ? d : 0.f};
      float hv[4] = {hh.x, hh.y, hh.z, hh.w};
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = fmaf(g[a], hv[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
      float w3 = p[kMlpOffW3 + j0 + a];
#pragma unroll
      for (int b = 0; b < 4; b++)
        red_add(grad + kMlpOffW2 + (j0 + a) * kMlpHidden + k0 + b, w3 * acc[a][b]);
    }
  }
  if (t < 112) {
    int j0 = (t / 7) * 4, i0 = (t % 7) * 4;
    float acc[4][4] = {};
    for (int r = 0; r < rows; r++) {
      float4 g = *reinterpret_cast<const float4*>(&S.g1[r][j0]);
      float4 xv = *reinterpret_cast<const float4*>(&S.x[r][i0]);
      float gv[4] = {g.x, g.y, g.z, g.w};
      float xs[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = fmaf(gv[a], xs[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) red_add(grad + kMlpOffW1 + (j0 + a) * kMlpIn + i0 + b, acc[a][b]);
  }
  // vectors: thread t < 64 -> db2[t] and dW3[t]; 64 <= t < 128 -> db1[t-64] (and db3)
  if (t < kMlpHidden) {
    float sb2 = 0.f, sw3 = 0.f;
    for (int r = 0; r < rows; r++) {
      float d = S.dout[r], h2 = S.h2[r][t];
      sb2 += h2 > 0.f ? d : 0.f;
      sw3 = fmaf(d, h2, sw3);
    }
    red_add(grad + kMlpOffB2 + t, p[kMlpOffW3 + t] * sb2);
    red_add(grad + kMlpOffW3 + t, sw3);
  } else {
    int j = t - kMlpHidden;
    float sb1 = 0.f;
    for (int r = 0; r < rows; r++) sb1 += S.g1[r][j];
    red_add(grad + kMlpOffB1 + j, sb1);
    if (j == 0) {
      float sb3 = 0.f;
      for (int r = 0; r < rows; r++) sb3 += S.dout[r];
      red_add(grad + kMlpOffB3, sb3);
    }
  }
}

// Adam on the trained entries [kMlpOffW1, kMlpParams); zeroes the gradient.
// bias1 = 1 / (1 - beta1^t), bias2 = 1 / (1 - beta2^t).
__global__ void mlp_adam_kernel(float* __restrict__ params, float* __restrict__ grad,
                                float* __restrict__ m, float* __restrict__ v, float lr, float beta1,
                                float beta2, float eps, float bias1, float bias2) {
  int i = kMlpOffW1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  float g = grad[i];
  float mi = fmaf(beta1, m[i], (1.f - beta1) * g);
  float vi = fmaf(beta2, v[i], (1.f - beta2) * g * g);
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi * bias1) / (sqrtf(vi * bias2) + eps);
  grad[i] = 0.f;
}

template <class Src>
int launch_train(const float* params, const Src& src, int n, float loss_scale, float* grad,
                 float* loss, cudaStream_t stream) {
  const int smem = (int)sizeof(TrainShared);
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(mlp_train_kernel<Src>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  unsigned blocks = (unsigned)((n + kTrainThreads - 1) / kTrainThreads);
  mlp_train_kernel<Src><<<blocks, kTrainThreads, smem, stream>>>(params, src, n, loss_scale, grad, loss);
  GTOMRLN_LAUNCH_CHECK("mlp_train_kernel");
  return GTOMRLN_OK;
}

}  // namespace

int mlp_predict_start(const float* d_params, const float* Fw, int P, int maskr2,
                      const double* scale_sums, float* Fnw, float2* convft, cudaStream_t stream) {
  const int64_t nc = (int64_t)(P / 2 + 1) * P * P;
  const int smem = (int)sizeof(StartShared);
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(mlp_start_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int dev = 0, sms = 0, per_sm = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  GTOMRLN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GTOMRLN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mlp_start_kernel, kStartThreads, smem));
  int64_t nchunks = (nc + kChunk - 1) / kChunk;
  int64_t blocks = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
  if (blocks > nchunks) blocks = nchunks;
  mlp_start_kernel<<<(unsigned)blocks, kStartThreads, smem, stream>>>(d_params, Fw, P, maskr2, scale_sums,
                                                                      Fnw, convft);
  GTOMRLN_LAUNCH_CHECK("mlp_start_kernel");
  mlp_start_mates_kernel<<<(P * P + 255) / 256, 256, 0, stream>>>(Fw, P, maskr2, Fnw, convft);
  GTOMRLN_LAUNCH_CHECK("mlp_start_mates_kernel");
  return GTOMRLN_OK;
}

int mlp_weight_scale(const float* Fw, int P, int maskr2, double* sums, cudaStream_t stream) {
  mlp_scale_kernel<<<4 * 148, 256, 0, stream>>>(Fw, P, maskr2, sums);
  GTOMRLN_LAUNCH_CHECK("mlp_scale_kernel");
  return GTOMRLN_OK;
}

}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_mlp_param_count(void) { return kMlpParams; }

int gtomrln_mlp_forward(const float* d_params, const float* d_features, int n, float* d_out,
                        void* stream) {
  clear_error();
  if (n < 0 || (n > 0 && (!d_params || !d_features || !d_out)))
    return set_error(GTOMRLN_ERR_INVALID, "mlp_forward: bad arguments");
  if (n == 0) return GTOMRLN_OK;
  mlp_forward_kernel<<<(n + kInferThreads - 1) / kInferThreads, kInferThreads, 0,
                       (cudaStream_t)stream>>>(d_params, d_features, n, d_out);
  GTOMRLN_LAUNCH_CHECK("mlp_forward_kernel");
  return GTOMRLN_OK;
}

int gtomrln_mlp_volume_features(const float* d_fw, int P, const float* d_inv_scale,
                                const long long* d_index, int n, float* d_features, void* stream) {
  clear_error();
  if (n < 0 || P < 4 || (P & 1) || (n > 0 && (!d_fw || !d_inv_scale || !d_index || !d_features)))
    return set_error(GTOMRLN_ERR_INVALID, "mlp_volume_features: bad arguments");
  if (n == 0) return GTOMRLN_OK;
  mlp_features_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_fw, P, d_inv_scale, d_index,
                                                                        n, d_features);
  GTOMRLN_LAUNCH_CHECK("mlp_features_kernel");
  return GTOMRLN_OK;
}

int gtomrln_mlp_gradients(const float* d_params, const float* d_features, const float* d_targets,
                          const float* d_weights, int n, float loss_scale, float* d_grad,
                          float* d_loss, void* stream) {
  clear_error();
  if (n < 0 || (n > 0 && (!d_params || !d_features || !d_targets || !d_weights || !d_grad || !d_loss)))
    return set_error(GTOMRLN_ERR_INVALID, "mlp_gradients: bad arguments");
  if (n == 0) return GTOMRLN_OK;
  MatrixSource src{d_features, d_targets, d_weights};
  return launch_train(d_params, src, n, loss_scale, d_grad, d_loss, (cudaStream_t)stream);
}

int gtomrln_mlp_train_batch(const float* d_params, const float* d_fw, const float* d_target,
                            const float* d_weight, const float* d_inv_scale, int P,
                            const long long* d_index, int n, float loss_scale, float* d_grad,
                            float* d_loss, void* stream) {
  clear_error();
  if (n < 0 || P < 4 || (P & 1) ||
      (n > 0 && (!d_params || !d_fw || !d_target || !d_weight || !d_inv_scale || !d_index || !d_grad ||
                 !d_loss)))
    return set_error(GTOMRLN_ERR_INVALID, "mlp_train_batch: bad arguments");
  if (n == 0) return GTOMRLN_OK;
  VolumeSource src{d_fw, d_target, d_weight, d_inv_scale, d_index, P};
  return launch_train(d_params, src, n, loss_scale, d_grad, d_loss, (cudaStream_t)stream);
}

int gtomrln_mlp_adam(float* d_params, float* d_grad, float* d_m, float* d_v, int step, float lr,
                     float beta1, float beta2, float eps, void* stream) {
  clear_error();
  if (!d_params || !d_grad || !d_m || !d_v || step < 1)
    return set_error(GTOMRLN_ERR_INVALID, "mlp_adam: bad arguments");
  float bias1 = (float)(1.0 / (1.0 - std::pow((double)beta1, step)));
  float bias2 = (float)(1.0 / (1.0 - std::pow((double)beta2, step)));
  int n = kMlpParams - kMlpOffW1;
  mlp_adam_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_params, d_grad, d_m, d_v, lr, beta1,
                                                                     beta2, eps, bias1, bias2);
  GTOMRLN_LAUNCH_CHECK("mlp_adam_kernel");
  return GTOMRLN_OK;
}

}  // extern "C"
