// Gridding reconstructor: RELION-style iterative gridding-weight correction
// followed by the inverse FFT, crop and sinc^2 correction — the B200
// replacement of gtom::d_ReconstructGridding
// (src/Reconstruction/RecFourier.cu:98-332).
//
// The reference makes 5 + 4 * iterations element-wise passes over the P-grid
// around its FFTs (decentre, sphere mask, fill, Iteration1, renormalise,
// blob multiply, Iteration2, ...).  Here they are fused into
//   init   : decentre + mask of the weights, Fnewweight = sphere mask, and
//            the first iteration's conv spectrum, in one pass;
//   blob   : 1/P^3 renormalisation and the real-space blob multiply, with
//            the blob computed on the fly from its radial table (no P^3
//            blob volume);
//   update : Iteration2 fused with the next iteration's Iteration1, plus the
//            optional relative-change reduction;
//   final  : decentre of the data, the weight product (or the division of
//            the iterations == 0 branch) and the centring shift as a sign;
//   crop   : centred crop, sinc^2 correction and the 1/(pad^3 ori) scale.
// On the grids gridsym.cu takes (the default there) the iterations and the
// final map (final, its inverse transform and crop) run on the library's own
// transforms, with no P^3 real grid; elsewhere, and on GTOMRLN_PATH_DIRECT,
// the P^3 R2C / C2R transforms are cuFFT library calls, plans cached per
// (device, P).
#include <cufft.h>
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "batch.cuh"
#include "gridfft.cuh"
#include "mlp.cuh"

namespace gtomrln {

double kaiser_fourier_value(double w, double a, double alpha, int m);  // below

// ---------------------------------------------------------------- kernels --
// RecFourier.cu:264-285 (DecenterKernel) for the weights + SphereMask.cu:167-189
// (Fnewweight = 1 inside r^2 < (r_max*pad)^2) + Iteration1Kernel
// (RecFourier.cu:287-291).  old* are the centred input dims.
// One warp per (y, z) row of the P grid (lanes along x; grid (rows / 8,
// volumes), 256 threads): the row's decentring and radii once, no index
// divisions per element.
constexpr int kInitWarps = 8;
__global__ void __launch_bounds__(32 * kInitWarps)
grid_init_kernel(const float* __restrict__ weight, int oldx, int oldy, int oldz, float* __restrict__ Fw,
                 float* __restrict__ Fnw, float2* __restrict__ convft, GridGeom g, int maskr2, int write_conv,
                 int64_t wstride) {
  const int64_t b = blockIdx.y;  // volume of a batch (stacks of equal volumes)
  weight += b * wstride;
  Fw += b * g.nc;
  Fnw += b * g.nc;
  convft += b * g.nc;
  const int row = blockIdx.x * kInitWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= g.P * g.P) return;
  const int z = row / g.P, y = row - z * g.P;
  const int zp = z < g.P / 2 + 1 ? z : z - g.P;
  const int yp = y < g.P / 2 + 1 ? y : y - g.P;
  const float r = (float)(zp * zp) + (float)(yp * yp);
  const int zi = zp + oldz / 2, yi = yp + oldy / 2;
  const bool in_yz = zi >= 0 && zi < oldz && yi >= 0 && yi < oldy;
  const float* wrow = weight + (in_yz ? ((int64_t)zi * oldy + yi) * (oldx / 2 + 1) : 0);
  const int64_t base = (int64_t)row * g.rowlen;
  const int yz2 = yp * yp + zp * zp;
  for (int x = lane; x < g.rowlen; x += 32) {
    const float rr = r + (float)(x * x);
    const float mask = rr < (float)(g.P * g.P / 4) ? 1.f : 0.f;
    float w = 0.f;
    if (in_yz && x < oldx / 2 + 1) w = __ldg(wrow + x) * mask;
    Fw[base + x] = w;
    // SphereMaskFTKernel uses y < dims.y/2+1 ? y : y - dims.x, the same split.
    const float nw = x * x + yz2 < maskr2 ? 1.f : 0.f;
    Fnw[base + x] = nw;
    if (write_conv) convft[base + x] = make_float2(w * nw, 0.f);
  }
}

// conv <- (conv * 1/P^3) * blob(r): d_IFFTC2R's renormalisation
// (IFFT.cu:36-46) and d_MultiplyByVector with PrecomputeBlobKernel's table
// lookup (RecFourier.cu:243-262), the radius evaluated as the reference does.
// A grid-stride kernel over units of kBlobRows rows (y) of one (volume, z)
// plane; each CTA stages the 10 000-entry table in shared memory once (read
// from global memory, lanes at consecutive x touch one cache line each).
// Each thread loads its kBlobRows elements of a column before using any
// (eight loads in flight per thread), and no index needs a 64-bit division.
constexpr int kBlobRows = 8;
constexpr int kBlobThreads = 512;
template <bool HOIST>
__global__ void __launch_bounds__(kBlobThreads, 3)
grid_blob_kernel(float* __restrict__ conv, const float* __restrict__ table, GridGeom g, int count, float inv_n,
                 float funcsampling) {
  __shared__ float stab[kBlobSamples];
  for (int i = threadIdx.x; i < kBlobSamples; i += blockDim.x) stab[i] = __ldg(table + i);
  __syncthreads();
  const int P = g.P;
  const int groups = (P + kBlobRows - 1) / kBlobRows;
  const int64_t units = (int64_t)count * P * groups;
  for (int64_t unit = blockIdx.x; unit < units; unit += gridDim.x) {
    const int64_t plane = unit / groups;  // volume * P + z
    const int y0 = (int)(unit - plane * groups) * kBlobRows;
    const int z = (int)(plane % P);
    const int rows = min(kBlobRows, P - y0);
    // HOIST (P <= 4096): grid_blob_index's radius with the conversions
    // hoisted: xp^2 + yp^2 + zp^2 is then an integer below 2^24, exact in
    // FP32 however it is summed, so the row part yp^2 + zp^2 is formed once
    // per row and only the square root, the divisions and the truncation
    // remain per voxel
    const int zp = z < P / 2 ? z : z - P;
    float c[kBlobRows];
#pragma unroll
    for (int r = 0; r < kBlobRows; r++) {
      const int y = y0 + r, yp = y < P / 2 ? y : y - P;
      c[r] = (float)(yp * yp + zp * zp);
    }
    for (int x = threadIdx.x; x < P; x += blockDim.x) {
      float* col = conv + (plane * P + y0) * P + x;
      float v[kBlobRows];
#pragma unroll
      for (int r = 0; r < kBlobRows; r++)
        if (r < rows) v[r] = col[r * P];
      const float xp = (float)(x < P / 2 ? x : x - P);
      const float xx = xp * xp;
#pragma unroll
      for (int r = 0; r < kBlobRows; r++) {
        if (r >= rows) break;
        int ti;
        if (HOIST) {
          ti = grid_blob_index_sq(xx + c[r], (float)P, funcsampling);
        } else {
          ti = grid_blob_index(P, x, y0 + r, z, funcsampling);
        }
        col[r * P] = v[r] * inv_n * stab[ti];
      }
    }
  }
}

// Launches grid_blob_kernel over `count` consecutive volumes: three CTAs per
// SM (40 registers, 40 KB of table each), striding over the row units.
static void launch_blob(float* conv, const float* table, const GridGeom& g, int count, cudaStream_t stream) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t units = (int64_t)count * g.P * ((g.P + kBlobRows - 1) / kBlobRows);
  const unsigned blocks = (unsigned)std::min<int64_t>(units, 3LL * sms);
  if (g.P <= 4096)
    grid_blob_kernel<true><<<blocks, kBlobThreads, 0, stream>>>(conv, table, g, count, 1.0f / (float)g.nr,
                                                              (float)(0.5 / kBlobSamples));
  else
    grid_blob_kernel<false><<<blocks, kBlobThreads, 0, stream>>>(conv, table, g, count, 1.0f / (float)g.nr,
                                                               (float)(0.5 / kBlobSamples));
}

// Iteration2Kernel (RecFourier.cu:293-308) fused with the next iteration's
// Iteration1Kernel.  Optionally accumulates the convergence measure
// sum((Fw*(new-old))^2) and sum((Fw*old)^2): the change of the corrected
// weight Fw*Fnw.  Unweighted, voxels with Fw = 0 would dominate: there
// Fnw grows by 1e4 per iteration until the 1e20 clamp and never matters.
// With ref (a single volume's reference weights, e.g. converged ones) it
// also accumulates sum((Fw*(new-ref))^2) and sum((Fw*ref)^2) into
// change[2..3]: the distance of the corrected weight from the reference's.
__global__ void grid_update_kernel(float2* __restrict__ convft, const float* __restrict__ Fw,
                                   float* __restrict__ Fnw, GridGeom g, int write_conv,
                                   double* __restrict__ change, const float* __restrict__ ref) {
  const int64_t b = blockIdx.y;  // change is only requested for a single volume
  convft += b * g.nc;
  Fw += b * g.nc;
  Fnw += b * g.nc;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0, o2 = 0, r2 = 0, q2 = 0;
  if (i < g.nc) {
    float old = Fnw[i];
    float nw = grid_update_value(convft[i].x, old);
    float fw = Fw[i];
    Fnw[i] = nw;
    if (write_conv) convft[i] = make_float2(fw * nw, 0.f);
    if (change) {
      double d = (double)fw * ((double)nw - (double)old);
      double o = (double)fw * (double)old;
      d2 = d * d;
      o2 = o * o;
      if (ref) {
        const double rf = (double)ref[i];
        const double e = (double)fw * ((double)nw - rf), q = (double)fw * rf;
        r2 = e * e;
        q2 = q * q;
      }
    }
  }
  if (change) grid_change_reduce(d2, o2, change);
  if (change && ref) {
    __syncthreads();  // grid_change_reduce's shared scratch is reused
    grid_change_reduce(r2, q2, change + 2);
  }
}

// The update of grid_update_kernel applied at an extrapolated point V
// (Nesterov-style momentum on the logarithm of the weights):
//   F' = min(1e20, V / max(1e-4, c)),   V' = min(1e20, F' (F' / F)^beta),
// where c is the real part of the spectrum computed from Fw * V.  Its fixed
// points are the plain iteration's (c = 1 wherever Fw * F is non-zero); it
// reaches them in far fewer iterations because the slowest modes of the
// plain iteration contract by 1 - blob(r) per step, with blob(r) down to
// ~0.007 at the edge of the box.  The change measure is the plain one,
// Fw * (F' - F) against Fw * F.
__global__ void grid_update_momentum_kernel(float2* __restrict__ convft, const float* __restrict__ Fw,
                                            float* __restrict__ Fnw, float* __restrict__ V, GridGeom g,
                                            float beta, int write_conv, double* __restrict__ change,
                                            const float* __restrict__ ref) {
  const int64_t b = blockIdx.y;
  convft += b * g.nc;
  Fw += b * g.nc;
  Fnw += b * g.nc;
  V += b * g.nc;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0, o2 = 0, r2 = 0, q2 = 0;
  if (i < g.nc) {
    float old = Fnw[i];
    float nw, ext;
    grid_update_momentum_value(convft[i].x, old, V[i], beta, nw, ext);
    float fw = Fw[i];
    Fnw[i] = nw;
    V[i] = ext;
    if (write_conv) convft[i] = make_float2(fw * ext, 0.f);
    if (change) {
      double d = (double)fw * ((double)nw - (double)old);
      double o = (double)fw * (double)old;
      d2 = d * d;
      o2 = o * o;
      if (ref) {
        const double rf = (double)ref[i];
        const double e = (double)fw * ((double)nw - rf), q = (double)fw * rf;
        r2 = e * e;
        q2 = q * q;
      }
    }
  }
  if (change) grid_change_reduce(d2, o2, change);
  if (change && ref) {
    __syncthreads();  // grid_change_reduce's shared scratch is reused
    grid_change_reduce(r2, q2, change + 2);
  }
}

// DecenterKernel<tcomplex> for the data (RecFourier.cu:175-179), then
// x Fnewweight (RecFourier.cu:206) or / max(|Fweight|, 1e-4) when no
// iteration ran (RecFourier.cu:200-202), then d_Shift by P/2 in every axis
// (RecFourier.cu:213-214), which is the factor (-1)^(x+y+z).
__global__ void grid_final_kernel(const float2* __restrict__ data, int oldx, int oldy, int oldz,
                                  const float* __restrict__ Fw, const float* __restrict__ Fnw,
                                  float2* __restrict__ convft, GridGeom g, int divide,
                                  int64_t wstride) {
  const int64_t b = blockIdx.y;
  data += b * wstride;
  Fw += b * g.nc;
  Fnw += b * g.nc;
  convft += b * g.nc;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nc) return;
  int x, y, z;
  split_index(i, g.rowlen, (int64_t)g.rowlen * g.P, g.nc, x, y, z);
  const float2 v = grid_final_value(data, oldx, oldy, oldz, Fw, Fnw, g.P, x, y, z, i, divide != 0);
  convft[i] = v;
}

// d_Pad T_PAD_VALUE centred crop P^3 -> ori^3 (Padding.cu:97-135),
// CorrectGriddingKernel (RecFourier.cu:310-332) and the final scale
// (RecFourier.cu:237).
__global__ void grid_crop_kernel(const float* __restrict__ conv, float* __restrict__ out, int P,
                                 int ori, int off, float scale, float* const* __restrict__ outs) {
  conv += (int64_t)blockIdx.y * P * P * P;
  if (outs) out = outs[blockIdx.y];
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t total = (int64_t)ori * ori * ori;
  if (i >= total) return;
  int x = (int)(i % ori);
  int64_t t = i / ori;
  int y = (int)(t % ori);
  int z = (int)(t / ori);
  const float v = conv[((int64_t)(z + off) * P + (y + off)) * P + (x + off)];
  out[i] = grid_crop_value(v, x, y, z, ori, P, scale);
}

// ----------------------------------------------------------------- plans --
struct PlanPair {
  cufftHandle r2c = 0, c2r = 0;
};
static std::mutex g_plan_mutex;
static std::map<std::tuple<int, unsigned long long, int>, PlanPair> g_plans;  // (device, context, P)

static int get_plans(int P, PlanPair* out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = g_plans.find(std::make_tuple(dev, ctx, P));
  if (it != g_plans.end()) {
    *out = it->second;
    return GTOMRLN_OK;
  }
  PlanPair pp;
  cufftResult r = cufftPlan3d(&pp.r2c, P, P, P, CUFFT_R2C);
  if (r != CUFFT_SUCCESS) return set_error(GTOMRLN_ERR_CUFFT, "cufftPlan3d R2C %d^3 failed (%d)", P, (int)r);
  r = cufftPlan3d(&pp.c2r, P, P, P, CUFFT_C2R);
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(pp.r2c);
    return set_error(GTOMRLN_ERR_CUFFT, "cufftPlan3d C2R %d^3 failed (%d)", P, (int)r);
  }
  g_plans[std::make_tuple(dev, ctx, P)] = pp;
  *out = pp;
  return GTOMRLN_OK;
}


// Blob tables are cached per (device, context, radius, alpha, order).
static std::mutex g_table_mutex;
static std::map<std::tuple<int, unsigned long long, double, double, int>, float*> g_tables;

// Destroys the plans and frees the tables of the current context on device
// dev, and forgets those of earlier contexts there (gone with their context).
int release_gridding_caches(int dev, unsigned long long ctx) {
  {
    std::lock_guard<std::mutex> lock(g_plan_mutex);
    for (auto it = g_plans.begin(); it != g_plans.end();) {
      if (std::get<0>(it->first) != dev) {
        ++it;
        continue;
      }
      if (std::get<1>(it->first) == ctx) {
        cufftDestroy(it->second.r2c);
        cufftDestroy(it->second.c2r);
      }
      it = g_plans.erase(it);
    }
  }
  std::lock_guard<std::mutex> lock(g_table_mutex);
  for (auto it = g_tables.begin(); it != g_tables.end();) {
    if (std::get<0>(it->first) != dev) {
      ++it;
      continue;
    }
    if (std::get<1>(it->first) == ctx) cudaFree(it->second);
    it = g_tables.erase(it);
  }
  return GTOMRLN_OK;
}

int build_blob_table(double radius, double alpha, int order, int nsamples, float* out) {
  if (order != 0 && order != 2)
    return set_error(GTOMRLN_ERR_INVALID, "blob order %d not supported (0 or 2)", order);
  double sampling = 0.5 / nsamples;
  // The reference stores the raw values as float and normalises in float
  // (RecFourier.cu:110-115).
  for (int i = 0; i < nsamples; i++) out[i] = (float)kaiser_fourier_value(i * sampling, radius, alpha, order);
  float norm = out[0];
  for (int i = 0; i < nsamples; i++) out[i] /= norm;
  return GTOMRLN_OK;
}

static int get_table(double radius, double alpha, int order, const float** out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  std::lock_guard<std::mutex> lock(g_table_mutex);
  auto key = std::make_tuple(dev, ctx, radius, alpha, order);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) {
    *out = it->second;
    return GTOMRLN_OK;
  }
  std::vector<float> h(kBlobSamples);
  int st = build_blob_table(radius, alpha, order, kBlobSamples, h.data());
  if (st) return st;
  float* d = nullptr;
  GTOMRLN_CUDA_TRY(cudaMalloc(&d, kBlobSamples * sizeof(float)));
  GTOMRLN_CUDA_TRY(cudaMemcpy(d, h.data(), kBlobSamples * sizeof(float), cudaMemcpyHostToDevice));
  g_tables[key] = d;
  *out = d;
  return GTOMRLN_OK;
}

// ------------------------------------------------------------- pipeline --
#define GTOMRLN_CUFFT_TRY(expr)                                                         \
  do {                                                                                  \
    cufftResult _r = (expr);                                                            \
    if (_r != CUFFT_SUCCESS) {                                                          \
      st = set_error(GTOMRLN_ERR_CUFFT, "%s failed (%d)", #expr, (int)_r);              \
      goto done;                                                                        \
    }                                                                                   \
  } while (0)

#define GTOMRLN_STEP(expr) \
  do {                     \
    st = (expr);           \
    if (st) goto done;     \
  } while (0)

static int launch_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(GTOMRLN_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return GTOMRLN_OK;
}

// Options beyond the reference's fixed iteration count.
struct GridOptions {
  double tolerance = 0;         // stop when the change measure is <= this (0: fixed count)
  float momentum = 0;           // beta of grid_update_momentum_kernel (0: the plain update)
  const float* mlp = nullptr;   // MLP parameters: predicted start instead of the sphere mask
  float residual_limit = 0.5f;  // the predicted start is kept only if its first change is <= this
  bool weights_only = false;    // stop after the weights (no map)
  float* out_fw = nullptr;      // copies of the final Fweight / Fnewweight on the P grid
  float* out_fnw = nullptr;
  const float* ref_fnw = nullptr;  // reference weights on the P grid: measure the distance to them
  double ref_tolerance = 0;        // and stop when it is <= this (cuFFT path)
};

struct GridResult {
  int iterations = 0;  // iterations run, including one from a rejected predicted start
  double change = 0;   // the last change measure
  int warm_used = 0;   // 1 if the predicted start was kept
  double distance = 0;  // the last distance from the reference weights (when given)
};

static int reconstruct(const float* d_dataft, const float* d_weight, float* d_out, int ori,
                       int oldx, int oldy, int oldz, int pad, cufftHandle planf, cufftHandle planb,
                       int iterations, double radius, int order, double alpha, const GridOptions& opt,
                       GridResult* res, cudaStream_t stream) {
  if (ori <= 0 || pad <= 0) return set_error(GTOMRLN_ERR_INVALID, "gridding: non-positive size");
  if (iterations < 0) return set_error(GTOMRLN_ERR_INVALID, "gridding: negative iteration count");
  if (!d_weight || (!opt.weights_only && (!d_dataft || !d_out)))
    return set_error(GTOMRLN_ERR_INVALID, "gridding: NULL pointer");
  if (!(opt.momentum >= 0.f && opt.momentum < 1.f))
    return set_error(GTOMRLN_ERR_INVALID, "gridding: momentum %g outside [0, 1)", (double)opt.momentum);
  const int P = ori * pad;
  GridGeom g;
  g.P = P;
  g.rowlen = P / 2 + 1;
  g.nc = (int64_t)g.rowlen * P * P;
  g.nr = (int64_t)P * P * P;
  int r_max = ori / 2;
  int maskr2 = (r_max * pad) * (r_max * pad);

  const float* table = nullptr;
  int st = get_table(radius * pad, alpha, order, &table);
  if (st) return st;
  PlanPair plans;

  const bool warm = opt.mlp != nullptr && iterations > 0;
  const bool momentum = opt.momentum > 0.f;
  float2* convft = nullptr;
  float* conv = nullptr;
  float *Fw = nullptr, *Fnw = nullptr, *V = nullptr;
  double* change = nullptr;
  double* sums = nullptr;
  double h_change[4] = {0, 0, 0, 0};  // change sums, then distance-to-reference sums
  const bool measure_ref = opt.ref_fnw != nullptr;
  double last_distance = 0;
  int total_iters = 0;
  double last_change = 0;
  bool warm_live = warm;
  const int T = 256;
  unsigned bc = (unsigned)((g.nc + T - 1) / T);
  const unsigned init_blocks = (unsigned)((P * P + kInitWarps - 1) / kInitWarps);
  // The symmetric-spectrum iteration (gridsym.cu; default on power-of-two
  // grids P = 64 .. 512) or, when the caller chose it, the fused FFT
  // iteration (gridfft.cu); cuFFT transforms otherwise and for the final map.
  const int gpath = path_choice(GTOMRLN_OP_GRIDDING);
  const bool sym = (gpath == GTOMRLN_PATH_SYMMETRIC || gpath == GTOMRLN_PATH_AUTO) && gridsym_available(P);
  const bool fused = !sym && gpath == GTOMRLN_PATH_FUSED && !measure_ref && gridfft_available(P, 1);
  bool need_first = true;  // both start with a transform along z
  if (!sym) {  // the symmetric path makes the final map with its own transforms too
    if (!planf || !planb) GTOMRLN_STEP(get_plans(P, &plans));
    if (planf) plans.r2c = planf;
    if (planb) plans.c2r = planb;
  }

  GTOMRLN_STEP(pool_alloc((void**)&convft, g.nc * sizeof(float2), stream));
  if (!sym) GTOMRLN_STEP(pool_alloc((void**)&conv, g.nr * sizeof(float), stream));
  GTOMRLN_STEP(pool_alloc((void**)&Fw, g.nc * sizeof(float), stream));
  GTOMRLN_STEP(pool_alloc((void**)&Fnw, g.nc * sizeof(float), stream));
  if (momentum) GTOMRLN_STEP(pool_alloc((void**)&V, g.nc * sizeof(float), stream));
  if (opt.tolerance > 0 || warm || measure_ref)
    GTOMRLN_STEP(pool_alloc((void**)&change, sizeof(h_change), stream));
  if (warm) GTOMRLN_STEP(pool_alloc((void**)&sums, 2 * sizeof(double), stream));

  if (!sym) {
    GTOMRLN_CUFFT_TRY(cufftSetStream(plans.r2c, stream));
    GTOMRLN_CUFFT_TRY(cufftSetStream(plans.c2r, stream));
  }

  // the first iteration's spectrum Fw * Fnw: the cuFFT and fused loops read
  // it; the symmetric loop makes its own first transform from Fw and Fnw
  grid_init_kernel<<<init_blocks, 32 * kInitWarps, 0, stream>>>(d_weight, oldx, oldy, oldz, Fw, Fnw, convft, g,
                                                                maskr2, iterations > 0 && !warm && !sym, 0);
  GTOMRLN_STEP(launch_check("grid_init_kernel"));
  if (warm) {
    GTOMRLN_CUDA_TRY(cudaMemsetAsync(sums, 0, 2 * sizeof(double), stream));
    GTOMRLN_STEP(mlp_weight_scale(Fw, P, maskr2, sums, stream));
    GTOMRLN_STEP(mlp_predict_start(opt.mlp, Fw, P, maskr2, sums, Fnw, convft, stream));
  }
  if (momentum) GTOMRLN_CUDA_TRY(cudaMemcpyAsync(V, Fnw, g.nc * sizeof(float), cudaMemcpyDeviceToDevice, stream));

  for (int it = 0; it < iterations; it++) {
    // the residual check of a predicted start needs the first change
    double* ch = (opt.tolerance > 0 || measure_ref || (warm_live && it == 0)) ? change : nullptr;
    if (sym) {
      if (need_first) GTOMRLN_STEP(gridsym_first(convft, g, 1, Fw, Fnw, momentum ? V : nullptr, stream));
      need_first = false;
      if (ch) GTOMRLN_CUDA_TRY(cudaMemsetAsync(ch, 0, sizeof(h_change), stream));
      GTOMRLN_STEP(gridsym_iteration(convft, g, 1, table, Fw, Fnw, momentum ? V : nullptr, opt.momentum,
                                     it + 1 < iterations, ch, opt.ref_fnw, stream));
    } else if (fused) {
      if (need_first) GTOMRLN_STEP(gridfft_first(convft, g, 1, stream));
      need_first = false;
      if (ch) GTOMRLN_CUDA_TRY(cudaMemsetAsync(ch, 0, sizeof(h_change), stream));
      GTOMRLN_STEP(gridfft_iteration(convft, g, 1, table, Fw, Fnw, momentum ? V : nullptr, opt.momentum,
                                     it + 1 < iterations, ch, stream));
    } else {
      GTOMRLN_CUFFT_TRY(cufftExecC2R(plans.c2r, (cufftComplex*)convft, conv));
      launch_blob(conv, table, g, 1, stream);
      GTOMRLN_STEP(launch_check("grid_blob_kernel"));
      GTOMRLN_CUFFT_TRY(cufftExecR2C(plans.r2c, conv, (cufftComplex*)convft));
      if (ch) GTOMRLN_CUDA_TRY(cudaMemsetAsync(ch, 0, sizeof(h_change), stream));
      if (momentum)
        grid_update_momentum_kernel<<<bc, T, 0, stream>>>(convft, Fw, Fnw, V, g, opt.momentum,
                                                          it + 1 < iterations, ch, opt.ref_fnw);
      else
        grid_update_kernel<<<bc, T, 0, stream>>>(convft, Fw, Fnw, g, it + 1 < iterations, ch, opt.ref_fnw);
      GTOMRLN_STEP(launch_check("grid_update_kernel"));
    }
    total_iters++;
    if (ch) {
      GTOMRLN_CUDA_TRY(cudaMemcpyAsync(h_change, ch, sizeof(h_change), cudaMemcpyDeviceToHost, stream));
      GTOMRLN_CUDA_TRY(cudaStreamSynchronize(stream));
      last_change = h_change[1] > 0 ? std::sqrt(h_change[0] / h_change[1]) : 0.0;
      if (measure_ref) last_distance = h_change[3] > 0 ? std::sqrt(h_change[2] / h_change[3]) : 0.0;
      if (warm_live && it == 0) {
        warm_live = false;
        if (!(last_change <= (double)opt.residual_limit)) {
          // Rejected predicted start: the cold start (sphere mask) from scratch.
          grid_init_kernel<<<init_blocks, 32 * kInitWarps, 0, stream>>>(d_weight, oldx, oldy, oldz, Fw, Fnw,
                                                                        convft, g, maskr2, !sym, 0);
          GTOMRLN_STEP(launch_check("grid_init_kernel"));
          need_first = true;
          if (momentum)
            GTOMRLN_CUDA_TRY(cudaMemcpyAsync(V, Fnw, g.nc * sizeof(float), cudaMemcpyDeviceToDevice, stream));
          if (res) res->warm_used = 0;
          it = -1;  // restart the count
          continue;
        }
        if (res) res->warm_used = 1;
      }
      if (opt.tolerance > 0 && last_change <= opt.tolerance) break;
      if (measure_ref && last_distance <= opt.ref_tolerance) break;
      if (it + 1 == iterations) break;
    }
  }

  if (opt.out_fw)
    GTOMRLN_CUDA_TRY(cudaMemcpyAsync(opt.out_fw, Fw, g.nc * sizeof(float), cudaMemcpyDeviceToDevice, stream));
  if (opt.out_fnw)
    GTOMRLN_CUDA_TRY(cudaMemcpyAsync(opt.out_fnw, Fnw, g.nc * sizeof(float), cudaMemcpyDeviceToDevice, stream));
  if (!opt.weights_only && sym) {
    GTOMRLN_STEP(gridsym_final(convft, g, 1, (const float2*)d_dataft, oldx, oldy, oldz, 0, Fw, Fnw,
                               iterations == 0, ori, 1.0f / (float)(pad * pad * pad * ori), d_out, nullptr,
                               stream));
  } else if (!opt.weights_only) {
    grid_final_kernel<<<bc, T, 0, stream>>>((const float2*)d_dataft, oldx, oldy, oldz, Fw, Fnw,
                                            convft, g, iterations == 0, 0);
    GTOMRLN_STEP(launch_check("grid_final_kernel"));
    GTOMRLN_CUFFT_TRY(cufftExecC2R(plans.c2r, (cufftComplex*)convft, conv));
    int64_t total = (int64_t)ori * ori * ori;
    grid_crop_kernel<<<(unsigned)((total + T - 1) / T), T, 0, stream>>>(
        conv, d_out, P, ori, P / 2 - ori / 2, 1.0f / (float)(pad * pad * pad * ori), nullptr);
    GTOMRLN_STEP(launch_check("grid_crop_kernel"));
  }
  if (res) {
    res->iterations = total_iters;
    res->change = last_change;
    res->distance = last_distance;
  }

done:
  pool_free(convft, stream);
  pool_free(conv, stream);
  pool_free(Fw, stream);
  pool_free(Fnw, stream);
  pool_free(V, stream);
  pool_free(change, stream);
  pool_free(sums, stream);
  return st;
}

// ----------------------------------------------------------- batches --
int gridding_batch_prepare(GridBatch* gb, int count, int ori, int pad, double blobradius,
                           int bloborder, double blobalpha) {
  if (count <= 0 || ori <= 0 || pad <= 0 || (ori * pad) % 2)
    return set_error(GTOMRLN_ERR_INVALID, "gridding batch: bad sizes");
  GridBatch b;
  b.count = count;
  b.ori = ori;
  b.pad = pad;
  b.P = ori * pad;
  b.D = b.P + 1;
  b.wstride = (int64_t)(b.D / 2 + 1) * b.D * b.D;
  const int64_t nc = (int64_t)(b.P / 2 + 1) * b.P * b.P, nr = (int64_t)b.P * b.P * b.P;
  int st = get_table(blobradius * pad, blobalpha, bloborder, &b.table);
  if (st) return st;
  // decided (and its tables and kernel attributes set up) here, outside the
  // stream capture of gridding_batch_run
  b.fused = gridfft_available(b.P, count);
  b.sym = gridsym_available(b.P);
  if (b.sym) {
    st = gridsym_prepare(b.P);
    if (st) return st;
  }
  *gb = b;  // so that gridding_batch_free releases what was made on failure
  GTOMRLN_CUDA_TRY(cudaMalloc(&gb->convft, count * nc * sizeof(float2)));
  GTOMRLN_CUDA_TRY(cudaMalloc(&gb->conv, count * nr * sizeof(float)));
  GTOMRLN_CUDA_TRY(cudaMalloc(&gb->Fw, count * nc * sizeof(float)));
  GTOMRLN_CUDA_TRY(cudaMalloc(&gb->Fnw, count * nc * sizeof(float)));
  int n[3] = {b.P, b.P, b.P};
  cufftResult r = cufftPlanMany(&gb->r2c, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, count);
  if (r != CUFFT_SUCCESS) {
    gb->r2c = 0;
    return set_error(GTOMRLN_ERR_CUFFT, "cufftPlanMany R2C %d^3 x %d failed (%d)", b.P, count, (int)r);
  }
  r = cufftPlanMany(&gb->c2r, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, count);
  if (r != CUFFT_SUCCESS) {
    gb->c2r = 0;
    return set_error(GTOMRLN_ERR_CUFFT, "cufftPlanMany C2R %d^3 x %d failed (%d)", b.P, count, (int)r);
  }
  return GTOMRLN_OK;
}

void gridding_batch_free(GridBatch* gb) {
  cudaFree(gb->convft);
  cudaFree(gb->conv);
  cudaFree(gb->Fw);
  cudaFree(gb->Fnw);
  if (gb->r2c) cufftDestroy(gb->r2c);
  if (gb->c2r) cufftDestroy(gb->c2r);
  *gb = GridBatch();
}

// The steps of reconstruct() with a fixed iteration count, each launched once
// over the stack (blockIdx.y = volume) and the transforms as batched plans;
// nothing synchronises the host, so the whole sequence can be captured.
int gridding_batch_run(const GridBatch& b, const float2* data, const float* weight,
                       float* const* outs, int iterations, cudaStream_t stream) {
  GridGeom g;
  g.P = b.P;
  g.rowlen = b.P / 2 + 1;
  g.nc = (int64_t)g.rowlen * b.P * b.P;
  g.nr = (int64_t)b.P * b.P * b.P;
  const int r_max = b.ori / 2;
  const int maskr2 = (r_max * b.pad) * (r_max * b.pad);
  const int T = 256;
  dim3 gc((unsigned)((g.nc + T - 1) / T), (unsigned)b.count);
  const dim3 gi((unsigned)((b.P * b.P + kInitWarps - 1) / kInitWarps), (unsigned)b.count);
  int st = GTOMRLN_OK;
  const int gpath = path_choice(GTOMRLN_OP_GRIDDING);
  const bool sym = b.sym && (gpath == GTOMRLN_PATH_AUTO || gpath == GTOMRLN_PATH_SYMMETRIC);
  const bool fused = !sym && b.fused && gpath == GTOMRLN_PATH_FUSED;
  GTOMRLN_CUFFT_TRY(cufftSetStream(b.r2c, stream));
  GTOMRLN_CUFFT_TRY(cufftSetStream(b.c2r, stream));
  grid_init_kernel<<<gi, 32 * kInitWarps, 0, stream>>>(weight, b.D, b.D, b.D, b.Fw, b.Fnw, b.convft, g, maskr2,
                                         iterations > 0 && !sym, b.wstride);
  GTOMRLN_STEP(launch_check("grid_init_kernel"));
  if (fused && iterations > 0) GTOMRLN_STEP(gridfft_first(b.convft, g, b.count, stream));
  if (sym && iterations > 0) GTOMRLN_STEP(gridsym_first(b.convft, g, b.count, b.Fw, b.Fnw, nullptr, stream));
  for (int it = 0; it < iterations; it++) {
    if (sym) {
      GTOMRLN_STEP(gridsym_iteration(b.convft, g, b.count, b.table, b.Fw, b.Fnw, nullptr, 0.f,
                                     it + 1 < iterations, nullptr, nullptr, stream));
      continue;
    }
    if (fused) {
      GTOMRLN_STEP(gridfft_iteration(b.convft, g, b.count, b.table, b.Fw, b.Fnw, nullptr, 0.f,
                                     it + 1 < iterations, nullptr, stream));
      continue;
    }
    GTOMRLN_CUFFT_TRY(cufftExecC2R(b.c2r, (cufftComplex*)b.convft, b.conv));
    launch_blob(b.conv, b.table, g, b.count, stream);
    GTOMRLN_STEP(launch_check("grid_blob_kernel"));
    GTOMRLN_CUFFT_TRY(cufftExecR2C(b.r2c, b.conv, (cufftComplex*)b.convft));
    grid_update_kernel<<<gc, T, 0, stream>>>(b.convft, b.Fw, b.Fnw, g, it + 1 < iterations, nullptr, nullptr);
    GTOMRLN_STEP(launch_check("grid_update_kernel"));
  }
  if (sym) {
    GTOMRLN_STEP(gridsym_final(b.convft, g, b.count, data, b.D, b.D, b.D, b.wstride, b.Fw, b.Fnw,
                               iterations == 0, b.ori, 1.0f / (float)(b.pad * b.pad * b.pad * b.ori), nullptr,
                               outs, stream));
    goto done;
  }
  grid_final_kernel<<<gc, T, 0, stream>>>(data, b.D, b.D, b.D, b.Fw, b.Fnw, b.convft, g, iterations == 0,
                                          b.wstride);
  GTOMRLN_STEP(launch_check("grid_final_kernel"));
  GTOMRLN_CUFFT_TRY(cufftExecC2R(b.c2r, (cufftComplex*)b.convft, b.conv));
  {
    int64_t total = (int64_t)b.ori * b.ori * b.ori;
    dim3 go((unsigned)((total + T - 1) / T), (unsigned)b.count);
    grid_crop_kernel<<<go, T, 0, stream>>>(b.conv, nullptr, b.P, b.ori, b.P / 2 - b.ori / 2,
                                           1.0f / (float)(b.pad * b.pad * b.pad * b.ori), outs);
    GTOMRLN_STEP(launch_check("grid_crop_kernel"));
  }
done:
  return st;
}

// ------------------------------------------------------- Kaiser-Bessel --
// Fourier transform of the generalised Kaiser-Bessel blob of radius a,
// taper alpha and order m (the function of src/Helpers/KaiserBessel.cpp:
// 357-376), from the closed forms of the Bessel functions of half-integer
// order:
//   I_{1/2}(x) = sqrt(2/(pi x)) sinh x,  I_{3/2}(x) = sqrt(2/(pi x))(cosh x - sinh x / x)
//   J_{1/2}(x) = sqrt(2/(pi x)) sin x,   J_{3/2}(x) = sqrt(2/(pi x))(sin x / x - cos x)
// with the recurrences I_{v+1} = I_{v-1} - (2v/x) I_v and
// J_{v+1} = (2v/x) J_v - J_{v-1}; I_0 by its power series.
static const double kPiD = 3.14159265358979323846;

static double bessel_i0(double x) {
  double t = x * x / 4, term = 1, sum = 1;
  for (int k = 1; k < 500; k++) {
    term *= t / ((double)k * k);
    sum += term;
    if (term < sum * 1e-18) break;
  }
  return sum;
}

static double bessel_half(double x, int twice_order, bool modified) {
  if (x == 0) return 0;
  double f = std::sqrt(2 / (kPiD * x));
  double lo, hi;  // orders 1/2 and 3/2
  if (modified) {
    lo = f * std::sinh(x);
    hi = f * (std::cosh(x) - std::sinh(x) / x);
  } else {
    lo = f * std::sin(x);
    hi = f * (std::sin(x) / x - std::cos(x));
  }
  if (twice_order == 1) return lo;
  for (int v2 = 3; v2 < twice_order; v2 += 2) {
    double next = modified ? lo - ((double)v2 / x) * hi : ((double)v2 / x) * hi - lo;
    lo = hi;
    hi = next;
  }
  return hi;
}

double kaiser_fourier_value(double w, double a, double alpha, int m) {
  double t = 2 * kPiD * a * w;
  double sigma = std::sqrt(std::fabs(alpha * alpha - t * t));
  int twice = m == 0 ? 3 : 7;
  double p = m == 0 ? 1.5 : 3.5;
  double bes = bessel_half(sigma, twice, !(t > alpha));
  double lead = std::pow(2 * kPiD, 1.5) * a * a * a * (m == 2 ? alpha * alpha : 1.0);
  return lead * bes / (bessel_i0(alpha) * std::pow(sigma, p));
}

}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_reconstruct_gridding(const float* d_dataft, const float* d_weight,
                                 float* d_reconstructed, int ox, int oy, int oz, int padx, int pady,
                                 int padz, int paddingfactor, int pre_planforw, int pre_planback,
                                 int iterations, double blobradius, int bloborder,
                                 double blobalpha, void* stream) {
  clear_error();
  (void)oy;
  (void)oz;
  GridOptions opt;
  return reconstruct(d_dataft, d_weight, d_reconstructed, ox, padx, pady, padz, paddingfactor,
                     (cufftHandle)pre_planforw, (cufftHandle)pre_planback, iterations, blobradius,
                     bloborder, blobalpha, opt, nullptr, (cudaStream_t)stream);
}

int gtomrln_reconstruct_gridding_tol(const float* d_dataft, const float* d_weight,
                                     float* d_reconstructed, int ox, int oy, int oz, int padx,
                                     int pady, int padz, int paddingfactor, int max_iterations,
                                     double tolerance, double blobradius, int bloborder,
                                     double blobalpha, int* iterations_done, double* final_change,
                                     void* stream) {
  clear_error();
  (void)oy;
  (void)oz;
  GridOptions opt;
  opt.tolerance = tolerance;
  GridResult res;
  int st = reconstruct(d_dataft, d_weight, d_reconstructed, ox, padx, pady, padz, paddingfactor, 0, 0,
                       max_iterations, blobradius, bloborder, blobalpha, opt, &res, (cudaStream_t)stream);
  if (iterations_done) *iterations_done = res.iterations;
  if (final_change) *final_change = res.change;
  return st;
}

int gtomrln_reconstruct_gridding_warm(const float* d_dataft, const float* d_weight,
                                      float* d_reconstructed, int ox, int oy, int oz, int padx,
                                      int pady, int padz, int paddingfactor, int max_iterations,
                                      double tolerance, float momentum, const float* d_mlp_params,
                                      float residual_limit, double blobradius, int bloborder,
                                      double blobalpha, int* iterations_done, double* final_change,
                                      int* warm_used, void* stream) {
  clear_error();
  (void)oy;
  (void)oz;
  GridOptions opt;
  opt.tolerance = tolerance;
  opt.momentum = momentum;
  opt.mlp = d_mlp_params;
  opt.residual_limit = residual_limit;
  GridResult res;
  int st = reconstruct(d_dataft, d_weight, d_reconstructed, ox, padx, pady, padz, paddingfactor, 0, 0,
                       max_iterations, blobradius, bloborder, blobalpha, opt, &res, (cudaStream_t)stream);
  if (iterations_done) *iterations_done = res.iterations;
  if (final_change) *final_change = res.change;
  if (warm_used) *warm_used = res.warm_used;
  return st;
}

int gtomrln_gridding_weights(const float* d_weight, int ox, int oy, int oz, int ori,
                             int paddingfactor, int max_iterations, double tolerance, float momentum,
                             const float* d_mlp_params, float residual_limit, double blobradius,
                             int bloborder, double blobalpha, float* d_fw, float* d_fnw,
                             int* iterations_done, double* final_change, int* warm_used,
                             const float* d_ref_fnw, double ref_tolerance, double* final_distance,
                             void* stream) {
  clear_error();
  if (!d_fnw) return set_error(GTOMRLN_ERR_INVALID, "gridding_weights: NULL output");
  if (d_ref_fnw && !(ref_tolerance >= 0))
    return set_error(GTOMRLN_ERR_INVALID, "gridding_weights: negative reference tolerance");
  GridOptions opt;
  opt.ref_fnw = d_ref_fnw;
  opt.ref_tolerance = ref_tolerance;
  opt.tolerance = tolerance;
  opt.momentum = momentum;
  opt.mlp = d_mlp_params;
  opt.residual_limit = residual_limit;
  opt.weights_only = true;
  opt.out_fw = d_fw;
  opt.out_fnw = d_fnw;
  GridResult res;
  int st = reconstruct(nullptr, d_weight, nullptr, ori, ox, oy, oz, paddingfactor, 0, 0, max_iterations,
                       blobradius, bloborder, blobalpha, opt, &res, (cudaStream_t)stream);
  if (iterations_done) *iterations_done = res.iterations;
  if (final_change) *final_change = res.change;
  if (warm_used) *warm_used = res.warm_used;
  if (final_distance) *final_distance = res.distance;
  return st;
}

int gtomrln_kaiser_bessel_table(double radius, double alpha, int order, int nsamples,
                                float* h_out) {
  clear_error();
  if (nsamples <= 0 || !h_out) return set_error(GTOMRLN_ERR_INVALID, "kaiser_bessel_table: bad arguments");
  return build_blob_table(radius, alpha, order, nsamples, h_out);
}

}  // extern "C"
