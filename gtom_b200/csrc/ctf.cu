// CTF simulation and particle preprocessing before insertion.
//
// gtomrln_ctf_simulate is the B200 replacement of gtom::d_CTFSimulate
// (include/CTF.cuh:317, src/CTF/Simulate.cu:22-47 and :117-139, with
// d_GetCTF of include/CTF.cuh:195-223 and the parameter conversion of
// CTFParamsLean, include/CTF.cuh:100-137).  gtomrln_preprocess_particles
// is the step every caller makes before d_rlnBackproject: batched R2C of
// the real-space particles, the phase that moves their centre to the
// origin, and the CTF: it writes CTF * FT (the data to insert) and CTF^2
// (the weights) in one pass over the transform, with the CTF evaluated in
// registers rather than stored.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"

namespace gtomrln {

// CTFParamsLean: lengths in Angstrom, the wavelength and K1..K3 derived in
// the reference's precision (float members, double intermediate terms).
struct CtfLean {
  float pixelsize, pixeldelta, pixelangle, lambda, defocus, astigmatismangle, defocusdelta, Cs,
      scale, phaseshift, K1, K2, K3, Bfactor, Bfactordelta, Bfactorangle;
};

static CtfLean make_lean(const gtomrln_ctf_params_t& p) {
  const float pi = 3.14159265358979323846f, pihalf = 1.57079632679489661923f;
  CtfLean l;
  l.pixelsize = (float)(p.pixelsize * 1e10);
  l.pixeldelta = (float)(p.pixeldelta * 0.5e10);
  l.pixelangle = p.pixelangle;
  l.lambda = (float)(12.2643247 / std::sqrt(p.voltage * (1.0 + p.voltage * 0.978466e-6)));
  l.defocus = (float)(p.defocus * 1e10);
  l.astigmatismangle = p.astigmatismangle;
  l.defocusdelta = (float)(p.defocusdelta * 0.5e10);
  l.Cs = (float)(p.Cs * 1e10);
  l.scale = p.scale;
  l.phaseshift = p.phaseshift;
  l.K1 = pi * l.lambda;
  l.K2 = (float)(pihalf * (p.Cs * 1e10) * l.lambda * l.lambda * l.lambda);
  l.K3 = (float)std::atan(p.amplitude / std::sqrt(1.0f - p.amplitude * p.amplitude));
  l.Bfactor = (float)(p.Bfactor * 0.25e20);
  l.Bfactordelta = (float)(p.Bfactordelta * 0.25e20);
  l.Bfactorangle = p.Bfactorangle;
  return l;
}

// d_GetCTF at spatial frequency r (1/Angstrom) and azimuth angle, with the
// reference's fast sine/cosine/exponential.
template <bool SQUARED_AMP, bool IGNORE_FIRST_PEAK>
__device__ __forceinline__ float ctf_value(float r, float angle, float gammacorr, const CtfLean& p) {
  float r2 = r * r;
  float r4 = r2 * r2;
  float deltaf = fmaf(p.defocusdelta, __cosf(2.f * (angle - p.astigmatismangle)), p.defocus);
  float gamma = fmaf(p.K1 * deltaf, r2, p.K2 * r4) - p.phaseshift - p.K3 + gammacorr;
  float v;
  if (IGNORE_FIRST_PEAK && fabsf(gamma) < 1.57079632679489661923f)
    v = 1.f;
  else
    v = -__sinf(gamma);
  if (p.Bfactor != 0.f || p.Bfactordelta != 0.f) {
    float b = p.Bfactor;
    if (p.Bfactordelta != 0.f) b = fmaf(p.Bfactordelta, __cosf(2.f * (angle - p.Bfactorangle)), b);
    v *= __expf(b * r2);
  }
  if (SQUARED_AMP) v = fabsf(v);
  return v * p.scale;
}

// CTFSimulateKernel: address = (frequency in 1/pixel, angle); the pixel
// size may vary with the angle.
template <bool SQ, bool IGN>
__global__ void ctf_simulate_kernel(float* __restrict__ out, const float2* __restrict__ addresses,
                                    const float* __restrict__ gammacorr, unsigned n,
                                    const CtfLean* __restrict__ params) {
  const CtfLean p = params[blockIdx.y];
  out += (size_t)blockIdx.y * n;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 a = addresses[i];
    float ps = fmaf(p.pixeldelta, __cosf(2.0f * (a.y - p.pixelangle)), p.pixelsize);
    float k = __fdividef(a.x, ps);
    float g = gammacorr ? gammacorr[i] : 0.f;
    out[i] = ctf_value<SQ, IGN>(k, a.y, g, p);
  }
}

// Particle preprocessing: x and y signed frequencies of the half-complex
// element, the CTF at (sqrt(x^2 + y^2) / n, atan2(y, x)) as
// ctf_simulate_kernel evaluates it for that address, the phase (-1)^(x+y)
// that moves the image centre (n/2, n/2) to the origin, and the products.
// One thread per element for kPrePB consecutive particles: the element's
// frequency, radius and azimuth are formed once, the particles' values are
// loaded before any is used (kPrePB loads in flight), and the CTF of each
// particle is evaluated as ctf_simulate_kernel does for that address.
constexpr int kPrePB = 4;
__global__ void __launch_bounds__(256, 4)
preprocess_kernel(float2* __restrict__ ft, float* __restrict__ weights, int n, int batch,
                  const CtfLean* __restrict__ params) {
  const int dimft = n / 2 + 1;
  const int e = dimft * n;  // the launcher keeps it below 2^31
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= e) return;
  const int x = i % dimft, idy = i / dimft;
  const int y = idy <= n / 2 ? idy : idy - n;
  const bool odd = (x + idy) & 1;
  float angle = 0.f, r = 0.f;
  if (params) {
    angle = atan2f((float)y, (float)x);
    r = sqrtf((float)(x * x + y * y)) / (float)n;
  }
  const int b0 = blockIdx.y * kPrePB;
  float2 v[kPrePB];
#pragma unroll
  for (int k = 0; k < kPrePB; k++)
    if (b0 + k < batch) v[k] = ft[(int64_t)(b0 + k) * e + i];
#pragma unroll
  for (int k = 0; k < kPrePB; k++) {
    const int b = b0 + k;
    if (b >= batch) break;
    float c = 1.f;
    if (params) {
      const CtfLean& p = params[b];
      const float ps = fmaf(p.pixeldelta, __cosf(2.0f * (angle - p.pixelangle)), p.pixelsize);
      c = ctf_value<false, false>(__fdividef(r, ps), angle, 0.f, p);
    }
    const float s = odd ? -c : c;
    const int64_t j = (int64_t)b * e + i;
    ft[j] = make_float2(v[k].x * s, v[k].y * s);
    if (weights) weights[j] = c * c;
  }
}

static std::mutex g_ctf_mutex;
// (device, context, n, batch)
static std::map<std::tuple<int, unsigned long long, int, unsigned>, cufftHandle> g_r2c_plans;

// Destroys the plans of the current context on device dev and forgets those
// of earlier contexts there (gone with their context).
int release_ctf_plans(int dev, unsigned long long ctx) {
  std::lock_guard<std::mutex> lock(g_ctf_mutex);
  for (auto it = g_r2c_plans.begin(); it != g_r2c_plans.end();) {
    if (std::get<0>(it->first) != dev) {
      ++it;
      continue;
    }
    if (std::get<1>(it->first) == ctx) cufftDestroy(it->second);
    it = g_r2c_plans.erase(it);
  }
  return GTOMRLN_OK;
}

static int r2c_plan(int n, unsigned batch, cufftHandle* out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  std::lock_guard<std::mutex> lock(g_ctf_mutex);
  auto key = std::make_tuple(dev, ctx, n, batch);
  auto it = g_r2c_plans.find(key);
  if (it != g_r2c_plans.end()) {
    *out = it->second;
    return GTOMRLN_OK;
  }
  int dims[2] = {n, n};
  cufftHandle h;
  cufftResult r = cufftPlanMany(&h, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, (int)batch);
  if (r != CUFFT_SUCCESS) return set_error(GTOMRLN_ERR_CUFFT, "cufftPlanMany R2C %d^2 x %u failed (%d)", n, batch, (int)r);
  g_r2c_plans[key] = h;
  *out = h;
  return GTOMRLN_OK;
}

static int upload_lean(const gtomrln_ctf_params_t* h_params, unsigned batch, cudaStream_t stream, CtfLean** d) {
  std::vector<CtfLean> lean(batch);
  for (unsigned i = 0; i < batch; i++) lean[i] = make_lean(h_params[i]);
  int st = pool_alloc((void**)d, batch * sizeof(CtfLean), stream);
  if (st) return st;
  cudaError_t e = cudaMemcpyAsync(*d, lean.data(), batch * sizeof(CtfLean), cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) {
    pool_free(*d, stream);
    return set_error(GTOMRLN_ERR_CUDA, "CTF parameter upload failed: %s", cudaGetErrorString(e));
  }
  return GTOMRLN_OK;
}

}  // namespace gtomrln

using namespace gtomrln;

extern "C" {

int gtomrln_ctf_simulate(const gtomrln_ctf_params_t* h_params, const float* d_addresses,
                         const float* d_gammacorrection, float* d_output, unsigned n,
                         int amplitudesquared, int ignorefirstpeak, int batch, void* stream) {
  clear_error();
  if (batch < 0) return set_error(GTOMRLN_ERR_INVALID, "ctf_simulate: negative batch");
  if (batch == 0 || n == 0) return GTOMRLN_OK;
  if (!h_params || !d_addresses || !d_output) return set_error(GTOMRLN_ERR_INVALID, "ctf_simulate: NULL pointer");
  if (batch > 65535) return set_error(GTOMRLN_ERR_INVALID, "ctf_simulate: batch above 65535");
  cudaStream_t s = (cudaStream_t)stream;
  CtfLean* d = nullptr;
  int st = upload_lean(h_params, (unsigned)batch, s, &d);
  if (st) return st;
  unsigned tpb = 128;
  dim3 grid((unsigned)std::min<unsigned>(1024u, (n + tpb - 1) / tpb), (unsigned)batch);
  const float2* a = (const float2*)d_addresses;
  if (amplitudesquared) {
    if (ignorefirstpeak) ctf_simulate_kernel<true, true><<<grid, tpb, 0, s>>>(d_output, a, d_gammacorrection, n, d);
    else ctf_simulate_kernel<true, false><<<grid, tpb, 0, s>>>(d_output, a, d_gammacorrection, n, d);
  } else {
    if (ignorefirstpeak) ctf_simulate_kernel<false, true><<<grid, tpb, 0, s>>>(d_output, a, d_gammacorrection, n, d);
    else ctf_simulate_kernel<false, false><<<grid, tpb, 0, s>>>(d_output, a, d_gammacorrection, n, d);
  }
  cudaError_t e = cudaGetLastError();
  pool_free(d, s);
  if (e != cudaSuccess) return set_error(GTOMRLN_ERR_CUDA, "launch of ctf_simulate_kernel failed: %s", cudaGetErrorString(e));
  return GTOMRLN_OK;
}

int gtomrln_preprocess_particles(const float* d_images, int n, unsigned batch,
                                 const gtomrln_ctf_params_t* h_params, float* d_projft,
                                 float* d_projweights, void* stream) {
  clear_error();
  if (n < 2 || (n & 1) || n > 32768)
    return set_error(GTOMRLN_ERR_INVALID, "preprocess_particles: n must be even, 2 .. 32768");
  if (batch == 0) return GTOMRLN_OK;
  if (!d_images || !d_projft) return set_error(GTOMRLN_ERR_INVALID, "preprocess_particles: NULL pointer");
  if (batch > 65535) return set_error(GTOMRLN_ERR_INVALID, "preprocess_particles: batch above 65535 (split it)");
  cudaStream_t s = (cudaStream_t)stream;
  cufftHandle plan;
  int st = r2c_plan(n, batch, &plan);
  if (st) return st;
  CtfLean* d = nullptr;
  if (h_params) {
    st = upload_lean(h_params, batch, s, &d);
    if (st) return st;
  }
  cufftResult r = cufftSetStream(plan, s);
  if (r == CUFFT_SUCCESS) r = cufftExecR2C(plan, (cufftReal*)d_images, (cufftComplex*)d_projft);
  if (r != CUFFT_SUCCESS) {
    pool_free(d, s);
    return set_error(GTOMRLN_ERR_CUFFT, "cufftExecR2C failed (%d)", (int)r);
  }
  const int64_t e = (int64_t)(n / 2 + 1) * n;
  dim3 grid((unsigned)((e + 255) / 256), (batch + kPrePB - 1) / kPrePB);
  preprocess_kernel<<<grid, 256, 0, s>>>((float2*)d_projft, d_projweights, n, (int)batch, d);
  cudaError_t ce = cudaGetLastError();
  pool_free(d, s);
  if (ce != cudaSuccess) return set_error(GTOMRLN_ERR_CUDA, "launch of preprocess_kernel failed: %s", cudaGetErrorString(ce));
  return GTOMRLN_OK;
}

}  // extern "C"
