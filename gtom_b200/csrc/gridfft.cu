// Fused FFT iteration of the gridding reconstructor for power-of-two grids
// (P = 64 .. 512): the replacement of d_ReconstructGridding's loop body
// (RecFourier.cu:158-180: Iteration1, C2R (normalised), blob multiply, R2C,
// Iteration2) by two kernels that each stream the working spectrum once.
//
// The 3D transforms of the half-complex spectrum X[z][y][x] (x < P/2 + 1)
// are split by axis.  Between iterations the spectrum is kept transformed
// back along z only.
//
//   gridfft_z_kernel   one CTA per 16 consecutive x at one y: the 16 columns
//                      along z in shared memory; forward transform along z
//                      (completing the 3D forward transform), Iteration2
//                      (the weight update, plain or with momentum, and the
//                      convergence sums), Iteration1 of the next iteration
//                      (Fw * Fnw, real), inverse transform along z;
//   gridfft_xy_kernel  one thread-block cluster of P/32 CTAs per z-plane,
//                      the plane (P x (P/2+1) complex) spread over the
//                      cluster's shared memory: inverse transform along y
//                      on column slabs, an exchange through distributed
//                      shared memory to row slabs, the inverse real
//                      transform along x, the blob multiply (with the
//                      in-loop 1/P^3), the forward real transform along x,
//                      the exchange back, the forward transform along y.
//
// HBM traffic per iteration: 28 B per spectrum element in the z pass
// (spectrum in and out, Fw and Fnw in, Fnw out) and 16 B in the plane pass,
// against the cuFFT path's six passes over the spectrum plus the real grid.
//
// The transforms are radix-8 Stockham FFTs in shared memory (a final radix-4
// or radix-2 stage for P = 256 or 128); each transform of length N is
// computed by N/8 threads holding 8 elements in registers per stage, with
// twiddle factors from a table computed in double precision on the host.
// The real transforms along x take two rows per complex transform: the
// inverse of A + iB (A, B the Hermitian extensions of two rows' half
// spectra, their x = 0 and x = P/2 terms taken as real, as a C2R does) is
// a + ib, and the forward transform of a + ib splits into the two rows'
// spectra by (Z[k] +- conj Z[N-k]) / 2.  Results equal the cuFFT path's to
// FP32 rounding of the transforms.
#include <cooperative_groups.h>

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "fftcore.cuh"
#include "gridfft.cuh"

namespace cg = cooperative_groups;

namespace gtomrln {

namespace {

constexpr int kColsPerCta = 16;  // x columns per CTA (z pass) and per cluster rank (plane pass)
constexpr int kRowsPerCta = 32;  // y rows per cluster rank in the plane pass

// Twiddle table exp(-2 pi i m / N), m < N, per (device, context, N), built
// in double.
std::mutex g_tw_mutex;
std::map<std::tuple<int, unsigned long long, int>, float2*> g_tw;

int twiddles(int N, const float2** out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long ctx = context_id();
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  auto key = std::make_tuple(dev, ctx, N);
  auto it = g_tw.find(key);
  if (it != g_tw.end()) {
    *out = it->second;
    return GTOMRLN_OK;
  }
  std::vector<float2> h(N);
  const double two_pi = 6.283185307179586476925286766559;
  for (int m = 0; m < N; m++) {
    const double a = two_pi * (double)m / (double)N;
    h[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
  }
  float2* d = nullptr;
  GTOMRLN_CUDA_TRY(cudaMalloc(&d, sizeof(float2) * N));
  GTOMRLN_CUDA_TRY(cudaMemcpy(d, h.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
  g_tw[key] = d;
  *out = d;
  return GTOMRLN_OK;
}

// Frees the twiddle tables of the current context on device dev and
// forgets those of earlier contexts there (gone with their context).
int release_tables(int dev, unsigned long long ctx) {
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  for (auto it = g_tw.begin(); it != g_tw.end();) {
    if (std::get<0>(it->first) != dev) {
      ++it;
      continue;
    }
    if (std::get<1>(it->first) == ctx) cudaFree(it->second);
    it = g_tw.erase(it);
  }
  return GTOMRLN_OK;
}

// Shared-memory layout of a transform: element i at i + i/8 (one spare
// slot per 8), which keeps every stage's strided side free of bank
// conflicts; transforms are kTS(N) apart (odd in 8-byte words).
__device__ __forceinline__ int phys(int i) { return i + (i >> 3); }
template <int N>
constexpr int kTS = N + N / 8 + 1;

// Barrier of the threads computing one transform: for N = 512 the 64-thread
// groups t and t + 8 share named barrier 1 + (t mod 8) (the block has 16
// groups, 1024 threads); smaller transforms live within a warp.
template <int N>
__device__ __forceinline__ void group_sync() {
  if (N == 512) {
    const int id = 1 + ((threadIdx.x / (N / 8)) & 7);
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(2 * (N / 8)) : "memory");
  } else {
    __syncwarp();
  }
}

// One Stockham stage of radix R over transforms of length N (Ns = the length
// of the sub-transforms already done).  Each of the N/8 threads of a
// transform takes 8/R butterflies; all reads precede all writes (barrier),
// so the stage runs in place.  Every thread of the block calls it.
template <int R, int N, bool INV>
__device__ __forceinline__ void fft_stage(float2* b, bool active, int j0, int Ns, const float2* tw) {
  constexpr int Q = 8 / R;
  float2 v[8];
  if (active) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const int j = j0 + q * (N / 8);
#pragma unroll
      for (int r = 0; r < R; r++) v[q * R + r] = b[phys(j + r * (N / R))];
    }
  }
  group_sync<N>();
  if (active) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const int j = j0 + q * (N / 8);
      const int k = j & (Ns - 1);
      const int step = N / (Ns * R);
      // W^(r k step) for r = 1 .. R-1 as powers of one table entry (one
      // shared load per butterfly; the table's lanes collide on banks)
      float2 w1 = tw[(k * step) & (N - 1)];
      if (INV) w1.y = -w1.y;
      float2 w = w1;
#pragma unroll
      for (int r = 1; r < R; r++) {
        v[q * R + r] = cmul(v[q * R + r], w);
        if (r + 1 < R) w = cmul(w, w1);
      }
      dft<R, INV>(v + q * R);
      const int d = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) b[phys(d + r * Ns)] = v[q * R + r];
    }
  }
  group_sync<N>();
}

// ntrans transforms of length N at buf + t * kTS<N> (layout phys), by the
// block's first ntrans * N / 8 threads; every thread of the block must call
// it, with the data in place (a block barrier before), and it ends with a
// block barrier.  Unnormalised in both directions (as cuFFT).  For N = 512
// the block must have 1024 threads (group_sync).
template <int N, bool INV>
__device__ __forceinline__ void block_fft(float2* buf, int ntrans, const float2* tw) {
  constexpr int per = N / 8;
  const int t = threadIdx.x / per, j0 = threadIdx.x - t * per;
  const bool active = t < ntrans;
  float2* b = buf + (active ? t : 0) * kTS<N>;
  fft_stage<8, N, INV>(b, active, j0, 1, tw);
  fft_stage<8, N, INV>(b, active, j0, 8, tw);
  if (N == 512) fft_stage<8, N, INV>(b, active, j0, 64, tw);
  if (N == 256) fft_stage<4, N, INV>(b, active, j0, 64, tw);
  if (N == 128) fft_stage<2, N, INV>(b, active, j0, 64, tw);
  __syncthreads();
}

}  // namespace

namespace {

enum : int { kZFirst = 0, kZIter = 1 };

// The z pass over kColsPerCta consecutive x at one y of one volume (grid:
// x groups, P, volumes; 2N threads, each holding 8 tile elements in the
// load, update and store phases, loads issued before use).  kZFirst:
// inverse transform along z.  kZIter: forward transform along z, the
// update, and (write_next) the inverse transform along z of the next
// iteration's Fw * Fnw.
template <int N, int MODE, bool MOM>
__global__ void __launch_bounds__(2 * N)
gridfft_z_kernel(float2* __restrict__ data, const float* __restrict__ Fw, float* __restrict__ Fnw,
                 float* __restrict__ V, GridGeom g, float beta, int write_next, double* __restrict__ change,
                 const float2* __restrict__ twg) {
  extern __shared__ float2 zsm[];
  constexpr int TS = kTS<N>;
  constexpr int U = kColsPerCta * N / (2 * N);  // tile elements per thread
  float2* tw = zsm;
  float2* buf = zsm + N;
  const int rowlen = g.rowlen;
  const int x0 = blockIdx.x * kColsPerCta;
  const int w = min(kColsPerCta, rowlen - x0);
  const int y = blockIdx.y;
  const int64_t vbase = (int64_t)blockIdx.z * g.nc;
  for (int m = threadIdx.x; m < N; m += blockDim.x) tw[m] = twg[m];
  // tile element u of this thread: column c = threadIdx.x mod 16 (the same
  // for all u: blockDim is a multiple of 16), z = threadIdx.x / 16 + u N/8
  // <-> global gbase + u zstep, shared c kTS + phys(z)
  constexpr int ZS = 2 * N / kColsPerCta;  // z step between a thread's elements (N/8)
  const int c = threadIdx.x & (kColsPerCta - 1), zt = threadIdx.x / kColsPerCta;
  const bool in = c < w;
  const int64_t zstep = (int64_t)ZS * g.P * rowlen;
  const int64_t gbase = vbase + ((int64_t)zt * g.P + y) * rowlen + x0 + c;
  float2* sb = buf + c * TS;
  if (in) {
    float2 v[U];
#pragma unroll
    for (int u = 0; u < U; u++) v[u] = data[gbase + u * zstep];
#pragma unroll
    for (int u = 0; u < U; u++) sb[phys(zt + u * ZS)] = v[u];
  }
  __syncthreads();
  if (MODE == kZFirst) {
    block_fft<N, true>(buf, w, tw);
  } else {
    block_fft<N, false>(buf, w, tw);
    double d2 = 0, o2 = 0;
    if (in) {
#pragma unroll
      for (int h = 0; h < U; h += U / 2) {  // two halves: loads of a half in flight together
        float fw[U / 2], old[U / 2], vv[U / 2];
#pragma unroll
        for (int u = 0; u < U / 2; u++) {
          const int64_t gi = gbase + (h + u) * zstep;
          fw[u] = Fw[gi];
          old[u] = Fnw[gi];
          if (MOM) vv[u] = V[gi];
        }
#pragma unroll
        for (int u = 0; u < U / 2; u++) {
          const int64_t gi = gbase + (h + u) * zstep;
          const int si = phys(zt + (h + u) * ZS);
          const float cval = sb[si].x;
          float nw, next;
          if (MOM) {
            grid_update_momentum_value(cval, old[u], vv[u], beta, nw, next);
            V[gi] = next;
          } else {
            nw = grid_update_value(cval, old[u]);
            next = nw;
          }
          Fnw[gi] = nw;
          sb[si] = make_float2(fw[u] * next, 0.f);
          if (change) {
            const double d = (double)fw[u] * ((double)nw - (double)old[u]);
            const double o = (double)fw[u] * (double)old[u];
            d2 += d * d;
            o2 += o * o;
          }
        }
      }
    }
    if (change) grid_change_reduce(d2, o2, change);  // change is uniform over the grid
    __syncthreads();
    if (!write_next) return;  // uniform
    block_fft<N, true>(buf, w, tw);
  }
  if (in) {
#pragma unroll
    for (int u = 0; u < U; u++) data[gbase + u * zstep] = sb[phys(zt + u * ZS)];
  }
}

// The plane pass: one cluster of N/32 CTAs per z-plane of one volume (grid:
// N/32, P, volumes; 2N threads).  Rank r holds x columns [16 r, 16 r + 16)
// (the last rank also x = N/2) for the y transforms and y rows
// [32 r, 32 r + 32) (as 16 pairs) for the x transforms.  Remote (and global)
// loads of a phase are all issued before any is used.
template <int N>
__global__ void __launch_bounds__(2 * N)
gridfft_xy_kernel(float2* __restrict__ data, GridGeom g, const float* __restrict__ table, float inv_n,
                  float funcsampling, const float2* __restrict__ twg) {
  constexpr int C = N / kRowsPerCta;  // cluster size
  constexpr int TS = kTS<N>;
  constexpr int NP = kRowsPerCta / 2;  // row pairs per rank
  constexpr int T = 2 * N;             // threads
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ float2 xsm[];
  float2* tw = xsm;
  float2* col = xsm + N;                       // kColsPerCta columns + the x = N/2 column (last rank)
  float2* row = col + (kColsPerCta + 1) * TS;  // NP row pairs
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int z = blockIdx.y;
  const int rowlen = g.rowlen;
  float2* plane = data + (int64_t)blockIdx.z * g.nc + (int64_t)z * g.P * rowlen;
  const int xa = rank * kColsPerCta;
  const bool last = rank == C - 1;
  const int ya = rank * kRowsPerCta;
  float2* nyq = col + kColsPerCta * TS;  // x = N/2 (last rank)
  for (int m = tid; m < N; m += T) tw[m] = twg[m];
  // column slab: thread column c = tid mod 16, rows y = tid/16 + u T/16
  constexpr int CU = kColsPerCta * N / T;  // 8
  constexpr int CY = T / kColsPerCta;      // N/8
  const int cc = tid & (kColsPerCta - 1), cy = tid / kColsPerCta;
  {
    float2 v[CU];
#pragma unroll
    for (int u = 0; u < CU; u++) v[u] = plane[(int64_t)(cy + u * CY) * rowlen + xa + cc];
    float2 vn = make_float2(0.f, 0.f);
    if (last && tid < N) vn = plane[(int64_t)tid * rowlen + N / 2];
#pragma unroll
    for (int u = 0; u < CU; u++) col[cc * TS + phys(cy + u * CY)] = v[u];
    if (last && tid < N) nyq[phys(tid)] = vn;
  }
  __syncthreads();
  // inverse along y on the column slab
  block_fft<N, true>(col, kColsPerCta, tw);
  block_fft<N, true>(nyq, last ? 1 : 0, tw);
  cluster.sync();
  // row pairs: Z = A + iB over the Hermitian extensions of rows ya + 2p, +1;
  // thread: spectrum index k = tid mod N, pairs p = tid / N + 2u
  constexpr int RU = NP * N / T;  // 8
  const int k = tid & (N - 1), p0 = tid / N;
  {
    const int kk = k <= N / 2 ? k : N - k;
    const int s = min(kk / kColsPerCta, C - 1), lc = kk - s * kColsPerCta;
    const float2* src = cluster.map_shared_rank(col, (unsigned)s) + lc * TS;
    const bool real = k == 0 || k == N / 2, mirror = k > N / 2;
    float2 zv[RU];
#pragma unroll
    for (int u = 0; u < RU; u++) {
      const int yr = ya + 2 * (p0 + 2 * u);
      float2 A = src[phys(yr)], B = src[phys(yr + 1)];
      if (real) {
        A.y = 0.f;
        B.y = 0.f;
      } else if (mirror) {
        A.y = -A.y;
        B.y = -B.y;
      }
      zv[u] = make_float2(A.x - B.y, A.y + B.x);
    }
#pragma unroll
    for (int u = 0; u < RU; u++) row[(p0 + 2 * u) * TS + phys(k)] = zv[u];
  }
  cluster.sync();  // every rank has read the column slabs it needs
  block_fft<N, true>(row, NP, tw);
  // the two real rows of each pair: blob multiply with the in-loop 1/P^3
#pragma unroll
  for (int u = 0; u < RU; u++) {
    const int pp = p0 + 2 * u, y0 = ya + 2 * pp;
    float2 v = row[pp * TS + phys(k)];
    v.x = v.x * inv_n * grid_blob_at(table, N, k, y0, z, funcsampling);
    v.y = v.y * inv_n * grid_blob_at(table, N, k, y0 + 1, z, funcsampling);
    row[pp * TS + phys(k)] = v;
  }
  __syncthreads();
  block_fft<N, false>(row, NP, tw);
  // the two rows' half spectra back to the column slabs,
  // A = (Z[k] + conj Z[N-k]) / 2, B = -i (Z[k] - conj Z[N-k]) / 2:
  // thread k = tid mod N/2, pairs tid / (N/2) + 4u; then k = N/2 for all pairs
  {
    const int kh = tid & (N / 2 - 1), ph = tid / (N / 2);
    const int s = min(kh / kColsPerCta, C - 1), lc = kh - s * kColsPerCta;
    float2* dst = cluster.map_shared_rank(col, (unsigned)s) + lc * TS;
#pragma unroll
    for (int u = 0; u < NP / 4; u++) {
      const int pp = ph + 4 * u;
      const float2 Z = row[pp * TS + phys(kh)], Zm = row[pp * TS + phys((N - kh) & (N - 1))];
      dst[phys(ya + 2 * pp)] = make_float2(0.5f * (Z.x + Zm.x), 0.5f * (Z.y - Zm.y));
      dst[phys(ya + 2 * pp + 1)] = make_float2(0.5f * (Z.y + Zm.y), -0.5f * (Z.x - Zm.x));
    }
    if (tid < NP) {
      const float2 Z = row[tid * TS + phys(N / 2)];  // conj Z[N - N/2] is conj Z[N/2]
      float2* dn = cluster.map_shared_rank(col, (unsigned)(C - 1)) + kColsPerCta * TS;
      dn[phys(ya + 2 * tid)] = make_float2(Z.x, 0.f);
      dn[phys(ya + 2 * tid + 1)] = make_float2(Z.y, 0.f);
    }
  }
  cluster.sync();
  block_fft<N, false>(col, kColsPerCta, tw);
  block_fft<N, false>(nyq, last ? 1 : 0, tw);
#pragma unroll
  for (int u = 0; u < CU; u++) plane[(int64_t)(cy + u * CY) * rowlen + xa + cc] = col[cc * TS + phys(cy + u * CY)];
  if (last && tid < N) plane[(int64_t)tid * rowlen + N / 2] = nyq[phys(tid)];
}

}  // namespace

// ------------------------------------------------------------------ host --
namespace {

template <int N>
size_t z_smem() {
  return sizeof(float2) * (size_t)(N + kColsPerCta * kTS<N>);
}
template <int N>
size_t xy_smem() {
  return sizeof(float2) * (size_t)(N + (kColsPerCta + 1) * kTS<N> + (kRowsPerCta / 2) * kTS<N>);
}

template <int N>
cudaError_t xy_prepare() {
  cudaError_t e = cudaFuncSetAttribute(gridfft_xy_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)xy_smem<N>());
  if (e == cudaSuccess && N / kRowsPerCta > 8)
    e = cudaFuncSetAttribute(gridfft_xy_kernel<N>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

template <int N>
cudaLaunchConfig_t xy_config(int count, cudaStream_t stream, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(N / kRowsPerCta, N, (unsigned)count);
  cfg.blockDim = dim3(2 * N);
  cfg.dynamicSmemBytes = xy_smem<N>();
  cfg.stream = stream;
  attr->id = cudaLaunchAttributeClusterDimension;
  attr->val.clusterDim.x = N / kRowsPerCta;
  attr->val.clusterDim.y = 1;
  attr->val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Sets the kernels' shared-memory limits, builds the twiddle table and tells
// whether a cluster of the plane pass fits this device (cached per device,
// N; to be called outside any stream capture).
template <int N>
bool xy_fits() {
  static std::mutex m;
  static std::map<std::pair<int, unsigned long long>, bool> cache;  // (device, context)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const auto key = std::make_pair(dev, context_id());
  std::lock_guard<std::mutex> lock(m);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  bool ok = false;
  const int zs = (int)z_smem<N>();
  if (xy_prepare<N>() == cudaSuccess &&
      cudaFuncSetAttribute(gridfft_z_kernel<N, kZFirst, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs) ==
          cudaSuccess &&
      cudaFuncSetAttribute(gridfft_z_kernel<N, kZIter, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs) ==
          cudaSuccess &&
      cudaFuncSetAttribute(gridfft_z_kernel<N, kZIter, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs) ==
          cudaSuccess) {
    cudaLaunchAttribute attr;
    cudaLaunchConfig_t cfg = xy_config<N>(1, nullptr, &attr);
    int clusters = 0;
    const float2* tw = nullptr;
    ok = cudaOccupancyMaxActiveClusters(&clusters, gridfft_xy_kernel<N>, &cfg) == cudaSuccess && clusters > 0 &&
         twiddles(N, &tw) == GTOMRLN_OK;
  }
  cudaGetLastError();
  cache[key] = ok;
  return ok;
}

template <int N, int MODE, bool MOM>
int launch_z(float2* data, const GridGeom& g, int count, const float* Fw, float* Fnw, float* V, float beta,
             bool write_next, double* change, cudaStream_t stream) {
  const float2* tw = nullptr;
  int st = twiddles(N, &tw);
  if (st) return st;
  auto kern = gridfft_z_kernel<N, MODE, MOM>;
  dim3 grid((unsigned)((g.rowlen + kColsPerCta - 1) / kColsPerCta), (unsigned)g.P, (unsigned)count);
  kern<<<grid, 2 * N, z_smem<N>(), stream>>>(data, Fw, Fnw, V, g, beta, write_next ? 1 : 0, change, tw);
  GTOMRLN_LAUNCH_CHECK("gridfft_z_kernel");
  return GTOMRLN_OK;
}

template <int N>
int launch_xy(float2* data, const GridGeom& g, int count, const float* table, cudaStream_t stream) {
  const float2* tw = nullptr;
  int st = twiddles(N, &tw);
  if (st) return st;
  cudaLaunchAttribute attr;
  cudaLaunchConfig_t cfg = xy_config<N>(count, stream, &attr);
  GTOMRLN_CUDA_TRY(cudaLaunchKernelEx(&cfg, gridfft_xy_kernel<N>, data, g, table, 1.0f / (float)g.nr,
                                      (float)(0.5 / kBlobSamples), tw));
  return GTOMRLN_OK;
}

template <int N>
int iteration_n(float2* data, const GridGeom& g, int count, const float* table, const float* Fw, float* Fnw,
                float* V, float beta, bool write_next, double* change, cudaStream_t stream) {
  int st = launch_xy<N>(data, g, count, table, stream);
  if (st) return st;
  if (V)
    return launch_z<N, kZIter, true>(data, g, count, Fw, Fnw, V, beta, write_next, change, stream);
  return launch_z<N, kZIter, false>(data, g, count, Fw, Fnw, nullptr, 0.f, write_next, change, stream);
}

}  // namespace

bool gridfft_available(int P, int count) {
  if (count < 1 || count > 65535) return false;
  switch (P) {
    case 64: return xy_fits<64>();
    case 128: return xy_fits<128>();
    case 256: return xy_fits<256>();
    case 512: return xy_fits<512>();
    default: return false;
  }
}

int gridfft_first(float2* data, const GridGeom& g, int count, cudaStream_t stream) {
  switch (g.P) {
    case 64: return launch_z<64, kZFirst, false>(data, g, count, nullptr, nullptr, nullptr, 0.f, false, nullptr, stream);
    case 128: return launch_z<128, kZFirst, false>(data, g, count, nullptr, nullptr, nullptr, 0.f, false, nullptr, stream);
    case 256: return launch_z<256, kZFirst, false>(data, g, count, nullptr, nullptr, nullptr, 0.f, false, nullptr, stream);
    case 512: return launch_z<512, kZFirst, false>(data, g, count, nullptr, nullptr, nullptr, 0.f, false, nullptr, stream);
    default: return set_error(GTOMRLN_ERR_INVALID, "fused gridding: grid %d not supported", g.P);
  }
}

int gridfft_iteration(float2* data, const GridGeom& g, int count, const float* table, const float* Fw,
                      float* Fnw, float* V, float beta, bool write_next, double* change, cudaStream_t stream) {
  switch (g.P) {
    case 64: return iteration_n<64>(data, g, count, table, Fw, Fnw, V, beta, write_next, change, stream);
    case 128: return iteration_n<128>(data, g, count, table, Fw, Fnw, V, beta, write_next, change, stream);
    case 256: return iteration_n<256>(data, g, count, table, Fw, Fnw, V, beta, write_next, change, stream);
    case 512: return iteration_n<512>(data, g, count, table, Fw, Fnw, V, beta, write_next, change, stream);
    default: return set_error(GTOMRLN_ERR_INVALID, "fused gridding: grid %d not supported", g.P);
  }
}

// Frees the fused transforms' tables of the current context on device dev
// (gtomrln_release_caches).
int release_gridfft_tables(int dev, unsigned long long ctx) { return release_tables(dev, ctx); }

int fft_twiddles(int N, const float2** out) { return twiddles(N, out); }

}  // namespace gtomrln
