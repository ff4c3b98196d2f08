// Gridding iteration on the symmetric half of the spectrum: the replacement
// of d_ReconstructGridding's loop body (RecFourier.cu:158-171: Iteration1,
// C2R, blob multiply, R2C, Iteration2) by four streaming passes over half
// the data the 3D transforms would touch.
//
// Why half.  The spectrum the loop transforms is real: Iteration1 writes
// (Fw * Fnw, 0), and Iteration2 reads only the real part of what the R2C
// returns.  For a real half spectrum S(kx, ky, kz) (kx <= P/2) the
// transform along z,
//   T1(kx, ky, z) = sum_kz S(kx, ky, kz) e(+kz z / P),     e(a) = exp(2 pi i a),
// is Hermitian in z (T1(., ., -z) = conj T1(., ., z)), so z in [0, P/2]
// holds all of it; the transforms along y and x keep that range (the real
// grid of the C2R is point-symmetric, f(-r) = f(r), as is the blob, so the
// planes z in [0, P/2] of the real grid determine the rest), and the last
// transform back along z is Hermitian-to-real.  Every intermediate array
// therefore has (P/2 + 1) x P x (P/2 + 1) complex elements, half the
// (P/2 + 1) x P x P of the cuFFT path's spectrum, and the real grid never
// leaves the chip.  The imaginary parts the cuFFT path computes and drops
// are zero up to rounding; the kept real parts are the same sums.
//
// Per iteration (W: the (P/2+1) x P x (P/2+1) complex work array, layout
// [z][y][x] with rows of P/2 + 1 like the reference's spectra):
//   gridsym_y_kernel<INV>  inverse transform along y of W (columns of 16
//                          consecutive x at one z, or of x = P/2 at 16 z);
//   gridsym_x_kernel       per row (y, z): C2R along x, times blob(r)/P^3
//                          (IFFT.cu:36-46 normalisation, RecFourier.cu:
//                          243-262 table), R2C along x;
//   gridsym_y_kernel<FWD>  forward transform along y;
//   gridsym_z_kernel       per column (x, y): Hermitian-to-real transform
//                          along z (the real part of the R2C), Iteration2
//                          (the weight update, plain or with momentum, the
//                          convergence sums), then Iteration1 of the next
//                          iteration and the real-to-Hermitian transform
//                          along z of Fw * Fnw.
// HBM bytes per iteration: W in and out in each pass (4 x 16 B per W
// element) plus Fw in, Fnw in and out in the z pass (12 B per spectrum
// element): 2.97 GB at P = 512, against ~8 GB for cuFFT's passes plus the
// blob and update kernels.
//
// The real transforms of length P run as complex transforms of length P/2
// on the packed pairs (x(2n), x(2n+1)) with the usual pre- and post-
// twiddles; the complex transforms are Stockham radix-8 (radix-4/2 last
// stage) FFTs over 16 columns in shared memory (element n of column c at
// n * 17 + c: conflict-free for the column-wise stages and for the row-wise
// loads of the x pass), 16 threads per column, twiddles read from a table
// e(-m/P) computed in double precision.  All transforms are unnormalised,
// as cuFFT's; the 1/P^3 of the reference's C2R rides with the blob.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "fftcore.cuh"
#include "gridfft.cuh"

namespace gtomrln {

namespace {

constexpr int kCols = 16;          // columns (rows in the x pass) per CTA
constexpr int kPitch = kCols + 1;  // shared-memory stride of element index n, in float2
constexpr int kThreads = 256;      // 16 threads per column

// Twiddle e(-m/N) (forward) or e(+m/N) (INV) of an N-point transform from
// the table e(-j/P) of the working grid, N = P/S.
template <int S, bool INV>
__device__ __forceinline__ float2 twiddle(const float2* tw, int m) {
  float2 w = tw[m * S];
  if (INV) w.y = -w.y;
  return w;
}

template <int N, int Ns>
constexpr int stage_radix() {
  return N / Ns >= 8 ? 8 : N / Ns;
}

// Stockham stages from sub-transform length Ns on over the CTA's 16
// columns (column c, thread t of the column's 16): each butterfly reads R
// elements, applies the twiddles and a radix-R DFT, and writes its R
// outputs to their sorted places; all reads of a stage precede all its
// writes (barrier), so the transform runs in place.
template <int N, int S, bool INV, int Ns>
__device__ __forceinline__ void fft_stages(float2* s, const float2* tw, int c, int t) {
  if constexpr (Ns < N) {
    constexpr int R = stage_radix<N, Ns>();
    constexpr int NB = N / R;                    // butterflies per column
    constexpr int Q = (NB + kCols - 1) / kCols;  // per thread
    float2 v[Q][R];
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const int j = t + kCols * q;
      if (NB % kCols == 0 || j < NB) {
#pragma unroll
        for (int r = 0; r < R; r++) v[q][r] = s[(j + r * NB) * kPitch + c];
        const int k = j & (Ns - 1);
#pragma unroll
        for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], twiddle<S, INV>(tw, r * k * (N / (Ns * R))));
        dft<R, INV>(v[q]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const int j = t + kCols * q;
      if (NB % kCols == 0 || j < NB) {
        const int k = j & (Ns - 1);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) s[(d + r * Ns) * kPitch + c] = v[q][r];
      }
    }
    __syncthreads();
    fft_stages<N, S, INV, Ns * R>(s, tw, c, t);
  }
}

// N-point transforms (unnormalised; INV: exp(+)) of the 16 columns.  The
// data must be in place (barrier before); ends with a barrier.
template <int N, int S, bool INV>
__device__ __forceinline__ void fft_cols(float2* s, const float2* tw, int c, int t) {
  fft_stages<N, S, INV, 1>(s, tw, c, t);
}

// Pre-twiddle of a Hermitian-to-real transform of length P computed as a
// complex transform of length H = P/2: from the half spectrum X(0..H) of a
// column, Z(k) = (X(k) + conj X(H-k)) + i e(sg k/P) (X(k) - conj X(H-k)),
// k < H (sg = +1: the inverse C2R, sg = -1: the forward sum).  The H-point
// transform of the same sign then gives x(2n) = Re z(n), x(2n+1) = Im z(n).
// In place; thread t of the column takes the pairs (k, H-k), k <= H/2.
template <int H, bool PLUS>
__device__ __forceinline__ void c2r_pre(float2* s, const float2* tw, int c, int t) {
  for (int k = t; k <= H / 2; k += kCols) {
    const float2 xk = s[k * kPitch + c], xm = s[(H - k) * kPitch + c];
    // e(sg k/P) with sg = +1 for PLUS, -1 otherwise; the table holds e(-j/P)
    float2 w = tw[k];
    if (PLUS) w.y = -w.y;
    {
      const float2 a = make_float2(xk.x + xm.x, xk.y - xm.y);  // X(k) + conj X(H-k)
      const float2 b = make_float2(xk.x - xm.x, xk.y + xm.y);  // X(k) - conj X(H-k)
      const float2 wb = cmul(w, b);
      s[k * kPitch + c] = make_float2(a.x - wb.y, a.y + wb.x);  // a + i wb
    }
    if (k != 0 && 2 * k != H) {
      // the partner H-k: e(sg (H-k)/P) = -conj e(sg k/P)
      const float2 w2 = make_float2(-w.x, w.y);
      const float2 a = make_float2(xm.x + xk.x, xm.y - xk.y);
      const float2 b = make_float2(xm.x - xk.x, xm.y + xk.y);
      const float2 wb = cmul(w2, b);
      s[(H - k) * kPitch + c] = make_float2(a.x - wb.y, a.y + wb.x);
    }
  }
  __syncthreads();
}

// Post-twiddle of a real-to-Hermitian transform of length P computed as a
// complex transform of length H of the packed pairs z(n) = x(2n) + i x(2n+1):
// Y(k) = (Z(k) + conj Z(H-k)) / 2 - (i/2) e(sg k/P) (Z(k) - conj Z(H-k)),
// k = 0 .. H (Z indices mod H; sg = -1: the forward R2C, sg = +1: the
// transform with exp(+)).  In place, Y(H) into row H.
template <int H, bool PLUS>
__device__ __forceinline__ void r2c_post(float2* s, const float2* tw, int c, int t) {
  for (int k = t; k <= H / 2; k += kCols) {
    const int km = k == 0 ? 0 : H - k;
    const float2 zk = s[k * kPitch + c], zm = s[km * kPitch + c];
    float2 w = tw[k];
    if (PLUS) w.y = -w.y;
    {
      const float2 a = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));  // (Z(k) + conj Z(H-k)) / 2
      const float2 b = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));  // (Z(k) - conj Z(H-k)) / 2
      const float2 wb = cmul(w, b);
      s[k * kPitch + c] = make_float2(a.x + wb.y, a.y - wb.x);  // a - i wb
    }
    // partner: H-k (k > 0), or H itself for k = 0, with e(sg (H-k)/P) = -conj e(sg k/P)
    if (2 * k != H) {
      const int kp = H - k;
      const float2 w2 = make_float2(-w.x, w.y);
      const float2 a = make_float2(0.5f * (zm.x + zk.x), 0.5f * (zm.y - zk.y));
      const float2 b = make_float2(0.5f * (zm.x - zk.x), 0.5f * (zm.y + zk.y));
      const float2 wb = cmul(w2, b);
      s[kp * kPitch + c] = make_float2(a.x + wb.y, a.y - wb.x);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void load_twiddles(float2* tw, const float2* __restrict__ twg, int P) {
  for (int m = threadIdx.x; m < P; m += blockDim.x) tw[m] = __ldg(twg + m);
}

// The transform along y of W (INV: exp(+), the inverse of the C2R; else
// the forward of the R2C).  Grid: (tiles, volumes); tiles are 16
// consecutive x < P/2 at one z, then x = P/2 at 16 consecutive z.
template <int P, bool INV>
__global__ void __launch_bounds__(kThreads, 3)
gridsym_y_kernel(float2* __restrict__ W, const float2* __restrict__ twg) {
  constexpr int H = P / 2, R = H + 1;
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* s = smem + P;
  load_twiddles(tw, twg, P);
  const int c = threadIdx.x & (kCols - 1), t = threadIdx.x / kCols;
  constexpr int kMain = (H / kCols) * (H + 1);
  const int b = blockIdx.x;
  int64_t base, cs;
  int ncols;
  if (b < kMain) {
    const int z = b / (H / kCols), xt = b - z * (H / kCols);
    base = (int64_t)z * P * R + xt * kCols;
    cs = 1;
    ncols = kCols;
  } else {
    const int z0 = (b - kMain) * kCols;
    base = (int64_t)z0 * P * R + H;
    cs = (int64_t)P * R;
    ncols = min(kCols, H + 1 - z0);
  }
  float2* col = W + (int64_t)blockIdx.y * ((int64_t)(H + 1) * P * R) + base + c * cs;
  const bool in = c < ncols;
  constexpr int U = P / kCols;  // elements per thread
  constexpr int UB = U < 8 ? U : 8;
#pragma unroll
  for (int u0 = 0; u0 < U; u0 += UB) {
    float2 v[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) v[u] = in ? col[(int64_t)(t + kCols * (u0 + u)) * R] : make_float2(0.f, 0.f);
#pragma unroll
    for (int u = 0; u < UB; u++) s[(t + kCols * (u0 + u)) * kPitch + c] = v[u];
  }
  __syncthreads();
  fft_cols<P, 1, INV>(s, tw, c, t);
  if (in) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int n = t + kCols * u;
      col[(int64_t)n * R] = s[n * kPitch + c];
    }
  }
}

// Per row (y, z), z <= P/2: C2R along x, times blob(r) / P^3, R2C along x.
// Grid: ((P/2 + 1) P / 16, volumes); a CTA takes 16 consecutive rows.
template <int P>
__global__ void __launch_bounds__(kThreads, 2)
gridsym_x_kernel(float2* __restrict__ W, const float2* __restrict__ twg, const float* __restrict__ table,
                 float inv_n, float funcsampling) {
  constexpr int H = P / 2, R = H + 1;
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* s = smem + P;
  float* stab = reinterpret_cast<float*>(s + (H + 1) * kPitch);
  load_twiddles(tw, twg, P);
  for (int i = threadIdx.x; i < kBlobSamples; i += blockDim.x) stab[i] = __ldg(table + i);
  const int c = threadIdx.x & (kCols - 1), t = threadIdx.x / kCols;
  const int64_t row0 = (int64_t)blockIdx.x * kCols;
  float2* rows = W + (int64_t)blockIdx.y * ((int64_t)(H + 1) * P * R) + row0 * R;
  // the 16 rows are 16 R consecutive elements
  constexpr int E = kCols * R;
  for (int e0 = 0; e0 < E; e0 += 4 * kThreads) {
    float2 v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int e = e0 + u * kThreads + threadIdx.x;
      if (e < E) v[u] = rows[e];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int e = e0 + u * kThreads + threadIdx.x;
      if (e < E) {
        const int r = e / R, x = e - r * R;
        s[x * kPitch + r] = v[u];
      }
    }
  }
  __syncthreads();
  c2r_pre<H, true>(s, tw, c, t);
  fft_cols<H, 2, true>(s, tw, c, t);
  {
    // blob: grid_blob_kernel's table index (radius sqrt(x^2 + y^2 + z^2) / P
    // / funcsampling in FP32 with the row part formed first)
    const int rg = (int)(row0 + c);  // z * P + y
    const int z = rg / P, y = rg - z * P;
    const int zp = z < H ? z : z - P, yp = y < H ? y : y - P;
    const float cyz = (float)(yp * yp + zp * zp);
    const float inv_p = __frcp_rn((float)P);
    for (int n = t; n < H; n += kCols) {
      float2 v = s[n * kPitch + c];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int x = 2 * n + h;
        const float xp = (float)(x < H ? x : x - P);
        const float sq = sqrtf(xp * xp + cyz);
        int ti = (int)((sq * inv_p) / funcsampling);
        ti = ti < kBlobSamples - 1 ? ti : kBlobSamples - 1;
        if (h == 0) v.x = v.x * inv_n * stab[ti];
        else v.y = v.y * inv_n * stab[ti];
      }
      s[n * kPitch + c] = v;
    }
  }
  __syncthreads();
  fft_cols<H, 2, false>(s, tw, c, t);
  r2c_post<H, false>(s, tw, c, t);
  for (int e0 = 0; e0 < E; e0 += kThreads) {
    const int e = e0 + threadIdx.x;
    if (e < E) {
      const int r = e / R, x = e - r * R;
      rows[e] = s[x * kPitch + r];
    }
  }
}

enum : int { kZFirst = 0, kZIter = 1 };

// Per column (x, y) along z.  kZFirst: the real-to-Hermitian transform
// (exp(+)) of S = Fw * Fnw (Fw * V with momentum) into W.  kZIter: the
// Hermitian-to-real transform (exp(-)) of W, the update of Fnw (and V) from
// its values, and with write_next the transform of the new S into W.
// change (single volume): sums of grid_update_kernel; ref: the distance sums
// to reference weights as well.  Grid: (tiles, volumes); tiles are 16
// consecutive x < P/2 at one y, then x = P/2 at 16 consecutive y.
template <int P, int MODE, bool MOM>
__global__ void __launch_bounds__(kThreads, 3)
gridsym_z_kernel(float2* __restrict__ W, const float* __restrict__ Fw, float* __restrict__ Fnw,
                 float* __restrict__ V, const float2* __restrict__ twg, float beta, int write_next,
                 double* __restrict__ change, const float* __restrict__ ref) {
  constexpr int H = P / 2, R = H + 1;
  constexpr int64_t NC = (int64_t)R * P * P;        // spectrum elements per volume
  constexpr int64_t NW = (int64_t)(H + 1) * P * R;  // W elements per volume
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* s = smem + P;
  load_twiddles(tw, twg, P);
  const int c = threadIdx.x & (kCols - 1), t = threadIdx.x / kCols;
  constexpr int kMain = P * (H / kCols);
  const int b = blockIdx.x;
  int64_t base, cs;
  int ncols;
  if (b < kMain) {
    const int y = b / (H / kCols), xt = b - y * (H / kCols);
    base = (int64_t)y * R + xt * kCols;
    cs = 1;
    ncols = kCols;
  } else {
    const int y0 = (b - kMain) * kCols;
    base = (int64_t)y0 * R + H;
    cs = R;
    ncols = min(kCols, P - y0);
  }
  constexpr int64_t ES = (int64_t)P * R;  // element stride along z (W and the weights)
  const bool in = c < ncols;
  const int64_t vol = blockIdx.y;
  float2* wc = W + vol * NW + base + c * cs;
  const int64_t wo = vol * NC + base + c * cs;
  if (MODE == kZIter) {
    constexpr int U = (H + 1 + kCols - 1) / kCols;
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int z = t + kCols * u;
      if (z <= H) s[z * kPitch + c] = in ? wc[z * ES] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    c2r_pre<H, false>(s, tw, c, t);
    fft_cols<H, 2, false>(s, tw, c, t);
  }
  // the update (kZIter) and S = Fw * Fnw (Fw * V), pairs (S(2n), S(2n+1))
  double d2 = 0, o2 = 0, r2 = 0, q2 = 0;
  constexpr int NQ = H / kCols;  // pairs (2n, 2n+1) per thread
  constexpr int CH = NQ < 4 ? NQ : 4;
  const bool dist = MODE == kZIter && change && ref;
#pragma unroll 1
  for (int q0 = 0; q0 < NQ; q0 += CH) {
    // loads of CH pairs first (in flight together), then the updates
    float fw[CH][2], old[CH][2], vv[CH][2], rf[CH][2];
#pragma unroll
    for (int q = 0; q < CH; q++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t gi = wo + (int64_t)(2 * (t + kCols * (q0 + q)) + h) * ES;
        fw[q][h] = in ? __ldg(Fw + gi) : 0.f;
        old[q][h] = in && (MODE == kZIter || !MOM) ? Fnw[gi] : 0.f;
        vv[q][h] = in && MOM ? V[gi] : 0.f;
        rf[q][h] = in && dist ? __ldg(ref + gi) : 0.f;
      }
    }
#pragma unroll
    for (int q = 0; q < CH; q++) {
      const int n = t + kCols * (q0 + q);
      const float2 cv = MODE == kZIter ? s[n * kPitch + c] : make_float2(0.f, 0.f);
      float sv[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t gi = wo + (int64_t)(2 * n + h) * ES;
        float next;
        if (MODE == kZIter) {
          const float cval = h ? cv.y : cv.x;
          float nw;
          if (MOM) {
            grid_update_momentum_value(cval, old[q][h], vv[q][h], beta, nw, next);
            if (in) V[gi] = next;
          } else {
            nw = grid_update_value(cval, old[q][h]);
            next = nw;
          }
          if (in) Fnw[gi] = nw;
          if (change) {
            const double d = (double)fw[q][h] * ((double)nw - (double)old[q][h]);
            const double o = (double)fw[q][h] * (double)old[q][h];
            d2 += d * d;
            o2 += o * o;
            if (dist) {
              const double e = (double)fw[q][h] * ((double)nw - (double)rf[q][h]);
              const double p = (double)fw[q][h] * (double)rf[q][h];
              r2 += e * e;
              q2 += p * p;
            }
          }
        } else {
          next = MOM ? vv[q][h] : old[q][h];
        }
        sv[h] = fw[q][h] * next;
      }
      s[n * kPitch + c] = make_float2(sv[0], sv[1]);
    }
  }
  if (MODE == kZIter && change) {
    grid_change_reduce(d2, o2, change);
    if (ref) {
      __syncthreads();  // grid_change_reduce's shared scratch is reused
      grid_change_reduce(r2, q2, change + 2);
    }
  }
  __syncthreads();
  if (MODE == kZIter && !write_next) return;  // uniform
  fft_cols<H, 2, true>(s, tw, c, t);
  r2c_post<H, true>(s, tw, c, t);
  if (in) {
    for (int z = t; z <= H; z += kCols) wc[z * ES] = s[z * kPitch + c];
  }
}

template <int P>
struct SymSizes {
  static constexpr int H = P / 2;
  static constexpr int y_tiles = (H / kCols) * (H + 1) + (H + 1 + kCols - 1) / kCols;
  static constexpr int x_tiles = (H + 1) * P / kCols;
  static constexpr int z_tiles = P * (H / kCols) + P / kCols;
  static constexpr size_t y_smem = sizeof(float2) * (P + (size_t)P * kPitch);
  static constexpr size_t x_smem = sizeof(float2) * (P + (size_t)(H + 1) * kPitch) + sizeof(float) * kBlobSamples;
  static constexpr size_t z_smem = sizeof(float2) * (P + (size_t)(H + 1) * kPitch);
};

template <int P>
int set_attributes() {
  using Z = SymSizes<P>;
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_y_kernel<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Z::y_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_y_kernel<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Z::y_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_x_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Z::x_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_z_kernel<P, kZFirst, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::z_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_z_kernel<P, kZFirst, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::z_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_z_kernel<P, kZIter, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::z_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_z_kernel<P, kZIter, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::z_smem));
  return GTOMRLN_OK;
}

template <int P>
int run_first(float2* W, int count, const float* Fw, float* Fnw, float* V, const float2* tw,
              cudaStream_t stream) {
  using Z = SymSizes<P>;
  const dim3 grid(Z::z_tiles, count);
  if (V)
    gridsym_z_kernel<P, kZFirst, true><<<grid, kThreads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, 0.f, 1,
                                                                              nullptr, nullptr);
  else
    gridsym_z_kernel<P, kZFirst, false><<<grid, kThreads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, 0.f, 1,
                                                                               nullptr, nullptr);
  GTOMRLN_LAUNCH_CHECK("gridsym_z_kernel (first)");
  return GTOMRLN_OK;
}

template <int P>
int run_iteration(float2* W, int count, const float* table, const float* Fw, float* Fnw, float* V, float beta,
                  bool write_next, double* change, const float* ref, const float2* tw, cudaStream_t stream) {
  using Z = SymSizes<P>;
  const float inv_n = 1.0f / ((float)P * (float)P * (float)P);
  const float funcsampling = (float)(0.5 / kBlobSamples);
  gridsym_y_kernel<P, true><<<dim3(Z::y_tiles, count), kThreads, Z::y_smem, stream>>>(W, tw);
  GTOMRLN_LAUNCH_CHECK("gridsym_y_kernel (inverse)");
  gridsym_x_kernel<P><<<dim3(Z::x_tiles, count), kThreads, Z::x_smem, stream>>>(W, tw, table, inv_n,
                                                                                funcsampling);
  GTOMRLN_LAUNCH_CHECK("gridsym_x_kernel");
  gridsym_y_kernel<P, false><<<dim3(Z::y_tiles, count), kThreads, Z::y_smem, stream>>>(W, tw);
  GTOMRLN_LAUNCH_CHECK("gridsym_y_kernel (forward)");
  const dim3 grid(Z::z_tiles, count);
  if (V)
    gridsym_z_kernel<P, kZIter, true><<<grid, kThreads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, beta,
                                                                             write_next, change, ref);
  else
    gridsym_z_kernel<P, kZIter, false><<<grid, kThreads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, beta,
                                                                              write_next, change, ref);
  GTOMRLN_LAUNCH_CHECK("gridsym_z_kernel");
  return GTOMRLN_OK;
}

// Dispatch over the supported grids.
template <typename F>
int with_grid(int P, F&& f) {
  switch (P) {
    case 64: return f(std::integral_constant<int, 64>());
    case 128: return f(std::integral_constant<int, 128>());
    case 256: return f(std::integral_constant<int, 256>());
    case 512: return f(std::integral_constant<int, 512>());
    default: return set_error(GTOMRLN_ERR_INVALID, "gridsym: unsupported grid %d", P);
  }
}

std::mutex g_attr_mutex;
std::map<std::tuple<int, unsigned long long, int>, bool> g_attr_done;

int ensure_attributes(int P) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, context_id(), P);
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  if (g_attr_done.count(key)) return GTOMRLN_OK;
  const int st = with_grid(P, [](auto p) { return set_attributes<decltype(p)::value>(); });
  if (st == GTOMRLN_OK) g_attr_done[key] = true;
  return st;
}

}  // namespace

bool gridsym_available(int P) { return P == 64 || P == 128 || P == 256 || P == 512; }

int gridsym_first(float2* W, const GridGeom& g, int count, const float* Fw, float* Fnw, float* V,
                  cudaStream_t stream) {
  int st = ensure_attributes(g.P);
  if (st) return st;
  const float2* tw = nullptr;
  st = fft_twiddles(g.P, &tw);
  if (st) return st;
  return with_grid(g.P, [&](auto p) { return run_first<decltype(p)::value>(W, count, Fw, Fnw, V, tw, stream); });
}

int gridsym_iteration(float2* W, const GridGeom& g, int count, const float* table, const float* Fw, float* Fnw,
                      float* V, float beta, bool write_next, double* change, const float* ref,
                      cudaStream_t stream) {
  int st = ensure_attributes(g.P);
  if (st) return st;
  const float2* tw = nullptr;
  st = fft_twiddles(g.P, &tw);
  if (st) return st;
  return with_grid(g.P, [&](auto p) {
    return run_iteration<decltype(p)::value>(W, count, table, Fw, Fnw, V, beta, write_next, change, ref, tw,
                                             stream);
  });
}

int release_gridsym_caches(int dev, unsigned long long /*ctx*/) {
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  for (auto it = g_attr_done.begin(); it != g_attr_done.end();) {
    if (std::get<0>(it->first) == dev) it = g_attr_done.erase(it);
    else ++it;
  }
  return GTOMRLN_OK;
}

}  // namespace gtomrln
