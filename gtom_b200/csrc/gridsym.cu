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
// [z][y][x] with rows of P/2 + 4, the last three elements padding, so that
// rows start on 32-byte boundaries):
//   gridsym_y_tma_kernel<INV>  inverse transform along y of W (columns of 16
//                          consecutive x at one z, staged in shared memory
//                          by tensor copies, or of x = P/2 at 16 z);
//   gridsym_x_kernel       per row (y, z): C2R along x, times blob(r)/P^3
//                          (IFFT.cu:36-46 normalisation, RecFourier.cu:
//                          243-262 table), R2C along x;
//   gridsym_y_tma_kernel<FWD>  forward transform along y;
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
// Transforms.  A real transform of length P runs as a complex transform of
// length H = P/2 on the packed pairs (x(2n), x(2n+1)) with the usual pre-
// and post-twiddles.  A complex transform of length N = N1 N2 is a four-step
// FFT over N2 threads per column: thread t holds the elements t + N2 m
// (m < N1) in registers, loaded straight from HBM; it transforms them with an
// in-register N1-point DFT, multiplies by e(-+ t k1 / N), exchanges through
// shared memory once (each thread then holds N1/N2 values of k1 for all N2
// threads' elements), and finishes with N1/N2 in-register N2-point DFTs, which
// leaves it holding the outputs t + N2 m again: loads and stores take the
// same coalesced pattern and the data crosses shared memory once per
// transform.  In the x pass the N2 threads of a row are consecutive lanes of
// one warp, so its exchanges need only the warp and the partners k, H - k of
// the pre- and post-twiddles are shuffles; in the y and z passes the lanes
// run over 16 consecutive columns (coalesced along x).  Twiddles come from a
// table e(-m/P) computed in double precision (runtime factors) and from
// compile-time constants (inside the in-register DFTs).  All transforms are
// unnormalised, as cuFFT's; the 1/P^3 of the reference's C2R rides with the
// blob.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is looked up at run time)

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "fftcore.cuh"
#include "gridfft.cuh"

namespace gtomrln {

namespace {

constexpr int kCols = 16;          // columns (y and z passes) or rows (x pass) per CTA
constexpr int kPitch = kCols + 1;  // shared-memory stride between element indices (y, z passes), in float2

// ---------------------------------------------- compile-time twiddles --
constexpr double kPiD = 3.14159265358979323846264338327950288;

// sin and cos by their Taylor series after reduction to [-pi, pi] (the
// remaining error is far below FP32 rounding); compile-time only.
constexpr double ce_sin(double x) {
  while (x > kPiD) x -= 2 * kPiD;
  while (x < -kPiD) x += 2 * kPiD;
  double term = x, sum = x;
  for (int k = 1; k < 20; k++) {
    term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double ce_cos(double x) { return ce_sin(x + kPiD / 2); }

// Odd prime DFT of length R in registers (R = 3, 5), unnormalised, forward
// (exp(-)) or inverse (exp(+)): X(k) = a(0) + sum over n = 1 .. (R-1)/2 of
// (a(n) + a(R-n)) cos(2 pi k n / R) -+ i (a(n) - a(R-n)) sin(2 pi k n / R).
template <int R, bool INV>
__device__ __forceinline__ void dft_odd(float2* v) {
  float2 sp[(R - 1) / 2], sm[(R - 1) / 2];
#pragma unroll
  for (int n = 1; n <= (R - 1) / 2; n++) {
    sp[n - 1] = cadd(v[n], v[R - n]);
    sm[n - 1] = csub(v[n], v[R - n]);
  }
  float2 out[R];
  out[0] = v[0];
#pragma unroll
  for (int n = 0; n < (R - 1) / 2; n++) out[0] = cadd(out[0], sp[n]);
#pragma unroll
  for (int k = 1; k < R; k++) {
    float2 re = v[0], im = make_float2(0.f, 0.f);  // re: cosine part, im: sine part (before the factor -+i)
#pragma unroll
    for (int n = 1; n <= (R - 1) / 2; n++) {
      const float cs = (float)ce_cos(2 * kPiD * ((k * n) % R) / R);
      const float sn = (float)ce_sin(2 * kPiD * ((k * n) % R) / R);
      re = make_float2(fmaf(cs, sp[n - 1].x, re.x), fmaf(cs, sp[n - 1].y, re.y));
      im = make_float2(fmaf(sn, sm[n - 1].x, im.x), fmaf(sn, sm[n - 1].y, im.y));
    }
    // forward: re - i im; inverse: re + i im
    out[k] = INV ? make_float2(re.x - im.y, re.y + im.x) : make_float2(re.x + im.y, re.y - im.x);
  }
#pragma unroll
  for (int k = 0; k < R; k++) v[k] = out[k];
}

// In-register DFT of length N (factors 2, 3, 5), unnormalised, forward
// (exp(-)) or inverse (exp(+)), natural order in and out: decimation in
// time by the smallest factor (2, then 3, then 5) down to the radix-8/4/2
// kernels of fftcore.cuh and the odd prime kernels above, with the
// combining twiddles as constants.
template <int N, bool INV>
__device__ __forceinline__ void dftr(float2* v) {
  if constexpr (N == 1) {
    return;
  } else if constexpr (N == 2 || N == 4 || N == 8) {
    dft<N, INV>(v);
  } else if constexpr (N == 3 || N == 5) {
    dft_odd<N, INV>(v);
  } else {
    constexpr int R = N % 2 == 0 ? 2 : (N % 3 == 0 ? 3 : 5);
    constexpr int M = N / R;
    static_assert(M * R == N, "dftr: lengths with factors 2, 3 and 5 only");
    float2 sub[R][M];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int i = 0; i < M; i++) sub[r][i] = v[R * i + r];
#pragma unroll
    for (int r = 0; r < R; r++) dftr<M, INV>(sub[r]);
#pragma unroll
    for (int k = 0; k < M; k++) {
      float2 u[R];
#pragma unroll
      for (int r = 0; r < R; r++) {
        if (r * k == 0) {
          u[r] = sub[r][k];
        } else if (4 * r * k == N) {
          u[r] = mul_mi<INV>(sub[r][k]);  // e(-+1/4) = -+i
        } else if (8 * r * k == N || 8 * r * k == 3 * N) {
          // e(-+1/8), e(-+3/8): (1 -+ i)/sqrt2, (-1 -+ i)/sqrt2, four operations
          const float h = 0.70710678118654752440f;
          const float2 a = sub[r][k];
          const float2 p = 8 * r * k == N ? a : mul_mi<INV>(a);  // e(-+3/8) = -+i e(-+1/8)
          u[r] = INV ? make_float2((p.x - p.y) * h, (p.x + p.y) * h) : make_float2((p.x + p.y) * h, (p.y - p.x) * h);
        } else {
          const float wr = (float)ce_cos(2 * kPiD * r * k / N);
          const float wi = (float)(INV ? ce_sin(2 * kPiD * r * k / N) : -ce_sin(2 * kPiD * r * k / N));
          u[r] = cmul(sub[r][k], make_float2(wr, wi));
        }
      }
      if constexpr (R == 2) {
        dft<2, INV>(u);
      } else {
        dft_odd<R, INV>(u);
      }
#pragma unroll
      for (int q = 0; q < R; q++) v[k + M * q] = u[q];
    }
  }
}

// ------------------------------------------------------ four-step FFT --
// N = N1 N2 with N2 threads per column and N1 a multiple of N2.
template <int N>
struct Split;
#define GTOMRLN_SPLIT(N_, A_, B_)            \
  template <>                               \
  struct Split<N_> {                        \
    static constexpr int N1 = A_, N2 = B_;  \
  };
GTOMRLN_SPLIT(32, 8, 4)
GTOMRLN_SPLIT(48, 12, 4)
GTOMRLN_SPLIT(64, 8, 8)
GTOMRLN_SPLIT(96, 24, 4)
GTOMRLN_SPLIT(128, 16, 8)
GTOMRLN_SPLIT(192, 24, 8)
GTOMRLN_SPLIT(256, 16, 16)
GTOMRLN_SPLIT(400, 20, 20)
GTOMRLN_SPLIT(512, 32, 16)
GTOMRLN_SPLIT(800, 40, 20)
#undef GTOMRLN_SPLIT

// Padded place of table entry i in the x passes' copy of the twiddle table
// (one spare entry after every 16): their lanes read entries 2 t k1 for
// t = 0 .. N2-1, strides that would put up to 16 lanes on one bank.
__host__ __device__ constexpr int tw_pad(int i) { return i + (i >> 4); }

// Runtime twiddle e(-m/N) (or e(+m/N), INV) from the table e(-j/P), N = P/S
// (PAD: the padded copy).
template <int S, bool INV, bool PAD = false>
__device__ __forceinline__ float2 twiddle(const float2* tw, int m) {
  float2 w = tw[PAD ? tw_pad(m * S) : m * S];
  if (INV) w.y = -w.y;
  return w;
}

// Shared-memory places of the exchange: element (k1, n2) of the transform of
// column c.  Columns-fast (y, z passes: lanes run over 16 columns and two
// threads, each half-warp's access contiguous) or rows (x pass: lanes run
// over the N2 threads of a row, each row in its own block; the odd stride
// N1 + 1 keeps both the write and the read conflict-free).
template <int N1, int N2, bool ROWS>
__device__ __forceinline__ int xplace(int k1, int n2, int c) {
  if constexpr (ROWS)
    return c * (N2 * (N1 + 1)) + n2 * (N1 + 1) + k1;
  else
    return (n2 * N1 + k1) * kPitch + c;
}

// The four-step transform of one column (thread t of its N2 threads holds
// elements t + N2 m in v[m]; afterwards outputs t + N2 m in v[m]).  ROWS:
// the row layout of xplace.  WSYNC: the column's threads share a warp and
// synchronise as a warp; else the block synchronises (every thread of the
// block must call it).  Begins with a barrier, so the exchange buffer may
// still be in use by the caller.
template <int N, bool INV, bool ROWS, bool WSYNC, int S>
__device__ __forceinline__ void four_step(float2* v, float2* xb, const float2* tw, int t, int c) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, J = N1 / N2;
  static_assert(J * N2 == N1, "four_step: N1 must be a multiple of N2");
  dftr<N1, INV>(v);
#pragma unroll
  for (int k1 = 1; k1 < N1; k1++) v[k1] = cmul(v[k1], twiddle<S, INV, ROWS>(tw, t * k1));
  if (WSYNC) __syncwarp(); else __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < N1; k1++) xb[xplace<N1, N2, ROWS>(k1, t, c)] = v[k1];
  if (WSYNC) __syncwarp(); else __syncthreads();
#pragma unroll
  for (int j = 0; j < J; j++) {
    float2 u[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) u[n2] = xb[xplace<N1, N2, ROWS>(t + N2 * j, n2, c)];
    dftr<N2, INV>(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) v[j + J * k2] = u[k2];
  }
}

// The same transform with the exchange in J = N1/N2 rounds of N2 x N2 values
// per column (round j: the outputs k1 = N2 j .. N2 j + N2 - 1 of every
// thread's N1-point DFT), so that the exchange buffer holds 16 N2^2 values
// instead of 16 N; columns-fast layout (16 columns per element, each
// half-warp's access one 128-byte row).  Round j's N2-point DFTs return
// X(k1 + N1 k2), k1 = N2 j + t, i.e. outputs t + N2 (j + J k2), written back
// into the registers the round's inputs left and renamed at the end.
// SYNC0: begin with a CTA barrier (a caller whose own last barrier already
// follows its threads' earlier reads of xb passes false).
template <int N, bool INV, bool SYNC0 = true>
__device__ __forceinline__ void four_step_rounds(float2* v, float2* xb, const float2* tw, int t, int c) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, J = N1 / N2;
  static_assert(J * N2 == N1, "four_step_rounds: N1 must be a multiple of N2");
  dftr<N1, INV>(v);
#pragma unroll
  for (int k1 = 1; k1 < N1; k1++) v[k1] = cmul(v[k1], twiddle<1, INV>(tw, t * k1));
#pragma unroll
  for (int j = 0; j < J; j++) {
    if (j > 0 || SYNC0) __syncthreads();  // the previous round's (or the caller's) reads of xb are done
#pragma unroll
    for (int k = 0; k < N2; k++) xb[(t * N2 + k) * kCols + c] = v[N2 * j + k];
    __syncthreads();
    float2 u[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) u[n2] = xb[(n2 * N2 + t) * kCols + c];
    dftr<N2, INV>(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) v[N2 * j + k2] = u[k2];
  }
  float2 w[N1];
#pragma unroll
  for (int j = 0; j < J; j++)
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) w[j + J * k2] = v[N2 * j + k2];
#pragma unroll
  for (int m = 0; m < N1; m++) v[m] = w[m];
}

// The pre-twiddle of a Hermitian-to-real transform of length P = 2H as an
// H-point complex transform: Z(k) = (X(k) + conj X(H-k)) + i e(sg k/P)
// (X(k) - conj X(H-k)) (sg = +1: the inverse C2R; -1: the forward sum); the
// H-point transform of the same sign then gives x(2n) = Re z(n),
// x(2n+1) = Im z(n).
template <bool PLUS>
__device__ __forceinline__ float2 c2r_pre(float2 xk, float2 xm, float2 w) {
  if (PLUS) w.y = -w.y;  // the table holds e(-k/P)
  const float2 a = make_float2(xk.x + xm.x, xk.y - xm.y);  // X(k) + conj X(H-k)
  const float2 b = make_float2(xk.x - xm.x, xk.y + xm.y);  // X(k) - conj X(H-k)
  const float2 wb = cmul(w, b);
  return make_float2(a.x - wb.y, a.y + wb.x);  // a + i wb
}

// The post-twiddle of a real-to-Hermitian transform of length P computed as
// an H-point complex transform of the packed pairs: Y(k) = (Z(k) + conj
// Z(H-k)) / 2 - (i/2) e(sg k/P) (Z(k) - conj Z(H-k)) (Z indices mod H;
// sg = -1: the forward R2C; +1: exp(+)).  Y(H) = Re Z(0) - Im Z(0).
template <bool PLUS>
__device__ __forceinline__ float2 r2c_post(float2 zk, float2 zm, float2 w) {
  if (PLUS) w.y = -w.y;
  const float2 a = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
  const float2 b = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
  const float2 wb = cmul(w, b);
  return make_float2(a.x + wb.y, a.y - wb.x);  // a - i wb
}

__device__ __forceinline__ void load_twiddles(float2* tw, const float2* __restrict__ twg, int P) {
  for (int m = threadIdx.x; m < P; m += blockDim.x) tw[m] = __ldg(twg + m);
}
// The padded copy (tw_pad) for the x passes: P + P/16 entries.
__device__ __forceinline__ void load_twiddles_padded(float2* tw, const float2* __restrict__ twg, int P) {
  for (int m = threadIdx.x; m < P; m += blockDim.x) tw[tw_pad(m)] = __ldg(twg + m);
}

// ------------------------------------------------------- TMA staging --
// Tensor copies global -> shared completed on an mbarrier (no multicast, no
// cluster).  Every wait is bounded: after kWaitLimitNs without completion
// the kernel records a fault (g_gridsym_fault), which the final map turns
// into NaN output.
constexpr unsigned long long kWaitLimitNs = 1000000000ull;  // 1 s
__device__ int g_gridsym_fault;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the phase of the given parity; false after kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
}
// Orders this thread's earlier shared-memory accesses (and, after a CTA
// barrier, the CTA's) before the following tensor copy's writes.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// ------------------------------------------------------------ y pass --
// W's rows hold P/2 + 4 complex elements (the last three padding), so that
// every row starts on a 32-byte boundary: tensor copies need 16, and a
// warp's run of 16 columns then covers whole sectors.
template <int P>
constexpr int w_pitch() { return P / 2 + 4; }

// Sizes of the staged y pass: a tile (16 columns x P rows) arrives as NB
// tensor boxes of BOX rows (a box has at most 256 rows).
template <int P>
struct YStage {
  static constexpr int NB = (P + 255) / 256;
  static constexpr int BOX = P / NB;
  static_assert(BOX * NB == P && BOX <= 256, "YStage: rows must split into equal boxes");
  static constexpr int N2 = Split<P>::N2;
  static constexpr size_t stage_bytes = sizeof(float2) * kCols * P;
  static constexpr size_t xb_bytes = sizeof(float2) * kCols * N2 * N2;
  // 1 KB for aligning the staging buffer, staging, exchange, twiddles
  static constexpr size_t smem = 1024 + stage_bytes + xb_bytes + sizeof(float2) * P;
};

// The y pass, persistent, over nyq + tiles work units: first the columns
// x = P/2 (16 consecutive z of one volume per unit, plain loads), then the
// tiles of 16 consecutive x < P/2 at one (volume, z), each of which arrives
// in shared memory by tensor copies (map: W as floats, dims {2 w_pitch, P,
// (P/2+1) volumes}, box {32, BOX, 1}).  CTA i starts with unit i and takes
// the next from a counter as soon as it holds its current unit in
// registers, starting the next tile's copy then, so the copy runs during the
// transform and the stores and the slower x = P/2 units leave no tail.  The
// counter and the count of finished CTAs sit in the padding element of W's
// first row (the last CTA zeroes both for the next launch; the first
// transform zeroes them once).  The transform is four_step_rounds (the
// exchange buffer and the staging buffer fit two CTAs per SM at P = 512).
template <int P, bool INV>
__global__ void __launch_bounds__(kCols * Split<P>::N2, (P > 512 ? 1 : 2))
gridsym_y_tma_kernel(const __grid_constant__ CUtensorMap map, float2* __restrict__ W,
                     const float2* __restrict__ twg, int tiles, int nyq) {
  using Y = YStage<P>;
  constexpr int H = P / 2, RW = w_pitch<P>();
  constexpr int N1 = Split<P>::N1, N2 = Split<P>::N2;
  constexpr int XT = H / kCols;                    // tiles per (volume, z)
  constexpr int NQ = (H + 1 + kCols - 1) / kCols;  // x = P/2 units per volume
  extern __shared__ unsigned char sraw[];
  __shared__ unsigned long long bar;
  __shared__ int next_s;
  float2* stage = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(sraw) + 1023) & ~(uintptr_t)1023);
  float2* xb = stage + kCols * P;
  float2* tw = xb + kCols * N2 * N2;
  int* sched = reinterpret_cast<int*>(W + H + 1);  // {counter, finished CTAs}
  load_twiddles(tw, twg, P);
  const int c = threadIdx.x & (kCols - 1), t = threadIdx.x / kCols;
  const int total = nyq + tiles;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  auto issue = [&](int tile) {  // one thread
    const int vz = tile / XT, xt = tile - vz * XT;
    fence_proxy_async();
    mbar_expect_tx(&bar, (unsigned)Y::stage_bytes);
#pragma unroll
    for (int k = 0; k < Y::NB; k++)
      tma_load_3d(stage + k * Y::BOX * kCols, &map, xt * 2 * kCols, k * Y::BOX, vz, &bar);
  };
  // the next unit, and its copy when it is a tile (one thread)
  auto take_next = [&]() {
    const int u = (int)gridDim.x + atomicAdd(sched, 1);
    next_s = u;
    if (u >= nyq && u < total) issue(u - nyq);
  };
  int u = blockIdx.x;
  if (threadIdx.x == 0 && u >= nyq && u < total) issue(u - nyq);
  unsigned parity = 0;
  bool fault = false;
  while (u < total) {
    float2 v[N1];
    float2* col;
    bool in = true;
    if (u >= nyq) {
      const bool ok = mbar_wait(&bar, parity);
      if (!__syncthreads_and(ok)) {
        if (threadIdx.x == 0) atomicExch(&g_gridsym_fault, 1);
        mbar_wait(&bar, parity);  // once more for the copy in flight, then leave
        fault = true;
        break;
      }
      parity ^= 1u;
#pragma unroll
      for (int m = 0; m < N1; m++) v[m] = stage[(t + N2 * m) * kCols + c];
      __syncthreads();  // the staging buffer is read
      if (threadIdx.x == 0) take_next();
      const int tile = u - nyq, vz = tile / XT, xt = tile - vz * XT;
      col = W + (int64_t)vz * P * RW + xt * kCols + c;
    } else {
      const int vol = u / NQ, z = (u - vol * NQ) * kCols + c;
      in = z <= H;
      col = W + ((int64_t)vol * (H + 1) + (in ? z : 0)) * P * RW + H;
#pragma unroll
      for (int m = 0; m < N1; m++) v[m] = in ? col[(int64_t)(t + N2 * m) * RW] : make_float2(0.f, 0.f);
      __syncthreads();  // every thread has read next_s
      if (threadIdx.x == 0) take_next();
    }
    // no leading barrier: both branches end with one after every thread's
    // reads of xb for the previous unit; next_s is visible after the rounds'
    // own barriers
    four_step_rounds<P, INV, false>(v, xb, tw, t, c);
    if (in) {
#pragma unroll
      for (int m = 0; m < N1; m++) col[(int64_t)(t + N2 * m) * RW] = v[m];
    }
    u = next_s;
  }
  // the last CTA to finish zeroes the counter for the next launch (a CTA
  // leaves the loop only once the counter is past the last unit)
  __syncthreads();
  if (threadIdx.x == 0 && !fault) {
    __threadfence();
    if (atomicAdd(sched + 1, 1) == (int)gridDim.x - 1) {
      sched[0] = 0;
      sched[1] = 0;
      __threadfence();
    }
  }
}

// ------------------------------------------------------------ x pass --
// Per row (y, z), z <= P/2: C2R along x, times blob(r) / P^3, R2C along x.
// Grid: ((P/2 + 1) P / 16, volumes); a CTA takes 16 consecutive rows, the
// N2 threads of a row consecutive lanes.  Where N2 divides 32 a row lies in
// one warp (warp-synchronous exchanges, shuffles for the Hermitian
// partners); else (P = 800) the block synchronises and the partners go
// through shared memory.
template <int P>
__global__ void __launch_bounds__(kCols * Split<P / 2>::N2, (P > 512 ? 2 : 3))
gridsym_x_kernel(float2* __restrict__ W, const float2* __restrict__ twg, const float* __restrict__ table,
                 float inv_n, float funcsampling) {
  constexpr int H = P / 2, RW = w_pitch<P>();
  constexpr int N1 = Split<H>::N1, N2 = Split<H>::N2;
  constexpr bool WROW = 32 % N2 == 0;    // a row's threads within one warp
  constexpr int XS = N2 * (N1 + 1);      // a row's block of the exchange buffer
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* xb = smem + P + P / 16;  // after the padded twiddle table
  load_twiddles_padded(tw, twg, P);
  const int t = threadIdx.x % N2, r = threadIdx.x / N2;
  const unsigned lane = threadIdx.x & 31;
  const unsigned partner = WROW ? (lane & ~(unsigned)(N2 - 1)) | ((unsigned)(N2 - t) & (N2 - 1)) : lane;
  const int64_t rg = (int64_t)blockIdx.x * kCols + r;  // z * P + y
  float2* row = W + (int64_t)blockIdx.y * ((int64_t)(H + 1) * P * RW) + rg * RW;
  float2 v[N1];
#pragma unroll
  for (int m = 0; m < N1; m++) v[m] = row[t + N2 * m];
  // a C2R takes the x = 0 and x = P/2 terms as real (their imaginary parts,
  // zero for a Hermitian spectrum, are dropped as cuFFT's C2R drops them)
  const float2 xH = t == 0 ? make_float2(row[H].x, 0.f) : make_float2(0.f, 0.f);
  if (t == 0) v[0].y = 0.f;
  __syncthreads();  // twiddles in place
  // pre-twiddle of the C2R.  The partner H - k of k = t + N2 m is element
  // N1-1-m of thread N2-t (t > 0), or element N1-m (H for m = 0) of thread 0
  // (into a second array: the partners' elements are read after this
  // thread's own have been replaced)
  {
    float2 z[N1];
    if constexpr (WROW) {
#pragma unroll
      for (int m = 0; m < N1; m++) {
        const float2 sh = make_float2(__shfl_sync(0xffffffffu, v[N1 - 1 - m].x, partner),
                                      __shfl_sync(0xffffffffu, v[N1 - 1 - m].y, partner));
        const float2 xm = t != 0 ? sh : (m == 0 ? xH : v[(N1 - m) % N1]);
        z[m] = c2r_pre<true>(v[m], xm, tw[tw_pad(t + N2 * m)]);
      }
    } else {
#pragma unroll
      for (int m = 0; m < N1; m++) xb[r * XS + t + N2 * m] = v[m];
      if (t == 0) xb[r * XS + H] = xH;
      __syncthreads();
#pragma unroll
      for (int m = 0; m < N1; m++) {
        const int k = t + N2 * m;
        z[m] = c2r_pre<true>(v[m], xb[r * XS + H - k], tw[tw_pad(k)]);
      }
    }
#pragma unroll
    for (int m = 0; m < N1; m++) v[m] = z[m];
  }
  four_step<H, true, true, WROW, 2>(v, xb, tw, t, r);
  {
    // blob: grid_blob_kernel's table index (the reference's radius
    // sqrt(x^2 + y^2 + z^2) / P / funcsampling with its fast-math square root
    // and divisions, the row part formed first)
    const int z = (int)(rg / P), y = (int)(rg - (int64_t)z * P);
    const int zp = z < H ? z : z - P, yp = y < H ? y : y - P;
    const float cyz = (float)(yp * yp + zp * zp);
    auto blob = [&](int x) {
      const float xp = (float)(x < H ? x : x - P);
      return __ldg(table + grid_blob_index_sq(xp * xp + cyz, (float)P, funcsampling));
    };
    if constexpr (WROW) {
      // x and P - x have the same radius, bit for bit: the blob values of
      // elements m <= N1/2 are computed, the others taken from the thread
      // holding P - x (x = 2n: element N1-1-m of thread N2-t, or element
      // N1-m of thread 0 for t = 0; x = 2n+1: element N1-1-m of thread
      // N2-1-t)
      constexpr int M0 = N1 / 2;
      const unsigned partner1 = (lane & ~(unsigned)(N2 - 1)) | (unsigned)(N2 - 1 - t);
      float bl[M0 + 1][2];
#pragma unroll
      for (int m = 0; m <= M0; m++) {
        bl[m][0] = blob(2 * (t + N2 * m));
        bl[m][1] = blob(2 * (t + N2 * m) + 1);
      }
#pragma unroll
      for (int m = 0; m < N1; m++) {
        float b0, b1;
        if (m <= M0) {
          b0 = bl[m][0];
          b1 = bl[m][1];
        } else {
          const float s0 = __shfl_sync(0xffffffffu, bl[N1 - 1 - m][0], partner);
          b0 = t != 0 ? s0 : bl[N1 - m][0];
          b1 = __shfl_sync(0xffffffffu, bl[N1 - 1 - m][1], partner1);
        }
        v[m].x = v[m].x * inv_n * b0;
        v[m].y = v[m].y * inv_n * b1;
      }
    } else {
#pragma unroll
      for (int m = 0; m < N1; m++) {
        const int n = t + N2 * m;
        v[m].x = v[m].x * inv_n * blob(2 * n);
        v[m].y = v[m].y * inv_n * blob(2 * n + 1);
      }
    }
  }
  four_step<H, false, true, WROW, 2>(v, xb, tw, t, r);
  // post-twiddle of the R2C: partner (H - k) mod H as above (thread 0:
  // element 0 for m = 0, else N1 - m)
  float2 y[N1];
  if constexpr (WROW) {
#pragma unroll
    for (int m = 0; m < N1; m++) {
      const float2 sh = make_float2(__shfl_sync(0xffffffffu, v[N1 - 1 - m].x, partner),
                                    __shfl_sync(0xffffffffu, v[N1 - 1 - m].y, partner));
      const float2 zm = t != 0 ? sh : v[(N1 - m) % N1];
      y[m] = r2c_post<false>(v[m], zm, tw[tw_pad(t + N2 * m)]);
    }
  } else {
    __syncthreads();  // the exchange buffer is free
#pragma unroll
    for (int m = 0; m < N1; m++) xb[r * XS + t + N2 * m] = v[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < N1; m++) {
      const int k = t + N2 * m;
      y[m] = r2c_post<false>(v[m], xb[r * XS + (k == 0 ? 0 : H - k)], tw[tw_pad(k)]);
    }
  }
#pragma unroll
  for (int m = 0; m < N1; m++) row[t + N2 * m] = y[m];
  if (t == 0) row[H] = make_float2(v[0].x - v[0].y, 0.f);
}

// ------------------------------------------------------------ z pass --
enum : int { kZFirst = 0, kZIter = 1 };

// Per column (x, y) along z.  kZFirst: the real-to-Hermitian transform
// (exp(+)) of S = Fw * Fnw (Fw * V with momentum) into W.  kZIter: the
// Hermitian-to-real transform (exp(-)) of W, the update of Fnw (and V) from
// its values, and with write_next the transform of the new S into W.
// change (single volume): sums of grid_update_kernel; ref: the distance sums
// to reference weights as well.  Grid: (tiles, volumes); tiles are 16
// consecutive x < P/2 at one y, then x = P/2 at 16 consecutive y.
template <int P, int MODE, bool MOM>
__global__ void __launch_bounds__(kCols * Split<P / 2>::N2, (P > 512 ? 2 : 3))
gridsym_z_kernel(float2* __restrict__ W, const float* __restrict__ Fw, float* __restrict__ Fnw,
                 float* __restrict__ V, const float2* __restrict__ twg, float beta, int write_next,
                 double* __restrict__ change, const float* __restrict__ ref) {
  constexpr int H = P / 2, R = H + 1, RW = w_pitch<P>();
  constexpr int N1 = Split<H>::N1, N2 = Split<H>::N2;
  constexpr int64_t NC = (int64_t)R * P * P;         // spectrum elements per volume
  constexpr int64_t NW = (int64_t)(H + 1) * P * RW;  // W elements per volume
  constexpr int64_t ES = (int64_t)P * R;             // element stride along z of the weights
  constexpr int64_t EW = (int64_t)P * RW;            // and of W
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* xb = smem + P;
  load_twiddles(tw, twg, P);
  const int c = threadIdx.x & (kCols - 1), t = threadIdx.x / kCols;
  constexpr int kMain = P * (H / kCols);
  const int b = blockIdx.x;
  int x, y;
  if (b < kMain) {
    y = b / (H / kCols);
    x = (b - y * (H / kCols)) * kCols + c;
  } else {
    y = (b - kMain) * kCols + c;
    x = H;
  }
  const int64_t vol = blockIdx.y;
  if (MODE == kZFirst && b == 0 && vol == 0 && threadIdx.x == 0) {
    // the y pass's work counter (padding of W's first row): zero for its first launch
    int* sched = reinterpret_cast<int*>(W + H + 1);
    sched[0] = 0;
    sched[1] = 0;
  }
  float2* wc = W + vol * NW + (int64_t)y * RW + x;
  const int64_t wo = vol * NC + (int64_t)y * R + x;
  float2 v[N1];
  if (MODE == kZIter) {
    float2 xH = make_float2(0.f, 0.f);
#pragma unroll
    for (int m = 0; m < N1; m++) v[m] = wc[(t + N2 * m) * EW];
    // the z = 0 and z = P/2 terms of a Hermitian column are real (their
    // imaginary parts are rounding, dropped as a C2R drops them)
    if (t == 0) {
      xH = make_float2(wc[H * EW].x, 0.f);
      v[0].y = 0.f;
    }
    // pre-twiddle (exp(-) sum) with the partners H - k through shared memory
    __syncthreads();  // twiddles in place
#pragma unroll
    for (int m = 0; m < N1; m++) xb[(t + N2 * m) * kPitch + c] = v[m];
    if (t == 0) xb[H * kPitch + c] = xH;
    __syncthreads();
#pragma unroll
    for (int m = 0; m < N1; m++) {
      const int k = t + N2 * m;
      v[m] = c2r_pre<false>(v[m], xb[(H - k) * kPitch + c], tw[k]);
    }
    four_step<H, false, false, false, 2>(v, xb, tw, t, c);
  }
  // the update (kZIter) and S = Fw * Fnw (Fw * V): element n = t + N2 m of
  // the packed pairs is (S(2n), S(2n+1))
  double d2 = 0, o2 = 0, r2 = 0, q2 = 0;
  const bool dist = MODE == kZIter && change && ref;
  constexpr int CH = N1 < 2 ? N1 : 2;
#pragma unroll
  for (int m0 = 0; m0 < N1; m0 += CH) {
    // loads of CH pairs first (in flight together), then the updates
    float fw[CH][2], old[CH][2], vv[CH][2], rf[CH][2];
#pragma unroll
    for (int q = 0; q < CH; q++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t gi = wo + (int64_t)(2 * (t + N2 * (m0 + q)) + h) * ES;
        fw[q][h] = __ldg(Fw + gi);
        old[q][h] = MODE == kZIter || !MOM ? Fnw[gi] : 0.f;
        vv[q][h] = MOM ? V[gi] : 0.f;
        rf[q][h] = dist ? __ldg(ref + gi) : 0.f;
      }
    }
#pragma unroll
    for (int q = 0; q < CH; q++) {
      const int m = m0 + q;
      float sv[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t gi = wo + (int64_t)(2 * (t + N2 * m) + h) * ES;
        float next;
        if (MODE == kZIter) {
          const float cval = h ? v[m].y : v[m].x;
          float nw;
          if (MOM) {
            grid_update_momentum_value(cval, old[q][h], vv[q][h], beta, nw, next);
            V[gi] = next;
          } else {
            nw = grid_update_value(cval, old[q][h]);
            next = nw;
          }
          Fnw[gi] = nw;
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
      v[m] = make_float2(sv[0], sv[1]);
    }
  }
  if (MODE == kZIter && change) {
    grid_change_reduce(d2, o2, change);
    if (ref) {
      __syncthreads();  // grid_change_reduce's shared scratch is reused
      grid_change_reduce(r2, q2, change + 2);
    }
  }
  if (MODE == kZIter && !write_next) return;  // uniform
  if (MODE == kZFirst) __syncthreads();  // twiddles in place
  four_step<H, true, false, false, 2>(v, xb, tw, t, c);
  // post-twiddle (exp(+)) with the partners (H - k) mod H through shared memory
  __syncthreads();
#pragma unroll
  for (int m = 0; m < N1; m++) xb[(t + N2 * m) * kPitch + c] = v[m];
  __syncthreads();
#pragma unroll
  for (int m = 0; m < N1; m++) {
    const int k = t + N2 * m, km = k == 0 ? 0 : H - k;
    wc[k * EW] = r2c_post<true>(v[m], xb[km * kPitch + c], tw[k]);
  }
  if (t == 0) wc[H * EW] = make_float2(v[0].x - v[0].y, 0.f);
}

// -------------------------------------------------------- final map --
// The final C2R of the corrected data (RecFourier.cu:175-216), cropped to
// the central ori^3 of the P grid (Padding.cu:22-42) and gridding-corrected
// (RecFourier.cu:310-332), as three passes of the same transforms: only the
// z planes and y rows of the crop are ever written.  T: the work array,
// (P/2+1) x P x ori complex per volume, layout [zc][y][x] (rows of P/2 + 1),
// inside the loop's W buffer.
struct FinalArgs {
  const float2* data;  // centred input spectra (old box), volume stride wstride
  int oldx, oldy, oldz;
  int64_t wstride;
  const float* Fw;     // P-grid weights, volume stride (P/2+1) P P
  const float* Fnw;
  int divide;          // no iteration ran: divide by max(|Fw|, 1e-4)
  int ori, off;        // output box and its offset in the P grid
  float scale;
  float* out;          // ori^3 output (one volume), or
  float* const* outs;  // one output per volume
};

// Pass 1, per column (x, y) along z: the final spectrum's elements
// (grid_final_value, straight from the caller's data), inverse transform,
// the crop's z planes written.  Tiles as in gridsym_z_kernel.
template <int P>
__global__ void __launch_bounds__(kCols * Split<P>::N2, (P > 512 ? 1 : 2))
gridsym_final_z_kernel(float2* __restrict__ T, FinalArgs f, const float2* __restrict__ twg) {
  constexpr int H = P / 2, R = H + 1;
  constexpr int N1 = Split<P>::N1, N2 = Split<P>::N2;
  constexpr int64_t NC = (int64_t)R * P * P;
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* xb = smem + P;
  load_twiddles(tw, twg, P);
  const int c = threadIdx.x & (kCols - 1), t = threadIdx.x / kCols;
  constexpr int kMain = P * (H / kCols);
  const int b = blockIdx.x;
  int x, y;
  if (b < kMain) {
    y = b / (H / kCols);
    x = (b - y * (H / kCols)) * kCols + c;
  } else {
    y = (b - kMain) * kCols + c;
    x = H;
  }
  const int64_t vol = blockIdx.y;
  const float2* data = f.data + vol * f.wstride;
  const float* Fw = f.Fw + vol * NC;
  const float* Fnw = f.Fnw + vol * NC;
  float2* tv = T + vol * ((int64_t)R * P * f.ori);
  // the loads of CH elements first (an index outside the input box reads
  // element 0, zeroed after), then their corrections
  const float* wsrc = f.divide ? Fw : Fnw;
  constexpr int CH = N1 <= 20 ? N1 : (N1 % 20 == 0 ? 20 : (N1 % 16 == 0 ? 16 : 12));
  static_assert(N1 % CH == 0, "gridsym_final_z_kernel: chunks");
  float2 v[N1];
#pragma unroll
  for (int m0 = 0; m0 < N1; m0 += CH) {
    float wt[CH];
#pragma unroll
    for (int q = 0; q < CH; q++) {
      const int z = t + N2 * (m0 + q);
      const int64_t src = grid_final_source(f.oldx, f.oldy, f.oldz, P, x, y, z);
      v[m0 + q] = __ldg(data + (src >= 0 ? src : 0));
      if (src < 0) v[m0 + q] = make_float2(0.f, 0.f);
      wt[q] = __ldg(wsrc + ((int64_t)z * P + y) * R + x);
    }
#pragma unroll
    for (int q = 0; q < CH; q++)
      v[m0 + q] = grid_final_apply(v[m0 + q], wt[q], P, x, y, t + N2 * (m0 + q), f.divide != 0);
  }
  __syncthreads();  // twiddles in place
  four_step<P, true, false, false, 1>(v, xb, tw, t, c);
#pragma unroll
  for (int m = 0; m < N1; m++) {
    const int z = t + N2 * m - f.off;
    if ((unsigned)z < (unsigned)f.ori) tv[((int64_t)z * P + y) * R + x] = v[m];
  }
}

// Pass 2, per column (x, zc) along y: inverse transform, the crop's rows
// written to rows 0 .. ori-1 of the plane (each CTA has read its whole
// column before it writes).  Tiles: 16 consecutive x < P/2 at one zc, then
// x = P/2 at 16 consecutive zc.
template <int P>
__global__ void __launch_bounds__(kCols * Split<P>::N2, (P > 512 ? 1 : 2))
gridsym_final_y_kernel(float2* __restrict__ T, int ori, int off, const float2* __restrict__ twg) {
  constexpr int H = P / 2, R = H + 1;
  constexpr int N1 = Split<P>::N1, N2 = Split<P>::N2;
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* xb = smem + P;
  load_twiddles(tw, twg, P);
  const int c = threadIdx.x & (kCols - 1), t = threadIdx.x / kCols;
  const int kMain = (H / kCols) * ori;
  const int b = blockIdx.x;
  int zc, x;
  if (b < kMain) {
    zc = b / (H / kCols);
    x = (b - zc * (H / kCols)) * kCols + c;
  } else {
    zc = (b - kMain) * kCols + c;
    x = H;
  }
  const bool in = zc < ori;
  float2* col = T + (int64_t)blockIdx.y * ((int64_t)R * P * ori) + (in ? ((int64_t)zc * P * R + x) : 0);
  float2 v[N1];
#pragma unroll
  for (int m = 0; m < N1; m++) v[m] = in ? col[(int64_t)(t + N2 * m) * R] : make_float2(0.f, 0.f);
  __syncthreads();  // twiddles in place
  four_step<P, true, false, false, 1>(v, xb, tw, t, c);
  if (in) {
#pragma unroll
    for (int m = 0; m < N1; m++) {
      const int yc = t + N2 * m - off;
      if ((unsigned)yc < (unsigned)ori) col[(int64_t)yc * R] = v[m];
    }
  }
}

// Pass 3, per row (yc, zc): C2R along x (the x = 0 and x = P/2 terms taken
// as real), the crop's x, the gridding correction and scale.  A CTA takes
// 16 consecutive rows of the ori x ori crop (rows past it idle).
template <int P>
__global__ void __launch_bounds__(kCols * Split<P / 2>::N2, (P > 512 ? 2 : 3))
gridsym_final_x_kernel(const float2* __restrict__ T, FinalArgs f, const float2* __restrict__ twg) {
  constexpr int H = P / 2, R = H + 1;
  constexpr int N1 = Split<H>::N1, N2 = Split<H>::N2;
  constexpr bool WROW = 32 % N2 == 0;
  constexpr int XS = N2 * (N1 + 1);
  extern __shared__ float2 smem[];
  float2* tw = smem;
  float2* xb = smem + P + P / 16;  // after the padded twiddle table
  load_twiddles_padded(tw, twg, P);
  const int t = threadIdx.x % N2, r = threadIdx.x / N2;
  const unsigned lane = threadIdx.x & 31;
  const unsigned partner = WROW ? (lane & ~(unsigned)(N2 - 1)) | ((unsigned)(N2 - t) & (N2 - 1)) : lane;
  const int ori = f.ori;
  const int64_t rr = (int64_t)blockIdx.x * kCols + r;  // zc * ori + yc
  const bool in = rr < (int64_t)ori * ori;
  const int zc = in ? (int)(rr / ori) : 0, yc = in ? (int)(rr - (int64_t)zc * ori) : 0;
  const int64_t vol = blockIdx.y;
  const float2* row = T + vol * ((int64_t)R * P * ori) + ((int64_t)zc * P + yc) * R;
  float2 v[N1];
#pragma unroll
  for (int m = 0; m < N1; m++) v[m] = in ? row[t + N2 * m] : make_float2(0.f, 0.f);
  const float2 xH = t == 0 && in ? make_float2(row[H].x, 0.f) : make_float2(0.f, 0.f);
  if (t == 0) v[0].y = 0.f;
  __syncthreads();  // twiddles in place
  {
    float2 z[N1];
    if constexpr (WROW) {
#pragma unroll
      for (int m = 0; m < N1; m++) {
        const float2 sh = make_float2(__shfl_sync(0xffffffffu, v[N1 - 1 - m].x, partner),
                                      __shfl_sync(0xffffffffu, v[N1 - 1 - m].y, partner));
        const float2 xm = t != 0 ? sh : (m == 0 ? xH : v[(N1 - m) % N1]);
        z[m] = c2r_pre<true>(v[m], xm, tw[tw_pad(t + N2 * m)]);
      }
    } else {
#pragma unroll
      for (int m = 0; m < N1; m++) xb[r * XS + t + N2 * m] = v[m];
      if (t == 0) xb[r * XS + H] = xH;
      __syncthreads();
#pragma unroll
      for (int m = 0; m < N1; m++) {
        const int k = t + N2 * m;
        z[m] = c2r_pre<true>(v[m], xb[r * XS + H - k], tw[tw_pad(k)]);
      }
    }
#pragma unroll
    for (int m = 0; m < N1; m++) v[m] = z[m];
  }
  four_step<H, true, true, WROW, 2>(v, xb, tw, t, r);
  if (!in) return;  // after the last collective of the row's warp / block
  // a y pass whose tensor copies did not complete left W unusable: NaN map
  const bool fault = g_gridsym_fault != 0;
  float* out = f.outs ? f.outs[vol] : f.out;
  float* orow = out + ((int64_t)zc * ori + yc) * ori;
#pragma unroll
  for (int m = 0; m < N1; m++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int xc = 2 * (t + N2 * m) + h - f.off;
      if ((unsigned)xc < (unsigned)ori)
        orow[xc] = fault ? __int_as_float(0x7fc00000) : grid_crop_value(h ? v[m].y : v[m].x, xc, yc, zc, ori, P,
                                                                        f.scale);
    }
  }
}

// ------------------------------------------------------------- launch --
template <int P>
struct SymSizes {
  static constexpr int H = P / 2;
  static constexpr int y_threads = kCols * Split<P>::N2;
  static constexpr int xz_threads = kCols * Split<H>::N2;
  static constexpr int x_tiles = (H + 1) * P / kCols;
  static constexpr int z_tiles = P * (H / kCols) + P / kCols;
  // twiddle table + exchange buffer
  static constexpr size_t y_smem = sizeof(float2) * (P + (size_t)P * kPitch);
  static constexpr size_t x_smem =
      sizeof(float2) * (P + P / 16 + (size_t)kCols * Split<H>::N2 * (Split<H>::N1 + 1));  // padded twiddles
  static constexpr size_t z_smem = sizeof(float2) * (P + (size_t)(H + 1) * kPitch);
};

template <int P>
int set_attributes() {
  using Z = SymSizes<P>;
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_y_tma_kernel<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)YStage<P>::smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_y_tma_kernel<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)YStage<P>::smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_final_z_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Z::y_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_final_y_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Z::y_smem));
  GTOMRLN_CUDA_TRY(cudaFuncSetAttribute(gridsym_final_x_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Z::x_smem));
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

// cuTensorMapEncodeTiled, looked up once through the runtime (no link
// against the driver library).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
std::once_flag g_encode_once;
EncodeTiledFn g_encode = nullptr;

// The tensor map of W for the staged y pass: floats, dims {2 w_pitch, P,
// (P/2+1) count} (the z planes of all volumes in one dimension), row stride
// w_pitch 8 bytes (a multiple of 32), box {32, BOX, 1}.
template <int P>
int w_tensor_map(float2* W, int count, CUtensorMap* map) {
  std::call_once(g_encode_once, [] {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&g_encode, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      g_encode = nullptr;
    cudaGetLastError();
  });
  if (!g_encode) return set_error(GTOMRLN_ERR_CUDA, "gridsym: cuTensorMapEncodeTiled is not available");
  if (reinterpret_cast<uintptr_t>(W) % 16)
    return set_error(GTOMRLN_ERR_INVALID, "gridsym: work array not 16-byte aligned");
  constexpr int RW = w_pitch<P>();
  const cuuint64_t dims[3] = {(cuuint64_t)2 * RW, (cuuint64_t)P, (cuuint64_t)(P / 2 + 1) * (cuuint64_t)count};
  const cuuint64_t strides[2] = {(cuuint64_t)RW * sizeof(float2), (cuuint64_t)P * RW * sizeof(float2)};
  const cuuint32_t box[3] = {2 * kCols, (cuuint32_t)YStage<P>::BOX, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, W, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(GTOMRLN_ERR_CUDA, "gridsym: tensor map encoding failed (%d)", (int)r);
  return GTOMRLN_OK;
}

// CTAs of the staged y pass resident on the device (both directions have the
// same resources), per (device, context, P).
std::mutex g_ctas_mutex;
std::map<std::tuple<int, unsigned long long, int>, int> g_ctas;

template <int P>
int y_stage_ctas(int* out) {
  int dev = 0;
  GTOMRLN_CUDA_TRY(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, context_id(), P);
  std::lock_guard<std::mutex> lock(g_ctas_mutex);
  auto it = g_ctas.find(key);
  if (it == g_ctas.end()) {
    int per_sm = 0, sms = 0;
    GTOMRLN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gridsym_y_tma_kernel<P, true>,
                                                                   SymSizes<P>::y_threads, YStage<P>::smem));
    GTOMRLN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return set_error(GTOMRLN_ERR_CUDA, "gridsym: staged y pass does not fit an SM");
    it = g_ctas.emplace(key, per_sm * sms).first;
  }
  *out = it->second;
  return GTOMRLN_OK;
}

template <int P>
int run_first(float2* W, int count, const float* Fw, float* Fnw, float* V, const float2* tw,
              cudaStream_t stream) {
  using Z = SymSizes<P>;
  const dim3 grid(Z::z_tiles, count);
  if (V)
    gridsym_z_kernel<P, kZFirst, true><<<grid, Z::xz_threads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, 0.f, 1,
                                                                                   nullptr, nullptr);
  else
    gridsym_z_kernel<P, kZFirst, false><<<grid, Z::xz_threads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, 0.f, 1,
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
  CUtensorMap map;
  int st = w_tensor_map<P>(W, count, &map);
  if (st) return st;
  int ctas = 0;
  st = y_stage_ctas<P>(&ctas);
  if (st) return st;
  const int tiles = (P / 2 / kCols) * (P / 2 + 1) * count;
  const unsigned grid_y = (unsigned)std::min(tiles, ctas);
  const int nyq = (P / 2 + 1 + kCols - 1) / kCols * count;
  gridsym_y_tma_kernel<P, true><<<grid_y, Z::y_threads, YStage<P>::smem, stream>>>(map, W, tw, tiles, nyq);
  GTOMRLN_LAUNCH_CHECK("gridsym_y_tma_kernel (inverse)");
  gridsym_x_kernel<P><<<dim3(Z::x_tiles, count), Z::xz_threads, Z::x_smem, stream>>>(W, tw, table, inv_n,
                                                                                     funcsampling);
  GTOMRLN_LAUNCH_CHECK("gridsym_x_kernel");
  gridsym_y_tma_kernel<P, false><<<grid_y, Z::y_threads, YStage<P>::smem, stream>>>(map, W, tw, tiles, nyq);
  GTOMRLN_LAUNCH_CHECK("gridsym_y_tma_kernel (forward)");
  const dim3 grid(Z::z_tiles, count);
  if (V)
    gridsym_z_kernel<P, kZIter, true><<<grid, Z::xz_threads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, beta,
                                                                                  write_next, change, ref);
  else
    gridsym_z_kernel<P, kZIter, false><<<grid, Z::xz_threads, Z::z_smem, stream>>>(W, Fw, Fnw, V, tw, beta,
                                                                                   write_next, change, ref);
  GTOMRLN_LAUNCH_CHECK("gridsym_z_kernel");
  return GTOMRLN_OK;
}

template <int P>
int run_final(float2* T, int count, const FinalArgs& f, const float2* tw, cudaStream_t stream) {
  using Z = SymSizes<P>;
  constexpr int H = P / 2;
  gridsym_final_z_kernel<P><<<dim3(Z::z_tiles, count), Z::y_threads, Z::y_smem, stream>>>(T, f, tw);
  GTOMRLN_LAUNCH_CHECK("gridsym_final_z_kernel");
  const unsigned ytiles = (unsigned)((H / kCols) * f.ori + (f.ori + kCols - 1) / kCols);
  gridsym_final_y_kernel<P><<<dim3(ytiles, count), Z::y_threads, Z::y_smem, stream>>>(T, f.ori, f.off, tw);
  GTOMRLN_LAUNCH_CHECK("gridsym_final_y_kernel");
  const unsigned xtiles = (unsigned)(((int64_t)f.ori * f.ori + kCols - 1) / kCols);
  gridsym_final_x_kernel<P><<<dim3(xtiles, count), Z::xz_threads, Z::x_smem, stream>>>(T, f, tw);
  GTOMRLN_LAUNCH_CHECK("gridsym_final_x_kernel");
  return GTOMRLN_OK;
}

// Dispatch over the supported grids.
template <typename F>
int with_grid(int P, F&& f) {
  switch (P) {
    case 64: return f(std::integral_constant<int, 64>());
    case 96: return f(std::integral_constant<int, 96>());
    case 128: return f(std::integral_constant<int, 128>());
    case 192: return f(std::integral_constant<int, 192>());
    case 256: return f(std::integral_constant<int, 256>());
    case 512: return f(std::integral_constant<int, 512>());
    case 800: return f(std::integral_constant<int, 800>());
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

bool gridsym_available(int P) {
  return P == 64 || P == 96 || P == 128 || P == 192 || P == 256 || P == 512 || P == 800;
}

int gridsym_prepare(int P) {
  int st = ensure_attributes(P);
  if (st) return st;
  const float2* tw = nullptr;
  return fft_twiddles(P, &tw);
}

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

int gridsym_final(float2* T, const GridGeom& g, int count, const float2* data, int oldx, int oldy, int oldz,
                  int64_t wstride, const float* Fw, const float* Fnw, bool divide, int ori, float scale, float* out,
                  float* const* outs, cudaStream_t stream) {
  if (ori <= 0 || ori > g.P) return set_error(GTOMRLN_ERR_INVALID, "gridsym_final: output box %d", ori);
  int st = ensure_attributes(g.P);
  if (st) return st;
  const float2* tw = nullptr;
  st = fft_twiddles(g.P, &tw);
  if (st) return st;
  FinalArgs f;
  f.data = data;
  f.oldx = oldx;
  f.oldy = oldy;
  f.oldz = oldz;
  f.wstride = wstride;
  f.Fw = Fw;
  f.Fnw = Fnw;
  f.divide = divide ? 1 : 0;
  f.ori = ori;
  f.off = g.P / 2 - ori / 2;
  f.scale = scale;
  f.out = out;
  f.outs = outs;
  return with_grid(g.P, [&](auto p) { return run_final<decltype(p)::value>(T, count, f, tw, stream); });
}

// Forgets the launch attributes set on device dev (a context reset drops
// them with the context).
int release_gridsym_caches(int dev, unsigned long long /*ctx*/) {
  {
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    for (auto it = g_attr_done.begin(); it != g_attr_done.end();) {
      if (std::get<0>(it->first) == dev) it = g_attr_done.erase(it);
      else ++it;
    }
  }
  {
    std::lock_guard<std::mutex> lock(g_ctas_mutex);
    for (auto it = g_ctas.begin(); it != g_ctas.end();) {
      if (std::get<0>(it->first) == dev) it = g_ctas.erase(it);
      else ++it;
    }
  }
  return GTOMRLN_OK;
}

}  // namespace gtomrln
