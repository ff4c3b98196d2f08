// CPU restatement of gtom's RELION-style Fourier projector / backprojector.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA library is
// compared against (and, in its single-precision instantiation, the CPU
// baseline that the benchmark times on the host cores).  Nothing in the
// product library links or calls it.
//
// Parity pin: the restatement is pinned against the reference's own CUDA
// path rebuilt from source (oracle/ref_harness.cu, built by oracle/Makefile
// into oracle/_ref/) through the golden fixtures in tests/golden/.  The
// reference ships no golden vectors of its own for this path
// (GTOMTest/RelionProject.cpp is commented out, GTOMTest/RecFourier.cpp
// asserts nothing).
//
// Two precisions are instantiated from one template:
//   R = double : the FP64 oracle (accumulation and interpolation in double),
//   R = float  : the FP32 OpenMP port timed as the CPU baseline.
//
// Layouts (identical to the reference):
//   volume   : half-complex (P/2+1) x P x P, x fastest, interleaved re/im,
//              decentred (FFT order in y and z) for the projector.
//   slices   : half-complex (n/2+1) x n [x n for 3D], FFT order in y (z).
//   matrices : 9 floats per slice, column-major (glm::mat3), M = s * A^T
//              with A the RELION ZYZ Euler matrix.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// The 1e-5 guard used by the reference (a float literal there).
const float kEps = 1e-5f;

// Round a single-precision value to IEEE binary16 and back (round to nearest
// even), as __float2half/__half2float do in Backproject.cu:224-238.
inline float round_half(float v) { return (float)(_Float16)v; }

template <class R>
struct Mat3 {
  R m[9];  // column-major: m[c*3 + r]
  explicit Mat3(const float* f) {
    for (int i = 0; i < 9; i++) m[i] = (R)f[i];
  }
  // glm's mat3 * vec3 (Project.cu:120, Backproject.cu:194):
  // m[0][0]*x + m[1][0]*y + m[2][0]*z, with the fused multiply-adds the
  // reference's compiled kernel performs (first product fused with the
  // rounded second, third fused onto that).  In single precision this
  // reproduces the reference's roundings; in double it is just accurate.
  inline void apply(R x, R y, R z, R& ox, R& oy, R& oz) const {
    ox = std::fma(m[6], z, std::fma(m[0], x, m[3] * y));
    oy = std::fma(m[7], z, std::fma(m[1], x, m[4] * y));
    oz = std::fma(m[8], z, std::fma(m[2], x, m[5] * y));
  }
};

// lerp of cutil_math_bugfixes.cuh:212: fma(b - a, t, a).
template <class R>
inline R lerp(R a, R b, R t) { return std::fma(b - a, t, a); }

// ---------------------------------------------------------------------------
// Projector: Project3DArraytoNDKernel (src/Relion/Project.cu:89-177).
// ---------------------------------------------------------------------------
template <class R, class OutT>
void project_impl(const float* vol, int P, OutT* out, int n, int ndims, int rmax,
                  const float* mats, int batch) {
  const int dimft = n / 2 + 1;
  const int64_t slice = (int64_t)dimft * n;
  const int64_t elements = ndims == 3 ? slice * n : slice;
  const int volft = P / 2 + 1;
  const int64_t nvox = (int64_t)volft * P * P;
  const int rmax2 = rmax * rmax;

#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < batch; b++) {
    Mat3<R> M(mats + 9 * (int64_t)b);
    OutT* o = out + 2 * elements * (int64_t)b;
    for (int64_t id = 0; id < elements; id++) {
      int idx = (int)(id % dimft);
      int idy = (int)((ndims == 3 ? id % slice : id) / dimft);
      int idz = ndims == 3 ? (int)(id / slice) : 0;
      int x = idx;
      int y = idy <= n / 2 ? idy : idy - n;
      int z = idz <= n / 2 ? idz : idz - n;
      int r2 = ndims == 3 ? z * z + y * y + x * x : y * y + x * x;
      if (r2 > rmax2) {
        o[2 * id] = 0;
        o[2 * id + 1] = 0;
        continue;
      }
      R px, py, pz;
      M.apply((R)x, (R)y, (R)z, px, py, pz);
      R sign = 1;
      if (px < -(R)kEps) {  // Friedel mate (Project.cu:124-131)
        px = std::fabs(px);
        py = -py;
        pz = -pz;
        sign = -1;
      }
      R fx0 = std::floor(px + (R)kEps);
      int x0 = (int)fx0;
      int x1 = x0 + 1;
      R fx = px - fx0;
      R fy0 = std::floor(py);
      int y0 = (int)fy0, y1 = y0 + 1;
      if (y0 < 0) y0 += P;
      if (y1 < 0) y1 += P;
      R fy = py - fy0;
      R fz0 = std::floor(pz);
      int z0 = (int)fz0, z1 = z0 + 1;
      if (z0 < 0) z0 += P;
      if (z1 < 0) z1 += P;
      R fz = pz - fz0;
      // Flat addressing exactly as the reference: x1 == P/2+1 reads the next
      // row's first element.  The single read past the end of the array that
      // the reference can make there is clamped to the last element.
      auto at = [&](int zz, int yy, int xx, R& re, R& im) {
        int64_t i = ((int64_t)zz * P + yy) * volft + xx;
        if (i < 0) i = 0;
        if (i >= nvox) i = nvox - 1;
        re = (R)vol[2 * i];
        im = (R)vol[2 * i + 1];
      };
      R r000, i000, r001, i001, r010, i010, r011, i011;
      R r100, i100, r101, i101, r110, i110, r111, i111;
      at(z0, y0, x0, r000, i000);
      at(z0, y0, x1, r001, i001);
      at(z0, y1, x0, r010, i010);
      at(z0, y1, x1, r011, i011);
      at(z1, y0, x0, r100, i100);
      at(z1, y0, x1, r101, i101);
      at(z1, y1, x0, r110, i110);
      at(z1, y1, x1, r111, i111);
      R rx00 = lerp(r000, r001, fx), ix00 = lerp(i000, i001, fx);
      R rx01 = lerp(r010, r011, fx), ix01 = lerp(i010, i011, fx);
      R rx10 = lerp(r100, r101, fx), ix10 = lerp(i100, i101, fx);
      R rx11 = lerp(r110, r111, fx), ix11 = lerp(i110, i111, fx);
      R rxy0 = lerp(rx00, rx01, fy), ixy0 = lerp(ix00, ix01, fy);
      R rxy1 = lerp(rx10, rx11, fy), ixy1 = lerp(ix10, ix11, fy);
      o[2 * id] = (OutT)lerp(rxy0, rxy1, fz);
      o[2 * id + 1] = (OutT)(lerp(ixy0, ixy1, fz) * sign);
    }
  }
}

// ---------------------------------------------------------------------------
// Backprojector: Backproject3DtoNDKernel (src/Relion/Backproject.cu:126-322).
// ---------------------------------------------------------------------------
struct BpParams {
  int P, n, ndims, rmax;
  float mag[4];          // float4 magnification: mat2 columns (Backproject.cu:57-61)
  float ewalddiaminv;    // 1 / (2 * ewaldradius * supersample), or 0
  int decentered, square, half_weights;
};

// Map a (possibly negative) neighbour coordinate to its stored location the
// way Backproject.cu:253-274 does, including the unsigned-comparison clamps.
inline void place(int& x, int& y, int& z, const BpParams& p) {
  if (p.decentered) {
    if (y < 0) y += p.P;
    if (z < 0) z += p.P;
  } else {
    y += p.P / 2;
    z += p.P / 2;
  }
  unsigned half = (unsigned)(p.P / 2), last = (unsigned)(p.P - 1);
  if ((unsigned)x > half) x = (int)half;
  if ((unsigned)y > last) y = (int)last;
  if ((unsigned)z > last) z = (int)last;
}

template <class R, bool Atomic>
inline void add_to(R* addr, R v) {
  if (Atomic) {
#pragma omp atomic
    *addr += v;
  } else {
    *addr += v;
  }
}

template <class R, bool Atomic>
void backproject_slice(R* volft, R* volw, const float* projft, const float* projw,
                       const float* mat, const BpParams& p) {
  const int n = p.n, P = p.P;
  const int dimft = n / 2 + 1;
  const int64_t slice = (int64_t)dimft * n;
  const int64_t elements = p.ndims == 3 ? slice * n : slice;
  const int rowlen = P / 2 + 1;
  const int rmax2 = p.rmax * p.rmax;
  Mat3<R> M(mat);
  // The float path mirrors the reference's single-precision arithmetic; the
  // double path keeps every intermediate in double.
  for (int64_t id = 0; id < elements; id++) {
    int idx = (int)(id % dimft);
    int idy = (int)((p.ndims == 3 ? id % slice : id) / dimft);
    int idz = p.ndims == 3 ? (int)(id / slice) : 0;
    int x = idx;
    int y = idy <= n / 2 ? idy : idy - n;
    int z = p.ndims == 3 ? (idz <= n / 2 ? idz : idz - n) : 0;
    if (p.ndims == 3) {
      if (x == 0 && y < 0 && z < 0) continue;
    } else {
      if (x == 0 && y < 0) continue;
    }
    R qx = (R)x, qy = (R)y, qz = (R)z;
    if (p.ndims == 2) {  // glm mat2 * vec2, fused like Mat3::apply
      qx = std::fma((R)p.mag[0], (R)x, (R)p.mag[2] * (R)y);
      qy = std::fma((R)p.mag[1], (R)x, (R)p.mag[3] * (R)y);
      qz = (R)p.ewalddiaminv * (R)(x * x + y * y);
    }
    int r2 = p.ndims == 3 ? (z * z + y * y + x * x)
                          : (int)std::fma(qz, qz, std::fma(qx, qx, qy * qy));
    if (r2 >= rmax2) continue;
    R px, py, pz;
    M.apply(qx, qy, qz, px, py, pz);
    int x0 = (int)(short)std::floor(px + (R)kEps);
    int y0 = (int)(short)std::floor(py);
    int z0 = (int)(short)std::floor(pz);
    R fx = px - (R)x0, fy = py - (R)y0, fz = pz - (R)z0;
    R c0 = 1 - fz, c1 = fz;
    R w[8];
    if (p.half_weights) {
      float c00 = round_half((float)((1 - fy) * c0));
      float c10 = round_half((float)(fy * c0));
      float c01 = round_half((float)((1 - fy) * c1));
      float c11 = round_half((float)(fy * c1));
      w[0] = round_half((float)((1 - fx) * (R)c00));
      w[1] = round_half((float)(fx * (R)c00));
      w[2] = round_half((float)((1 - fx) * (R)c10));
      w[3] = round_half((float)(fx * (R)c10));
      w[4] = round_half((float)((1 - fx) * (R)c01));
      w[5] = round_half((float)(fx * (R)c01));
      w[6] = round_half((float)((1 - fx) * (R)c11));
      w[7] = round_half((float)(fx * (R)c11));
    } else {
      R c00 = (1 - fy) * c0, c10 = fy * c0, c01 = (1 - fy) * c1, c11 = fy * c1;
      w[0] = (1 - fx) * c00; w[1] = fx * c00;
      w[2] = (1 - fx) * c10; w[3] = fx * c10;
      w[4] = (1 - fx) * c01; w[5] = fx * c01;
      w[6] = (1 - fx) * c11; w[7] = fx * c11;
    }
    R vre = 1, vim = 0, pw = 1;
    if (projft) { vre = (R)projft[2 * id]; vim = (R)projft[2 * id + 1]; }
    if (projw) pw = (R)projw[id];
    for (int i = 0; i < 8; i++) {
      int nx = x0 + (i & 1), ny = y0 + ((i >> 1) & 1), nz = z0 + ((i >> 2) & 1);
      R iw = w[i];
      if (p.square) iw *= iw;
      R sre = vre, sim = vim;
      int tx = nx, ty = ny, tz = nz;
      if (tx < 0) { tx = -tx; ty = -ty; tz = -tz; sim = -sim; }
      place(tx, ty, tz, p);
      int64_t o = ((int64_t)tz * P + ty) * rowlen + tx;
      if (volft) {
        add_to<R, Atomic>(volft + 2 * o, iw * sre);
        add_to<R, Atomic>(volft + 2 * o + 1, iw * sim);
      }
      if (volw) add_to<R, Atomic>(volw + o, iw * pw);
      if (nx == 0 && (ny != 0 || nz != 0)) {  // x = 0 plane: Backproject.cu:289-319
        tx = 0; ty = -ny; tz = -nz;
        place(tx, ty, tz, p);
        o = ((int64_t)tz * P + ty) * rowlen + tx;
        if (volft) {
          add_to<R, Atomic>(volft + 2 * o, iw * sre);
          add_to<R, Atomic>(volft + 2 * o + 1, -iw * sim);
        }
        if (volw) add_to<R, Atomic>(volw + o, iw * pw);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Kaiser-Bessel blob, Fourier transform (src/Helpers/KaiserBessel.cpp:357-376).
// Restated from the closed forms of the half-integer-order Bessel functions:
//   I_{1/2}(x) = sqrt(2/(pi x)) sinh x,  I_{3/2}(x) = sqrt(2/(pi x)) (cosh x - sinh x / x)
//   J_{1/2}(x) = sqrt(2/(pi x)) sin x,   J_{3/2}(x) = sqrt(2/(pi x)) (sin x / x - cos x)
// and the recurrences Z_{v+1} = Z_{v-1} -/+ (2v/x) Z_v.  I_0 uses its power series.
// ---------------------------------------------------------------------------
const double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Shifted variants (src/Relion/ProjectShifted.cu:124-224,
// src/Relion/BackprojectShifted.cu:67-186), in float64.  shifts are the
// per-slice 2*pi/n-scaled shifts the matrix overloads take; the phase is
// exp(i phi), phi = -(x sx + y sy [+ z sz]), and the global weight scales
// the value (and, for insertion, the weight).
// ---------------------------------------------------------------------------
void project_shifted_f64(const float* vol, int P, double* out, int n, int ndims, int rmax,
                         const float* mats, const float* shifts, const float* gw, int batch) {
  project_impl<double, double>(vol, P, out, n, ndims, rmax, mats, batch);
  const int dimft = n / 2 + 1;
  const int64_t slice = (int64_t)dimft * n;
  const int64_t elements = ndims == 3 ? slice * n : slice;
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < batch; b++) {
    double* o = out + 2 * elements * (int64_t)b;
    double sx = shifts[3 * b], sy = shifts[3 * b + 1], sz = shifts[3 * b + 2], w = gw[b];
    for (int64_t id = 0; id < elements; id++) {
      int x = (int)(id % dimft);
      int idy = (int)((ndims == 3 ? id % slice : id) / dimft);
      int idz = ndims == 3 ? (int)(id / slice) : 0;
      int y = idy <= n / 2 ? idy : idy - n;
      int z = idz <= n / 2 ? idz : idz - n;
      if ((ndims == 3 ? z * z : 0) + y * y + x * x > rmax * rmax) continue;  // stays 0
      double phase = -(x * sx + y * sy + (ndims == 3 ? z * sz : 0.0));
      double c = std::cos(phase), sn = std::sin(phase);
      double re = o[2 * id], im = o[2 * id + 1];
      o[2 * id] = (re * c - im * sn) * w;
      o[2 * id + 1] = (re * sn + im * c) * w;
    }
  }
}

// BackprojectShifted3DtoNDKernel: plain (not binary16-rounded) trilinear
// weights, no mirroring of neighbours and no second insertion on x = 0 (the
// whole x = 0 column is inserted), r^2 <= rmax^2, centred output.  The
// reference writes without bounds checks; here every index is clamped as
// in the unshifted backprojector (x <= V/2, y, z <= V-1, compared unsigned).
void backproject_shifted_f64(double* volft, double* volw, int V, const float* projft,
                             const float* projw, int n, int ndims, int rmax, const float* mats,
                             const float* shifts, const float* gw, int batch) {
  const int dimft = n / 2 + 1;
  const int64_t slice = (int64_t)dimft * n;
  const int64_t elements = ndims == 3 ? slice * n : slice;
  const int rowlen = V / 2 + 1;
  for (int b = 0; b < batch; b++) {
    Mat3<double> M(mats + 9 * (int64_t)b);
    double sx = shifts[3 * b], sy = shifts[3 * b + 1], sz = shifts[3 * b + 2], w = gw[b];
    for (int64_t id = 0; id < elements; id++) {
      int x = (int)(id % dimft);
      int idy = (int)((ndims == 3 ? id % slice : id) / dimft);
      int idz = ndims == 3 ? (int)(id / slice) : 0;
      int y = idy <= rmax ? idy : idy - n;
      int z = ndims == 3 ? (idz <= rmax ? idz : idz - n) : 0;
      int r2 = ndims == 3 ? z * z + y * y + x * x : y * y + x * x;
      if (r2 > rmax * rmax) continue;
      double px, py, pz;
      M.apply(x, y, z, px, py, pz);
      double sign = 1;
      if (px + kEps < 0) {
        px = std::fabs(px);
        py = -py;
        pz = -pz;
        sign = -1;
      }
      int x0 = (int)std::floor(px + kEps);
      double fx = px - x0;
      int y0 = (int)std::floor(py);
      double fy = py - y0;
      int z0 = (int)std::floor(pz);
      double fz = pz - z0;
      y0 += V / 2;
      z0 += V / 2;
      double re = projft ? projft[2 * (elements * b + id)] : 1.0;
      double im = projft ? projft[2 * (elements * b + id) + 1] : 0.0;
      double phase = -(x * sx + y * sy + (ndims == 3 ? z * sz : 0.0));
      double c = std::cos(phase), sn = std::sin(phase);
      double vr = (re * c - im * sn) * w;
      double vi = (re * sn + im * c) * w * sign;
      double wt = (projw ? projw[elements * b + id] : 1.0) * w;
      for (int i = 0; i < 8; i++) {
        int dx = i & 1, dy = (i >> 1) & 1, dz = (i >> 2) & 1;
        double cw = (dx ? fx : 1 - fx) * (dy ? fy : 1 - fy) * (dz ? fz : 1 - fz);
        unsigned tx = (unsigned)(x0 + dx), ty = (unsigned)(y0 + dy), tz = (unsigned)(z0 + dz);
        if (tx > (unsigned)(V / 2)) tx = V / 2;
        if (ty > (unsigned)(V - 1)) ty = V - 1;
        if (tz > (unsigned)(V - 1)) tz = V - 1;
        int64_t o = ((int64_t)tz * V + ty) * rowlen + tx;
        if (volft) {
          volft[2 * o] += cw * vr;
          volft[2 * o + 1] += cw * vi;
        }
        if (volw) volw[o] += cw * wt;
      }
    }
  }
}

double bessel_i0(double x) {
  double t = x * x / 4, term = 1, sum = 1;
  for (int k = 1; k < 500; k++) {
    term *= t / ((double)k * k);
    sum += term;
    if (term < sum * 1e-18) break;
  }
  return sum;
}

double bessel_i_half(double x, int twice_order) {  // order 1/2, 3/2, 5/2, 7/2
  if (x == 0) return 0;
  double f = std::sqrt(2 / (kPi * x));
  double im = f * std::sinh(x);                        // I_{1/2}
  double i = f * (std::cosh(x) - std::sinh(x) / x);    // I_{3/2}
  if (twice_order == 1) return im;
  for (int v2 = 3; v2 < twice_order; v2 += 2) {        // I_{v+1} = I_{v-1} - (2v/x) I_v
    double next = im - ((double)v2 / x) * i;
    im = i;
    i = next;
  }
  return i;
}

double bessel_j_half(double x, int twice_order) {
  if (x == 0) return 0;
  double f = std::sqrt(2 / (kPi * x));
  double jm = f * std::sin(x);                         // J_{1/2}
  double j = f * (std::sin(x) / x - std::cos(x));      // J_{3/2}
  if (twice_order == 1) return jm;
  for (int v2 = 3; v2 < twice_order; v2 += 2) {        // J_{v+1} = (2v/x) J_v - J_{v-1}
    double next = ((double)v2 / x) * j - jm;
    jm = j;
    j = next;
  }
  return j;
}

}  // namespace

extern "C" {

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// RELION ZYZ Euler matrix A (src/Helpers/Euler.cu:39-68) for angles
// (rot, tilt, psi) in radians; returns M = s * A^T column-major, in double.
void orc_matrices_f64(const float* angles, int batch, double s, double* out) {
  for (int b = 0; b < batch; b++) {
    double a = angles[3 * b], be = angles[3 * b + 1], g = angles[3 * b + 2];
    double ca = std::cos(a), sa = std::sin(a), cb = std::cos(be), sb = std::sin(be);
    double cg = std::cos(g), sg = std::sin(g);
    double cc = cb * ca, cs = cb * sa, sc = sb * ca, ss = sb * sa;
    double A[3][3] = {{cg * cc - sg * sa, cg * cs + sg * ca, -cg * sb},
                      {-sg * cc - cg * sa, -sg * cs + cg * ca, sg * sb},
                      {sc, ss, cb}};
    double* o = out + 9 * (int64_t)b;
    // M(r, c) = s * A(c, r); column-major o[c*3 + r]
    for (int c = 0; c < 3; c++)
      for (int r = 0; r < 3; r++) o[c * 3 + r] = s * A[c][r];
  }
}

void orc_project_f64(const float* vol, int P, double* out, int n, int ndims, int rmax,
                     const float* mats, int batch) {
  project_impl<double, double>(vol, P, out, n, ndims, rmax, mats, batch);
}

void orc_project_f32(const float* vol, int P, float* out, int n, int ndims, int rmax,
                     const float* mats, int batch) {
  project_impl<float, float>(vol, P, out, n, ndims, rmax, mats, batch);
}

// FP64 backprojection.  Deterministic: slices are inserted in order on one
// thread.  volft (complex128) and volw (float64) are accumulated in place.
void orc_backproject_f64(double* volft, double* volw, int P, const float* projft,
                         const float* projw, int n, int ndims, int rmax, const float* mats,
                         const int* ivolume, const float* mag4, float ewalddiaminv,
                         int decentered, int square, int half_weights, int batch) {
  BpParams p{P, n, ndims, rmax, {mag4[0], mag4[1], mag4[2], mag4[3]}, ewalddiaminv,
             decentered, square, half_weights};
  const int dimft = n / 2 + 1;
  const int64_t elements = (int64_t)dimft * n * (ndims == 3 ? n : 1);
  const int64_t nvox = (int64_t)(P / 2 + 1) * P * P;
  for (int b = 0; b < batch; b++) {
    int64_t off = ivolume ? (int64_t)ivolume[b] * nvox : 0;
    backproject_slice<double, false>(volft ? volft + 2 * off : nullptr, volw ? volw + off : nullptr,
                                     projft ? projft + 2 * elements * b : nullptr,
                                     projw ? projw + elements * b : nullptr, mats + 9 * (int64_t)b, p);
  }
}

// FP32 OpenMP backprojection (the CPU baseline): slices in parallel, atomic
// single-precision adds into the shared volume, like the GPU reference.
void orc_backproject_f32(float* volft, float* volw, int P, const float* projft,
                         const float* projw, int n, int ndims, int rmax, const float* mats,
                         const int* ivolume, const float* mag4, float ewalddiaminv,
                         int decentered, int square, int half_weights, int batch) {
  BpParams p{P, n, ndims, rmax, {mag4[0], mag4[1], mag4[2], mag4[3]}, ewalddiaminv,
             decentered, square, half_weights};
  const int dimft = n / 2 + 1;
  const int64_t elements = (int64_t)dimft * n * (ndims == 3 ? n : 1);
  const int64_t nvox = (int64_t)(P / 2 + 1) * P * P;
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < batch; b++) {
    int64_t off = ivolume ? (int64_t)ivolume[b] * nvox : 0;
    backproject_slice<float, true>(volft ? volft + 2 * off : nullptr, volw ? volw + off : nullptr,
                                   projft ? projft + 2 * elements * b : nullptr,
                                   projw ? projw + elements * b : nullptr, mats + 9 * (int64_t)b, p);
  }
}

// kaiser_Fourier_value(w, a, alpha, m) for m in {0, 2}; returns NaN otherwise.
// ProjectShifted.cu:124-224 / BackprojectShifted.cu:67-186 (float64).
void orc_project_shifted_f64(const float* vol, int P, double* out, int n, int ndims, int rmax,
                             const float* mats, const float* shifts, const float* gw, int batch) {
  project_shifted_f64(vol, P, out, n, ndims, rmax, mats, shifts, gw, batch);
}

void orc_backproject_shifted_f64(double* volft, double* volw, int V, const float* projft,
                                 const float* projw, int n, int ndims, int rmax, const float* mats,
                                 const float* shifts, const float* gw, int batch) {
  backproject_shifted_f64(volft, volw, V, projft, projw, n, ndims, rmax, mats, shifts, gw, batch);
}

double orc_kaiser_fourier_value(double w, double a, double alpha, int m) {
  double t = 2 * kPi * a * w;
  double sigma = std::sqrt(std::fabs(alpha * alpha - t * t));
  int twice = m == 0 ? 3 : (m == 2 ? 7 : -1);
  if (twice < 0) return std::nan("");
  double pw = m == 0 ? 1.5 : 3.5;
  double bes = t > alpha ? bessel_j_half(sigma, twice) : bessel_i_half(sigma, twice);
  double lead = std::pow(2 * kPi, 1.5) * std::pow(a, 3.0) * (m == 2 ? alpha * alpha : 1.0);
  return lead * bes / (bessel_i0(alpha) * std::pow(sigma, pw));
}

// The gridding blob table: nsamples values at w = i * 0.5 / nsamples,
// normalised by the value at w = 0 (RecFourier.cu:104-116).
void orc_kb_table(double radius, double alpha, int order, int nsamples, double* out) {
  double sampling = 0.5 / nsamples;
  for (int i = 0; i < nsamples; i++) out[i] = orc_kaiser_fourier_value(i * sampling, radius, alpha, order);
  double norm = out[0];
  for (int i = 0; i < nsamples; i++) out[i] /= norm;
}

}  // extern "C"
