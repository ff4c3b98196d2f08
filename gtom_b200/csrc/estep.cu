// RELION E-step consumers of the projections: squared differences between
// CTF-weighted reference projections and shifted particles, their remapping
// into the weight layout with the minimum per particle, the conversion to
// weights, sorting and compaction, the inverse noise spectra, and the
// weighted accumulation of the shifted particles (gtom's src/Relion/
// ConvertWeights.cu, DiffRemap.cu, Misc.cu, StoreWeights.cu; the squared
// differences are declared in include/Relion.cuh:46-48 but their source,
// src/Relion/SquaredDifferences.cu, is empty, and are defined here from the
// CPU computation in GTOMTest/RelionSquaredDiff.cpp:55-69).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "common.cuh"

namespace gtomrln {

namespace {

constexpr int kDiffThreads = 256;

// diff2 for a group of refs x shifts of one particle over n elements:
//   plain: 0.5 sum_i w_i |c_i ref_i - p_i shift_i|^2
//   cc:    -sum_i Re((c_i ref_i) conj(p_i shift_i)) / sqrt(sum_i |c_i ref_i|^2)
// (w = minvsigma2, c = ctf, p = particle).  One CTA per group; each thread
// strides over the elements holding the group's G x G partial sums.
template <int G, bool CC>
__global__ void __launch_bounds__(kDiffThreads)
diff2_group_kernel(const float2* __restrict__ particle, const float* __restrict__ minvsigma2,
                   const float* __restrict__ ctf, int64_t elements, const float2* __restrict__ shifts,
                   const float2* __restrict__ refs, float* __restrict__ diff2,
                   const uint3* __restrict__ combos, unsigned nrefs, unsigned nshifts, unsigned nparticles) {
  // group -> (first shift, particle, first ref) and output base
  unsigned s0, part, r0;
  int64_t out0;
  int rstride;  // output stride between refs of the group
  if (combos) {
    uint3 c = combos[blockIdx.x];
    s0 = c.x;
    part = c.y;
    r0 = c.z;
    out0 = (int64_t)blockIdx.x * G * G;
    rstride = G;
  } else {  // dense: blocks over (particle, ref group, shift group)
    unsigned ng_s = (nshifts + G - 1) / G, ng_r = (nrefs + G - 1) / G;
    unsigned b = blockIdx.x;
    unsigned gs = b % ng_s;
    b /= ng_s;
    unsigned gr = b % ng_r;
    part = b / ng_r;
    s0 = gs * G;
    r0 = gr * G;
    out0 = ((int64_t)part * nrefs + r0) * nshifts + s0;
    rstride = (int)nshifts;
  }
  const float2* p = particle + elements * part;
  const float* cp = ctf ? ctf + elements * part : nullptr;
  float acc[G][G];
  float aa[G];
#pragma unroll
  for (int r = 0; r < G; r++) {
    aa[r] = 0.f;
#pragma unroll
    for (int s = 0; s < G; s++) acc[r][s] = 0.f;
  }
  for (int64_t i = threadIdx.x; i < elements; i += kDiffThreads) {
    float2 pv = p[i];
    float w = minvsigma2 ? minvsigma2[i] : 1.f;
    float c = cp ? cp[i] : 1.f;
    float2 b[G];
#pragma unroll
    for (int s = 0; s < G; s++) {
      float2 sh = (combos || s0 + s < nshifts) ? shifts[elements * (s0 + s) + i] : make_float2(0.f, 0.f);
      b[s] = make_float2(pv.x * sh.x - pv.y * sh.y, pv.x * sh.y + pv.y * sh.x);
    }
#pragma unroll
    for (int r = 0; r < G; r++) {
      float2 rv = (combos || r0 + r < nrefs) ? refs[elements * (r0 + r) + i] : make_float2(0.f, 0.f);
      float2 a = make_float2(rv.x * c, rv.y * c);
      if (CC) aa[r] = fmaf(a.x, a.x, fmaf(a.y, a.y, aa[r]));
#pragma unroll
      for (int s = 0; s < G; s++) {
        if (CC) {
          acc[r][s] = fmaf(a.x, b[s].x, fmaf(a.y, b[s].y, acc[r][s]));
        } else {
          float dx = a.x - b[s].x, dy = a.y - b[s].y;
          acc[r][s] = fmaf(w, fmaf(dx, dx, dy * dy), acc[r][s]);
        }
      }
    }
  }
  // block reduction of the G x G (+ G) partial sums
  __shared__ float red[kDiffThreads / 32][G * G + G];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < G; r++) {
#pragma unroll
    for (int s = 0; s < G; s++) {
      float v = acc[r][s];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][r * G + s] = v;
    }
    if (CC) {
      float v = aa[r];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][G * G + r] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < G * G) {
    const int r = threadIdx.x / G, s = threadIdx.x % G;
    float v = 0.f, n = 0.f;
    for (int k = 0; k < kDiffThreads / 32; k++) {
      v += red[k][threadIdx.x];
      if (CC) n += red[k][G * G + r];
    }
    bool inside = combos || (r0 + r < nrefs && s0 + s < nshifts);
    if (inside) diff2[out0 + (int64_t)r * rstride + s] = CC ? -v / sqrtf(n) : 0.5f * v;
  }
}

// Dense layout [particle][reference][shift] (gtomrln_squared_differences):
// one CTA per 64 references x 64 shifts of one particle.  Chunks of 32
// elements of c * ref and particle * shift are staged in shared memory
// (element-major, rows padded against bank conflicts); each thread holds
// 4 x 4 outputs (references tr + 16 k, shifts ts + 16 k).  For the squared
// differences both staged operands are scaled by sqrt(w) of their element,
// so that a term w |a - b|^2 = |sqrt(w) a - sqrt(w) b|^2 costs four FP32
// instructions instead of five (the extra rounding of the scaled operands
// is of the order of the products' own; the expanded form, which would
// cancel for close matches, is not used).
constexpr int kDT = 64;        // references and shifts per tile
constexpr int kDK = 32;        // elements per staged chunk
constexpr int kDThreads = 256;
template <bool CC>
__global__ void __launch_bounds__(kDThreads)
diff2_dense_tiled_kernel(const float2* __restrict__ particle, const float* __restrict__ minvsigma2,
                         const float* __restrict__ ctf, int64_t elements, const float2* __restrict__ shifts,
                         const float2* __restrict__ refs, float* __restrict__ diff2, unsigned nrefs,
                         unsigned nshifts) {
  __shared__ float2 As[kDK][kDT + 1];  // c * ref
  __shared__ float2 Bs[kDK][kDT + 1];  // particle * shift
  const unsigned part = blockIdx.z, r0 = blockIdx.y * kDT, s0 = blockIdx.x * kDT;
  const int tid = threadIdx.x, tr = tid >> 4, ts = tid & 15;
  const int li = tid & (kDK - 1), lrow = tid / kDK;  // loader: element li, rows lrow + 8 k
  const float2* pp = particle + elements * part;
  const float* cp = ctf ? ctf + elements * part : nullptr;
  float acc[4][4], nn[4];
  // (x, y) partial sums per output as packed pairs, added at the end
  unsigned long long acc2[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    nn[a] = 0.f;
#pragma unroll
    for (int b = 0; b < 4; b++) {
      acc[a][b] = 0.f;
      acc2[a][b] = 0ull;
    }
  }
  for (int64_t i0 = 0; i0 < elements; i0 += kDK) {
    const int64_t gi = i0 + li;
    const bool ok = gi < elements;
    const float2 pv = ok ? pp[gi] : make_float2(0.f, 0.f);
    const float c = ok ? (cp ? cp[gi] : 1.f) : 0.f;
    float2 rv[kDT / (kDThreads / kDK)], sv[kDT / (kDThreads / kDK)];
#pragma unroll
    for (int k = 0; k < kDT / (kDThreads / kDK); k++) {
      const unsigned row = lrow + k * (kDThreads / kDK);
      rv[k] = ok && r0 + row < nrefs ? refs[elements * (r0 + row) + gi] : make_float2(0.f, 0.f);
      sv[k] = ok && s0 + row < nshifts ? shifts[elements * (s0 + row) + gi] : make_float2(0.f, 0.f);
    }
    // sqrt(w) of the loader's element (squared differences only)
    const float sw = CC ? 1.f : (ok ? (minvsigma2 ? sqrtf(minvsigma2[gi]) : 1.f) : 0.f);
    const float cs = c * sw;
#pragma unroll
    for (int k = 0; k < kDT / (kDThreads / kDK); k++) {
      const int row = lrow + k * (kDThreads / kDK);
      As[li][row] = make_float2(rv[k].x * cs, rv[k].y * cs);
      float2 bv = make_float2(pv.x * sv[k].x - pv.y * sv[k].y, pv.x * sv[k].y + pv.y * sv[k].x);
      if (!CC) bv = make_float2(bv.x * sw, bv.y * sw);
      Bs[li][row] = bv;
    }
    __syncthreads();
#pragma unroll 4
    for (int i = 0; i < kDK; i++) {
      float2 a[4], b[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        a[k] = As[i][tr + 16 * k];
        b[k] = Bs[i][ts + 16 * k];
      }
#pragma unroll
      for (int x = 0; x < 4; x++) {
        if (CC) nn[x] = fmaf(a[x].x, a[x].x, fmaf(a[x].y, a[x].y, nn[x]));
#pragma unroll
        for (int y = 0; y < 4; y++) {
          if (CC) {
            // (sx, sy) += (a.x b.x, a.y b.y): one packed FMA
            const unsigned long long av = *reinterpret_cast<const unsigned long long*>(&a[x]);
            const unsigned long long bv = *reinterpret_cast<const unsigned long long*>(&b[y]);
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc2[x][y]) : "l"(av), "l"(bv));
          } else {
            // (dx, dy) = a - b and (sx, sy) += (dx^2, dy^2) as one packed
            // subtraction and one packed FMA (two issue slots, IEEE per lane)
            const unsigned long long av = *reinterpret_cast<const unsigned long long*>(&a[x]);
            const unsigned long long bv = *reinterpret_cast<const unsigned long long*>(&b[y]);
            unsigned long long d;
            asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(av), "l"(bv));
            asm("fma.rn.f32x2 %0, %1, %1, %0;" : "+l"(acc2[x][y]) : "l"(d));
          }
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const float2 v = *reinterpret_cast<const float2*>(&acc2[x][y]);
      acc[x][y] = v.x + v.y;
    }
#pragma unroll
  for (int x = 0; x < 4; x++) {
    const unsigned r = r0 + tr + 16 * x;
    if (r >= nrefs) continue;
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const unsigned s2 = s0 + ts + 16 * y;
      if (s2 < nshifts)
        diff2[((int64_t)part * nrefs + r) * nshifts + s2] = CC ? -acc[x][y] / sqrtf(nn[x]) : 0.5f * acc[x][y];
    }
  }
}

template <int G>
int launch_diff2(bool cc, unsigned blocks, cudaStream_t stream, const float2* particle, const float* w,
                 const float* ctf, int64_t elements, const float2* shifts, const float2* refs, float* diff2,
                 const uint3* combos, unsigned nrefs, unsigned nshifts, unsigned nparticles) {
  if (cc)
    diff2_group_kernel<G, true><<<blocks, kDiffThreads, 0, stream>>>(particle, w, ctf, elements, shifts, refs,
                                                                     diff2, combos, nrefs, nshifts, nparticles);
  else
    diff2_group_kernel<G, false><<<blocks, kDiffThreads, 0, stream>>>(particle, w, ctf, elements, shifts, refs,
                                                                      diff2, combos, nrefs, nshifts, nparticles);
  GTOMRLN_LAUNCH_CHECK("diff2_group_kernel");
  return GTOMRLN_OK;
}

int diff2_dispatch(unsigned G, bool cc, unsigned blocks, cudaStream_t stream, const float2* particle,
                   const float* w, const float* ctf, int64_t elements, const float2* shifts, const float2* refs,
                   float* diff2, const uint3* combos, unsigned nrefs, unsigned nshifts, unsigned nparticles) {
  switch (G) {
    case 1: return launch_diff2<1>(cc, blocks, stream, particle, w, ctf, elements, shifts, refs, diff2, combos, nrefs, nshifts, nparticles);
    case 2: return launch_diff2<2>(cc, blocks, stream, particle, w, ctf, elements, shifts, refs, diff2, combos, nrefs, nshifts, nparticles);
    case 4: return launch_diff2<4>(cc, blocks, stream, particle, w, ctf, elements, shifts, refs, diff2, combos, nrefs, nshifts, nparticles);
    case 8: return launch_diff2<8>(cc, blocks, stream, particle, w, ctf, elements, shifts, refs, diff2, combos, nrefs, nshifts, nparticles);
    default: return set_error(GTOMRLN_ERR_INVALID, "squared differences: group size %u not 1, 2, 4 or 8", G);
  }
}

// ConvertWeightsDenseKernel (ConvertWeights.cu:23-44): in place,
// w = pdfrot[class, rot] * pdftrans[particle, class, trans] * exp(-(diff2 - mindiff2[particle])).
__global__ void convert_dense_kernel(float* __restrict__ w, uint64_t elements, unsigned perpart,
                                     unsigned perclass, unsigned nclasses, unsigned nrot, unsigned ntrans,
                                     const float* __restrict__ pdfrot, const float* __restrict__ pdftrans,
                                     const float* __restrict__ mindiff2) {
  for (uint64_t id = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; id < elements;
       id += (uint64_t)gridDim.x * blockDim.x) {
    unsigned ipart = (unsigned)(id / perpart), iclass = (unsigned)((id % perpart) / perclass);
    unsigned irot = (unsigned)((id % perclass) / ntrans), itrans = (unsigned)(id % ntrans);
    float d = w[id] - mindiff2[ipart];
    float weight = pdfrot[iclass * nrot + irot] * pdftrans[((uint64_t)ipart * nclasses + iclass) * ntrans + itrans];
    w[id] = weight * __expf(-d);
  }
}

// ConvertWeightsSparseKernel (ConvertWeights.cu:53-73); combination =
// (class, rot, trans, index into the dense array).
__global__ void convert_sparse_kernel(float* __restrict__ dense, float* __restrict__ sparse,
                                      const uint4* __restrict__ combos, unsigned nsparse, unsigned nrot,
                                      unsigned ntrans, const float* __restrict__ pdfrot,
                                      const float* __restrict__ pdftrans, const float* __restrict__ mindiff2) {
  for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < nsparse; id += gridDim.x * blockDim.x) {
    uint4 c = combos[id];
    float d = dense[c.w] - *mindiff2;
    float weight = pdfrot[c.x * nrot + c.y] * pdftrans[c.x * ntrans + c.z] * __expf(-d);
    dense[c.w] = weight;
    sparse[id] = weight;
  }
}

// DiffRemapDenseKernel (DiffRemap.cu:30-51).
template <bool CC>
__global__ void remap_dense_kernel(const float* __restrict__ in, float* __restrict__ out,
                                   const uint3* __restrict__ orient, uint64_t elements, unsigned iclass,
                                   unsigned nparticles, unsigned nclasses, unsigned nrot, unsigned ntrans,
                                   unsigned ntranspadded, const float* __restrict__ xi2,
                                   const float* __restrict__ sqrtxi2) {
  for (uint64_t id = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; id < elements;
       id += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t per = (uint64_t)nparticles * ntrans;
    unsigned irot = (unsigned)(id / per);
    unsigned ipart = (unsigned)((id - irot * per) / ntrans), itrans = (unsigned)(id % ntrans);
    unsigned iorient = orient[irot].y;
    float v = in[((uint64_t)irot * nparticles + ipart) * ntranspadded + itrans];
    v = CC ? v * sqrtxi2[ipart] : v + xi2[ipart];
    out[(((uint64_t)ipart * nclasses + iclass) * nrot + iorient) * ntrans + itrans] = v;
  }
}

__device__ __forceinline__ void atomic_min_float(float* addr, float v) {
  int* a = (int*)addr;
  int old = *a, assumed;
  do {
    assumed = old;
    old = atomicCAS(a, assumed, __float_as_int(fminf(v, __int_as_float(assumed))));
  } while (assumed != old);
}

// DiffRemapSparseKernel (DiffRemap.cu:65-88): values placed at
// weightsperpart * particle + hiddenover[id]; the per-particle minimum is
// folded into mindiff2 (minimum within the warp first, then one atomic per
// run of lanes of the same particle).
template <bool CC>
__global__ void remap_sparse_kernel(const float* __restrict__ in, float* __restrict__ out,
                                    float* __restrict__ mindiff2, const uint3* __restrict__ combos,
                                    const unsigned* __restrict__ hiddenover, unsigned elements,
                                    unsigned tileelements, unsigned weightsperpart,
                                    const float* __restrict__ xi2, const float* __restrict__ sqrtxi2) {
  for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < elements; id += gridDim.x * blockDim.x) {
    unsigned ipart = combos[id / tileelements].y;
    float v = in[id];
    v = CC ? v * sqrtxi2[ipart] : v + xi2[ipart];
    out[(uint64_t)weightsperpart * ipart + hiddenover[id]] = v;
    atomic_min_float(mindiff2 + ipart, v);
  }
}

// CreateMinvsigma2sKernel (Misc.cu:19-29).
__global__ void minvsigma2_kernel(float* __restrict__ out, const int* __restrict__ mresol, unsigned elements,
                                  const float* __restrict__ sigma2noise, float fudge) {
  for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < elements; id += gridDim.x * blockDim.x) {
    int r = mresol[id];
    out[id] = r > 0 ? 1.f / (fudge * sigma2noise[r]) : 0.f;
  }
}

// StoreWeightsAddKernel (StoreWeights.cu:20-63); blockIdx.y = translation.
template <bool SCALE>
__global__ void store_weights_kernel(const float2* __restrict__ input, const float* __restrict__ ctf,
                                     const float2* __restrict__ ref, const float* __restrict__ minvsigma2,
                                     const int* __restrict__ mresol, unsigned elements,
                                     const float* __restrict__ weights, float sigweight, float invsum,
                                     float2* __restrict__ output, float* __restrict__ outweights,
                                     float* __restrict__ sigma2noise, float* __restrict__ normcorr,
                                     const float* __restrict__ priorclass, float* __restrict__ corrxa,
                                     float* __restrict__ corraa) {
  float weight = weights[blockIdx.y];
  input += (uint64_t)elements * blockIdx.y;
  output += (uint64_t)elements * blockIdx.y;
  outweights += (uint64_t)elements * blockIdx.y;
  float norm = 0.f;
  if (weight >= sigweight) {
    weight *= invsum;
    for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < elements; id += gridDim.x * blockDim.x) {
      float c = ctf[id];
      float wx = weight * c * minvsigma2[id];
      float2 sh = input[id];
      float2 o = output[id];
      output[id] = make_float2(o.x + sh.x * wx, o.y + sh.y * wx);
      outweights[id] += wx * c;
      int ires = mresol[id];
      if (ires > -1) {
        float2 r = ref[id];
        float dx = r.x - sh.x, dy = r.y - sh.y;
        float wd = weight * (dx * dx + dy * dy);
        atomicAdd(sigma2noise + ires, wd);
        norm += wd;
        if (SCALE && priorclass[ires] > 3.f) {
          atomicAdd(corrxa + ires, weight * (r.x * sh.x + r.y * sh.y));
          atomicAdd(corraa + ires, weight * (r.x * r.x + r.y * r.y));
        }
      }
    }
  } else {
    for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < elements; id += gridDim.x * blockDim.x) {
      output[id] = make_float2(0.f, 0.f);
      outweights[id] = 0.f;
    }
  }
  // the normalisation correction: one atomic per warp instead of per element
  for (int o = 16; o > 0; o >>= 1) norm += __shfl_down_sync(0xffffffffu, norm, o);
  if ((threadIdx.x & 31) == 0 && norm != 0.f) atomicAdd(normcorr, norm);
}

struct Positive {
  __device__ __forceinline__ bool operator()(const float& x) const { return x > 0.f; }
};

}  // namespace
}  // namespace gtomrln

using namespace gtomrln;

static unsigned grid_for(uint64_t n, unsigned tpb = 256) {
  uint64_t b = (n + tpb - 1) / tpb;
  return (unsigned)(b < 148 * 32 ? (b ? b : 1) : 148 * 32);
}

extern "C" {

int gtomrln_squared_differences_sparse(const float* d_particleft, const float* d_minvsigma2,
                                       const float* d_ctf, int dx, int dy, int dz,
                                       const float* d_precalcshifts, const float* d_refft,
                                       float* d_diff2, const unsigned* d_combination,
                                       unsigned ncombinations, unsigned groupsize,
                                       int dofirstitercc, void* stream) {
  clear_error();
  if (groupsize == 0 || ncombinations % (groupsize * groupsize))
    return set_error(GTOMRLN_ERR_INVALID, "squared_differences_sparse: %u outputs not a multiple of %u^2",
                     ncombinations, groupsize);
  if (ncombinations == 0) return GTOMRLN_OK;
  if (!d_particleft || !d_precalcshifts || !d_refft || !d_diff2 || !d_combination)
    return set_error(GTOMRLN_ERR_INVALID, "squared_differences_sparse: NULL pointer");
  int64_t elements = (int64_t)(dx / 2 + 1) * dy * (dz > 1 ? dz : 1);
  unsigned groups = ncombinations / (groupsize * groupsize);
  return diff2_dispatch(groupsize, dofirstitercc != 0, groups, (cudaStream_t)stream, (const float2*)d_particleft,
                        d_minvsigma2, d_ctf, elements, (const float2*)d_precalcshifts, (const float2*)d_refft,
                        d_diff2, (const uint3*)d_combination, 0, 0, 0);
}

int gtomrln_squared_differences(const float* d_particleft, const float* d_minvsigma2, const float* d_ctf,
                                int dx, int dy, int dz, unsigned nparticles, const float* d_precalcshifts,
                                unsigned nshifts, const float* d_refft, unsigned nrefs, unsigned tile,
                                float* d_diff2, int dofirstitercc, void* stream) {
  clear_error();
  if (nparticles == 0 || nshifts == 0 || nrefs == 0) return GTOMRLN_OK;
  if (!d_particleft || !d_precalcshifts || !d_refft || !d_diff2)
    return set_error(GTOMRLN_ERR_INVALID, "squared_differences: NULL pointer");
  int64_t elements = (int64_t)(dx / 2 + 1) * dy * (dz > 1 ? dz : 1);
  if (tile != 1 && tile != 2 && tile != 4 && tile != 8)
    return set_error(GTOMRLN_ERR_INVALID, "squared_differences: group size %u not 1, 2, 4 or 8", tile);
  if (nparticles > 65535)
    return set_error(GTOMRLN_ERR_INVALID, "squared_differences: more than 65535 particles per call");
  // The dense layout does not depend on the group size: one tiled kernel.
  dim3 grid((nshifts + kDT - 1) / kDT, (nrefs + kDT - 1) / kDT, nparticles);
  if (dofirstitercc)
    diff2_dense_tiled_kernel<true><<<grid, kDThreads, 0, (cudaStream_t)stream>>>(
        (const float2*)d_particleft, d_minvsigma2, d_ctf, elements, (const float2*)d_precalcshifts,
        (const float2*)d_refft, d_diff2, nrefs, nshifts);
  else
    diff2_dense_tiled_kernel<false><<<grid, kDThreads, 0, (cudaStream_t)stream>>>(
        (const float2*)d_particleft, d_minvsigma2, d_ctf, elements, (const float2*)d_precalcshifts,
        (const float2*)d_refft, d_diff2, nrefs, nshifts);
  GTOMRLN_LAUNCH_CHECK("diff2_dense_tiled_kernel");
  return GTOMRLN_OK;
}

int gtomrln_convert_weights_dense(float* d_weights, unsigned nparticles, unsigned nclasses, unsigned nrot,
                                  unsigned ntrans, const float* d_pdfrot, const float* d_pdftrans,
                                  const float* d_mindiff2, void* stream) {
  clear_error();
  uint64_t perclass = (uint64_t)nrot * ntrans, perpart = perclass * nclasses, n = perpart * nparticles;
  if (n == 0) return GTOMRLN_OK;
  if (!d_weights || !d_pdfrot || !d_pdftrans || !d_mindiff2 || perpart > 0xffffffffULL)
    return set_error(GTOMRLN_ERR_INVALID, "convert_weights_dense: bad arguments");
  convert_dense_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_weights, n, (unsigned)perpart,
                                                                      (unsigned)perclass, nclasses, nrot, ntrans,
                                                                      d_pdfrot, d_pdftrans, d_mindiff2);
  GTOMRLN_LAUNCH_CHECK("convert_dense_kernel");
  return GTOMRLN_OK;
}

int gtomrln_convert_weights_sparse(float* d_weightsdense, float* d_weightssparse,
                                   const unsigned* d_combinations, unsigned nsparse, unsigned nrot,
                                   unsigned ntrans, const float* d_pdfrot, const float* d_pdftrans,
                                   const float* d_mindiff2, void* stream) {
  clear_error();
  if (nsparse == 0) return GTOMRLN_OK;
  if (!d_weightsdense || !d_weightssparse || !d_combinations || !d_pdfrot || !d_pdftrans || !d_mindiff2)
    return set_error(GTOMRLN_ERR_INVALID, "convert_weights_sparse: NULL pointer");
  convert_sparse_kernel<<<grid_for(nsparse), 256, 0, (cudaStream_t)stream>>>(
      d_weightsdense, d_weightssparse, (const uint4*)d_combinations, nsparse, nrot, ntrans, d_pdfrot, d_pdftrans,
      d_mindiff2);
  GTOMRLN_LAUNCH_CHECK("convert_sparse_kernel");
  return GTOMRLN_OK;
}

int gtomrln_convert_weights_sort(float* d_input, unsigned n, void* stream) {
  clear_error();
  if (n < 2) return GTOMRLN_OK;
  if (!d_input) return set_error(GTOMRLN_ERR_INVALID, "convert_weights_sort: NULL pointer");
  cudaStream_t s = (cudaStream_t)stream;
  size_t tbytes = 0;
  GTOMRLN_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tbytes, d_input, d_input, (int)n, 0, 32, s));
  char* buf = nullptr;
  int st = pool_alloc((void**)&buf, tbytes + 256 + (size_t)n * 4, s);
  if (st) return st;
  float* tmp = (float*)(buf + ((tbytes + 255) & ~(size_t)255));
  cudaError_t e = cub::DeviceRadixSort::SortKeys(buf, tbytes, d_input, tmp, (int)n, 0, 32, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_input, tmp, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);
  pool_free(buf, s);
  if (e != cudaSuccess) return set_error(GTOMRLN_ERR_CUDA, "convert_weights_sort: %s", cudaGetErrorString(e));
  return GTOMRLN_OK;
}

int gtomrln_convert_weights_compact(const float* d_input, float* d_output, unsigned* n, void* stream) {
  clear_error();
  if (!n) return set_error(GTOMRLN_ERR_INVALID, "convert_weights_compact: NULL count");
  if (*n == 0) return GTOMRLN_OK;
  if (!d_input || !d_output) return set_error(GTOMRLN_ERR_INVALID, "convert_weights_compact: NULL pointer");
  cudaStream_t s = (cudaStream_t)stream;
  size_t tbytes = 0;
  GTOMRLN_CUDA_TRY(cub::DeviceSelect::If(nullptr, tbytes, d_input, d_output, (int*)nullptr, (int)*n, Positive(), s));
  char* buf = nullptr;
  int st = pool_alloc((void**)&buf, tbytes + 256, s);
  if (st) return st;
  int* d_num = (int*)buf;
  cudaError_t e = cub::DeviceSelect::If(buf + 256, tbytes, d_input, d_output, d_num, (int)*n, Positive(), s);
  int h_num = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_num, d_num, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  pool_free(buf, s);
  if (e != cudaSuccess) return set_error(GTOMRLN_ERR_CUDA, "convert_weights_compact: %s", cudaGetErrorString(e));
  *n = (unsigned)h_num;
  return GTOMRLN_OK;
}

int gtomrln_diff_remap_dense(const float* d_input, float* d_output, const unsigned* d_orientationindices,
                             unsigned norientations, unsigned iclass, unsigned nparticles, unsigned nclasses,
                             unsigned nrot, unsigned ntrans, unsigned ntranspadded, const float* d_xi2imgs,
                             const float* d_sqrtxi2, int docc, void* stream) {
  clear_error();
  uint64_t n = (uint64_t)norientations * nparticles * ntrans;
  if (n == 0) return GTOMRLN_OK;
  if (!d_input || !d_output || !d_orientationindices || (docc ? !d_sqrtxi2 : !d_xi2imgs))
    return set_error(GTOMRLN_ERR_INVALID, "diff_remap_dense: NULL pointer");
  auto s = (cudaStream_t)stream;
  const uint3* o = (const uint3*)d_orientationindices;
  if (docc)
    remap_dense_kernel<true><<<grid_for(n), 256, 0, s>>>(d_input, d_output, o, n, iclass, nparticles, nclasses, nrot,
                                                         ntrans, ntranspadded, d_xi2imgs, d_sqrtxi2);
  else
    remap_dense_kernel<false><<<grid_for(n), 256, 0, s>>>(d_input, d_output, o, n, iclass, nparticles, nclasses,
                                                          nrot, ntrans, ntranspadded, d_xi2imgs, d_sqrtxi2);
  GTOMRLN_LAUNCH_CHECK("remap_dense_kernel");
  return GTOMRLN_OK;
}

int gtomrln_diff_remap_sparse(const float* d_input, float* d_output, float* d_mindiff2,
                              const unsigned* d_combinations, const unsigned* d_hiddenover, unsigned elements,
                              unsigned tileelements, unsigned weightsperpart, unsigned nparticles,
                              const float* d_xi2imgs, const float* d_sqrtxi2, int docc, void* stream) {
  clear_error();
  (void)nparticles;
  if (elements == 0) return GTOMRLN_OK;
  if (!d_input || !d_output || !d_mindiff2 || !d_combinations || !d_hiddenover || tileelements == 0 ||
      (docc ? !d_sqrtxi2 : !d_xi2imgs))
    return set_error(GTOMRLN_ERR_INVALID, "diff_remap_sparse: bad arguments");
  auto s = (cudaStream_t)stream;
  const uint3* c = (const uint3*)d_combinations;
  if (docc)
    remap_sparse_kernel<true><<<grid_for(elements), 256, 0, s>>>(d_input, d_output, d_mindiff2, c, d_hiddenover,
                                                                 elements, tileelements, weightsperpart, d_xi2imgs,
                                                                 d_sqrtxi2);
  else
    remap_sparse_kernel<false><<<grid_for(elements), 256, 0, s>>>(d_input, d_output, d_mindiff2, c, d_hiddenover,
                                                                  elements, tileelements, weightsperpart,
                                                                  d_xi2imgs, d_sqrtxi2);
  GTOMRLN_LAUNCH_CHECK("remap_sparse_kernel");
  return GTOMRLN_OK;
}

int gtomrln_create_minvsigma2s(float* d_output, const int* d_mresol, unsigned elements,
                               const float* d_sigma2noise, float sigma2fudge, void* stream) {
  clear_error();
  if (elements == 0) return GTOMRLN_OK;
  if (!d_output || !d_mresol || !d_sigma2noise) return set_error(GTOMRLN_ERR_INVALID, "create_minvsigma2s: NULL pointer");
  minvsigma2_kernel<<<grid_for(elements), 256, 0, (cudaStream_t)stream>>>(d_output, d_mresol, elements,
                                                                          d_sigma2noise, sigma2fudge);
  GTOMRLN_LAUNCH_CHECK("minvsigma2_kernel");
  return GTOMRLN_OK;
}

int gtomrln_store_weights_add(const float* d_input, const float* d_ctf, const float* d_ref,
                              const float* d_minvsigma2, const int* d_mresol, unsigned elements,
                              unsigned ntrans, const float* d_weights, float sigweight, float sumweight,
                              float* d_output, float* d_outputweights, float* d_sigma2noise,
                              float* d_normcorrection, const float* d_priorclass, float* d_correctionxa,
                              float* d_correctionaa, int doscale, void* stream) {
  clear_error();
  if (elements == 0 || ntrans == 0) return GTOMRLN_OK;
  if (!d_input || !d_ctf || !d_ref || !d_minvsigma2 || !d_mresol || !d_weights || !d_output ||
      !d_outputweights || !d_sigma2noise || !d_normcorrection ||
      (doscale && (!d_priorclass || !d_correctionxa || !d_correctionaa)))
    return set_error(GTOMRLN_ERR_INVALID, "store_weights_add: NULL pointer");
  if (ntrans > 65535) return set_error(GTOMRLN_ERR_INVALID, "store_weights_add: more than 65535 translations");
  dim3 grid((elements + 127) / 128, ntrans);
  float invsum = (float)(1.0 / sumweight);  // the reference passes 1.0 / sumweight
  auto s = (cudaStream_t)stream;
  if (doscale)
    store_weights_kernel<true><<<grid, 128, 0, s>>>((const float2*)d_input, d_ctf, (const float2*)d_ref,
                                                    d_minvsigma2, d_mresol, elements, d_weights, sigweight, invsum,
                                                    (float2*)d_output, d_outputweights, d_sigma2noise,
                                                    d_normcorrection, d_priorclass, d_correctionxa, d_correctionaa);
  else
    store_weights_kernel<false><<<grid, 128, 0, s>>>((const float2*)d_input, d_ctf, (const float2*)d_ref,
                                                     d_minvsigma2, d_mresol, elements, d_weights, sigweight, invsum,
                                                     (float2*)d_output, d_outputweights, d_sigma2noise,
                                                     d_normcorrection, d_priorclass, d_correctionxa, d_correctionaa);
  GTOMRLN_LAUNCH_CHECK("store_weights_kernel");
  return GTOMRLN_OK;
}

}  // extern "C"
