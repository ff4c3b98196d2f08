// Batched gridding of many equal-size volumes (one size class of a batch of
// uneven reconstructions): stacks of working buffers, batched cuFFT plans
// and the gridding kernels launched once per step over the whole stack
// (gridding.cu).  Used by the batched reconstructor (batch.cu).
#pragma once

#include <cufft.h>

#include <cstdint>

namespace gtomrln {

struct GridBatch {
  int count = 0;       // volumes in the stack
  int ori = 0;         // output box
  int pad = 0;         // padding factor
  int P = 0;           // working grid ori * pad
  int D = 0;           // centred input box (P + 1)
  int64_t wstride = 0; // elements between input volumes, (D/2+1) D D
  float2* convft = nullptr;
  float* conv = nullptr;
  float* Fw = nullptr;
  float* Fnw = nullptr;
  cufftHandle r2c = 0, c2r = 0;
  const float* table = nullptr;
  bool fused = false;  // the fused FFT iteration is prepared (outside any capture) and available
  bool sym = false;    // the symmetric-spectrum iteration is prepared (outside any capture) and available
};

// Allocates the stacks (cudaMalloc) and makes the batched plans.
int gridding_batch_prepare(GridBatch* gb, int count, int ori, int pad, double blobradius,
                           int bloborder, double blobalpha);
// Enqueues `iterations` gridding iterations and the final maps on stream:
// data / weight are stacks of centred (D/2+1) x D x D volumes, outs[i]
// (device array of device pointers) receives volume i's ori^3 map.
int gridding_batch_run(const GridBatch& gb, const float2* data, const float* weight,
                       float* const* outs, int iterations, cudaStream_t stream);
void gridding_batch_free(GridBatch* gb);

}  // namespace gtomrln
