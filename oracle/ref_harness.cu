// C entry points over the reference's own CUDA implementation of the
// projector / backprojector / gridding reconstructor, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libgtomref.so.
//
// TEST INFRASTRUCTURE ONLY: used to pin the CPU oracle and to generate the
// golden fixtures in tests/golden/.  The product library never links it.
//
// Each wrapper calls the reference overload named beside it unchanged and
// returns cudaGetLastError() after a device synchronise.
#include "Prerequisites.cuh"
#include "Angles.cuh"
#include "Helper.cuh"
#include "Relion.cuh"
#include "Reconstruction.cuh"
#include "CTF.cuh"

using namespace gtom;

extern "C" {

// The host matrices of the h_angles overloads (src/Relion/Project.cu:14-16,
// src/Relion/Backproject.cu:29-31): the same expression, column-major glm
// layout, 9 floats per slice.
int ref_matrices(float* h_angles, float supersample, int batch, float* h_matrices) {
  for (int i = 0; i < batch; i++) {
    glm::mat3 m = glm::transpose(Matrix3Euler(((tfloat3*)h_angles)[i])) * Matrix3Scale(supersample);
    memcpy(h_matrices + 9 * (size_t)i, &m, sizeof(glm::mat3));
  }
  return 0;
}

// include/Relion.cuh:35 -> src/Relion/Project.cu:25-43
int ref_project(float* d_volumeft, int P, float* d_proj, int n, int ndims, int rmax,
                float* d_matrices, int batch) {
  int3 dv = toInt3(P, P, P);
  int3 dp = toInt3(n, n, ndims == 3 ? n : 1);
  d_rlnProject((tcomplex*)d_volumeft, dv, (tcomplex*)d_proj, dp, (uint)rmax,
               (glm::mat3*)d_matrices, (uint)batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:34 -> src/Relion/Project.cu:12-23
int ref_project_angles(float* d_volumeft, int P, float* d_proj, int n, int ndims,
                       float* h_angles, float supersample, int batch) {
  int3 dv = toInt3(P, P, P);
  int3 dp = toInt3(n, n, ndims == 3 ? n : 1);
  d_rlnProject((tcomplex*)d_volumeft, dv, (tcomplex*)d_proj, dp, (tfloat3*)h_angles,
               supersample, (uint)batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:9 -> src/Relion/Backproject.cu:48-124
int ref_backproject(float* d_volumeft, float* d_volumeweights, int P, float* d_projft,
                    float* d_projweights, int n, int ndims, int rmax, float* d_matrices,
                    int* d_ivolume, float mx, float my, float mz, float mw,
                    float ewaldradiussuper, int outputdecentered, int squareinterpweights,
                    int batch) {
  int3 dv = toInt3(P, P, P);
  int3 dp = toInt3(n, n, ndims == 3 ? n : 1);
  d_rlnBackproject((tcomplex*)d_volumeft, d_volumeweights, dv, (tcomplex*)d_projft,
                   d_projweights, dp, (uint)rmax, (glm::mat3*)d_matrices, d_ivolume,
                   make_float4(mx, my, mz, mw), ewaldradiussuper, outputdecentered != 0,
                   squareinterpweights != 0, (uint)batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:10 -> src/Relion/Backproject.cu:23-46
int ref_backproject_angles(float* d_volumeft, float* d_volumeweights, int P, float* d_projft,
                           float* d_projweights, int n, int ndims, int rmax, float* h_angles,
                           int* h_ivolume, float mx, float my, float mz, float mw,
                           float ewaldradius, float supersample, int outputdecentered,
                           int squareinterpweights, int batch) {
  int3 dv = toInt3(P, P, P);
  int3 dp = toInt3(n, n, ndims == 3 ? n : 1);
  d_rlnBackproject((tcomplex*)d_volumeft, d_volumeweights, dv, (tcomplex*)d_projft,
                   d_projweights, dp, (uint)rmax, (tfloat3*)h_angles, h_ivolume,
                   make_float4(mx, my, mz, mw), ewaldradius, supersample,
                   outputdecentered != 0, squareinterpweights != 0, (uint)batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:41 -> src/Relion/ProjectShifted.cu:58-75
int ref_project_shifted(float* d_volumeft, int P, float* d_proj, int n, int ndims, int rmax,
                        float* d_matrices, float* d_shifts, float* d_globalweights, int batch) {
  d_rlnProjectShifted((tcomplex*)d_volumeft, toInt3(P, P, P), (tcomplex*)d_proj,
                      toInt3(n, n, ndims == 3 ? n : 1), (uint)rmax, (glm::mat3*)d_matrices,
                      (tfloat3*)d_shifts, d_globalweights, (uint)batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:18 -> src/Relion/BackprojectShifted.cu:37-58
int ref_backproject_shifted(float* d_volumeft, float* d_volumeweights, int V, float* d_projft,
                            float* d_projweights, int n, int ndims, int rmax, float* d_matrices,
                            float* d_shifts, float* d_globalweights, int batch) {
  d_rlnBackprojectShifted((tcomplex*)d_volumeft, d_volumeweights, toInt3(V, V, V), (tcomplex*)d_projft,
                          d_projweights, toInt3(n, n, ndims == 3 ? n : 1), (uint)rmax,
                          (glm::mat3*)d_matrices, (tfloat3*)d_shifts, d_globalweights, (uint)batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/CTF.cuh:317 -> src/CTF/Simulate.cu:22-47 (h_params: 14 floats per
// CTFParams, in the struct's order)
int ref_ctf_simulate(float* h_params, float* d_addresses, float* d_gammacorrection, float* d_output,
                     int n, int amplitudesquared, int ignorefirstpeak, int batch) {
  d_CTFSimulate((CTFParams*)h_params, (float2*)d_addresses, d_gammacorrection, d_output, (uint)n,
                amplitudesquared != 0, ignorefirstpeak != 0, batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:14 -> src/Relion/BackprojectTomo.cu:30-46
int ref_backproject_tomo(float* d_volumeft, int V, float* d_projft, float* d_projweights, int n, int rmax,
                         float* d_matrices, int batch) {
  d_BackprojectTomo((tcomplex*)d_volumeft, toInt3(V, V, V), (tcomplex*)d_projft, d_projweights, toInt3(n, n, 1),
                    (uint)rmax, (glm::mat3*)d_matrices, (uint)batch);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:21-24 -> src/Relion/ConvertWeights.cu
int ref_convert_weights_dense(float* d_weights, int nparticles, int nclasses, int nrot, int ntrans,
                              float* d_pdfrot, float* d_pdftrans, float* d_mindiff2) {
  d_rlnConvertWeightsDense(d_weights, nparticles, nclasses, nrot, ntrans, d_pdfrot, d_pdftrans, d_mindiff2);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

int ref_convert_weights_sparse(float* d_dense, float* d_sparse, unsigned* d_combinations, int nsparse, int nrot,
                               int ntrans, float* d_pdfrot, float* d_pdftrans, float* d_mindiff2) {
  d_rlnConvertWeightsSparse(d_dense, d_sparse, (uint4*)d_combinations, nsparse, nrot, ntrans, d_pdfrot, d_pdftrans,
                            d_mindiff2);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:27-28 -> src/Relion/DiffRemap.cu
int ref_diff_remap_dense(float* d_input, float* d_output, unsigned* d_orient, int norient, int iclass,
                         int nparticles, int nclasses, int nrot, int ntrans, int ntranspadded, float* d_xi2,
                         float* d_sqrtxi2, int docc) {
  d_rlnDiffRemapDense(d_input, d_output, (uint3*)d_orient, norient, iclass, nparticles, nclasses, nrot, ntrans,
                      ntranspadded, d_xi2, d_sqrtxi2, docc != 0);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

int ref_diff_remap_sparse(float* d_input, float* d_output, float* d_mindiff2, unsigned* d_combinations,
                          unsigned* d_hiddenover, int elements, int tileelements, int weightsperpart,
                          int nparticles, float* d_xi2, float* d_sqrtxi2, int docc) {
  d_rlnDiffRemapSparse(d_input, d_output, d_mindiff2, (uint3*)d_combinations, d_hiddenover, elements, tileelements,
                       weightsperpart, nparticles, d_xi2, d_sqrtxi2, docc != 0);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:31 -> src/Relion/Misc.cu:12-17
int ref_create_minvsigma2s(float* d_output, int* d_mresol, int elements, float* d_sigma2noise, float fudge) {
  d_rlnCreateMinvsigma2s(d_output, d_mresol, elements, d_sigma2noise, fudge);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Relion.cuh:51-57 -> src/Relion/StoreWeights.cu:9-18
int ref_store_weights_add(float* d_input, float* d_ctf, float* d_ref, float* d_minvsigma2, int* d_mresol,
                          int elements, int ntrans, float* d_weights, float sigweight, float sumweight,
                          float* d_output, float* d_outputweights, float* d_sigma2noise, float* d_normcorrection,
                          float* d_priorclass, float* d_correctionxa, float* d_correctionaa, int doscale) {
  d_rlnStoreWeightsAdd((tcomplex*)d_input, d_ctf, (tcomplex*)d_ref, d_minvsigma2, d_mresol, elements, ntrans,
                       d_weights, sigweight, sumweight, (tcomplex*)d_output, d_outputweights, d_sigma2noise,
                       d_normcorrection, d_priorclass, d_correctionxa, d_correctionaa, doscale != 0);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

// include/Reconstruction.cuh:16 -> src/Reconstruction/RecFourier.cu:98-241
int ref_reconstruct_gridding(float* d_dataft, float* d_weight, float* d_reconstructed, int ori,
                             int padded, int paddingfactor, int iterations, double blobradius,
                             int bloborder, double blobalpha) {
  d_ReconstructGridding((tcomplex*)d_dataft, d_weight, d_reconstructed, toInt3(ori, ori, ori),
                        toInt3(padded, padded, padded), paddingfactor, NULL, NULL, iterations,
                        blobradius, bloborder, blobalpha);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

}  // extern "C"
